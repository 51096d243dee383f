"""Per-scenario Ybus values on one pattern (parameter and contingency sweeps).

The reference's storage carries a per-case Ybus value stride
(cuda_batched_storage.hpp:84-89) that its Ibus kernel rejects
(compute_ibus.cu:45-48).  Here every scenario may bring its own values:
each scenario must match the FP64 oracle solved with that scenario's Ybus,
and values that equal the shared ones must give the shared solve bit for bit.
"""
import types

import numpy as np
import pytest

import cupf
from cupf import grids as G
from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def make_solver(g, compute, graph=False):
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = compute
    o.use_cuda_graph = graph
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    return s


def cfg(tol=1e-8, max_iter=10):
    return cupf.NRConfig(tolerance=tol, max_iter=max_iter)


def with_data(g, data):
    return types.SimpleNamespace(indptr=g.indptr, indices=g.indices, data=data, pv=g.pv, pq=g.pq, n_bus=g.n_bus,
                                 dim_f=g.dim_f)


@pytest.mark.parametrize("policy", [cupf.ComputePolicy.FP64, cupf.ComputePolicy.Mixed])
@pytest.mark.parametrize("graph", [False, True])
def test_replicated_values_equal_the_shared_solve(policy, graph):
    g = G.grid_2000()
    S, V0 = g.scenarios(40, seed=3), g.flat_start(40)
    s = make_solver(g, policy, graph)
    shared = s.solve_batch(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, S, V0, g.pv, g.pq, cfg())
    rep = np.repeat(g.data[None, :], 40, axis=0)
    per = s.solve_batch(g.indptr, g.indices, rep, g.n_bus, g.n_bus, S, V0, g.pv, g.pq, cfg())
    assert np.array_equal(per.V_numpy, shared.V_numpy)
    assert np.array_equal(per.final_mismatch_numpy, shared.final_mismatch_numpy)


@pytest.mark.parametrize("policy", [cupf.ComputePolicy.FP64, cupf.ComputePolicy.Mixed])
def test_branch_sweep_matches_oracle(oracle, policy):
    g = G.grid_2000()
    B = 40
    Y = g.branch_scaled_ybus(B, 0.8, 1.2, seed=11)
    S, V0 = g.scenarios(B, seed=12), g.flat_start(B)
    s = make_solver(g, policy)
    r = s.solve_batch(g.indptr, g.indices, Y, g.n_bus, g.n_bus, S, V0, g.pv, g.pq, cfg())
    assert r.converged_numpy.all()
    for b in (0, 13, 31, 39):
        o = oracle.solve(with_data(g, Y[b]), S[b], V0[b], tol=1e-12, max_iter=30)
        assert np.abs(r.V_numpy[b] - o["V"]).max() <= 1e-8
    # the same scenarios with the shared Ybus land elsewhere: the values are used
    base = s.solve_batch(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, S, V0, g.pv, g.pq, cfg())
    assert np.abs(base.V_numpy - r.V_numpy).max() > 1e-4


def test_device_entry_and_graph_switching(oracle):
    """Device tensors; a graph-mode handle alternating shared and per-scenario
    values recaptures its iteration and keeps every result exact."""
    import torch

    g = G.grid_118()
    B = 33
    Y = g.branch_scaled_ybus(B, 0.7, 1.3, seed=5)
    S, V0 = g.scenarios(B, seed=6), g.flat_start(B)
    dS, dV0, dY = (torch.tensor(a, device="cuda") for a in (S, V0, Y))
    s = make_solver(g, cupf.ComputePolicy.Mixed, graph=True)
    fresh_shared = make_solver(g, cupf.ComputePolicy.Mixed, graph=True)
    ref_shared, _, _ = fresh_shared.solve_batch_device(dS, dV0, config=cfg())
    for _ in range(2):
        v1, fm1, _ = s.solve_batch_device(dS, dV0, config=cfg())
        v2, fm2, _ = s.solve_batch_device(dS, dV0, config=cfg(), ybus=dY)
        assert torch.equal(v1, ref_shared)
        assert bool((fm2 <= 1e-8).all())
    v2 = v2.cpu().numpy()
    for b in (0, 32):
        o = oracle.solve(with_data(g, Y[b]), S[b], V0[b], tol=1e-12, max_iter=30)
        assert np.abs(v2[b] - o["V"]).max() <= 1e-8


def test_adjoint_uses_the_scenario_values(oracle):
    g = G.grid_118()
    B = 6
    Y = g.branch_scaled_ybus(B, 0.8, 1.2, seed=8)
    S, V0 = g.scenarios(B, seed=9), g.flat_start(B)
    s = make_solver(g, cupf.ComputePolicy.FP64)
    so = cupf.SolveOptions(prepare_adjoint_cache=True)
    r = s.solve_batch(g.indptr, g.indices, Y, g.n_bus, g.n_bus, S, V0, g.pv, g.pq, cfg(1e-12, 30), so)
    rng = np.random.default_rng(4)
    ga, gm = rng.standard_normal((B, g.n_bus)), rng.standard_normal((B, g.n_bus))
    a = s.solve_adjoint(ga, gm, g.pv, g.pq)
    for b in range(B):
        o = oracle.adjoint(with_data(g, Y[b]), r.V_numpy[b], ga[b], gm[b])
        for mine, ref in ((a.grad_load_p_numpy[b], o["grad_p"]), (a.grad_load_q_numpy[b], o["grad_q"])):
            assert np.abs(mine - ref).max() <= 1e-6 * np.abs(ref).max()


def test_bad_shapes_are_rejected():
    g = G.grid_118()
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    S, V0 = g.scenarios(4), g.flat_start(4)
    with pytest.raises(ValueError):
        s.solve_batch(g.indptr, g.indices, np.repeat(g.data[None, :], 3, axis=0), g.n_bus, g.n_bus, S, V0, g.pv,
                      g.pq, cfg())
