"""Batched Newton-Raphson on the GPU against the oracle and the reference's goldens.

Bars: V within 1e-8 of the FP64 oracle run to 1e-12; with FP64 factors the
iteration counts equal the oracle's on the same stopping rule (the NR loop
semantics of newton_solver.cpp:245-342: iterations = norm evaluations,
convergence tested before the Jacobian, final mismatch = last evaluated norm).
"""
from pathlib import Path

import numpy as np
import pytest

import cupf
from cupf import grids as G
from conftest import gpu_available, max_dv_vs_oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]
GOLD = Path(__file__).resolve().parent / "golden"
POLICIES = {"FP64": cupf.ComputePolicy.FP64, "Mixed": cupf.ComputePolicy.Mixed}


def make_solver(g, compute, graph=False, serial_nd=True, autotune=False):
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = compute
    o.use_cuda_graph = graph
    o.custom.serial_nd = serial_nd
    o.custom.autotune = autotune
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    return s


def cfg(tol=1e-8, max_iter=10):
    c = cupf.NRConfig()
    c.tolerance = tol
    c.max_iter = max_iter
    return c


def solve(s, g, S, V0, c):
    return s.solve_batch(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, S, V0, g.pv, g.pq, c)


class TwoBus:
    def __init__(self):
        c = G.two_bus_case()
        self.c = c
        self.indptr, self.indices, self.data = c["indptr"], c["indices"], c["data"]
        self.pv, self.pq, self.n_bus = c["pv"], c["pq"], 2


@pytest.mark.parametrize("policy", list(POLICIES))
@pytest.mark.parametrize("graph", [False, True])
def test_two_bus(policy, graph):
    """cuPF/tests/unit/test_minimal_solver.cpp:100-346 (FP64/FP32/Mixed, batch 2, graph)."""
    g = TwoBus()
    s = make_solver(g, POLICIES[policy], graph=graph)
    S = np.stack([g.c["sbus"]] * 2)
    V0 = np.stack([g.c["v0"]] * 2)
    r = solve(s, g, S, V0, cfg(1e-10, 20))
    assert r.converged_numpy.all()
    assert np.abs(r.V_numpy - g.c["expected_v"][None, :]).max() <= 1e-8
    single = s.solve(g.indptr, g.indices, g.data, 2, 2, g.c["sbus"], g.c["v0"], g.pv, g.pq, cfg(1e-10, 20))
    assert single.converged and abs(single.V_numpy - g.c["expected_v"]).max() <= 1e-8


@pytest.mark.parametrize("policy", list(POLICIES))
def test_118_matches_oracle(oracle, policy):
    g = G.grid_118()
    B = 40  # more than one warp of scenarios, ragged last warp
    S = g.scenarios(B, seed=17)
    V0 = g.flat_start(B)
    s = make_solver(g, POLICIES[policy])
    r = solve(s, g, S, V0, cfg())
    assert r.converged_numpy.all()
    for b in range(0, B, 7):
        tight = oracle.solve(g, S[b], V0[b], tol=1e-12, max_iter=30)
        assert np.abs(r.V_numpy[b] - tight["V"]).max() <= 1e-8
        same = oracle.solve(g, S[b], V0[b], tol=1e-8, max_iter=10)
        if policy == "FP64":
            assert r.iterations_numpy[b] == same["iterations"]
            assert r.final_mismatch_numpy[b] == pytest.approx(same["final_mismatch"], rel=1e-3, abs=1e-13)
        assert r.final_mismatch_numpy[b] <= 1e-8


def test_118_matches_reference_golden():
    """The reference CPU NewtonSolver's answers (tests/golden/nr_118.npz)."""
    g = G.grid_118()
    gold = np.load(GOLD / "nr_118.npz")
    s = make_solver(g, cupf.ComputePolicy.FP64)
    r = solve(s, g, gold["sbus"], gold["v0"], cfg(1e-8, 10))
    assert np.array_equal(r.iterations_numpy, gold["it_t8"])
    assert np.abs(r.V_numpy - gold["V_t8"]).max() <= 1e-10
    r12 = solve(s, g, gold["sbus"], gold["v0"], cfg(1e-12, 30))
    assert np.abs(r12.V_numpy - gold["V_t12"]).max() <= 1e-11


@pytest.mark.parametrize("policy", ["FP64", "Mixed"])
def test_2000_matches_oracle(oracle, policy):
    """The benchmark's workload at full size (2,000 buses x 1,024 scenarios,
    flat start): every scenario converges and lies within 1e-8 of the FP64
    oracle solved to 1e-12; in FP64 the batch's iteration count is the
    oracle's largest at the same stopping rule."""
    import os

    g = G.grid_2000()
    B = 1024
    S = g.scenarios(B, seed=23)
    V0 = g.flat_start(B)
    s = make_solver(g, POLICIES[policy], graph=True)
    r = solve(s, g, S, V0, cfg())
    assert r.converged_numpy.all()
    dv = max_dv_vs_oracle(oracle, g, S, V0, r.V_numpy)
    assert dv.max() <= 1e-8, (int(dv.argmax()), float(dv.max()))
    if policy == "FP64":
        its = oracle.solve_many(g, S, V0, tol=1e-8, max_iter=10, threads=os.cpu_count() or 1)["iterations"]
        assert r.iterations_numpy[0] == its.max()


def test_2000_matches_reference_golden():
    g = G.grid_2000()
    gold = np.load(GOLD / "nr_2000.npz")
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    r = solve(s, g, gold["sbus"], gold["v0"], cfg(1e-8, 10))
    assert r.converged_numpy.all()
    assert np.abs(r.V_numpy - gold["V_t12"]).max() <= 1e-8


def test_10000_mixed_matches_oracle(oracle):
    """The 10,000-bus x 64 workload: every scenario within 1e-8 of the oracle."""
    g = G.grid_10000()
    B = 64
    S = g.scenarios(B, seed=29)
    V0 = g.flat_start(B)
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    r = solve(s, g, S, V0, cfg())
    assert r.converged_numpy.all()
    dv = max_dv_vs_oracle(oracle, g, S, V0, r.V_numpy)
    assert dv.max() <= 1e-8, (int(dv.argmax()), float(dv.max()))


def test_10000_nominal_state_warm_start(oracle):
    """The 10,000-bus x 64 workload started from the converged nominal-load
    state (cupf.warm_start.nominal_state): fewer Newton norms than from the
    flat start, and every scenario within 1e-8 of the oracle's flat-start
    solution."""
    from cupf.warm_start import nominal_state

    g = G.grid_10000()
    B = 64
    S = g.scenarios(B, seed=29)
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    vnom = nominal_state(s, g).cpu().numpy()
    flat = solve(s, g, S, g.flat_start(B), cfg(max_iter=20))
    warm = solve(s, g, S, np.repeat(vnom[None, :], B, axis=0), cfg(max_iter=20))
    assert warm.converged_numpy.all() and flat.converged_numpy.all()
    assert warm.iterations_numpy.max() < flat.iterations_numpy.max()
    dv = max_dv_vs_oracle(oracle, g, S, g.flat_start(B), warm.V_numpy)
    assert dv.max() <= 1e-8, (int(dv.argmax()), float(dv.max()))


def test_identical_rows_agree():
    """test_cpu_solver.cpp:355-359: batch rows of the same case agree."""
    g = G.grid_118()
    S = np.repeat(g.scenarios(1, seed=3), 37, axis=0)
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    r = solve(s, g, S, g.flat_start(37), cfg())
    assert np.abs(r.V_numpy - r.V_numpy[0:1]).max() == 0.0
    assert len(set(r.iterations_numpy.tolist())) == 1


def test_graph_mode_matches_stream_mode():
    g = G.grid_2000()
    S = g.scenarios(64, seed=41)
    V0 = g.flat_start(64)
    a = solve(make_solver(g, cupf.ComputePolicy.Mixed), g, S, V0, cfg())
    b = solve(make_solver(g, cupf.ComputePolicy.Mixed, graph=True), g, S, V0, cfg())
    assert np.array_equal(a.V_numpy, b.V_numpy)
    assert np.array_equal(a.iterations_numpy, b.iterations_numpy)


def test_not_converged_reports_last_norm(oracle):
    """max_iter too small: converged False and final_mismatch = the last norm evaluated."""
    g = G.grid_118()
    S = g.scenarios(4, seed=5)
    V0 = g.flat_start(4)
    s = make_solver(g, cupf.ComputePolicy.FP64)
    r = solve(s, g, S, V0, cfg(1e-8, 2))
    assert not r.converged_numpy.any()
    assert (r.iterations_numpy == 2).all()
    for b in range(4):
        o = oracle.solve(g, S[b], V0[b], tol=1e-8, max_iter=2)
        assert r.final_mismatch_numpy[b] == pytest.approx(o["final_mismatch"], rel=1e-9)
        assert np.abs(r.V_numpy[b] - o["V"]).max() <= 1e-12


def test_device_entry_point_matches_host():
    import torch

    g = G.grid_2000()
    S = g.scenarios(33, seed=8)
    V0 = g.flat_start(33)
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    host = solve(s, g, S, V0, cfg())
    v, fm, it = s.solve_batch_device(torch.tensor(S, device="cuda"), torch.tensor(V0, device="cuda"), config=cfg())
    assert np.array_equal(v.cpu().numpy(), host.V_numpy)
    assert np.array_equal(fm.cpu().numpy(), host.final_mismatch_numpy)


def test_evaluate_matches_oracle(oracle):
    """Mismatch F and Jacobian values at arbitrary states (FP64 kernels)."""
    g = G.grid_2000()
    rng = np.random.default_rng(4)
    B = 3
    V = (1 + 0.05 * rng.standard_normal((B, g.n_bus))) * np.exp(1j * 0.1 * rng.standard_normal((B, g.n_bus)))
    S = g.scenarios(B, seed=9)
    s = make_solver(g, cupf.ComputePolicy.FP64)
    F, J = s.evaluate(V, S)
    for b in range(B):
        Fo, _ = oracle.mismatch(g, S[b], V[b])
        Jo = oracle.jacobian_values(g, V[b])
        assert np.abs(F[b] - Fo).max() <= 1e-12 * max(1.0, np.abs(Fo).max())
        assert np.abs(J[b] - Jo).max() <= 1e-12 * np.abs(Jo).max()


def test_stage_profiling_counts_launches():
    g = G.grid_118()
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    s.set_profiling(True)
    r = solve(s, g, g.scenarios(8), g.flat_start(8), cfg())
    st = s.stage_times()
    s.set_profiling(False)
    it = int(r.iterations_numpy[0])
    assert st["mismatch"][1] == it
    assert st["jacobian"][1] == it - 1
    assert all(v[0] >= 0.0 for v in st.values())


def test_uneven_multi_grid_batch(oracle):
    """The uneven batch at its full size (118/500/2,000/10,000 buses x
    256/128/96/32 instances): solved concurrently, one engine and stream per
    grid; every one of the 512 instances converges, equals the same grid
    solved alone, and lies within 1e-8 of the oracle."""
    import torch
    from cupf.batching import UnevenBatch

    inst = G.uneven_grids()
    counts = [c for _, c in inst]
    grids = [g for g, _ in inst]
    ub = UnevenBatch(grids)
    S = [torch.tensor(g.scenarios(c, seed=31 + i), device="cuda") for i, (g, c) in enumerate(zip(grids, counts))]
    V0 = [torch.tensor(g.flat_start(c), device="cuda") for g, c in zip(grids, counts)]
    res = ub.solve(S, V0, cfg())
    alone = ub.solve(S, V0, cfg(), concurrent=False)
    for i, (g, c) in enumerate(zip(grids, counts)):
        V, fm, it = res[i]
        assert bool((fm <= 1e-8).all())
        assert torch.equal(V, alone[i][0])
        dv = max_dv_vs_oracle(oracle, g, S[i].cpu().numpy(), V0[i].cpu().numpy(), V.cpu().numpy())
        assert dv.size == c and dv.max() <= 1e-8, (g.n_bus, int(dv.argmax()), float(dv.max()))


def test_dump_case_solves_like_the_grid(tmp_path):
    """A grid written in the dump-case format and read back solves to the
    same voltages, bit for bit, on the batch cupf_bench builds from a case
    (load scale 1 + step * b, cuPF/tests/cupf_bench.cpp:188-198)."""
    from cupf import case_io

    g = G.grid_2000()
    c = case_io.load_dump_case(case_io.save_grid(tmp_path, g))
    S, V0 = case_io.replicate_scenarios(c, 40, load_scale_step=0.001)
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    a = s.solve_batch(c.indptr, c.indices, c.ybus_data, c.rows, c.cols, S, V0, c.pv, c.pq, cfg())
    b = solve(s, g, S, V0, cfg())
    assert a.converged_numpy.all()
    assert np.array_equal(a.V_numpy, b.V_numpy)


def test_structural_matching_gives_the_same_solution():
    """CustomMatchingMode::Structural on a Newton Jacobian (its diagonal is
    structurally full, so the matching is the identity): the same voltages,
    bit for bit."""
    g = G.grid_2000()
    S, V0 = g.scenarios(40, seed=19), g.flat_start(40)
    a = solve(make_solver(g, cupf.ComputePolicy.Mixed), g, S, V0, cfg())
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.serial_nd = True
    o.custom.matching = cupf.CustomMatchingMode.Structural
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    b = solve(s, g, S, V0, cfg())
    assert np.array_equal(a.V_numpy, b.V_numpy)


@pytest.mark.parametrize("kind", ["Edge", "EdgeAtomic", "VertexWarp"])
def test_jacobian_kinds_match_oracle(oracle, kind):
    """CudaJacobianKind (newton_solver_types.hpp:96-100): every fill gives the
    oracle's Jacobian values, and the Newton solve converges to the oracle's
    voltages with each of them."""
    g = G.grid_2000()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.FP64
    o.custom.serial_nd = True
    o.cuda_jacobian = getattr(cupf.CudaJacobianKind, kind)
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    rng = np.random.default_rng(21)
    V = (1 + 0.05 * rng.standard_normal((3, g.n_bus))) * np.exp(1j * 0.1 * rng.standard_normal((3, g.n_bus)))
    _, J = s.evaluate(V, g.scenarios(3, seed=2))
    for b in range(3):
        Jo = oracle.jacobian_values(g, V[b])
        assert np.abs(J[b] - Jo).max() <= 1e-12 * np.abs(Jo).max()
    S = g.scenarios(40, seed=24)
    o.compute = cupf.ComputePolicy.Mixed
    m = cupf.NewtonSolver(o)
    m.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    r = solve(m, g, S, g.flat_start(40), cfg())
    assert r.converged_numpy.all()
    for b in (0, 39):
        ref = oracle.solve(g, S[b], g.v0, tol=1e-12, max_iter=30)["V"]
        assert np.abs(r.V_numpy[b] - ref).max() <= 1e-8


def test_graph_loop_capped_and_failed_scenarios_match_stream_mode():
    """The device-side Newton loop (one graph per solve, conditional WHILE
    node) keeps the host loop's semantics: with the iteration cap reached it
    reports the cap, the last evaluated norms and the state after the last
    update; a warm-started scenario whose state goes non-finite fails alone
    (final mismatch inf) and the solve reports not all converged."""
    import torch

    g = G.grid_2000()
    S, V0 = g.scenarios(40, seed=45), g.flat_start(40)
    for mi in (1, 2, 3):
        a = solve(make_solver(g, cupf.ComputePolicy.Mixed), g, S, V0, cfg(1e-8, mi))
        b = solve(make_solver(g, cupf.ComputePolicy.Mixed, graph=True), g, S, V0, cfg(1e-8, mi))
        assert np.array_equal(a.iterations_numpy, b.iterations_numpy) and (b.iterations_numpy == mi).all()
        assert np.array_equal(a.final_mismatch_numpy, b.final_mismatch_numpy)
        assert np.array_equal(a.V_numpy, b.V_numpy)
        assert not b.converged_numpy.any()
    dS = torch.tensor(S, device="cuda")
    v0 = torch.tensor(g.v0, device="cuda")
    pvpq = torch.tensor(np.concatenate([g.pv, g.pq]), device="cuda")
    pq = torch.tensor(g.pq, device="cuda")
    ref, _, _ = make_solver(g, cupf.ComputePolicy.FP64).solve_batch_device(
        dS, torch.tensor(V0, device="cuda"), config=cfg(1e-10, 20))
    pred = torch.cat([torch.angle(ref)[:, pvpq], torch.abs(ref)[:, pq]], 1).float().contiguous()
    pred[7, 3] = float("nan")
    out = {}
    for graph in (False, True):
        s = make_solver(g, cupf.ComputePolicy.Mixed, graph=graph)
        V, fm, it = s.solve_batch_warm_device(dS, v0, pred, config=cfg(1e-8, 10))
        out[graph] = (V, fm, it, s.last_all_converged)
    for graph in (False, True):
        V, fm, it, allc = out[graph]
        assert np.isinf(fm[7].item()) and not allc
        ok = torch.ones(40, dtype=torch.bool, device="cuda")
        ok[7] = False
        assert bool((fm[ok] <= 1e-8).all())
    assert torch.equal(out[False][1], out[True][1]) and out[False][2] == out[True][2]


@pytest.mark.parametrize("policy", ["FP64", "Mixed"])
@pytest.mark.parametrize("graph", [False, True])
def test_autotuned_factor_launches_give_identical_solves(policy, graph):
    """CustomSolverConfig.autotune: the warps per block of every factor level
    and backward-sweep launch are timed and chosen at the first solve of each
    batch size; the solves stay bit for bit those of the built-in rule."""
    g = G.grid_2000()
    S, V0 = g.scenarios(256, seed=77), g.flat_start(256)
    base = make_solver(g, POLICIES[policy], graph)
    tuned = make_solver(g, POLICIES[policy], graph, autotune=True)
    assert not tuned.plan_array("factor_level_warps").any()  # nothing tuned before a solve
    for B in (256, 96, 256):  # a new batch size tunes again
        a = solve(base, g, S[:B], V0[:B], cfg())
        b = solve(tuned, g, S[:B], V0[:B], cfg())
        assert np.array_equal(a.V_numpy, b.V_numpy)
        assert np.array_equal(a.final_mismatch_numpy, b.final_mismatch_numpy)
        w = tuned.plan_array("factor_level_warps")
        assert w.size > 0 and set(w.tolist()) <= {0, 1, 2, 4, 8, 16, 32}
        wb = tuned.plan_array("backward_launch_warps")
        assert wb.size > 0 and set(wb.tolist()) <= {0, 1, 2, 4, 8}
    assert not base.plan_array("factor_level_warps").any()
    assert not base.plan_array("backward_launch_warps").any()


@pytest.mark.parametrize("width,serial", [(1, True), (4, True), (8, False)])
def test_other_plans_solve_like_the_oracle(oracle, width, serial):
    """The numeric path on plans other than the default: relaxed panels capped
    at 1 or 4 columns, and a separator-recursion ordering split down to
    500-vertex parts.  V within 1e-8 of the FP64 oracle on the 2,000-bus grid."""
    g = G.grid_2000()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.serial_nd = serial
    o.custom.max_panel_width = width
    o.custom.parallel_nd_depth = 4
    o.custom.parallel_nd_base_small = 500
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    B = 16
    S, V0 = g.scenarios(B, seed=61), g.flat_start(B)
    r = solve(s, g, S, V0, cfg())
    assert r.converged_numpy.all()
    for b in (0, 7, 15):
        ref = oracle.solve(g, S[b], V0[b], tol=1e-12, max_iter=30)
        assert np.abs(r.V_numpy[b] - ref["V"]).max() <= 1e-8


def test_tf32_factors_on_the_10000_bus_grid(oracle):
    """CustomPrecision.TF32 in the Newton loop (Mixed state), tensor-core
    threshold 33: the launches whose fronts reach 33 rows (the top of the
    10,000-bus grid's tree, fronts
    up to 38 rows) run their trailing updates on the tensor cores; every
    scenario still converges to 1e-8 and lies within 1e-8 of the oracle, the
    Newton iteration being the refinement back to FP64 accuracy."""
    g = G.grid_10000()
    B = 64
    S = g.scenarios(B, seed=29)
    V0 = g.flat_start(B)
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.precision = cupf.CustomPrecision.TF32
    o.custom.tc_min_front = 33
    o.custom.serial_nd = True
    o.custom.autotune = False
    o.use_cuda_graph = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    assert 2 in s.plan_array("factor_level_tiers")
    r = solve(s, g, S, V0, cfg())
    assert r.converged_numpy.all()
    dv = max_dv_vs_oracle(oracle, g, S, V0, r.V_numpy)
    assert dv.max() <= 1e-8, float(dv.max())
