"""Adjoint load gradients on the GPU: J^T lambda = dL/dx on the final-state
factors, grad_load = -lambda (newton_solver_adjoint.cpp:33-153,
adjoint_math.cpp:62-154).  Bars: within 1e-6 relative of the reference's own
solve_adjoint (tests/golden/adjoint_*.npz) and of central differences (h=1e-6)."""
from pathlib import Path

import numpy as np
import pytest

import cupf
from cupf import grids as G
from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]
GOLD = Path(__file__).resolve().parent / "golden"


def make_solver(g, compute):
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = compute
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    return s


def forward(s, g, S, V0, tol=1e-12, max_iter=30, prepare=True):
    c = cupf.NRConfig(tolerance=tol, max_iter=max_iter)
    so = cupf.SolveOptions(prepare_adjoint_cache=prepare)
    return s.solve_batch(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, S, V0, g.pv, g.pq, c, so)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", ["118", "2000"])
@pytest.mark.parametrize("policy", [cupf.ComputePolicy.FP64, cupf.ComputePolicy.Mixed])
def test_adjoint_matches_reference(name, policy):
    g = {"118": G.grid_118, "2000": G.grid_2000}[name]()
    gold = np.load(GOLD / f"adjoint_{name}.npz")
    s = make_solver(g, policy)
    tol = 1e-12 if policy == cupf.ComputePolicy.FP64 else 1e-10
    r = forward(s, g, gold["sbus"][None, :], gold["v0"][None, :], tol=tol)
    assert r.converged_numpy.all()
    a = s.solve_adjoint(gold["grad_va"], gold["grad_vm"], g.pv, g.pq)
    assert a.success and a.jt_residual_norm <= 1e-10
    assert rel(a.lambda_numpy[0], gold["lam"]) <= 1e-6
    assert rel(a.grad_load_p_numpy[0], gold["grad_p"]) <= 1e-6
    assert rel(a.grad_load_q_numpy[0], gold["grad_q"]) <= 1e-6


def test_adjoint_batch_matches_oracle(oracle):
    g = G.grid_2000()
    B = 40
    S = g.scenarios(B, seed=13)
    V0 = g.flat_start(B)
    rng = np.random.default_rng(2)
    ga, gm = rng.standard_normal((B, g.n_bus)), rng.standard_normal((B, g.n_bus))
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    r = forward(s, g, S, V0, tol=1e-10)
    a = s.solve_adjoint(ga, gm, g.pv, g.pq)
    for b in (0, 17, 39):
        o = oracle.adjoint(g, r.V_numpy[b], ga[b], gm[b])
        assert rel(a.grad_load_p_numpy[b], o["grad_p"]) <= 1e-6
        assert rel(a.grad_load_q_numpy[b], o["grad_q"]) <= 1e-6
        assert rel(a.lambda_numpy[b], o["lambda"]) <= 1e-6


def test_adjoint_matches_central_differences():
    g = G.grid_118()
    S0 = g.scenarios(1, seed=6)[0]
    rng = np.random.default_rng(3)
    ga, gm = rng.standard_normal(g.n_bus), rng.standard_normal(g.n_bus)
    s = make_solver(g, cupf.ComputePolicy.FP64)
    r = forward(s, g, S0[None, :], g.flat_start(1))
    a = s.solve_adjoint(ga, gm, g.pv, g.pq)
    h = 1e-6
    buses = list(g.pq[:4]) + list(g.pv[:2])
    rows, labels = [], []
    for bus in buses:
        for kind, unit in (("p", 1.0), ("q", 1.0j)):
            e = np.zeros(g.n_bus, complex)
            e[bus] = unit * h
            rows += [S0 - e, S0 + e]  # load up = Sbus down
            labels.append((kind, bus))
    fd_solver = make_solver(g, cupf.ComputePolicy.FP64)
    rr = forward(fd_solver, g, np.stack(rows), g.flat_start(len(rows)), prepare=False)
    L = ga @ np.angle(rr.V_numpy).T + gm @ np.abs(rr.V_numpy).T
    for k, (kind, bus) in enumerate(labels):
        fd = (L[2 * k] - L[2 * k + 1]) / (2 * h)
        an = (a.grad_load_p_numpy if kind == "p" else a.grad_load_q_numpy)[0, bus]
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)) + 1e-7, (kind, bus, fd, an)


def test_adjoint_without_cache_raises():
    g = G.grid_118()
    s = make_solver(g, cupf.ComputePolicy.Mixed)
    forward(s, g, g.scenarios(2), g.flat_start(2), tol=1e-8, prepare=False)
    with pytest.raises(RuntimeError):
        s.solve_adjoint(np.zeros((2, g.n_bus)), np.zeros((2, g.n_bus)), g.pv, g.pq)


def test_torch_autograd_two_bus():
    """cuPF/tests/smoke/test_torch_autograd.py:32-105 on the custom backend:
    shapes, dtypes and finite gradients; here also their values."""
    import torch

    c = G.two_bus_case()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    s = cupf.NewtonSolver(o)
    s.initialize(c["indptr"], c["indices"], c["data"], 2, 2, c["pv"], c["pq"])
    dev, dt = torch.device("cuda"), torch.float32
    load_p = torch.zeros((1, 2), device=dev, dtype=dt, requires_grad=True)
    load_q = torch.zeros((1, 2), device=dev, dtype=dt, requires_grad=True)
    base_re = torch.tensor(c["sbus"].real, device=dev, dtype=dt)
    base_im = torch.tensor(c["sbus"].imag, device=dev, dtype=dt)
    v0 = torch.tensor(c["v0"], device=dev, dtype=torch.complex64)
    va, vm = cupf.solve(load_p, load_q, s, sbus_base_re=base_re, sbus_base_im=base_im,
                        v0_va=torch.angle(v0).to(dt), v0_vm=torch.abs(v0).to(dt),
                        config=cupf.NRConfig(tolerance=1e-6, max_iter=20), solve_options=cupf.SolveOptions())
    assert va.shape == load_p.shape and vm.shape == load_q.shape and va.dtype == dt
    loss = va[:, 1].sum() + vm[:, 1].sum()
    loss.backward()
    assert torch.isfinite(load_p.grad).all() and torch.isfinite(load_q.grad).all()
    assert float(load_p.grad[0, 0]) == 0.0  # the slack bus carries no gradient
    assert abs(float(load_p.grad[0, 1])) > 0.0


def test_torch_autograd_matches_oracle(oracle):
    """CuPFFunction on the 118-bus grid (float64, FP64 policy): gradients of
    L = sum(w_a * Va + w_m * Vm) against the oracle adjoint."""
    import torch

    g = G.grid_118()
    s = make_solver(g, cupf.ComputePolicy.FP64)
    B = 3
    dev, dt = torch.device("cuda"), torch.float64
    rng = np.random.default_rng(7)
    lp = 0.05 * rng.random((B, g.n_bus))
    lq = 0.02 * rng.random((B, g.n_bus))
    load_p = torch.tensor(lp, device=dev, dtype=dt, requires_grad=True)
    load_q = torch.tensor(lq, device=dev, dtype=dt, requires_grad=True)
    base = g.sbus
    v0 = torch.tensor(g.v0, device=dev)
    va, vm = cupf.solve(load_p, load_q, s, sbus_base_re=torch.tensor(base.real, device=dev),
                        sbus_base_im=torch.tensor(base.imag, device=dev), v0_va=torch.angle(v0),
                        v0_vm=torch.abs(v0), config=cupf.NRConfig(tolerance=1e-12, max_iter=30))
    wa = torch.tensor(rng.standard_normal((B, g.n_bus)), device=dev)
    wm = torch.tensor(rng.standard_normal((B, g.n_bus)), device=dev)
    ((wa * va).sum() + (wm * vm).sum()).backward()
    for b in range(B):
        S = base - (lp[b] + 1j * lq[b])
        V = oracle.solve(g, S, g.v0, tol=1e-12, max_iter=30)["V"]
        assert np.abs(np.angle(V) - va[b].detach().cpu().numpy()).max() <= 1e-9
        o = oracle.adjoint(g, V, wa[b].cpu().numpy(), wm[b].cpu().numpy())
        assert rel(load_p.grad[b].cpu().numpy(), o["grad_p"]) <= 1e-6
        assert rel(load_q.grad[b].cpu().numpy(), o["grad_q"]) <= 1e-6


@pytest.mark.parametrize("compute", [cupf.ComputePolicy.FP64, cupf.ComputePolicy.Mixed])
def test_torch_autograd_graph_mode_matches_stream_mode(compute):
    """NewtonOptions.use_cuda_graph on the torch path (the whole forward solve
    as one graph launch, then the adjoint cache): the same Va, Vm and load
    gradients, bit for bit, as host-driven iterations, on the 2,000-bus grid
    at 40 scenarios (a ragged second lane group)."""
    import torch

    g = G.grid_2000()
    B = 40
    dev = torch.device("cuda")
    dt = torch.float64 if compute == cupf.ComputePolicy.FP64 else torch.float32
    lp, lq = g.load_scenarios(B, seed=91)
    v0 = torch.tensor(g.v0, device=dev)
    out = []
    for graph in (False, True):
        o = cupf.NewtonOptions()
        o.backend = cupf.BackendKind.CUDA
        o.compute = compute
        o.custom.serial_nd = True
        o.use_cuda_graph = graph
        s = cupf.NewtonSolver(o)
        s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
        res = []
        for rep in range(2):  # the second pass replays the captured graph
            load_p = torch.tensor(lp, device=dev, dtype=dt, requires_grad=True)
            load_q = torch.tensor(lq, device=dev, dtype=dt, requires_grad=True)
            va, vm = cupf.solve(load_p, load_q, s, sbus_base_re=torch.tensor(g.sgen.real, device=dev, dtype=dt),
                                sbus_base_im=torch.tensor(g.sgen.imag, device=dev, dtype=dt),
                                v0_va=torch.angle(v0).to(dt), v0_vm=torch.abs(v0).to(dt),
                                config=cupf.NRConfig(tolerance=1e-10, max_iter=20))
            ((vm - 1.0) ** 2).sum().backward()
            res.append([t.detach().cpu().numpy() for t in (va, vm, load_p.grad, load_q.grad)])
        for a, b in zip(res[0], res[1]):
            assert np.array_equal(a, b)
        out.append(res[1])
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_torch_generation_guard():
    import torch

    c = G.two_bus_case()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.FP64
    s = cupf.NewtonSolver(o)
    s.initialize(c["indptr"], c["indices"], c["data"], 2, 2, c["pv"], c["pq"])
    dev = torch.device("cuda")
    kw = dict(sbus_base_re=torch.tensor(c["sbus"].real, device=dev),
              sbus_base_im=torch.tensor(c["sbus"].imag, device=dev),
              v0_va=torch.zeros(2, device=dev, dtype=torch.float64),
              v0_vm=torch.ones(2, device=dev, dtype=torch.float64))
    lp = torch.zeros((1, 2), device=dev, dtype=torch.float64, requires_grad=True)
    lq = torch.zeros((1, 2), device=dev, dtype=torch.float64, requires_grad=True)
    va1, _ = cupf.solve(lp, lq, s, **kw)
    cupf.solve(lp, lq, s, **kw)
    with pytest.raises(RuntimeError):
        va1.sum().backward()


def test_c5_10000_bus_vm_loss_gradients(oracle):
    """The differentiable large case: 10,000-bus grid x 64 scenarios, forward
    Newton in mixed precision, loss = sum of squared Vm deviations from 1 pu,
    dLoss/dP and dLoss/dQ through the adjoint.  Checked against the CPU
    oracle's FP64 adjoint and against central differences (h = 1e-6) of the
    loss computed with tightly converged FP64 solves."""
    import torch

    g = G.grid_10000()
    B = 64
    S = g.scenarios(B, seed=55)
    mixed = make_solver(g, cupf.ComputePolicy.Mixed)
    r = forward(mixed, g, S, g.flat_start(B), tol=1e-10, max_iter=20)
    assert r.converged_numpy.all()
    vm = np.abs(r.V_numpy)
    ga = np.zeros_like(vm)
    gm = 2.0 * (vm - 1.0)
    a = mixed.solve_adjoint(ga, gm, g.pv, g.pq)
    assert a.success
    for b in (0, 37):
        o = oracle.adjoint(g, r.V_numpy[b], ga[b], gm[b])
        assert rel(a.grad_load_p_numpy[b], o["grad_p"]) <= 1e-6
        assert rel(a.grad_load_q_numpy[b], o["grad_q"]) <= 1e-6
    # central differences on scenario 0 for a few PQ buses, FP64 engine, all
    # perturbed cases in one batch
    fp64 = make_solver(g, cupf.ComputePolicy.FP64)
    h = 1e-6
    buses = list(g.pq[[0, 100, 4000, 7998]])
    rows, labels = [], []
    for bus in buses:
        for kind, unit in (("p", 1.0), ("q", 1.0j)):
            e = np.zeros(g.n_bus, complex)
            e[bus] = unit * h
            rows += [S[0] - e, S[0] + e]
            labels.append((kind, bus))
    rr = forward(fp64, g, np.stack(rows), g.flat_start(len(rows)), tol=1e-12, prepare=False)
    assert rr.converged_numpy.all()
    L = ((np.abs(rr.V_numpy) - 1.0) ** 2).sum(axis=1)
    for k, (kind, bus) in enumerate(labels):
        fd = (L[2 * k] - L[2 * k + 1]) / (2 * h)
        an = (a.grad_load_p_numpy if kind == "p" else a.grad_load_q_numpy)[0, bus]
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)) + 1e-6 * np.abs(a.grad_load_p_numpy[0]).max(), (kind, bus, fd, an)
