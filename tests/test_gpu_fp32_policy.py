"""ComputePolicy.FP32 on the GPU: the reference's CudaFp32CustomPipeline
(cuPF/cpp/src/newton_solver/core/pipeline.hpp:261-299; semantics at
cuPF/cpp/inc/newton_solver/core/newton_solver_types.hpp:63-80), where the
state V, Sbus, Ibus, the mismatch F and the voltage update are FP32 along
with the Jacobian and the factors.

Bars.  FP32 state leaves a mismatch floor of about 1e-5 pu on the 118- and
2,000-bus grids: Ibus sums terms |y||V| of up to a few hundred pu in FP32
and the mismatch cancels them.  So the Newton tests run at the tolerance the
reference's own FP32 tests use (1e-6 on the two-bus case,
cuPF/tests/unit/test_minimal_solver.cpp:140-180 and 270-306) or at 1e-4 on
the grids, above that floor.  Voltages are compared with the FP64 oracle run
to 1e-12: within 1e-6 pu on the two-bus case, 5e-5 pu on the 118-bus grid and
1e-4 pu on the 2,000-bus grid (the floor divided through the Jacobian gives
errors of a few 1e-6 and a few 1e-5 there).
"""
import numpy as np
import pytest

import cupf
from cupf import grids as G
from conftest import gpu_available, max_dv_vs_oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def make_solver(g, compute=cupf.ComputePolicy.FP32, graph=False, kind=None, precision=None):
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = compute
    o.use_cuda_graph = graph
    o.custom.serial_nd = True
    if kind is not None:
        o.cuda_jacobian = getattr(cupf.CudaJacobianKind, kind)
    if precision is not None:
        o.custom.precision = precision
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    return s


def cfg(tol, max_iter=10):
    c = cupf.NRConfig()
    c.tolerance = tol
    c.max_iter = max_iter
    return c


def solve(s, g, S, V0, c):
    return s.solve_batch(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, S, V0, g.pv, g.pq, c)


def is_fp32(x: np.ndarray) -> bool:
    """Every real and imaginary part is a float32 value (the state was FP32)."""
    x = np.asarray(x)
    return bool(np.array_equal(x.real.astype(np.float32).astype(np.float64), x.real)
                and np.array_equal(x.imag.astype(np.float32).astype(np.float64), x.imag))


class TwoBus:
    def __init__(self):
        c = G.two_bus_case()
        self.c = c
        self.indptr, self.indices, self.data = c["indptr"], c["indices"], c["data"]
        self.pv, self.pq, self.n_bus = c["pv"], c["pq"], 2


@pytest.mark.parametrize("graph", [False, True])
def test_fp32_two_bus(graph):
    """The reference's custom CUDA FP32 two-bus tests, stream and graph mode:
    converged, final mismatch finite and within the 1e-6 tolerance."""
    g = TwoBus()
    s = make_solver(g, graph=graph)
    single = s.solve(g.indptr, g.indices, g.data, 2, 2, g.c["sbus"], g.c["v0"], g.pv, g.pq, cfg(1e-6, 20))
    assert single.converged
    assert np.isfinite(single.final_mismatch) and single.final_mismatch <= 1e-6
    assert np.abs(single.V_numpy - g.c["expected_v"]).max() <= 1e-6
    S = np.stack([g.c["sbus"]] * 2)
    V0 = np.stack([g.c["v0"]] * 2)
    r = solve(s, g, S, V0, cfg(1e-6, 20))
    assert r.converged_numpy.all() and (r.final_mismatch_numpy <= 1e-6).all()
    assert np.abs(r.V_numpy - g.c["expected_v"][None, :]).max() <= 1e-6
    assert is_fp32(r.V_numpy)


def test_fp32_118_matches_oracle(oracle):
    """40 scenarios (a ragged second warp): every one within 5e-5 pu of the
    FP64 oracle; the voltages are FP32 values and differ from the Mixed
    policy's (the option is not an alias)."""
    g = G.grid_118()
    B = 40
    S = g.scenarios(B, seed=17)
    V0 = g.flat_start(B)
    r = solve(make_solver(g), g, S, V0, cfg(1e-4))
    assert r.converged_numpy.all()
    assert (r.final_mismatch_numpy <= 1e-4).all()
    assert max_dv_vs_oracle(oracle, g, S, V0, r.V_numpy).max() <= 5e-5
    assert is_fp32(r.V_numpy)
    m = solve(make_solver(g, cupf.ComputePolicy.Mixed), g, S, V0, cfg(1e-4))
    assert not is_fp32(m.V_numpy)
    assert np.abs(r.V_numpy - m.V_numpy).max() > 0.0


def test_fp32_2000_graph_equals_stream_and_matches_oracle(oracle):
    """2,000-bus x 64: graph mode (device-side loop) gives the stream-mode
    solve bit for bit; every scenario within 1e-4 pu of the FP64 oracle."""
    g = G.grid_2000()
    B = 64
    S = g.scenarios(B, seed=41)
    V0 = g.flat_start(B)
    a = solve(make_solver(g), g, S, V0, cfg(1e-4))
    b = solve(make_solver(g, graph=True), g, S, V0, cfg(1e-4))
    assert a.converged_numpy.all()
    assert np.array_equal(a.V_numpy, b.V_numpy)
    assert np.array_equal(a.iterations_numpy, b.iterations_numpy)
    assert max_dv_vs_oracle(oracle, g, S, V0, a.V_numpy).max() <= 1e-4


@pytest.mark.parametrize("kind", ["Edge", "EdgeAtomic", "VertexWarp"])
def test_fp32_mismatch_and_jacobian_kinds(oracle, kind):
    """F and J under FP32 state, at voltages that are FP32 values, against the
    FP64 oracle at the same voltages: J within 2e-6 of max|J| for every
    CudaJacobianKind, F within 1e-4 pu; each kind's Newton solve converges."""
    g = G.grid_118()
    s = make_solver(g, kind=kind)
    rng = np.random.default_rng(21)
    V = (1 + 0.05 * rng.standard_normal((3, g.n_bus))) * np.exp(1j * 0.1 * rng.standard_normal((3, g.n_bus)))
    V = V.real.astype(np.float32).astype(np.float64) + 1j * V.imag.astype(np.float32).astype(np.float64)
    S = g.scenarios(3, seed=2)
    S = S.real.astype(np.float32).astype(np.float64) + 1j * S.imag.astype(np.float32).astype(np.float64)
    F, J = s.evaluate(V, S)
    for b in range(3):
        Jo = oracle.jacobian_values(g, V[b])
        assert np.abs(J[b] - Jo).max() <= 2e-6 * np.abs(Jo).max()
        Fo, _ = oracle.mismatch(g, S[b], V[b])
        assert np.abs(F[b] - Fo).max() <= 1e-4
    B = 8
    r = solve(s, g, g.scenarios(B, seed=24), g.flat_start(B), cfg(1e-4))
    assert r.converged_numpy.all()


def test_fp32_tf32_factors_converge(oracle):
    """CustomPrecision.TF32 is available on FP32 state (newton_solver_types.hpp:
    136); an FP64 factor precision falls back to FP32 factors, as the
    reference's custom solver does (cuda_custom_solver.cpp:71-72), so its
    solve equals the FP32-factor solve bit for bit."""
    g = G.grid_118()
    B = 16
    S = g.scenarios(B, seed=5)
    V0 = g.flat_start(B)
    t = solve(make_solver(g, precision=cupf.CustomPrecision.TF32), g, S, V0, cfg(1e-4))
    assert t.converged_numpy.all()
    assert max_dv_vs_oracle(oracle, g, S, V0, t.V_numpy).max() <= 5e-5
    f32 = solve(make_solver(g, precision=cupf.CustomPrecision.FP32), g, S, V0, cfg(1e-4))
    f64 = solve(make_solver(g, precision=cupf.CustomPrecision.FP64), g, S, V0, cfg(1e-4))
    assert np.array_equal(f32.V_numpy, f64.V_numpy)


def test_fp32_adjoint_is_refused_with_its_reason():
    """The adjoint's FP64 residual refinement needs FP64 state, so under
    ComputePolicy.FP32 solve_adjoint raises, naming the policy (the
    reference's custom backend raises for every adjoint)."""
    g = G.grid_118()
    s = make_solver(g)
    so = cupf.SolveOptions()
    so.prepare_adjoint_cache = True
    r = s.solve_batch(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.scenarios(2, seed=1), g.flat_start(2),
                      g.pv, g.pq, cfg(1e-4), so)
    assert r.converged_numpy.all()
    ga = np.ones((2, g.n_bus))
    with pytest.raises(RuntimeError, match="FP32"):
        s.solve_adjoint(ga, ga, g.pv, g.pq)


def test_fp32_torch_forward():
    """cupf.solve on float32 tensors (the dtype the reference's torch bridge
    wants for FP32, torch_bridge.cpp:133-141): the same voltages as
    solve_batch on the same problem."""
    torch = pytest.importorskip("torch")
    g = G.grid_118()
    s = make_solver(g)
    dev, dt = torch.device("cuda"), torch.float32
    rng = np.random.default_rng(7)
    B = 3
    lp = (0.05 * rng.random((B, g.n_bus))).astype(np.float32)
    lq = (0.02 * rng.random((B, g.n_bus))).astype(np.float32)
    base = g.sbus
    bre, bim = base.real.astype(np.float32), base.imag.astype(np.float32)
    va0, vm0 = np.angle(g.v0).astype(np.float32), np.abs(g.v0).astype(np.float32)
    va, vm = cupf.solve(torch.tensor(lp, device=dev), torch.tensor(lq, device=dev), s,
                        sbus_base_re=torch.tensor(bre, device=dev), sbus_base_im=torch.tensor(bim, device=dev),
                        v0_va=torch.tensor(va0, device=dev), v0_vm=torch.tensor(vm0, device=dev),
                        config=cupf.NRConfig(tolerance=1e-4, max_iter=10))
    assert va.dtype == dt and vm.dtype == dt
    V = vm.double().cpu().numpy() * np.exp(1j * va.double().cpu().numpy())
    S = (bre.astype(np.float64) - lp) + 1j * (bim.astype(np.float64) - lq)
    V0 = np.repeat((vm0.astype(np.float64) * np.exp(1j * va0.astype(np.float64)))[None, :], B, axis=0)
    ref = solve(make_solver(g), g, S, V0, cfg(1e-4))
    assert ref.converged_numpy.all()
    # two FP32 solves from starts rounded differently, each within 5e-5 pu of the solution
    assert np.abs(V - ref.V_numpy).max() <= 1e-4
