"""The single-system schedule (a batch of one: one block per front, threads
over the front's rows; the reference's single-system path,
custom_linear_solver/src/factorize/single.cuh) against the batched lane
kernels at batch 1 (batch1_schedule = 1): the same factors, bit for bit, so
the same solutions, Newton iterates and adjoints; and the oracle's answers.
Without tensor-core launches the whole factorization is one launch over the
front tree; with them (TF32) each level is its own launch."""
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

import cupf
from cupf import grids as G
from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]
GOLD = Path(__file__).resolve().parent / "golden"


def _factor_solve(d, precision, schedule, tc_min_front=0, serial_nd=True, matching=0):
    import torch

    ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(precision), serial_nd=serial_nd, batch1_schedule=schedule,
                                             tc_min_front=tc_min_front, matching=matching))
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze()
    ls.setup(1)
    dt = torch.float64 if precision == cupf.CustomPrecision.FP64 else torch.float32
    ls.factorize(torch.tensor(d["values"][None, :], dtype=dt, device="cuda"))
    rhs = torch.tensor(d["F"][None, :], dtype=torch.float64, device="cuda")
    x = ls.solve(rhs).cpu().numpy()[0]
    xt = ls.solve_transpose(rhs).cpu().numpy()[0]
    return x, xt, ls.singular_flags().copy(), ls.plan_array("fp_fsz").max()


@pytest.mark.parametrize("case", ["case118", "case1354pegase", "case3120sp", "case6468rte", "case8387pegase"])
@pytest.mark.parametrize("precision", [cupf.CustomPrecision.FP64, cupf.CustomPrecision.FP32])
def test_single_system_factors_equal_the_lane_kernels(case, precision):
    """Every dataset of the reference (fronts up to 77 rows on case8387pegase):
    solve and transpose solve bit-identical between the schedules, and the
    FP64 residual at the dataset's right-hand side small."""
    d = np.load(GOLD / f"linsys_{case}.npz")
    x1, xt1, s1, fmax = _factor_solve(d, precision, 0)
    x0, xt0, s0, _ = _factor_solve(d, precision, 1)
    assert np.array_equal(x1, x0) and np.array_equal(xt1, xt0)
    assert np.array_equal(s1, s0)
    if precision == cupf.CustomPrecision.FP64:
        n = d["row_ptr"].size - 1
        A = sp.csr_matrix((d["values"], d["col_idx"], d["row_ptr"]), shape=(n, n))
        r = np.linalg.norm(A @ x1 - d["F"]) / np.linalg.norm(d["F"])
        assert r <= 1e-10, (case, r, fmax)


@pytest.mark.parametrize("serial_nd,matching", [(False, 0), (True, 1)])
def test_single_system_with_other_orderings(serial_nd, matching):
    """The separator-recursion ordering and the structural matching (other
    front trees and assembly lists): still the lane kernels' bits."""
    d = np.load(GOLD / "linsys_case1354pegase.npz")
    for precision in (cupf.CustomPrecision.FP64, cupf.CustomPrecision.FP32):
        x1, xt1, _, _ = _factor_solve(d, precision, 0, serial_nd=serial_nd, matching=matching)
        x0, xt0, _, _ = _factor_solve(d, precision, 1, serial_nd=serial_nd, matching=matching)
        assert np.array_equal(x1, x0) and np.array_equal(xt1, xt0)


def test_single_system_with_tensor_core_launches():
    """TF32 at batch 1: the launches past the tensor-core threshold keep the
    tensor-core kernel, the others take the single-system kernel; the
    solution equals the lane schedule's."""
    d = np.load(GOLD / "linsys_case8387pegase.npz")
    x1, xt1, _, _ = _factor_solve(d, cupf.CustomPrecision.TF32, 0, tc_min_front=33)
    x0, xt0, _, _ = _factor_solve(d, cupf.CustomPrecision.TF32, 1, tc_min_front=33)
    assert np.array_equal(x1, x0) and np.array_equal(xt1, xt0)


def _nr(g, compute, schedule, graph):
    import torch

    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = compute
    o.custom.serial_nd = True
    o.custom.batch1_schedule = schedule
    o.use_cuda_graph = graph
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    S = torch.tensor(g.scenarios(1, seed=21), device="cuda")
    V0 = torch.tensor(g.flat_start(1), device="cuda")
    V, fm, it = s.solve_batch_device(S, V0, config=cupf.NRConfig(tolerance=1e-8, max_iter=10))
    return s, V.cpu().numpy(), fm.cpu().numpy(), it, s.info()["last_kernel_launches"]


@pytest.mark.parametrize("name", ["118", "2000"])
@pytest.mark.parametrize("compute", [cupf.ComputePolicy.FP64, cupf.ComputePolicy.Mixed])
def test_single_system_newton_solve(name, compute, oracle):
    """A batch-1 Newton solve: the same iterates as the lane schedule (graph
    and stream mode), and the oracle's voltages within 1e-8."""
    g = {"118": G.grid_118, "2000": G.grid_2000}[name]()
    _, V1, fm1, it1, _ = _nr(g, compute, 0, True)
    _, V1s, _, it1s, n1 = _nr(g, compute, 0, False)
    _, V0, fm0, it0, _ = _nr(g, compute, 1, True)
    _, _, _, _, n0 = _nr(g, compute, 1, False)
    assert it1 == it0 == it1s and np.array_equal(V1, V0) and np.array_equal(V1, V1s)
    assert n1 < n0  # one factor launch per iteration instead of one per level
    assert fm1[0] <= 1e-8
    ref = oracle.solve(g, g.scenarios(1, seed=21)[0], g.flat_start(1)[0], tol=1e-12, max_iter=30)["V"]
    assert np.abs(V1[0] - ref).max() <= 1e-8


def test_batch_size_changes_switch_the_schedule():
    """One solver alternating between batch 1 and batch 3 (the same 32-lane
    workspace): each solve matches a fresh solver of its batch size."""
    import torch

    g = G.grid_118()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.serial_nd = True
    o.use_cuda_graph = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    cfg = cupf.NRConfig(tolerance=1e-8, max_iter=10)
    S3 = torch.tensor(g.scenarios(3, seed=4), device="cuda")
    V3 = torch.tensor(g.flat_start(3), device="cuda")
    outs = []
    for B in (1, 3, 1, 3):
        V, _, _ = s.solve_batch_device(S3[:B].contiguous(), V3[:B].contiguous(), config=cfg)
        outs.append(V.cpu().numpy())
    for B, out in zip((1, 3), outs[:2]):
        f = cupf.NewtonSolver(o)
        f.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
        V, _, _ = f.solve_batch_device(S3[:B].contiguous(), V3[:B].contiguous(), config=cfg)
        assert np.array_equal(out, V.cpu().numpy()), B
    assert np.array_equal(outs[0], outs[2]) and np.array_equal(outs[1], outs[3])
