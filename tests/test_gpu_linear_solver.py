"""The batched sparse solver (cls_* ABI, custom_linear_solver::Solver phases) on
the reference's own linear-system datasets: real Newton Jacobians of case118
and case1354pegase (custom_linear_solver/tests/datasets/power/<case>/J.mtx, F.mtx).

The reference checks these with a relative residual (run_custom_solver.cu); the
same check here, plus agreement with a FP64 SuperLU solve.
"""
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import cupf
from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]
GOLD = Path(__file__).resolve().parent / "golden"


def load(case):
    d = np.load(GOLD / f"linsys_{case}.npz")
    n = d["row_ptr"].size - 1
    A = sp.csr_matrix((d["values"], d["col_idx"], d["row_ptr"]), shape=(n, n))
    return d, A


def batch_values(d, B, rng):
    """B value sets on the same pattern: the dataset J with +-2 % perturbations."""
    base = d["values"]
    v = np.repeat(base[None, :], B, axis=0)
    if B > 1:
        v[1:] *= 1.0 + 0.02 * rng.uniform(-1, 1, size=(B - 1, base.size))
    return v


@pytest.mark.parametrize("case", ["case118", "case1354pegase"])
@pytest.mark.parametrize("precision,tol", [(cupf.CustomPrecision.FP64, 1e-11), (cupf.CustomPrecision.FP32, 2e-4)])
def test_factor_solve_residual(case, precision, tol):
    import torch

    d, A = load(case)
    rng = np.random.default_rng(1)
    B = 35
    vals = batch_values(d, B, rng)
    rhs = np.repeat(d["F"][None, :], B, axis=0) + 0.1 * rng.standard_normal((B, A.shape[0]))
    ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(precision), serial_nd=True))
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze()
    ls.setup(B)
    dt = torch.float64 if precision == cupf.CustomPrecision.FP64 else torch.float32
    ls.factorize(torch.tensor(vals, dtype=dt, device="cuda"))
    x = ls.solve(torch.tensor(rhs, dtype=torch.float64, device="cuda")).cpu().numpy()
    xt = ls.solve_transpose(torch.tensor(rhs, dtype=torch.float64, device="cuda")).cpu().numpy()
    assert not ls.singular_flags().any()
    for b in range(B):
        Ab = sp.csr_matrix((vals[b], d["col_idx"], d["row_ptr"]), shape=A.shape)
        r = np.linalg.norm(Ab @ x[b] - rhs[b]) / np.linalg.norm(rhs[b])
        rt = np.linalg.norm(Ab.T @ xt[b] - rhs[b]) / np.linalg.norm(rhs[b])
        assert r <= tol and rt <= tol, (b, r, rt)
    if precision == cupf.CustomPrecision.FP64:
        ref = spla.spsolve(sp.csc_matrix(A), rhs[0])
        assert np.abs(x[0] - ref).max() <= 1e-9 * np.abs(ref).max()


def test_float32_solution_buffers():
    """rhs/solution type pairs f64/f32 and f32/f32 (solver.cpp:192-210)."""
    import torch

    d, A = load("case118")
    ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(cupf.CustomPrecision.FP32)))
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze()
    ls.setup(2)
    ls.factorize(torch.tensor(np.stack([d["values"]] * 2), dtype=torch.float32, device="cuda"))
    rhs = torch.tensor(np.stack([d["F"]] * 2), dtype=torch.float64, device="cuda")
    x64 = ls.solve(rhs).cpu().numpy()
    x32 = ls.solve(rhs, out=torch.empty(rhs.shape, dtype=torch.float32, device="cuda")).cpu().numpy()
    xf = ls.solve(rhs.float()).cpu().numpy()
    assert np.abs(x32 - x64).max() <= 1e-5 * np.abs(x64).max()
    assert np.abs(xf - x64).max() <= 1e-3 * np.abs(x64).max()


def test_device_pattern_upload():
    import torch

    d, A = load("case118")
    ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(cupf.CustomPrecision.FP64)))
    ls.set_data(torch.tensor(d["row_ptr"], device="cuda"), torch.tensor(d["col_idx"], device="cuda"))
    ls.analyze()
    ls.setup(1)
    ls.factorize(torch.tensor(d["values"][None, :], device="cuda"))
    x = ls.solve(torch.tensor(d["F"][None, :], device="cuda")).cpu().numpy()[0]
    assert np.linalg.norm(A @ x - d["F"]) <= 1e-11 * np.linalg.norm(d["F"])


def test_zero_pivot_sets_singular_flag():
    """A structurally present but numerically zero row: the static diagonal shift
    (PivotStrategy::StaticDiagonalShift) replaces the zero pivot and flags the
    scenario, the other scenarios stay unflagged."""
    import torch

    d, A = load("case118")
    vals = np.stack([d["values"]] * 3)
    r0, r1 = d["row_ptr"][5], d["row_ptr"][6]
    vals[1, r0:r1] = 0.0
    ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(cupf.CustomPrecision.FP64)))
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze()
    ls.setup(3)
    ls.factorize(torch.tensor(vals, device="cuda"))
    flags = ls.singular_flags()
    assert flags[1] != 0 and flags[0] == 0 and flags[2] == 0
    x = ls.solve(torch.tensor(np.stack([d["F"]] * 3), device="cuda")).cpu().numpy()
    assert np.isfinite(x[0]).all() and np.isfinite(x[2]).all()


def test_state_errors():
    import torch

    d, _ = load("case118")
    ls = cupf.LinearSolver()
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze()
    ls.setup(2)
    with pytest.raises(cupf.linear_solver.CustomSolverError):
        ls.solve(torch.zeros((2, 181), dtype=torch.float64, device="cuda"))  # before factorize
    with pytest.raises(ValueError):
        ls.factorize(torch.zeros((2, d["col_idx"].size), dtype=torch.int32, device="cuda"))


def _row_permuted(d, seed):
    """case118's J with its rows in a seeded random order: the diagonal is
    structurally incomplete, so only a matching makes the pivots nonzero."""
    rp0, ci0, v0 = d["row_ptr"], d["col_idx"], d["values"]
    n = rp0.size - 1
    order = np.random.default_rng(seed).permutation(n)
    rp = np.concatenate([[0], np.cumsum(np.diff(rp0)[order])]).astype(np.int32)
    ci = np.concatenate([ci0[rp0[r]:rp0[r + 1]] for r in order]).astype(np.int32)
    v = np.concatenate([v0[rp0[r]:rp0[r + 1]] for r in order])
    return rp, ci, v, order


@pytest.mark.parametrize("precision,tol,tol_t", [(cupf.CustomPrecision.FP64, 1e-8, 1e-8)])
def test_structural_matching_solves_a_row_permuted_system(precision, tol, tol_t):
    """MatchingMode::Structural (analyze/pipeline.cpp:77-160, 222-272) on a
    row-shuffled Jacobian (structurally zero diagonal entries; ordered
    without a matching, its A + A^T graph fills in past the 64-row front
    limit): factor, solve and transpose solve are accurate.  The matched
    diagonal is not the Jacobian's own, so the unpivoted LU grows elements
    (185x to 1,049x over these nine systems; the exact FP64 LU in this order
    leaves relative residuals up to 1e-9 (solve) and 3e-9 (transpose)),
    hence the looser bars than on the natural row order.  FP32 factors are
    not tested on this system: an exact FP32 LU in the matched order already
    leaves a 1 % residual (growth times FP32 roundoff), whatever the kernel;
    the FP32 kernels share the permutation code checked here."""
    import torch

    d = np.load(GOLD / "linsys_case118.npz")
    rp, ci, v, order = _row_permuted(d, 118)
    n = rp.size - 1
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    rng = np.random.default_rng(5)
    B = 9
    vals = np.repeat(v[None, :], B, axis=0) * (1.0 + 0.02 * rng.uniform(-1, 1, size=(B, v.size)))
    rhs = rng.standard_normal((B, n))
    dt = torch.float64 if precision == cupf.CustomPrecision.FP64 else torch.float32
    ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(precision), serial_nd=True, matching=1))
    ls.set_data(rp, ci)
    ls.analyze()
    ls.setup(B)
    ls.factorize(torch.tensor(vals, dtype=dt, device="cuda"))
    assert not ls.singular_flags().any()
    x = ls.solve(torch.tensor(rhs, device="cuda")).cpu().numpy()
    xt = ls.solve_transpose(torch.tensor(rhs, device="cuda")).cpu().numpy()
    for b in range(B):
        Ab = sp.csr_matrix((vals[b], ci, rp), shape=A.shape)
        assert np.linalg.norm(Ab @ x[b] - rhs[b]) <= tol * np.linalg.norm(rhs[b])
        assert np.linalg.norm(Ab.T @ xt[b] - rhs[b]) <= tol_t * np.linalg.norm(rhs[b])


def test_pivot_strategy_none_keeps_small_pivots():
    """PivotStrategy::None (front_ops.cuh:147-161): a pivot below the shift
    threshold is used as it is and no system is flagged; the default static
    shift replaces it and flags the system."""
    import torch

    # a path 0 - 1 - 2 whose leaf 0 has the small diagonal: whatever the
    # nested-dissection order, bus 0 is eliminated before its neighbour 1,
    # so its pivot is 1e-4, below the 1e-3 threshold
    n = 3
    rp = np.array([0, 2, 5, 7], np.int32)
    ci = np.array([0, 1, 0, 1, 2, 1, 2], np.int32)
    vals = np.array([[1e-4, 1.0, 1.0, 2.0, 1.0, 1.0, 3.0]])
    rhs = np.array([[1.0, 2.0, 3.0]])
    A = sp.csr_matrix((vals[0], ci, rp), shape=(n, n))
    exact = np.linalg.solve(A.toarray(), rhs[0])
    out = {}
    for strat in (0, 1):
        ls = cupf.LinearSolver(cupf.SolverConfig(precision=0, serial_nd=True, pivot_strategy=strat,
                                                 shift_retry_epsilon=1e-3))
        ls.set_data(rp, ci)
        ls.analyze()
        ls.setup(1)
        ls.factorize(torch.tensor(vals, device="cuda"))
        out[strat] = (ls.solve(torch.tensor(rhs, device="cuda")).cpu().numpy()[0], ls.singular_flags()[0])
    x0, f0 = out[0]
    assert not f0 and np.abs(x0 - exact).max() <= 1e-9 * np.abs(exact).max()
    x1, f1 = out[1]
    assert f1 and np.abs(x1 - exact).max() > 1e-6 * np.abs(exact).max()


@pytest.mark.parametrize("case", ["case1354pegase", "case8387pegase"])
def test_autotuned_factorization_is_bit_identical(case):
    """SolverConfig(autotune=True): the first factorization of a batch size
    times the factor levels' block shapes (and, for launches of large fronts,
    the any-size tier with 8 to 32 warps) on the given values and keeps the
    fastest per level; the factors, and so the solutions, do not change."""
    import torch

    d, A = load(case)
    rng = np.random.default_rng(3)
    B = 64
    vals = batch_values(d, B, rng)
    rhs = np.repeat(d["F"][None, :], B, axis=0) + 0.1 * rng.standard_normal((B, A.shape[0]))
    out = []
    for tune in (False, True):
        ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(cupf.CustomPrecision.FP32), serial_nd=True,
                                                 autotune=tune))
        ls.set_data(d["row_ptr"], d["col_idx"])
        ls.analyze()
        ls.setup(B)
        for _ in range(2):
            ls.factorize(torch.tensor(vals, dtype=torch.float32, device="cuda"))
        out.append(ls.solve(torch.tensor(rhs, dtype=torch.float64, device="cuda")).cpu().numpy())
    assert np.array_equal(out[0], out[1])


# The reference's three larger Newton Jacobians (5,890 / 12,293 / 14,908
# unknowns).  case8387pegase has fronts of 66, 69 and 77 rows, past the
# register kernels' 64: the any-size tier factors them.  Residual bars: FP64
# 1e-11 (an unpivoted LU in the engine's ordering, computed by SuperLU, leaves
# at most 3.3e-13 on these systems); FP32 and TF32 factors: at most 4x the
# residual of SuperLU's FP32 unpivoted LU of the same system in the same
# ordering (floor 1e-5).  The +-2 % perturbed value sets reach 3.2e-3 there:
# that is what FP32 factors without pivoting can do on them, whatever the
# kernel.
LARGER = ["case3120sp", "case6468rte", "case8387pegase"]
PRECISIONS = {"FP64": (cupf.CustomPrecision.FP64, 1e-11), "FP32": (cupf.CustomPrecision.FP32, None),
              "TF32": (cupf.CustomPrecision.TF32, None)}


def _fp32_lu_residuals(d, perm, vals, rhs):
    """Relative residual of SuperLU's FP32 LU without pivoting, in the
    engine's ordering, per value set: the accuracy FP32 factors can reach."""
    n = d["row_ptr"].size - 1
    out = []
    for b in range(vals.shape[0]):
        A = sp.csr_matrix((vals[b], d["col_idx"], d["row_ptr"]), shape=(n, n))
        Ap = sp.csc_matrix(A[perm][:, perm])
        lu = spla.splu(Ap.astype(np.float32), permc_spec="NATURAL", diag_pivot_thresh=0.0,
                       options={"SymmetricMode": True})
        x = np.empty(n)
        x[perm] = lu.solve(rhs[b][perm].astype(np.float32)).astype(np.float64)
        out.append(np.linalg.norm(A @ x - rhs[b]) / np.linalg.norm(rhs[b]))
    return np.array(out)


def _factor_solve(d, B, precision, rng, **cfg):
    import torch

    vals = batch_values(d, B, rng)
    n = d["row_ptr"].size - 1
    rhs = np.repeat(d["F"][None, :], B, axis=0) + 0.1 * rng.standard_normal((B, n))
    ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(precision), serial_nd=True, **cfg))
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze()
    ls.setup(B)
    dt = torch.float64 if precision == cupf.CustomPrecision.FP64 else torch.float32
    ls.factorize(torch.tensor(vals, dtype=dt, device="cuda"))
    r = torch.tensor(rhs, dtype=torch.float64, device="cuda")
    return ls, vals, rhs, ls.solve(r).cpu().numpy(), ls.solve_transpose(r).cpu().numpy()


def _residuals(d, vals, rhs, x, xt):
    n = d["row_ptr"].size - 1
    out = []
    for b in range(vals.shape[0]):
        Ab = sp.csr_matrix((vals[b], d["col_idx"], d["row_ptr"]), shape=(n, n))
        nb = np.linalg.norm(rhs[b])
        out.append((np.linalg.norm(Ab @ x[b] - rhs[b]) / nb, np.linalg.norm(Ab.T @ xt[b] - rhs[b]) / nb))
    return np.array(out)


@pytest.mark.parametrize("case", LARGER)
@pytest.mark.parametrize("prec", list(PRECISIONS))
def test_larger_reference_datasets_factor_and_solve(case, prec):
    """Factor, solve and transpose solve of the larger reference datasets in
    every precision, 8 value sets each (+-2 % perturbations), within the
    residual bars; the launch plan shows which kernel tier factored what
    (any-size tier on case8387pegase; with TF32 the tensor-core tier on the
    launches whose fronts reach 65 rows, the default threshold)."""
    precision, tol = PRECISIONS[prec]
    d, _ = load(case)
    ls, vals, rhs, x, xt = _factor_solve(d, 8, precision, np.random.default_rng(2), autotune=False)
    assert not ls.singular_flags().any()
    res = _residuals(d, vals, rhs, x, xt)
    if tol is None:
        bar = np.maximum(4.0 * _fp32_lu_residuals(d, ls.plan_array("perm"), vals, rhs), 1e-5)
        assert (res[:, 0] <= bar).all() and (res[:, 1] <= 4 * bar).all(), (res, bar)
    else:
        assert res.max() <= tol, res.max(axis=0)
    tiers = ls.plan_array("factor_level_tiers")
    fsz = ls.plan_array("fp_fsz")
    if prec == "TF32":
        assert int(ls.plan_array("tc_threshold")[0]) == 65
        assert (2 in tiers) == (fsz.max() >= 65)
    else:
        assert 2 not in tiers and (1 in tiers) == (fsz.max() > 64)


@pytest.mark.parametrize("precision", [cupf.CustomPrecision.FP64, cupf.CustomPrecision.FP32])
@pytest.mark.parametrize("case", ["case1354pegase", "case8387pegase"])
def test_any_size_tier_gives_the_register_kernels_factors(case, precision):
    """wide_min_front = 1 runs every launch on the any-size tier: the same
    operations in the same order per element as the register kernels, so the
    solutions are bit for bit those of the default plan.  At 33 scenarios (two
    groups) the tier's rule gives the launches 8, 16 and 32 warps (many,
    some and few blocks); above 8 warps the assembly ranges are split at
    destination changes."""
    d, _ = load(case)
    out = []
    for wide in (0, 1):
        ls, vals, rhs, x, xt = _factor_solve(d, 33, precision, np.random.default_rng(4), autotune=False,
                                             wide_min_front=wide)
        tiers = ls.plan_array("factor_level_tiers")
        assert (tiers == 1).all() if wide else (0 in tiers)
        out.append((x, xt))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_tensor_core_tier_on_every_front_size():
    """TF32 with tc_min_front = 1: every launch of case1354pegase (fronts of
    3 to 35 rows, 1 to 8 pivots) runs its trailing update on the tensor cores
    (split tf32 products, fp32 accumulation); the residuals stay within the
    FP32 bar (4x SuperLU's unpivoted FP32 LU) and within 8x of the FP32
    factors' residuals on the same systems."""
    d, _ = load("case1354pegase")
    ls, vals, rhs, x, xt = _factor_solve(d, 40, cupf.CustomPrecision.TF32, np.random.default_rng(6), autotune=False,
                                         tc_min_front=1)
    assert (ls.plan_array("factor_level_tiers") == 2).all()
    assert not ls.singular_flags().any()
    res = _residuals(d, vals, rhs, x, xt)
    bar = np.maximum(4.0 * _fp32_lu_residuals(d, ls.plan_array("perm"), vals, rhs), 1e-5)
    assert (res[:, 0] <= bar).all() and (res[:, 1] <= 4 * bar).all(), (res, bar)
    # against the FP32 factors of the same systems: the residuals (backward
    # errors) of the split-tf32 factors are within 8x of theirs; each split
    # operand keeps about 21 of FP32's 24 bits, so the products carry about
    # 8x the FP32 rounding.  (Forward errors of two such factorizations can
    # differ far more on ill-conditioned systems; the residual is the check.)
    _, v32, r32, x32, xt32 = _factor_solve(d, 40, cupf.CustomPrecision.FP32, np.random.default_rng(6),
                                           autotune=False)
    res32 = _residuals(d, v32, r32, x32, xt32)
    assert (res[:, 0] <= 8.0 * res32[:, 0] + 1e-6).all(), (res[:, 0], res32[:, 0])


def test_tensor_core_threshold_is_autotuned():
    """TF32 with autotune: the first factorization times the tensor-core
    threshold (33, 49 or 65 rows) on the actual values and keeps the fastest;
    any choice factors within the bars."""
    d, _ = load("case8387pegase")
    ls, vals, rhs, x, xt = _factor_solve(d, 64, cupf.CustomPrecision.TF32, np.random.default_rng(8), autotune=True)
    t = int(ls.plan_array("tc_threshold")[0])
    assert t in (33, 49, 65)
    tiers, fsz = ls.plan_array("factor_level_tiers"), ls.plan_array("fp_fsz")
    assert 2 in tiers  # case8387pegase has fronts beyond every candidate
    res = _residuals(d, vals[:8], rhs[:8], x[:8], xt[:8])
    bar = np.maximum(4.0 * _fp32_lu_residuals(d, ls.plan_array("perm"), vals[:8], rhs[:8]), 1e-5)
    assert (res[:, 0] <= bar).all() and (res[:, 1] <= 4 * bar).all(), (res, bar)
