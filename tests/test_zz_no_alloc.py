"""cls_factorize_static_scratch: the allocation-free factorization entry point.

Kept in its own file, collected last, so it runs both on its own in a fresh
process and after every other GPU test.  The case is the reference dataset
case1354pegase in FP64, whose largest fronts (34-35 rows) exceed shared memory
and so do use the front scratch that this entry point takes from its static
area."""
from pathlib import Path

import numpy as np
import pytest

import cupf
from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]
GOLD = Path(__file__).resolve().parent / "golden"


def _solver(d, B, autotune=True):
    ls = cupf.LinearSolver(cupf.SolverConfig(precision=int(cupf.CustomPrecision.FP64), serial_nd=True,
                                             autotune=autotune))
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze()
    ls.setup(B)
    return ls


def test_static_scratch_factorize_matches_regular_twice_in_a_row():
    import torch

    d = np.load(GOLD / "linsys_case1354pegase.npz")
    B = 2
    rng = np.random.default_rng(11)
    rhs = torch.tensor(np.stack([d["F"]] * B) + 0.1 * rng.standard_normal((B, d["F"].size)), device="cuda")
    ref = _solver(d, B)
    ls = _solver(d, B, autotune=False)
    ls.factorize(torch.tensor(np.stack([d["values"]] * B), device="cuda"))  # workspace for this batch size
    # the case exercises the static area: some launches keep their fronts in
    # the global scratch under the built-in placement the entry point uses
    # (2: register rows over the scratch, 3: the any-size tier)
    assert set(ls.plan_array("factor_level_placement").tolist()) & {2, 3}
    for call in range(2):
        vals = np.stack([d["values"]] * B) * (1.0 + 0.01 * rng.uniform(-1, 1, (B, d["values"].size)))
        tv = torch.tensor(vals, device="cuda")
        ref.factorize(tv)
        x_ref = ref.solve(rhs).cpu().numpy()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        ls.factorize_static_scratch(tv)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (call, free0 - free1)  # the call allocated no device memory
        x = ls.solve(rhs).cpu().numpy()
        assert np.isfinite(x).all(), call
        assert np.abs(x - x_ref).max() <= 1e-12 * np.abs(x_ref).max(), call


def test_static_scratch_requires_existing_workspace():
    import torch

    d = np.load(GOLD / "linsys_case1354pegase.npz")
    ls = _solver(d, 2)
    with pytest.raises(cupf.linear_solver.CustomSolverError) as e:
        ls.factorize_static_scratch(torch.tensor(np.stack([d["values"]] * 2), device="cuda"))
    assert "allocates nothing" in str(e.value)


def test_static_scratch_rejects_a_batch_beyond_its_size():
    import torch

    d = np.load(GOLD / "linsys_case1354pegase.npz")
    B = 256
    ls = _solver(d, B)
    vals = torch.tensor(np.stack([d["values"]] * B), device="cuda")
    ls.factorize(vals)
    with pytest.raises(cupf.linear_solver.CustomSolverError) as e:
        ls.factorize_static_scratch(vals)
    assert "bytes of front scratch" in str(e.value) and e.value.status == 1


def test_static_scratch_at_batch_one():
    """A batch of one factors with the single-system tree launch, which keeps
    every front in shared memory: the entry point allocates nothing and
    gives the regular call's solution."""
    import torch

    d = np.load(GOLD / "linsys_case1354pegase.npz")
    ls = _solver(d, 1)
    vals = torch.tensor(d["values"][None, :], device="cuda")
    rhs = torch.tensor(d["F"][None, :], device="cuda")
    ls.factorize(vals)
    x_ref = ls.solve(rhs).cpu().numpy()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    ls.factorize_static_scratch(vals)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(ls.solve(rhs).cpu().numpy(), x_ref)
