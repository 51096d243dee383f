"""Case I/O in the reference's dump-case format (CPU only).

The engine's reader (pf_case_*) is checked against the reference's own loader
(cuPF/tests/dump_case_loader.cpp, compiled into oracle/_ref) on the same
directories: identical arrays, and the same error message for each defect
the reference checks.
"""
from pathlib import Path

import numpy as np
import pytest

from cupf import case_io
from cupf import grids as G
from oracle.oracle import LIB_REF

needs_ref = pytest.mark.skipif(not LIB_REF.exists(), reason="oracle/_ref not built (reference sources absent)")


@pytest.fixture(scope="module")
def reference():
    from oracle.oracle import Reference
    return Reference()


def _write(d: Path, name: str, text: str) -> None:
    (d / name).write_text(text)


def _small_case(d: Path, mtx: str, sbus="1 0\n-0.5 -0.1\n-0.4 -0.2\n", v0="1 0\n1 0\n1 0\n", pv="", pq="1\n2\n"):
    d.mkdir(parents=True, exist_ok=True)
    _write(d, "dump_Ybus.mtx", mtx)
    _write(d, "dump_Sbus.txt", sbus)
    _write(d, "dump_V.txt", v0)
    _write(d, "dump_pv.txt", pv)
    _write(d, "dump_pq.txt", pq)
    return d


GENERAL = """%%MatrixMarket matrix coordinate complex general
% a comment line
3 3 8

1 1 10.0 -30.0
1 2 -5.0 15.0
2 1 -5.0 15.0
# another comment
2 2 9.0 -28.0
2 3 -4.0 13.0
3 2 -4.0 13.0
3 3 4.0 -13.0
3 3 0.5 -0.25
"""

SYMMETRIC = """%%MatrixMarket matrix coordinate complex symmetric
3 3 5
1 1 10.0 -30.0
2 1 -5.0 15.0
2 2 9.0 -28.0
3 2 -4.0 13.0
3 3 4.5 -13.25
"""


def _same(ours, ref):
    assert ours.rows == ref["rows"]
    for k in ("indptr", "indices", "pv", "pq"):
        assert np.array_equal(getattr(ours, k), ref[k]), k
    for k in ("ybus_data", "sbus", "v0"):
        assert np.array_equal(getattr(ours, k).view(np.float64), ref[k].view(np.float64)), k


def test_round_trip_synthetic_grid(tmp_path):
    g = G.grid_118()
    vref = g.v0 * np.exp(0.01j)
    d = case_io.save_grid(tmp_path, g, vref=vref)
    c = case_io.load_dump_case(d)
    assert c.case_name == "synthetic_118" and c.rows == c.cols == 118
    assert np.array_equal(c.indptr, g.indptr) and np.array_equal(c.indices, g.indices)
    assert np.array_equal(c.ybus_data, g.data)
    assert np.array_equal(c.sbus, g.sbus) and np.array_equal(c.v0, g.v0)
    assert np.array_equal(c.pv, g.pv) and np.array_equal(c.pq, g.pq)
    assert np.array_equal(c.vref, vref)
    assert c.metadata["n_bus"] == 118 and c.metadata["n_pv"] == len(g.pv)


@needs_ref
@pytest.mark.parametrize("n", [118, 2000])
def test_matches_reference_loader_on_grids(tmp_path, reference, n):
    g = G.grid_118() if n == 118 else G.grid_2000()
    d = case_io.save_grid(tmp_path, g)
    _same(case_io.load_dump_case(d), reference.load_dump_case(d))


@needs_ref
@pytest.mark.parametrize("mtx", [GENERAL, SYMMETRIC], ids=["general_dup_comments", "symmetric"])
def test_matches_reference_loader_on_format_cases(tmp_path, reference, mtx):
    d = _small_case(tmp_path / "c", mtx)
    ours = case_io.load_dump_case(d)
    _same(ours, reference.load_dump_case(d))
    assert ours.vref is None
    if mtx is GENERAL:  # the duplicate (3, 3) entries are summed
        assert ours.ybus_data[-1] == complex(4.5, -13.25)
    else:  # the lower triangle is mirrored
        assert ours.indptr.tolist() == [0, 2, 5, 7]


DEFECTS = {
    "missing_dir": None,
    "missing_file": ("dump_pq.txt", None),
    "bad_header": ("dump_Ybus.mtx", "%%MatrixMarket matrix coordinate real general\n1 1 1\n1 1 1.0\n"),
    "bad_dims": ("dump_Ybus.mtx", "%%MatrixMarket matrix coordinate complex general\n3 x 1\n"),
    "truncated": ("dump_Ybus.mtx", "%%MatrixMarket matrix coordinate complex general\n3 3 2\n1 1 1 0\n"),
    "bad_entry": ("dump_Ybus.mtx", "%%MatrixMarket matrix coordinate complex general\n3 3 1\n1 1 1.0\n"),
    "out_of_bounds": ("dump_Ybus.mtx", "%%MatrixMarket matrix coordinate complex general\n3 3 1\n4 1 1 0\n"),
    "not_square": ("dump_Ybus.mtx", "%%MatrixMarket matrix coordinate complex general\n3 2 1\n1 1 1 0\n"),
    "bad_pair": ("dump_Sbus.txt", "1 0\n2\n3 0\n"),
    "bad_int": ("dump_pv.txt", "x\n"),
    "sbus_size": ("dump_Sbus.txt", "1 0\n"),
    "v0_size": ("dump_V.txt", "1 0\n1 0\n"),
}


@needs_ref
@pytest.mark.parametrize("defect", list(DEFECTS))
def test_errors_match_reference_loader(tmp_path, reference, defect):
    d = tmp_path / "case"
    if DEFECTS[defect] is not None:
        _small_case(d, GENERAL)
        name, text = DEFECTS[defect]
        if text is None:
            (d / name).unlink()
        else:
            _write(d, name, text)
    with pytest.raises(RuntimeError) as ref_err:
        reference.load_dump_case(d)
    with pytest.raises(RuntimeError) as our_err:
        case_io.load_dump_case(d)
    assert str(our_err.value) == str(ref_err.value)


def test_vref_size_is_checked(tmp_path):
    d = _small_case(tmp_path / "c", GENERAL)
    _write(d, "dump_Vref.txt", "1 0\n")
    with pytest.raises(RuntimeError, match="Vref size does not match Ybus rows"):
        case_io.load_dump_case(d)


def test_replicate_scenarios_follows_the_bench_recipe(tmp_path):
    g = G.grid_118()
    c = case_io.load_dump_case(case_io.save_grid(tmp_path, g))
    sbus, v0 = case_io.replicate_scenarios(c, 5, load_scale_step=0.01)
    for b in range(5):
        assert np.array_equal(sbus[b], g.sbus * (1.0 + 0.01 * b))
        assert np.array_equal(v0[b], g.v0)
