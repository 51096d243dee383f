"""Host-side analysis of the engine, bit-exact against the reference (no GPU needed).

The engine's Jacobian analysis (make_jacobian_indexing / JacobianPatternGenerator /
JacobianMapBuilder, cuPF/cpp/src/newton_solver/ops/jacobian/jacobian_analysis.cpp)
and its symbolic plan (custom_linear_solver/src/analyze/pipeline.cpp steps 5-8,
elimination_tree.cpp, supernode.cpp, multifrontal.cpp, host parts of lower.cu)
are compared array by array with what the reference produced on the same
inputs with serial nested dissection (hashes and full arrays in tests/golden/).
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import cupf
from cupf import grids as G

GOLD = Path(__file__).resolve().parent / "golden"
HASHES = json.loads((GOLD / "hashes.json").read_text())

# engine plan_array name -> reference symbolic array name
SYMBOLIC = {"perm": "perm", "iperm": "iperm", "parent": "parent", "Lp": "Lp", "Li": "Li_sorted",
            "panel_first": "panel_first", "panel_ncols": "panel_ncols", "panel_width": "panel_width",
            "panel_of": "panel_of", "front_ptr": "front_ptr", "front_rows": "front_rows",
            "panel_parent": "panel_parent", "asm_ptr": "asm_ptr", "asm_idx": "asm_idx", "asm_local": "asm_local",
            "plevel": "plevel", "level_ptr": "panel_level_ptr", "plcols_level": "plcols_level",
            "front_off": "front_off", "a_pos_csr": "a_pos_csr", "graph_xadj": "graph_xadj",
            "graph_adjncy": "graph_adjncy", "sym_col_ptr": "sym_col_ptr", "sym_row_idx": "sym_row_idx"}
JACOBIAN = {"jac_row_ptr": "row_ptr", "jac_col_idx": "col_idx", "map11": "map11", "map21": "map21",
            "map12": "map12", "map22": "map22", "diag11": "diag11", "diag21": "diag21", "diag12": "diag12",
            "diag22": "diag22"}
GRIDS = {"118": G.grid_118, "500": G.grid_500, "2000": G.grid_2000, "10000": G.grid_10000}


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a), dtype=np.int64).tobytes()).hexdigest()


def _analyzed(g, serial_nd=True):
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.custom.serial_nd = serial_nd
    s = cupf.NewtonSolver(o)
    s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, g.pq)
    return s


@pytest.fixture(scope="module")
def analyzed():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = _analyzed(GRIDS[name]())
        return cache[name]
    return get


@pytest.mark.parametrize("name", list(GRIDS))
def test_jacobian_analysis_bit_exact(analyzed, name):
    s = analyzed(name)
    gold = HASHES[f"grid{name}"]
    for ours, ref in JACOBIAN.items():
        assert digest(s.plan_array(ours)) == gold["jacobian"][ref], ours
    inf = s.info()
    assert inf["dim_f"] == gold["dim"] and inf["nnz_jacobian"] == gold["nnz"]


@pytest.mark.parametrize("name", list(GRIDS))
def test_symbolic_plan_bit_exact(analyzed, name):
    s = analyzed(name)
    gold = HASHES[f"grid{name}"]
    bad = [ours for ours, ref in SYMBOLIC.items() if digest(s.plan_array(ours)) != gold["symbolic"][ref]]
    assert not bad, f"arrays differing from the reference: {bad}"


def test_symbolic_plan_118_arrays(analyzed):
    """Full-array comparison on the 118-bus grid (readable diff on failure)."""
    s = analyzed("118")
    gold = np.load(GOLD / "symbolic_118.npz")
    for ours, ref in SYMBOLIC.items():
        np.testing.assert_array_equal(s.plan_array(ours), gold[ref], err_msg=ours)
    jg = np.load(GOLD / "jacobian_118.npz")
    for ours, ref in JACOBIAN.items():
        np.testing.assert_array_equal(s.plan_array(ours), jg[ref], err_msg=ours)


@pytest.mark.parametrize("case", ["case118", "case1354pegase"])
def test_linear_solver_symbolic_on_reference_datasets(case):
    """cls_analyze_host on the reference's own J.mtx patterns."""
    d = np.load(GOLD / f"linsys_{case}.npz")
    ls = cupf.LinearSolver(cupf.SolverConfig(serial_nd=True))
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze_host()
    gold = HASHES[case]
    bad = [ours for ours, ref in SYMBOLIC.items()
           if digest(ls.plan_array(ours)) != gold["symbolic"][ref]]
    assert not bad, f"arrays differing from the reference: {bad}"


@pytest.mark.parametrize("name", ["118", "2000"])
def test_factor_program_invariants(analyzed, name):
    """The dense-front program the kernels run: every Jacobian position reaches
    exactly one front slot; children are factored in earlier levels; sizes agree."""
    s = analyzed(name)
    fsz = s.plan_array("fp_fsz")
    nc = s.plan_array("fp_nc")
    front_ptr = s.plan_array("front_ptr")
    assert np.array_equal(fsz, np.diff(front_ptr))
    assert np.array_equal(nc, s.plan_array("panel_ncols"))
    assert (nc >= 1).all() and (nc <= fsz).all() and (nc <= 8).all()
    # assembly of J: every CSR position appears once in the A-row program
    arow_q = s.plan_array("fp_arow_q")
    nnz = s.info()["nnz_jacobian"]
    assert np.array_equal(np.sort(arow_q), np.arange(nnz))
    # level order: a panel's parent is in a later level
    plevel = s.plan_array("plevel")
    parent = s.plan_array("panel_parent")
    has = parent >= 0
    assert (plevel[parent[has]] > plevel[has]).all()
    lf = s.plan_array("fp_level_fronts")
    assert np.array_equal(np.sort(lf), np.arange(fsz.size))


def test_parallel_nd_matches_reference_below_threshold():
    """Parallel nested dissection reduces to one METIS call below 4,000 vertices
    (metis_nd.cpp:241-278), so it equals the serial plan there."""
    g = G.grid_500()
    a, b = _analyzed(g, True), _analyzed(g, False)
    for ours in ("perm", "front_ptr", "asm_local"):
        assert np.array_equal(a.plan_array(ours), b.plan_array(ours))


def test_analysis_is_deterministic_across_threads():
    """METIS calls are serialized: concurrent analyses give the same plan."""
    import threading
    g = G.grid_2000()
    out = [None] * 4

    def run(i):
        out[i] = _analyzed(g, False).plan_array("perm")
    ts = [threading.Thread(target=run, args=(i,)) for i in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert all(np.array_equal(out[0], o) for o in out[1:])


def test_front_launch_records(analyzed):
    """front_meta: one 24-int32 record per front in level order, consistent
    with the plan arrays it summarises (the kernels read only the record)."""
    s = analyzed("2000")
    meta = s.plan_array("front_meta").reshape(-1, 24)
    lf = s.plan_array("fp_level_fronts")
    fsz, nc = s.plan_array("fp_fsz"), s.plan_array("fp_nc")
    front_ptr = s.plan_array("front_ptr")
    fe_ptr, u_off, cb_off = s.plan_array64("fe_ptr"), s.plan_array64("u_off"), s.plan_array64("cb_off")
    split = s.plan_array64("fe_split").reshape(-1, 9)
    wide = meta[:, 4:12].copy().view(np.int64)
    assert np.array_equal(meta[:, 3], lf)
    assert np.array_equal(meta[:, 0], fsz[lf]) and np.array_equal(meta[:, 1], nc[lf])
    assert np.array_equal(wide[:, 0], fe_ptr[lf]) and np.array_equal(wide[:, 1], u_off[lf])
    assert np.array_equal(wide[:, 3], cb_off[lf])
    assert np.array_equal(meta[:, 12:20], (split[lf, 1:] - split[lf, :1]).astype(np.int32))
    assert np.array_equal(meta[:, 20], front_ptr[lf])


MATCHING = dict(SYMBOLIC, row_iperm="row_iperm", col_perm="col_perm", row_to_col="row_to_col")


def _row_permuted(row_ptr, col_idx, seed):
    """The rows of a CSR pattern in a seeded random order (tests/golden/make_golden.py)."""
    n = row_ptr.size - 1
    order = np.random.default_rng(seed).permutation(n)
    lens = np.diff(row_ptr)[order]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([col_idx[row_ptr[r]:row_ptr[r + 1]] for r in order]).astype(np.int32)
    return rp, ci


@pytest.mark.parametrize("name", ["118", "2000", "10000"])
def test_symbolic_plan_with_matching_bit_exact(name):
    """Structural matching (CustomMatchingMode::Structural): the Hopcroft-Karp
    matching, both permutations and every plan array equal the reference's
    (analyze/pipeline.cpp:77-160, 222-272)."""
    g = GRIDS[name]()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.custom.serial_nd = True
    o.custom.matching = cupf.CustomMatchingMode.Structural
    s = cupf.NewtonSolver(o)
    s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, g.pq)
    gold = HASHES[f"grid{name}"]["symbolic_matching"]
    bad = [ours for ours, ref in MATCHING.items() if digest(s.plan_array(ours)) != gold[ref]]
    assert not bad, f"arrays differing from the reference: {bad}"


@pytest.mark.parametrize("case", ["case118", "case1354pegase", "case118_rowperm"])
def test_linear_solver_matching_bit_exact(case):
    """Matching on the reference datasets, and on case118's J with its rows
    shuffled, where the diagonal is structurally incomplete and the matching
    is not the identity."""
    d = np.load(GOLD / f"linsys_{case.split('_')[0]}.npz")
    rp, ci = d["row_ptr"], d["col_idx"]
    if case.endswith("rowperm"):
        rp, ci = _row_permuted(rp, ci, HASHES[case]["seed"])
    ls = cupf.LinearSolver(cupf.SolverConfig(serial_nd=True, matching=1))
    ls.set_data(rp, ci)
    ls.analyze_host()
    gold = HASHES[case]["symbolic_matching"]
    bad = [ours for ours, ref in MATCHING.items() if digest(ls.plan_array(ours)) != gold[ref]]
    assert not bad, f"arrays differing from the reference: {bad}"
    if case.endswith("rowperm"):
        r2c = ls.plan_array("row_to_col")
        assert np.array_equal(np.sort(r2c), np.arange(rp.size - 1))
        assert (r2c != np.arange(rp.size - 1)).any()


def test_matching_fails_without_a_perfect_matching():
    """Two rows whose only column is the same: no perfect matching exists; the
    analysis fails (the reference's Analyze returns false there)."""
    rp = np.array([0, 1, 2, 4], np.int32)
    ci = np.array([0, 0, 1, 2], np.int32)
    ls = cupf.LinearSolver(cupf.SolverConfig(serial_nd=True, matching=1))
    ls.set_data(rp, ci)
    with pytest.raises(Exception):
        ls.analyze_host()


def _sha(text: str) -> str:
    return hashlib.sha256(text.encode()).hexdigest()


def _rows_without_q(text: str) -> str:
    return "\n".join(sorted(",".join(line.split(",")[1:]) for line in text.splitlines()[1:]))


@pytest.mark.parametrize("name", list(GRIDS))
def test_fronts_csv_matches_the_reference_dump(analyzed, name, tmp_path):
    """pf_dump_fronts_csv writes, byte for byte, the reference's front dump
    under analyze_fronts_only (MaybeDumpFronts, analyze/pipeline.cpp:162-193);
    its full analysis lists the same rows in its own order inside each
    level."""
    path = tmp_path / "fronts.csv"
    analyzed(name).dump_fronts_csv(path)
    text = path.read_text()
    assert text.startswith("q,p,fsz,nc,uc,level,parent,asm_len,extend_elems\n")
    gold = HASHES[f"grid{name}"]["fronts"]
    assert _sha(text) == gold["fronts_csv_level"]
    assert _sha(_rows_without_q(text)) == gold["fronts_rows_full"]


@pytest.mark.parametrize("case", ["case118", "case1354pegase"])
def test_linear_solver_fronts_csv_on_reference_datasets(case, tmp_path):
    d = np.load(GOLD / f"linsys_{case}.npz")
    ls = cupf.LinearSolver(cupf.SolverConfig(serial_nd=True))
    ls.set_data(d["row_ptr"], d["col_idx"])
    ls.analyze_host()
    path = tmp_path / "fronts.csv"
    ls.dump_fronts_csv(path)
    text = path.read_text()
    assert _sha(text) == HASHES[case]["fronts"]["fronts_csv_level"]
    assert _sha(_rows_without_q(text)) == HASHES[case]["fronts"]["fronts_rows_full"]
    with pytest.raises(Exception):
        ls.dump_fronts_csv(tmp_path / "no_such_dir" / "fronts.csv")


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["LIB_REF"]).LIB_REF.exists(),
                    reason="oracle/_ref not built (reference sources absent)")
def test_fronts_csv_against_the_live_reference(analyzed, tmp_path):
    """The same on the 118-bus grid against the reference run here: the text
    itself, so a difference shows where it is."""
    from oracle.oracle import Reference

    g = GRIDS["118"]()
    s = analyzed("118")
    ref = Reference()
    sym = ref.symbolic(s.plan_array("jac_row_ptr"), s.plan_array("jac_col_idx"), parallel_nd=False)
    path = tmp_path / "fronts.csv"
    s.dump_fronts_csv(path)
    assert path.read_text() == sym["fronts_csv_level"]
    assert _rows_without_q(path.read_text()) == _rows_without_q(sym["fronts_csv_full"])
    assert g.n_bus == 118


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["LIB_REF"]).LIB_REF.exists(),
                    reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("name,depth,small", [("2000", 2, 500), ("2000", 4, 1000), ("10000", 4, 4000)])
def test_parallel_nd_matches_the_reference_recursion(name, depth, small):
    """Separator recursion (serial_nd = False) with SolverConfig's
    parallel_nd_depth / parallel_nd_base_small (metis_nd.cpp:241-278), at
    sizes where the Jacobian's graph is split: every plan array equals the
    reference's own recursion.  The oracle runs the reference with its METIS
    calls serialised (oracle/ref_shim/metis_lock_shim.c), which makes its
    threaded recursion deterministic; the engine runs the halves one after
    the other."""
    from oracle.oracle import Reference

    g = GRIDS[name]()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.custom.serial_nd = False
    o.custom.parallel_nd_depth = depth
    o.custom.parallel_nd_base_small = small
    s = cupf.NewtonSolver(o)
    s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, g.pq)
    ref = Reference()
    rp, ci = s.plan_array("jac_row_ptr"), s.plan_array("jac_col_idx")
    r1 = ref.symbolic(rp, ci, parallel_nd=True, nd_depth=depth, nd_base_small=small)
    r2 = ref.symbolic(rp, ci, parallel_nd=True, nd_depth=depth, nd_base_small=small)
    assert np.array_equal(r1["perm"], r2["perm"])  # the serialised reference is deterministic
    bad = [ours for ours, r in SYMBOLIC.items() if not np.array_equal(s.plan_array(ours), r1[r])]
    assert not bad, f"arrays differing from the reference: {bad}"
    serial = _analyzed(g, True)
    assert not np.array_equal(s.plan_array("perm"), serial.plan_array("perm"))  # the graph was split


def test_parallel_nd_parameters_are_validated():
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.custom.parallel_nd_depth = -1
    with pytest.raises(ValueError):
        cupf.NewtonSolver(o)


@pytest.mark.parametrize("name,depth,small", [("2000", 2, 500), ("2000", 4, 1000), ("10000", 4, 4000)])
def test_parallel_nd_matches_the_reference_golden(name, depth, small):
    """The same cases against the committed hashes of the reference's plan
    (tests/golden/make_golden.py), so the check stands without the reference."""
    g = GRIDS[name]()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.custom.serial_nd = False
    o.custom.parallel_nd_depth = depth
    o.custom.parallel_nd_base_small = small
    s = cupf.NewtonSolver(o)
    s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, g.pq)
    gold = HASHES["parallel_nd"][f"grid{name}_d{depth}_b{small}"]
    bad = [ours for ours, ref in SYMBOLIC.items() if digest(s.plan_array(ours)) != gold[ref]]
    assert not bad, f"arrays differing from the reference: {bad}"


@pytest.mark.parametrize("name,width", [("118", 1), ("118", 2), ("118", 4), ("2000", 1), ("2000", 2), ("2000", 4)])
def test_symbolic_plan_at_other_panel_widths(name, width):
    """Relaxed panels capped below 8 (SolverConfig::max_panel_width,
    supernode.cpp:55-92): every plan array equals the reference's."""
    g = GRIDS[name]()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.custom.serial_nd = True
    o.custom.max_panel_width = width
    s = cupf.NewtonSolver(o)
    s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, g.pq)
    gold = HASHES["panel_width"][f"grid{name}_w{width}"]
    bad = [ours for ours, ref in SYMBOLIC.items() if digest(s.plan_array(ours)) != gold[ref]]
    assert not bad, f"arrays differing from the reference: {bad}"
    assert int(s.plan_array("panel_ncols").max()) <= width


REF_DATASETS = __import__("oracle.oracle", fromlist=["REFERENCE_ROOT"]).REFERENCE_ROOT / "custom_linear_solver/tests/datasets/power"


@pytest.mark.skipif(not (REF_DATASETS.exists() and
                         __import__("oracle.oracle", fromlist=["LIB_REF"]).LIB_REF.exists()),
                    reason="the reference's datasets and oracle/_ref are needed")
@pytest.mark.parametrize("case", ["case118", "case1354pegase", "case3120sp", "case6468rte", "case8387pegase"])
@pytest.mark.parametrize("serial", [True, False])
def test_symbolic_plan_on_every_reference_dataset(case, serial):
    """cls_analyze_host on the reference's five linear-system patterns (real
    Newton Jacobians up to 8,387 unknowns), serial and parallel nested
    dissection at SolverConfig's defaults, against the reference's own plan
    computed here (the larger two are split by the parallel ordering)."""
    import scipy.io
    import scipy.sparse as sp
    from oracle.oracle import Reference

    J = sp.csr_matrix(scipy.io.mmread(str(REF_DATASETS / case / "J.mtx")))
    J.sort_indices()
    rp, ci = J.indptr.astype(np.int32), J.indices.astype(np.int32)
    ls = cupf.LinearSolver(cupf.SolverConfig(serial_nd=serial))
    ls.set_data(rp, ci)
    ls.analyze_host()
    ref = Reference().symbolic(rp, ci, parallel_nd=not serial)
    bad = [ours for ours, r in SYMBOLIC.items() if not np.array_equal(ls.plan_array(ours), ref[r])]
    assert not bad, f"arrays differing from the reference: {bad}"


@pytest.mark.skipif(not (REF_DATASETS.exists() and
                         __import__("oracle.oracle", fromlist=["LIB_REF"]).LIB_REF.exists()),
                    reason="the reference's datasets and oracle/_ref are needed")
@pytest.mark.parametrize("case", ["case3120sp", "case6468rte", "case8387pegase"])
def test_matching_plan_on_the_larger_reference_datasets(case):
    """Structural matching (MatchingMode::Structural) on the larger reference
    datasets: the matching, both permutations and every plan array equal the
    reference's own, computed here."""
    import scipy.io
    import scipy.sparse as sp
    from oracle.oracle import Reference

    J = sp.csr_matrix(scipy.io.mmread(str(REF_DATASETS / case / "J.mtx")))
    J.sort_indices()
    rp, ci = J.indptr.astype(np.int32), J.indices.astype(np.int32)
    ls = cupf.LinearSolver(cupf.SolverConfig(serial_nd=True, matching=1))
    ls.set_data(rp, ci)
    ls.analyze_host()
    ref = Reference().symbolic(rp, ci, parallel_nd=False, use_matching=True)
    bad = [ours for ours, r in MATCHING.items() if not np.array_equal(ls.plan_array(ours), ref[r])]
    assert not bad, f"arrays differing from the reference: {bad}"
