"""Regenerate the golden fixtures in this folder.

    python tests/golden/make_golden.py [--ref-root PATH]

Every number here comes from the REFERENCE itself, built from its own sources
by oracle/Makefile into oracle/_ref/libcupf_ref.so (its CPU NewtonSolver,
cuPF/cpp/src/newton_solver/core/newton_solver.cpp, and its symbolic analysis,
custom_linear_solver/src/analyze/pipeline.cpp + lower.cu host code), or from the
reference's own linear-system datasets
(custom_linear_solver/tests/datasets/power/<case>/{J.mtx,F.mtx}).

Outputs:
  two_bus.npz            reference NR on the analytic 2-bus case
                         (cuPF/tests/unit/small_cases.cpp:9-31)
  nr_<grid>.npz          reference NR (V, iterations, final mismatch) on seeded
                         scenarios of the synthetic grids, tol 1e-8 / max 10 and
                         tol 1e-12 / max 30
  adjoint_<grid>.npz     reference solve_adjoint (lambda, grad_p, grad_q) at the
                         converged state for seeded dL/dVa, dL/dVm
  jacobian_118.npz       reference Jacobian pattern + scatter maps (118-bus)
  symbolic_118.npz       every reference symbolic-plan array for the 118-bus
                         Jacobian (serial nested dissection)
  linsys_<case>.npz      the reference datasets' J (CSR) and F
  hashes.json            sha256 of every Jacobian-analysis and symbolic-plan
                         array for all synthetic grids and dataset patterns
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for p in (ROOT / "gpu-powerflow_b200", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

from cupf import grids as G  # noqa: E402
from oracle import oracle as orc  # noqa: E402

DATASETS = ("case118", "case1354pegase")
SYMBOLIC_KEYS = ("perm", "iperm", "parent", "Lp", "Li_sorted", "panel_first", "panel_ncols", "panel_width",
                 "panel_of", "front_ptr", "front_rows", "panel_parent", "asm_ptr", "asm_idx", "asm_local",
                 "plevel", "panel_level_ptr", "plcols_level", "front_off", "a_pos_csr", "graph_xadj",
                 "graph_adjncy", "sym_col_ptr", "sym_row_idx")
# with structural matching the plan also carries the matching and both inverses
MATCHING_KEYS = SYMBOLIC_KEYS + ("row_iperm", "col_perm", "row_to_col")
JAC_KEYS = ("row_ptr", "col_idx", "map11", "map21", "map12", "map22", "diag11", "diag21", "diag12", "diag22")


ROWPERM_SEED = 118


def row_permuted_pattern(row_ptr, col_idx, seed: int):
    """CSR pattern with its rows in a seeded random order (columns kept)."""
    n = row_ptr.size - 1
    order = np.random.default_rng(seed).permutation(n)
    lens = np.diff(row_ptr)[order]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([col_idx[row_ptr[r]:row_ptr[r + 1]] for r in order]).astype(np.int32)
    return rp, ci


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a), dtype=np.int64).tobytes()).hexdigest()


class _Case:
    """Minimal grid-like view of the 2-bus case for the oracle wrappers."""

    def __init__(self, c: dict):
        self.indptr, self.indices, self.data = c["indptr"], c["indices"], c["data"]
        self.pv, self.pq, self.n_bus = c["pv"], c["pq"], 2
        self.dim_f = self.pv.size + 2 * self.pq.size


def fronts_hashes(sym: dict) -> dict:
    """The reference's front CSVs (MaybeDumpFronts, pipeline.cpp:162-193):
    the analyze_fronts_only dump as text, and the full analysis's rows with
    their dispatch position q dropped, sorted (the same rows, another order)."""
    level = sym["fronts_csv_level"]
    rows = sorted(",".join(line.split(",")[1:]) for line in sym["fronts_csv_full"].splitlines()[1:])
    return {"fronts_csv_level": hashlib.sha256(level.encode()).hexdigest(),
            "fronts_rows_full": hashlib.sha256("\n".join(rows).encode()).hexdigest()}


# separator recursion (SolverConfig::parallel_nd_*) where the Jacobian's graph
# is split: (grid, depth, base_small); the oracle serialises the reference's
# METIS calls, so its threaded recursion is deterministic
PARALLEL_ND_CASES = (("2000", 2, 500), ("2000", 4, 1000), ("10000", 4, 4000))


def parallel_nd_hashes(ref) -> dict:
    grids = {"2000": G.grid_2000, "10000": G.grid_10000}
    out = {}
    for name, depth, small in PARALLEL_ND_CASES:
        ja = ref.jacobian_analysis(grids[name]())
        sym = ref.symbolic(ja["row_ptr"], ja["col_idx"], parallel_nd=True, nd_depth=depth, nd_base_small=small)
        out[f"grid{name}_d{depth}_b{small}"] = {k: digest(sym[k]) for k in SYMBOLIC_KEYS}
    return out


# relaxed-panel caps below the default 8 (SolverConfig::max_panel_width)
PANEL_WIDTH_CASES = (("118", 1), ("118", 2), ("118", 4), ("2000", 1), ("2000", 2), ("2000", 4))


def panel_width_hashes(ref) -> dict:
    grids = {"118": G.grid_118, "2000": G.grid_2000}
    out = {}
    for name, w in PANEL_WIDTH_CASES:
        ja = ref.jacobian_analysis(grids[name]())
        sym = ref.symbolic(ja["row_ptr"], ja["col_idx"], max_panel_width=w, parallel_nd=False)
        out[f"grid{name}_w{w}"] = {k: digest(sym[k]) for k in SYMBOLIC_KEYS}
    return out


def read_mtx(path: Path):
    import scipy.io
    import scipy.sparse as sp

    m = scipy.io.mmread(str(path))
    if sp.issparse(m):
        m = sp.csr_matrix(m)
        m.sort_indices()
        return m
    return np.asarray(m).reshape(-1)


def write_linsys(droot: Path, case: str) -> tuple[np.ndarray, np.ndarray]:
    """linsys_<case>.npz: a reference dataset's Newton Jacobian (CSR, FP64
    values) and mismatch vector, as its J.mtx / F.mtx hold them."""
    J = read_mtx(droot / case / "J.mtx")
    F = read_mtx(droot / case / "F.mtx")
    meta = json.loads((droot / case / "metadata.json").read_text())
    rp, ci = J.indptr.astype(np.int32), J.indices.astype(np.int32)
    np.savez_compressed(HERE / f"linsys_{case}.npz", row_ptr=rp, col_idx=ci, values=J.data, F=F,
                        mismatch_inf_norm=meta["mismatch_inf_norm"])
    return rp, ci


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=str(orc.REFERENCE_ROOT))
    ap.add_argument("--added-only", action="store_true",
                    help="only add the front-CSV, parallel-ND and panel-width hashes to the existing hashes.json "
                         "(other fixtures untouched)")
    ap.add_argument("--linsys", nargs="*", default=None, metavar="CASE",
                    help="only write linsys_<case>.npz for these reference datasets (other fixtures untouched)")
    args = ap.parse_args()
    if args.linsys is not None:
        droot = Path(args.ref_root) / "custom_linear_solver/tests/datasets/power"
        for case in args.linsys:
            write_linsys(droot, case)
        print("linear-system fixtures written:", ", ".join(args.linsys))
        return
    ref = orc.Reference()
    if args.added_only:
        hashes = json.loads((HERE / "hashes.json").read_text())
        hashes["parallel_nd"] = parallel_nd_hashes(ref)
        hashes["panel_width"] = panel_width_hashes(ref)
        for name, mk in {"118": G.grid_118, "500": G.grid_500, "2000": G.grid_2000, "10000": G.grid_10000}.items():
            ja = ref.jacobian_analysis(mk())
            hashes[f"grid{name}"]["fronts"] = fronts_hashes(ref.symbolic(ja["row_ptr"], ja["col_idx"],
                                                                         parallel_nd=False))
        for case in DATASETS:
            d = np.load(HERE / f"linsys_{case}.npz")
            hashes[case]["fronts"] = fronts_hashes(ref.symbolic(d["row_ptr"], d["col_idx"], parallel_nd=False))
        (HERE / "hashes.json").write_text(json.dumps(hashes, indent=1, sort_keys=True) + "\n")
        print("front-CSV, parallel-ND and panel-width hashes added to", HERE / "hashes.json")
        return
    hashes: dict = {}

    c2 = G.two_bus_case()
    g2 = _Case(c2)
    r = ref.solve(g2, c2["sbus"], c2["v0"], 1e-8, 20)
    np.savez(HERE / "two_bus.npz", V=r["V"], iterations=r["iterations"], final_mismatch=r["final_mismatch"],
             expected=c2["expected_v"])

    grids = {"118": G.grid_118, "500": G.grid_500, "2000": G.grid_2000, "10000": G.grid_10000}
    for name, mk in grids.items():
        g = mk()
        ja = ref.jacobian_analysis(g)
        sym = ref.symbolic(ja["row_ptr"], ja["col_idx"], parallel_nd=False)
        hashes[f"grid{name}"] = {"jacobian": {k: digest(ja[k]) for k in JAC_KEYS},
                                 "symbolic": {k: digest(sym[k]) for k in SYMBOLIC_KEYS},
                                 "front_total": int(sym["front_total"][0]), "dim": int(ja["row_ptr"].size - 1),
                                 "nnz": int(ja["col_idx"].size), "fronts": fronts_hashes(sym)}
        symm = ref.symbolic(ja["row_ptr"], ja["col_idx"], parallel_nd=False, use_matching=True)
        hashes[f"grid{name}"]["symbolic_matching"] = {k: digest(symm[k]) for k in MATCHING_KEYS}
        if name == "118":
            np.savez_compressed(HERE / "jacobian_118.npz", **{k: ja[k] for k in JAC_KEYS})
            np.savez_compressed(HERE / "symbolic_118.npz", **{k: sym[k] for k in SYMBOLIC_KEYS})
        if name in ("118", "2000"):
            nsc = 4 if name == "118" else 2
            S = g.scenarios(nsc, seed=777)
            out = {"sbus": S, "v0": g.flat_start(nsc)}
            for tag, tol, mi in (("t8", 1e-8, 10), ("t12", 1e-12, 30)):
                rs = [ref.solve(g, S[b], out["v0"][b], tol, mi) for b in range(nsc)]
                out[f"V_{tag}"] = np.stack([x["V"] for x in rs])
                out[f"it_{tag}"] = np.array([x["iterations"] for x in rs], np.int32)
                out[f"fm_{tag}"] = np.array([x["final_mismatch"] for x in rs])
            np.savez_compressed(HERE / f"nr_{name}.npz", **out)
            rng = np.random.default_rng(31 + int(name))
            ga, gm = rng.standard_normal(g.n_bus), rng.standard_normal(g.n_bus)
            ad = ref.adjoint(g, S[0], out["v0"][0], ga, gm, 1e-12, 30)
            np.savez_compressed(HERE / f"adjoint_{name}.npz", sbus=S[0], v0=out["v0"][0], grad_va=ga, grad_vm=gm,
                                V=ad["V"], lam=ad["lambda"], grad_p=ad["grad_p"], grad_q=ad["grad_q"],
                                residual=ad["residual"])

    droot = Path(args.ref_root) / "custom_linear_solver/tests/datasets/power"
    for case in DATASETS:
        rp, ci = write_linsys(droot, case)
        sym = ref.symbolic(rp, ci, parallel_nd=False)
        hashes[case] = {"symbolic": {k: digest(sym[k]) for k in SYMBOLIC_KEYS},
                        "front_total": int(sym["front_total"][0]), "dim": int(rp.size - 1), "nnz": int(ci.size),
                        "fronts": fronts_hashes(sym)}
        symm = ref.symbolic(rp, ci, parallel_nd=False, use_matching=True)
        hashes[case]["symbolic_matching"] = {k: digest(symm[k]) for k in MATCHING_KEYS}

    # a pattern whose diagonal is structurally incomplete: case118's J with
    # its rows shuffled (seeded); structural matching has to find columns
    d = np.load(HERE / "linsys_case118.npz")
    rp, ci = row_permuted_pattern(d["row_ptr"], d["col_idx"], ROWPERM_SEED)
    symm = ref.symbolic(rp, ci, parallel_nd=False, use_matching=True)
    hashes["case118_rowperm"] = {"symbolic_matching": {k: digest(symm[k]) for k in MATCHING_KEYS},
                                 "seed": ROWPERM_SEED}

    hashes["parallel_nd"] = parallel_nd_hashes(ref)
    hashes["panel_width"] = panel_width_hashes(ref)
    (HERE / "hashes.json").write_text(json.dumps(hashes, indent=1, sort_keys=True) + "\n")
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
