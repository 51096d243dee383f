"""Command-line runner of the batched sparse solver on one linear system.

The counterpart of the reference's runner
(custom_linear_solver/tests/runners/run_custom_solver.cu): read a matrix and
a right-hand side, analyse, factor and solve a uniform batch of B systems
sharing the pattern (system b's values scaled by 1 + 1e-3 b), time the
phases with CUDA events, and report the relative residual of every system.

    python -m cupf.run_solver --matrix J.mtx --rhs F.mtx --batch 256 --precision tf32
    python -m cupf.run_solver --npz tests/golden/linsys_case8387pegase.npz --batch 256
    python -m cupf.run_solver --npz tests/golden/linsys_case8387pegase.npz --batch 64 --transpose

Prints one JSON object: dimensions, the plan's front sizes and per-launch
kernel tiers, the median factorization and solve times, and the largest
relative residual ||A_b x_b - r|| / ||r|| over the batch (FP64 on the host).
With --transpose it also times the transposed solve A^T x = r on the same
factors (the adjoint's U^T and L^T sweeps) and reports its residual.
"""
from __future__ import annotations

import argparse
import json
import statistics
import sys
from pathlib import Path

import numpy as np

PRECISION = {"fp64": 0, "fp32": 1, "tf32": 2}


def load_system(args) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(row_ptr, col_idx, values, rhs) from an .npz fixture or MatrixMarket files."""
    if args.npz:
        d = np.load(args.npz)
        return d["row_ptr"].astype(np.int32), d["col_idx"].astype(np.int32), d["values"], np.asarray(d["F"])
    import scipy.io
    import scipy.sparse as sp

    A = sp.csr_matrix(scipy.io.mmread(str(args.matrix)))
    A.sort_indices()
    n = A.shape[0]
    rhs = np.ones(n) if not args.rhs else np.asarray(scipy.io.mmread(str(args.rhs))).reshape(-1)
    return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64), rhs


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    src = ap.add_mutually_exclusive_group(required=True)
    src.add_argument("--npz", type=Path, help="fixture with row_ptr, col_idx, values, F")
    src.add_argument("--matrix", type=Path, help="MatrixMarket matrix (real, square)")
    ap.add_argument("--rhs", type=Path, help="MatrixMarket right-hand side (default: all ones)")
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--repeat", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--precision", choices=list(PRECISION), default="fp64")
    ap.add_argument("--parallel-nd", action="store_true", help="separator recursion instead of one METIS call")
    ap.add_argument("--max-panel-width", type=int, default=8)
    ap.add_argument("--matching", action="store_true", help="structural row/column matching")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--wide-min-front", type=int, default=0)
    ap.add_argument("--tc-min-front", type=int, default=0)
    ap.add_argument("--batch1-schedule", type=int, choices=(0, 1), default=0,
                    help="batch 1: 0 the single-system tree launch, 1 the batched lane kernels")
    ap.add_argument("--transpose", action="store_true",
                    help="also time the transposed solve A^T x = b on the same factors (the adjoint's sweeps)")
    args = ap.parse_args(argv)

    import scipy.sparse as sp
    import torch

    import cupf

    if not torch.cuda.is_available():
        sys.exit("run_solver: needs a CUDA device")
    rp, ci, vals, rhs = load_system(args)
    n, B = rp.size - 1, args.batch
    dev = torch.device("cuda")
    cfg = cupf.SolverConfig(precision=PRECISION[args.precision], serial_nd=not args.parallel_nd,
                            max_panel_width=args.max_panel_width, matching=int(args.matching),
                            autotune=not args.no_autotune, wide_min_front=args.wide_min_front,
                            tc_min_front=args.tc_min_front, batch1_schedule=args.batch1_schedule)
    ls = cupf.LinearSolver(cfg)
    ls.set_data(rp, ci)
    ls.analyze()
    ls.setup(B)
    scale = 1.0 + 1e-3 * np.arange(B)[:, None]
    V = vals[None, :] * scale
    dt = torch.float64 if args.precision == "fp64" else torch.float32
    Vd = torch.tensor(V, dtype=dt, device=dev)
    R = torch.tensor(np.repeat(rhs[None, :], B, axis=0), dtype=torch.float64, device=dev)
    tf, ts, tt = [], [], []
    x = xt = None
    for k in range(args.warmup + args.repeat):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record()
        ls.factorize(Vd)
        e[1].record()
        x = ls.solve(R)
        e[2].record()
        if args.transpose:
            xt = ls.solve_transpose(R)
        e[3].record()
        e[3].synchronize()
        if k >= args.warmup:
            tf.append(e[0].elapsed_time(e[1]))
            ts.append(e[1].elapsed_time(e[2]))
            tt.append(e[2].elapsed_time(e[3]))
    xh = x.cpu().numpy()
    xth = xt.cpu().numpy() if xt is not None else None
    res, rest = [], []
    for b in range(B):
        A = sp.csr_matrix((V[b], ci, rp), shape=(n, n))
        res.append(float(np.linalg.norm(A @ xh[b] - rhs) / max(np.linalg.norm(rhs), 1e-300)))
        if xth is not None:
            rest.append(float(np.linalg.norm(A.T @ xth[b] - rhs) / max(np.linalg.norm(rhs), 1e-300)))
    fsz = ls.plan_array("fp_fsz")
    extra = {"solve_transpose_ms": round(statistics.median(tt), 4),
             "max_relative_residual_transpose": max(rest)} if args.transpose else {}
    print(json.dumps({
        "n": int(n), "nnz": int(ci.size), "batch": B, "precision": args.precision, "fronts": int(fsz.size),
        "max_front": int(fsz.max()), "factor_level_tiers": ls.plan_array("factor_level_tiers").tolist(),
        "tc_threshold": int(ls.plan_array("tc_threshold")[0]),
        "factorize_ms": round(statistics.median(tf), 4), "solve_ms": round(statistics.median(ts), 4),
        "max_relative_residual": max(res), **extra, "singular": int(ls.singular_flags().sum())}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
