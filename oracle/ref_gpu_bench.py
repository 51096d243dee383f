"""The reference's own GPU linear solver beside this engine's, on one GPU
(TEST INFRASTRUCTURE ONLY: a timing comparison; the engine never calls it).

    python -m oracle.ref_gpu_bench [--batch 1024] [--reps 10]

Both factor and solve the same batch of Newton Jacobians of the synthetic
2,000-bus grid (the Jacobian at the nominal solution, system b scaled by
1 + 1e-3 b) with the same serial nested-dissection ordering, in FP32 and in
FP64.  The reference is custom_linear_solver built from its sources
(oracle/_ref/libcls_refgpu.so, compute_86 PTX JIT-compiled for this GPU, its
standalone mode with internal CUDA graphs); the engine is the cls_* C ABI.
Each side is timed per Factorize + Solve pair with host timers around
synchronized calls (the reference synchronizes inside its calls), median of
--reps after 2 warm-up pairs, and the largest relative residual of its
solutions is reported.  Prints one JSON object; exits non-zero when the
reference library is missing or fails.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import statistics
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libcls_refgpu.so"


def _load():
    lib = C.CDLL(str(LIB))
    lib.rg_create.restype = C.c_void_p
    lib.rg_create.argtypes = [C.c_int, C.c_int]
    lib.rg_destroy.argtypes = [C.c_void_p]
    lib.rg_setup.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                             C.c_int, C.c_void_p, C.c_int, C.c_int]
    lib.rg_factorize.argtypes = [C.c_void_p]
    lib.rg_solve.argtypes = [C.c_void_p]
    lib.rg_last_error.restype = C.c_char_p
    return lib


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--reps", type=int, default=10)
    args = ap.parse_args(argv)
    root = HERE.parent
    for p in (root / "gpu-powerflow_b200", root):
        if str(p) not in sys.path:
            sys.path.insert(0, str(p))
    import scipy.sparse as sp
    import torch

    import cupf
    from cupf import grids
    from oracle.oracle import Oracle

    if not LIB.exists():
        print(json.dumps({"unavailable": "oracle/_ref/libcls_refgpu.so was not built (reference sources absent)"}))
        return 1
    lib = _load()
    g = grids.grid_2000()
    orc = Oracle()
    V = orc.solve(g, g.sbus, g.v0, tol=1e-12, max_iter=30)["V"]
    J1 = orc.jacobian_values(g, V)
    s = cupf.NewtonSolver(_opts(cupf))
    s.analyze_host(g.indptr, g.indices, g.n_bus, g.pv, g.pq)
    rp, ci = s.plan_array("jac_row_ptr"), s.plan_array("jac_col_idx")
    n, nnz, B = rp.size - 1, ci.size, args.batch
    vals = J1[None, :] * (1.0 + 1e-3 * np.arange(B)[:, None])
    rhs = np.random.default_rng(7).standard_normal((B, n))
    dev = torch.device("cuda")
    d_rp = torch.tensor(rp, device=dev)
    d_ci = torch.tensor(ci, device=dev)
    out = {"workload": f"2,000-bus Newton Jacobian (n {n}, nnz {nnz}) x {B} systems, serial nested dissection",
           "timing": "median Factorize+Solve pair, synchronized host timers", "reps": args.reps}
    for prec, name, dt in ((1, "fp32", torch.float32), (0, "fp64", torch.float64)):
        d_vals = torch.tensor(vals, dtype=dt, device=dev)
        d_rhs = torch.tensor(rhs, dtype=torch.float64, device=dev)
        d_x = torch.zeros(B, n, dtype=torch.float64, device=dev)
        # the reference
        h = lib.rg_create(prec, 1)
        if not h:
            raise RuntimeError("rg_create: " + lib.rg_last_error().decode())
        rc = lib.rg_setup(h, n, nnz, d_rp.data_ptr(), d_ci.data_ptr(), d_vals.data_ptr(), int(prec == 1),
                          d_rhs.data_ptr(), 0, d_x.data_ptr(), 0, B)
        if rc:
            raise RuntimeError("reference setup: " + lib.rg_last_error().decode())

        def ref_pair():
            if lib.rg_factorize(h) or lib.rg_solve(h):
                raise RuntimeError("reference: " + lib.rg_last_error().decode())
        t_ref = _time(ref_pair, args.reps)
        x_ref = d_x.cpu().numpy()
        lib.rg_destroy(h)
        # the engine
        ls = cupf.LinearSolver(cupf.SolverConfig(precision=prec, serial_nd=True))
        ls.set_data(rp, ci)
        ls.analyze()
        ls.setup(B)
        x_ours = [None]

        def our_pair():
            ls.factorize(d_vals)
            x_ours[0] = ls.solve(d_rhs)
        t_ours = _time(our_pair, args.reps)
        res = {}
        for who, x in (("reference", x_ref), ("engine", x_ours[0].cpu().numpy())):
            r = 0.0
            for b in range(0, B, max(1, B // 16)):
                A = sp.csr_matrix((vals[b], ci, rp), shape=(n, n))
                r = max(r, float(np.linalg.norm(A @ x[b] - rhs[b]) / np.linalg.norm(rhs[b])))
            res[who] = r
        out[name] = {"reference_ms": round(t_ref, 4), "engine_ms": round(t_ours, 4),
                     "speedup": round(t_ref / t_ours, 2),
                     "max_relative_residual": res, "systems_checked": len(range(0, B, max(1, B // 16)))}
    print(json.dumps(out))
    return 0


def _opts(cupf):
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    return o


def _time(fn, reps: int) -> float:
    import torch

    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        ts.append((time.perf_counter() - t0) * 1e3)
    return statistics.median(ts)


if __name__ == "__main__":
    raise SystemExit(main())
