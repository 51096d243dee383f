"""ctypes bindings for the test oracle (TEST INFRASTRUCTURE ONLY).

``Oracle``     -- this repository's C restatement of the reference's CPU FP64
                  Newton-Raphson path (oracle/pf_oracle.c, liboracle.so).
``Reference``  -- the reference's own CPU NewtonSolver and symbolic analysis
                  compiled from its sources (oracle/_ref/libcupf_ref.so), present
                  only where the reference sources were available at build time.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_ORACLE = HERE / "liboracle.so"
LIB_REF = HERE / "_ref" / "libcupf_ref.so"
# The reference checkout the oracle/_ref build and the live comparisons read:
# $CUPF_REFERENCE_ROOT, else a checkout named `reference` beside this repository.
REFERENCE_ROOT = Path(os.environ.get("CUPF_REFERENCE_ROOT") or (HERE.parent.parent / "reference"))

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    targets = ["oracle"] + (["ref", "refgpu"] if ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE), "-j8", *targets], check=True)


def _cplx(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).view(np.float64)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class _NRConfig(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iter", C.c_int32)]


class _NRResult(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("final_mismatch", C.c_double),
                ("converged", C.c_int32), ("status", C.c_int32)]


class Oracle:
    """The C restatement (pf_oracle.c)."""

    def __init__(self, path: Path = LIB_ORACLE):
        if not Path(path).exists():
            build(ref=False)
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.orc_jacobian_nnz.restype = C.c_int
        L.orc_jacobian_nnz.argtypes = [C.c_int, _i32p, _i32p, _i32p, C.c_int, _i32p, C.c_int, C.POINTER(C.c_int)]
        L.orc_jacobian_analysis.restype = C.c_int
        L.orc_jacobian_analysis.argtypes = [C.c_int, _i32p, _i32p, _i32p, C.c_int, _i32p, C.c_int,
                                            _i32p, _i32p] + [_i32p] * 8
        L.orc_nr_solve.restype = C.c_int
        L.orc_nr_solve.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _i32p, C.c_int, _i32p, C.c_int,
                                   _NRConfig, _f64p, C.POINTER(_NRResult)]
        L.orc_adjoint.restype = C.c_double
        L.orc_adjoint.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _i32p, C.c_int, _i32p, C.c_int,
                                  _f64p, _f64p, _f64p, _f64p, _f64p]
        L.orc_mismatch.restype = C.c_double
        L.orc_mismatch.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _i32p, C.c_int, _i32p, C.c_int, _f64p]
        L.orc_jacobian_values.restype = C.c_int
        L.orc_jacobian_values.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _i32p, C.c_int, _i32p, C.c_int, _f64p]
        L.orc_nr_solve_many.restype = C.c_int
        L.orc_nr_solve_many.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int, _i32p, C.c_int,
                                        _i32p, C.c_int, _NRConfig, C.c_int, _f64p, _i32p, _f64p]
        L.orc_nd_order.restype = C.c_int
        L.orc_nd_order.argtypes = [C.c_int, _i32p, _i32p, _i32p]

    # -- analysis --
    def jacobian_analysis(self, g) -> dict:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        nnz = C.c_int(0)
        dim = self.lib.orc_jacobian_nnz(g.n_bus, ip, ix, pv, pv.size, pq, pq.size, C.byref(nnz))
        if dim <= 0:
            raise ValueError("invalid pv/pq for Jacobian analysis")
        out = {"row_ptr": np.zeros(dim + 1, np.int32), "col_idx": np.zeros(nnz.value, np.int32)}
        for k in ("map11", "map21", "map12", "map22"):
            out[k] = np.zeros(ix.size, np.int32)
        for k in ("diag11", "diag21", "diag12", "diag22"):
            out[k] = np.zeros(g.n_bus, np.int32)
        self.lib.orc_jacobian_analysis(g.n_bus, ip, ix, pv, pv.size, pq, pq.size, out["row_ptr"], out["col_idx"],
                                       out["map11"], out["map21"], out["map12"], out["map22"],
                                       out["diag11"], out["diag21"], out["diag12"], out["diag22"])
        return out

    # -- NR --
    def solve(self, g, sbus, v0, tol: float = 1e-8, max_iter: int = 50) -> dict:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        v = np.zeros(2 * g.n_bus)
        r = _NRResult()
        self.lib.orc_nr_solve(g.n_bus, ip, ix, _cplx(g.data), _cplx(sbus), _cplx(v0), pv, pv.size, pq, pq.size,
                              _NRConfig(tol, max_iter), v, C.byref(r))
        return {"V": v.view(np.complex128).copy(), "iterations": r.iterations,
                "final_mismatch": r.final_mismatch, "converged": bool(r.converged), "status": r.status}

    def solve_many(self, g, sbus, v0, tol: float = 1e-8, max_iter: int = 50, threads: int = 1) -> dict:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        sbus = np.ascontiguousarray(sbus, dtype=np.complex128)
        v0 = np.ascontiguousarray(v0, dtype=np.complex128)
        b = sbus.shape[0]
        v = np.zeros(2 * g.n_bus * b)
        its = np.zeros(b, np.int32)
        fm = np.zeros(b)
        self.lib.orc_nr_solve_many(g.n_bus, ip, ix, _cplx(g.data), sbus.reshape(-1).view(np.float64),
                                   v0.reshape(-1).view(np.float64), b, pv, pv.size, pq, pq.size,
                                   _NRConfig(tol, max_iter), threads, v, its, fm)
        return {"V": v.view(np.complex128).reshape(b, g.n_bus), "iterations": its, "final_mismatch": fm}

    def mismatch(self, g, sbus, v) -> tuple[np.ndarray, float]:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        F = np.zeros(g.dim_f)
        nrm = self.lib.orc_mismatch(g.n_bus, ip, ix, _cplx(g.data), _cplx(sbus), _cplx(v), pv, pv.size, pq,
                                    pq.size, F)
        return F, nrm

    def jacobian_values(self, g, v) -> np.ndarray:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        nnz = C.c_int(0)
        self.lib.orc_jacobian_nnz(g.n_bus, ip, ix, pv, pv.size, pq, pq.size, C.byref(nnz))
        out = np.zeros(nnz.value)
        self.lib.orc_jacobian_values(g.n_bus, ip, ix, _cplx(g.data), _cplx(v), pv, pv.size, pq, pq.size, out)
        return out

    def adjoint(self, g, v, grad_va, grad_vm) -> dict:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        lam = np.zeros(g.dim_f)
        gp = np.zeros(g.n_bus)
        gq = np.zeros(g.n_bus)
        res = self.lib.orc_adjoint(g.n_bus, ip, ix, _cplx(g.data), _cplx(v), pv, pv.size, pq, pq.size,
                                   np.ascontiguousarray(grad_va, np.float64), np.ascontiguousarray(grad_vm, np.float64),
                                   lam, gp, gq)
        return {"lambda": lam, "grad_p": gp, "grad_q": gq, "residual": res}


class Reference:
    """The reference's own CPU NewtonSolver + symbolic analysis (oracle/_ref)."""

    def __init__(self, path: Path = LIB_REF):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (reference sources absent at build time)")
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.ref_last_error.restype = C.c_char_p
        L.ref_nr_solve.restype = C.c_int
        L.ref_nr_solve.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _i32p, C.c_int, _i32p, C.c_int,
                                   C.c_double, C.c_int, _f64p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                   C.POINTER(C.c_int32)]
        L.ref_nr_adjoint.restype = C.c_int
        L.ref_nr_adjoint.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _i32p, C.c_int, _i32p, C.c_int,
                                     C.c_double, C.c_int, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                     C.POINTER(C.c_double)]
        L.ref_jacobian_analysis.restype = C.c_int
        L.ref_jacobian_analysis.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p, C.c_int, _i32p, C.c_int,
                                            C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p, C.c_void_p,
                                            C.c_void_p]
        L.ref_nr_solve_many.restype = C.c_int
        L.ref_nr_solve_many.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int, _i32p, C.c_int, _i32p,
                                        C.c_int, C.c_double, C.c_int, C.c_int, _f64p, _i32p, _f64p]
        L.ref_symbolic_run.restype = C.c_void_p
        L.ref_symbolic_run.argtypes = [C.c_int, _i32p, _i32p, C.c_int, C.c_int, C.c_int]
        L.ref_symbolic_run_m.restype = C.c_void_p
        L.ref_symbolic_run_m.argtypes = [C.c_int, _i32p, _i32p, C.c_int, C.c_int, C.c_int, C.c_int]
        L.ref_symbolic_run_p.restype = C.c_void_p
        L.ref_symbolic_run_p.argtypes = [C.c_int, _i32p, _i32p] + [C.c_int] * 7
        L.ref_symbolic_len.restype = C.c_int
        L.ref_symbolic_len.argtypes = [C.c_void_p, C.c_char_p]
        L.ref_symbolic_copy.restype = C.c_int
        L.ref_symbolic_copy.argtypes = [C.c_void_p, C.c_char_p, _i32p]
        L.ref_symbolic_names.restype = C.c_int
        L.ref_symbolic_names.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.ref_symbolic_free.restype = None
        L.ref_symbolic_free.argtypes = [C.c_void_p]
        L.ref_symbolic_text.restype = C.c_int
        L.ref_symbolic_text.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int]
        L.ref_load_dump_case.restype = C.c_int
        L.ref_load_dump_case.argtypes = [C.c_char_p] + [C.POINTER(C.c_int32)] * 4 + [C.c_void_p] * 7

    def _err(self, rc: int) -> None:
        if rc:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def solve(self, g, sbus, v0, tol: float = 1e-8, max_iter: int = 50) -> dict:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        v = np.zeros(2 * g.n_bus)
        it, fm, cv = C.c_int32(0), C.c_double(0), C.c_int32(0)
        self._err(self.lib.ref_nr_solve(g.n_bus, ip, ix, _cplx(g.data), _cplx(sbus), _cplx(v0), pv, pv.size, pq,
                                        pq.size, tol, max_iter, v, C.byref(it), C.byref(fm), C.byref(cv)))
        return {"V": v.view(np.complex128).copy(), "iterations": it.value, "final_mismatch": fm.value,
                "converged": bool(cv.value)}

    def solve_many(self, g, sbus, v0, tol: float = 1e-8, max_iter: int = 50, threads: int = 1) -> dict:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        sbus = np.ascontiguousarray(sbus, dtype=np.complex128)
        v0 = np.ascontiguousarray(v0, dtype=np.complex128)
        b = sbus.shape[0]
        v = np.zeros(2 * g.n_bus * b)
        its = np.zeros(b, np.int32)
        fm = np.zeros(b)
        self._err(self.lib.ref_nr_solve_many(g.n_bus, ip, ix, _cplx(g.data), sbus.reshape(-1).view(np.float64),
                                             v0.reshape(-1).view(np.float64), b, pv, pv.size, pq, pq.size, tol,
                                             max_iter, threads, v, its, fm))
        return {"V": v.view(np.complex128).reshape(b, g.n_bus), "iterations": its, "final_mismatch": fm}

    def adjoint(self, g, sbus, v0, grad_va, grad_vm, tol: float = 1e-8, max_iter: int = 50) -> dict:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        v = np.zeros(2 * g.n_bus)
        lam, gp, gq = np.zeros(g.dim_f), np.zeros(g.n_bus), np.zeros(g.n_bus)
        res = C.c_double(0)
        self._err(self.lib.ref_nr_adjoint(g.n_bus, ip, ix, _cplx(g.data), _cplx(sbus), _cplx(v0), pv, pv.size, pq,
                                          pq.size, tol, max_iter, np.ascontiguousarray(grad_va, np.float64),
                                          np.ascontiguousarray(grad_vm, np.float64), v, lam, gp, gq, C.byref(res)))
        return {"V": v.view(np.complex128).copy(), "lambda": lam, "grad_p": gp, "grad_q": gq,
                "residual": res.value}

    def jacobian_analysis(self, g) -> dict:
        ip, ix, pv, pq = _i32(g.indptr), _i32(g.indices), _i32(g.pv), _i32(g.pq)
        dim, nnz = C.c_int32(0), C.c_int32(0)
        self._err(self.lib.ref_jacobian_analysis(g.n_bus, ip, ix, _cplx(g.data), pv, pv.size, pq, pq.size,
                                                 C.byref(dim), C.byref(nnz), None, None, None))
        rp = np.zeros(dim.value + 1, np.int32)
        ci = np.zeros(nnz.value, np.int32)
        maps = np.zeros(4 * ix.size + 4 * g.n_bus, np.int32)
        self._err(self.lib.ref_jacobian_analysis(g.n_bus, ip, ix, _cplx(g.data), pv, pv.size, pq, pq.size,
                                                 C.byref(dim), C.byref(nnz), rp.ctypes.data, ci.ctypes.data,
                                                 maps.ctypes.data))
        m = ix.size
        out = {"row_ptr": rp, "col_idx": ci}
        for i, k in enumerate(("map11", "map21", "map12", "map22")):
            out[k] = maps[i * m:(i + 1) * m].copy()
        base = 4 * m
        for i, k in enumerate(("diag11", "diag21", "diag12", "diag22")):
            out[k] = maps[base + i * g.n_bus: base + (i + 1) * g.n_bus].copy()
        return out

    def symbolic(self, row_ptr, col_idx, max_panel_width: int = 8, parallel_nd: bool = False,
                 float_front: bool = True, use_matching: bool = False, nd_depth: int = 4,
                 nd_base_small: int = 4000, nd_base_large: int = 20000) -> dict:
        """The reference's symbolic analysis; nd_* are SolverConfig's
        parallel_nd_depth / parallel_nd_base_small / parallel_nd_base_large."""
        rp, ci = _i32(row_ptr), _i32(col_idx)
        n = rp.size - 1
        h = self.lib.ref_symbolic_run_p(n, rp, ci, max_panel_width, int(parallel_nd), int(float_front),
                                        int(use_matching), nd_depth, nd_base_small, nd_base_large)
        if not h:
            raise RuntimeError("reference symbolic analysis failed")
        try:
            buf = C.create_string_buffer(1 << 16)
            self.lib.ref_symbolic_names(h, buf, len(buf))
            names = [x for x in buf.value.decode().split(",") if x]
            out = {}
            for nm in names:
                ln = self.lib.ref_symbolic_len(h, nm.encode())
                a = np.zeros(max(ln, 0), np.int32)
                if ln > 0:
                    self.lib.ref_symbolic_copy(h, nm.encode(), a)
                out[nm] = a
            # the reference's own front CSVs (MaybeDumpFronts): the
            # analyze_fronts_only order and the full analysis's order
            for nm in ("fronts_csv_level", "fronts_csv_full"):
                ln = self.lib.ref_symbolic_text(h, nm.encode(), None, 0)
                if ln >= 0:
                    tb = C.create_string_buffer(ln + 1)
                    self.lib.ref_symbolic_text(h, nm.encode(), tb, ln + 1)
                    out[nm] = tb.value.decode()
            return out
        finally:
            self.lib.ref_symbolic_free(h)


    def load_dump_case(self, case_dir) -> dict:
        """cupf::tests::load_dump_case (cuPF/tests/dump_case_loader.cpp:210-232)."""
        rows, nnz, npv, npq = (C.c_int32(0) for _ in range(4))
        d = str(case_dir).encode()
        self._err(self.lib.ref_load_dump_case(d, C.byref(rows), C.byref(nnz), C.byref(npv), C.byref(npq),
                                              *([None] * 7)))
        n = rows.value
        out = {"indptr": np.zeros(n + 1, np.int32), "indices": np.zeros(nnz.value, np.int32),
               "ybus_data": np.zeros(nnz.value, np.complex128), "sbus": np.zeros(n, np.complex128),
               "v0": np.zeros(n, np.complex128), "pv": np.zeros(npv.value, np.int32),
               "pq": np.zeros(npq.value, np.int32)}
        keys = ("indptr", "indices", "ybus_data", "sbus", "v0", "pv", "pq")
        self._err(self.lib.ref_load_dump_case(d, C.byref(rows), C.byref(nnz), C.byref(npv), C.byref(npq),
                                              *[out[k].ctypes.data for k in keys]))
        out["rows"] = n
        return out


def reference_available() -> bool:
    return LIB_REF.exists() and os.environ.get("CUPF_NO_REF_ORACLE") != "1"
