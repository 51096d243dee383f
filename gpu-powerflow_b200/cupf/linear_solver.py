"""Batched sparse direct solver: the phase API of custom_linear_solver::Solver
(custom_linear_solver/src/solver.hpp:67-114) over the cls_* C ABI.

    s = LinearSolver(SolverConfig(precision=CustomPrecision.FP64))
    s.set_data(row_ptr, col_idx)          # CSR pattern (host numpy or device tensor)
    s.analyze(); s.setup(batch)
    s.factorize(values)                   # CUDA tensor [batch, nnz] float64/float32
    x = s.solve(rhs)                      # CUDA tensor [batch, n]
    y = s.solve_transpose(rhs)            # A^T y = rhs on the same factors

Status codes become exceptions carrying StatusString (solver.cpp:214-232).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi


class SolverConfig:
    """SolverConfig (solver.hpp:35-65); precision uses CustomPrecision values."""

    def __init__(self, precision: int = 0, pivot_strategy: int = 1, serial_nd: bool = True,
                 max_panel_width: int = 8, shift_retry_epsilon: float = 1e-8, matching: int = 0,
                 autotune: bool = True, parallel_nd_depth: int = 4, parallel_nd_base_small: int = 4000,
                 parallel_nd_base_large: int = 20000, wide_min_front: int = 0, tc_min_front: int = 0,
                 batch1_schedule: int = 0):
        self.precision = int(precision)
        self.matching = int(matching)  # MatchingMode: 0 None, 1 Structural
        self.pivot_strategy = int(pivot_strategy)
        self.serial_nd = bool(serial_nd)
        self.max_panel_width = int(max_panel_width)
        self.shift_retry_epsilon = float(shift_retry_epsilon)
        self.autotune = bool(autotune)  # per-level factor launch shapes timed at the first factorization
        # separator recursion when serial_nd is False (SolverConfig::parallel_nd_*)
        self.parallel_nd_depth = int(parallel_nd_depth)
        self.parallel_nd_base_small = int(parallel_nd_base_small)
        self.parallel_nd_base_large = int(parallel_nd_base_large)
        # fronts from this size on: the any-size tier (0: 65), and with TF32 the
        # tensor-core trailing update (0: 65, or autotuned among 33, 49, 65)
        self.wide_min_front = int(wide_min_front)
        self.tc_min_front = int(tc_min_front)
        # a batch of one system: 0 one block per front (threads over its rows), 1 the batched lane kernels
        self.batch1_schedule = int(batch1_schedule)


class CustomSolverError(RuntimeError):
    def __init__(self, status: int, text: str, detail: str):
        super().__init__(f"custom solver {text}" + (f": {detail}" if detail else ""))
        self.status = status


class LinearSolver:
    def __init__(self, config: SolverConfig | None = None):
        self._lib = _capi.load()
        c = config or SolverConfig()
        cfg = _capi.ClsConfig(c.precision, c.matching, c.pivot_strategy, int(c.serial_nd), c.max_panel_width,
                              c.shift_retry_epsilon, int(c.autotune), c.parallel_nd_depth, c.parallel_nd_base_small,
                              c.parallel_nd_base_large, c.wide_min_front, c.tc_min_front, c.batch1_schedule)
        h = C.c_void_p()
        st = self._lib.cls_create(C.byref(cfg), C.byref(h))
        if st:
            raise CustomSolverError(st, self._lib.cls_status_string(st).decode(), "")
        self._h = h
        self.n = 0
        self.batch = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.cls_destroy(h)
            self._h = None

    def _check(self, st: int) -> None:
        if st:
            raise CustomSolverError(st, self._lib.cls_status_string(st).decode(),
                                    self._lib.cls_last_error(self._h).decode())

    def set_data(self, row_ptr, col_idx) -> None:
        try:
            import torch
            is_dev = isinstance(row_ptr, torch.Tensor) and row_ptr.is_cuda
        except ImportError:
            is_dev = False
        if is_dev:
            n = row_ptr.numel() - 1
            self._check(self._lib.cls_set_data(self._h, n, col_idx.numel(), row_ptr.data_ptr(), col_idx.data_ptr(), 1))
        else:
            rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
            ci = np.ascontiguousarray(col_idx, dtype=np.int32)
            n = rp.size - 1
            self._check(self._lib.cls_set_data(self._h, n, ci.size, rp.ctypes.data_as(C.c_void_p),
                                               ci.ctypes.data_as(C.c_void_p), 0))
        self.n = n

    def analyze(self) -> None:
        self._check(self._lib.cls_analyze(self._h))

    def analyze_host(self) -> None:
        """Symbolic analysis without device memory (plan introspection only)."""
        self._check(self._lib.cls_analyze_host(self._h))

    def setup(self, batch: int = 1) -> None:
        self._check(self._lib.cls_setup(self._h, batch))
        self.batch = batch

    def set_stream(self, stream) -> None:
        """cls_set_stream; 0 / None is the legacy default stream."""
        self._check(self._lib.cls_set_stream(self._h, C.c_void_p(int(stream or 0))))

    @staticmethod
    def _vt(t) -> int:
        import torch
        if t.dtype == torch.float64:
            return 0
        if t.dtype == torch.float32:
            return 1
        raise ValueError("values must be float64 or float32")

    def _bind_stream(self, t) -> None:
        """Run on torch's current stream of the tensor's device (ordered after
        the work that produced the inputs)."""
        import torch
        self.set_stream(torch.cuda.current_stream(t.device).cuda_stream)

    def factorize(self, values) -> None:
        self._bind_stream(values)
        self._check(self._lib.cls_factorize(self._h, values.data_ptr(), self._vt(values)))

    def factorize_static_scratch(self, values) -> None:
        """cls_factorize_static_scratch: same factorization, no device allocation
        in the call (needs a prior regular factorize at this batch size)."""
        self._bind_stream(values)
        self._check(self._lib.cls_factorize_static_scratch(self._h, values.data_ptr(), self._vt(values)))

    def solve(self, rhs, out=None, transpose: bool = False):
        import torch
        if out is None:
            out = torch.empty_like(rhs)
        fn = self._lib.cls_solve_transpose if transpose else self._lib.cls_solve
        self._bind_stream(rhs)
        self._check(fn(self._h, rhs.data_ptr(), self._vt(rhs), out.data_ptr(), self._vt(out)))
        return out

    def solve_transpose(self, rhs, out=None):
        return self.solve(rhs, out, transpose=True)

    def singular_flags(self) -> np.ndarray:
        out = np.zeros(self.batch, dtype=np.int32)
        self._check(self._lib.cls_singular_flags(self._h, out.ctypes.data_as(C.c_void_p), self.batch))
        return out

    def dump_fronts_csv(self, path) -> None:
        """Per-front structure of the analysed plan as CSV (the columns of
        SolverConfig::analyze_dump_fronts_path, solver.cpp:120)."""
        self._check(self._lib.cls_dump_fronts_csv(self._h, str(path).encode()))

    def plan_array(self, name: str) -> np.ndarray:
        ln = C.c_int64(0)
        self._check(self._lib.cls_plan_array(self._h, name.encode(), None, 0, C.byref(ln)))
        out = np.zeros(ln.value, dtype=np.int32)
        self._check(self._lib.cls_plan_array(self._h, name.encode(), out.ctypes.data_as(C.c_void_p), out.size,
                                             C.byref(ln)))
        return out
