"""cuPF-compatible Python API of the B200 batched Newton-Raphson power-flow engine.

Same names, fields, defaults and argument meaning as the reference's ``cupf``
package and its ``_cupf`` pybind module (cuPF/python/cupf/__init__.py,
cuPF/bindings/pybind_cupf.cpp:162-657), so code written against
``cupf.NewtonSolver`` with the CUDA backend runs unchanged.  Underneath is the
C ABI of include/cupf_b200.h (libcupf_b200.so), reached through ctypes.

Differences a user can see:
  * only ``BackendKind.CUDA`` with ``CudaLinearSolverKind.Custom`` is provided
    (the CPU/KLU and cuDSS backends are other libraries); constructing a
    solver with another backend raises ``ValueError``;
  * ``ComputePolicy.FP32`` keeps V, Sbus, Ibus, the mismatch and the
    voltage update in FP32 along with the Jacobian and the factors (an FP64
    factor precision falls back to FP32, as in the reference); its mismatch
    floor is about 1e-5 pu on 100-2,000-bus grids, so tolerances below that
    do not converge.  The adjoint raises under it (its FP64 residual
    refinement needs FP64 state); ``ComputePolicy.Mixed`` keeps the state in
    FP64 with FP32 factors;
  * ``CustomSolverConfig.max_panel_width`` is limited to 1..8;
  * ``CustomSolverConfig.autotune`` (not in the reference, on by default)
    times each factor level's block shape at the first solve of a batch size
    and keeps the fastest; the results do not depend on it;
  * ``CustomSolverConfig.wide_min_front`` and ``tc_min_front`` (not in the
    reference) set where the any-size front tier (default 65 rows) and, with
    ``CustomPrecision.TF32``, the tensor-core trailing update (default 65
    rows, autotuned among 33, 49 and 65) take over;
  * ``CustomSolverConfig.batch1_schedule`` (not in the reference's config;
    its solver picks its single-system path by itself at batch 1): 0 (the
    default) factors a batch of one system with one block per front and its
    threads over the front's rows, 1 with the batched lane kernels; the
    factors are the same.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum
from typing import Any

import numpy as np

from . import _capi

# ---------------------------------------------------------------------------
# Enums (newton_solver_types.hpp:55-150; pybind_cupf.cpp:167-240)
# ---------------------------------------------------------------------------


class BackendKind(IntEnum):
    CPU = 0
    CUDA = 1


class ComputePolicy(IntEnum):
    FP64 = 0
    FP32 = 1
    Mixed = 2


class CudaLinearSolverKind(IntEnum):
    CuDSS = 0
    Custom = 1


class CustomPrecision(IntEnum):
    FP64 = 0
    FP32 = 1
    TF32 = 2


CustomMatchingMode = IntEnum("CustomMatchingMode", [("None", 0), ("Structural", 1)])
CustomPivotStrategy = IntEnum("CustomPivotStrategy", [("None", 0), ("StaticDiagonalShift", 1)])


class CpuLinearSolverKind(IntEnum):
    KLU = 0
    UMFPACK = 1


class CudaJacobianKind(IntEnum):
    Edge = 0
    EdgeAtomic = 1
    VertexWarp = 2


AdjointCacheMode = IntEnum("AdjointCacheMode", [("None", 0), ("FinalStateFactorization", 1),
                                                 ("ReuseLastNewtonFactorizationIfExact", 2)])


class CuDSSAlgorithm(IntEnum):
    DEFAULT = 0
    ALG_1 = 1
    ALG_2 = 2
    ALG_3 = 3
    ALG_4 = 4
    ALG_5 = 5


# ---------------------------------------------------------------------------
# Option / config structs (defaults as newton_solver_types.hpp)
# ---------------------------------------------------------------------------


class _Struct:
    _fields: dict[str, Any] = {}

    def __init__(self, **kw):
        for k, v in self._fields.items():
            setattr(self, k, v() if callable(v) and not isinstance(v, IntEnum) else v)
        for k, v in kw.items():
            if k not in self._fields:
                raise AttributeError(f"{type(self).__name__} has no field {k!r}")
            setattr(self, k, v)

    def __repr__(self) -> str:
        return f"{type(self).__name__}(" + ", ".join(f"{k}={getattr(self, k)!r}" for k in self._fields) + ")"


class NRConfig(_Struct):
    """Newton-Raphson stopping rule: ||F||_inf <= tolerance within max_iter."""
    _fields = {"tolerance": 1e-8, "max_iter": 50}


class CuDSSOptions(_Struct):
    _fields = {"use_matching": False, "matching_alg": CuDSSAlgorithm.DEFAULT, "auto_pivot_epsilon": True,
               "pivot_epsilon": 0.0}


class CustomSolverConfig(_Struct):
    _fields = {"precision": CustomPrecision.FP32, "matching": CustomMatchingMode["None"],
               "pivot_strategy": CustomPivotStrategy.StaticDiagonalShift, "serial_nd": False,
               "max_panel_width": 8, "shift_retry_epsilon": 1.0e-8, "autotune": True,
               "parallel_nd_depth": 4, "parallel_nd_base_small": 4000, "parallel_nd_base_large": 20000,
               "wide_min_front": 0, "tc_min_front": 0, "batch1_schedule": 0}


class NewtonOptions(_Struct):
    _fields = {"backend": BackendKind.CPU, "compute": ComputePolicy.Mixed,
               "cpu_linear_solver": CpuLinearSolverKind.KLU, "cuda_jacobian": CudaJacobianKind.Edge,
               "cuda_linear_solver": CudaLinearSolverKind.Custom, "cudss": CuDSSOptions,
               "custom": CustomSolverConfig, "use_cuda_graph": False}


class SolveOptions(_Struct):
    _fields = {"prepare_adjoint_cache": False,
               "adjoint_cache_mode": AdjointCacheMode.FinalStateFactorization,
               "allow_explicit_transpose_fallback": False}


class AdjointOptions(_Struct):
    _fields = {"reuse_forward_factorization": False, "allow_refactorize": True,
               "require_cached_factorization": False, "allow_refactorize_for_backward": True,
               "allow_inexact_last_newton_factorization": False, "use_transpose_solve": True,
               "allow_explicit_transpose_fallback": False, "compute_load_gradients": True,
               "check_residual": True}


# ---------------------------------------------------------------------------
# Results (newton_solver_types.hpp:198-290)
# ---------------------------------------------------------------------------


class NRResult:
    def __init__(self, V, iterations, final_mismatch, converged):
        self.V_numpy = np.asarray(V, dtype=np.complex128)
        self.iterations = int(iterations)
        self.final_mismatch = float(final_mismatch)
        self.converged = bool(converged)

    @property
    def V(self) -> list:
        return self.V_numpy.tolist()


class NRBatchResult:
    def __init__(self, V, n_bus, batch_size, iterations, final_mismatch, converged):
        self.V_numpy = V
        self.n_bus = int(n_bus)
        self.batch_size = int(batch_size)
        self.iterations_numpy = iterations
        self.final_mismatch_numpy = final_mismatch
        self.converged_numpy = converged

    @property
    def V(self) -> list:
        return self.V_numpy.reshape(-1).tolist()

    @property
    def iterations(self) -> list:
        return self.iterations_numpy.tolist()

    @property
    def final_mismatch(self) -> list:
        return self.final_mismatch_numpy.tolist()

    @property
    def converged(self) -> list:
        return self.converged_numpy.tolist()


class AdjointResult:
    sign_convention = "F=S_calc-S_spec; load increase decreases Sbus; grad_load=-lambda"

    def __init__(self, raw: _capi.PfAdjointResult, lam=None, grad_p=None, grad_q=None, backend="cuda_custom",
                 zero_copy=False):
        self.n_bus = raw.n_bus
        self.batch_size = raw.batch_size
        self.dimF = raw.dim_f
        self.success = bool(raw.success)
        self.used_adjoint_cache = bool(raw.used_adjoint_cache)
        self.adjoint_cache_matches_final_state = bool(raw.used_adjoint_cache)
        self.reused_forward_factorization = False
        self.reused_final_state_factorization = bool(raw.reused_final_state_factorization)
        self.refactorized_for_backward = bool(raw.refactorized_for_backward)
        self.used_explicit_transpose = False
        self.used_python_scipy = False
        self.includes_host_device_transfer = not zero_copy
        self.zero_copy = zero_copy
        self.torch_extension_zero_copy = zero_copy
        self.raw_pointer_api_used = False
        self.current_stream_integrated = zero_copy
        self.jt_symbolic_analyzed_at_initialize = True
        self.jt_values_transposed_on_device = False
        self.jt_factorized_during_forward_cache = True
        self.jt_refactorized_during_backward = False
        self.host_roundtrip_for_jt_transpose = False
        self.jt_residual_norm = raw.jt_residual_norm
        self.solve_time_ms = 0.0
        self.transpose_solve_time_ms = 0.0
        self.factorization_time_ms = 0.0
        self.total_time_ms = 0.0
        self.backend = backend
        self.transpose_solve_backend = "cuda_custom_multifrontal_transpose_sweeps"
        self.iterations = raw.iterations
        self.max_final_mismatch = raw.max_final_mismatch
        self.all_converged = bool(raw.all_converged)
        self.lambda_numpy = lam
        self.grad_load_p_numpy = grad_p
        self.grad_load_q_numpy = grad_q

    @property
    def lambda_(self) -> list:
        return [] if self.lambda_numpy is None else self.lambda_numpy.reshape(-1).tolist()

    @property
    def grad_load_p(self) -> list:
        return [] if self.grad_load_p_numpy is None else self.grad_load_p_numpy.reshape(-1).tolist()

    @property
    def grad_load_q(self) -> list:
        return [] if self.grad_load_q_numpy is None else self.grad_load_q_numpy.reshape(-1).tolist()


# ---------------------------------------------------------------------------
# NewtonSolver
# ---------------------------------------------------------------------------


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.int32)


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.complex128)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a.size else None


def _check(lib, h, st: int) -> None:
    if st == 0:
        return
    msg = lib.pf_last_error(h).decode(errors="replace")
    if st == 1:
        raise ValueError(msg)
    raise RuntimeError(msg)


def _cls_config(c: CustomSolverConfig) -> _capi.ClsConfig:
    return _capi.ClsConfig(int(c.precision), int(c.matching), int(c.pivot_strategy), int(bool(c.serial_nd)),
                           int(c.max_panel_width), float(c.shift_retry_epsilon), int(bool(c.autotune)),
                           int(c.parallel_nd_depth), int(c.parallel_nd_base_small), int(c.parallel_nd_base_large),
                           int(c.wide_min_front), int(c.tc_min_front), int(c.batch1_schedule))


def _nr_config(cfg: NRConfig | None) -> _capi.PfNRConfig:
    cfg = cfg or NRConfig()
    return _capi.PfNRConfig(float(cfg.tolerance), int(cfg.max_iter))


def _solve_options(so: SolveOptions | None) -> _capi.PfSolveOptions:
    so = so or SolveOptions()
    return _capi.PfSolveOptions(int(bool(so.prepare_adjoint_cache)), int(so.adjoint_cache_mode),
                                int(bool(so.allow_explicit_transpose_fallback)))


def _adjoint_options(o: AdjointOptions | None) -> _capi.PfAdjointOptions:
    o = o or AdjointOptions()
    return _capi.PfAdjointOptions(*[int(bool(getattr(o, f[0]))) for f in _capi.PfAdjointOptions._fields_])


class NewtonSolver:
    """Batched Newton-Raphson power-flow solver (NewtonSolver, newton_solver.hpp:26-102)."""

    def __init__(self, options: NewtonOptions | None = None):
        self._lib = _capi.load()
        self.options = options or NewtonOptions()
        o = self.options
        if o.backend != BackendKind.CUDA:
            raise ValueError("NewtonSolver: this engine provides BackendKind.CUDA only "
                             "(the reference's CPU/KLU backend is a different library)")
        if o.cuda_linear_solver != CudaLinearSolverKind.Custom:
            raise ValueError("NewtonSolver: this engine provides CudaLinearSolverKind.Custom only")
        po = _capi.PfOptions(int(o.backend), int(o.compute), int(o.cuda_linear_solver), int(o.cuda_jacobian),
                             _cls_config(o.custom), int(bool(o.use_cuda_graph)))
        h = C.c_void_p()
        st = self._lib.pf_create(C.byref(po), C.byref(h))
        self._h = h
        if st != 0:
            msg = self._lib.pf_last_error(h).decode() if h else "pf_create failed"
            if h:
                self._lib.pf_destroy(h)
                self._h = None
            raise ValueError(msg) if st == 1 else RuntimeError(msg)
        self._n_bus = 0
        self._batch = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.pf_destroy(h)
            self._h = None

    @property
    def dtype_name(self) -> str:
        return "float64" if self.options.compute == ComputePolicy.FP64 else "float32"

    # -- initialize --
    def initialize(self, indptr, indices, data, rows, cols, pv, pq) -> None:
        ip, ix, dt = _i32(indptr), _i32(indices), _c128(data)
        pv, pq = _i32(pv), _i32(pq)
        if rows <= 0 or cols <= 0:
            raise ValueError("Ybus rows/cols must be positive")
        if ip.ndim != 1 or ix.ndim != 1 or dt.ndim != 1:
            raise ValueError("Ybus indptr, indices, and data must be 1D arrays")
        if ip.size != rows + 1:
            raise ValueError("Ybus indptr length must be rows + 1")
        if ix.size != dt.size:
            raise ValueError("Ybus indices and data must have the same length")
        _check(self._lib, self._h, self._lib.pf_initialize(self._h, _ptr(ip), _ptr(ix), _ptr(dt), rows, cols, dt.size,
                                                           _ptr(pv), pv.size, _ptr(pq), pq.size))
        self._n_bus = rows

    def analyze_host(self, indptr, indices, rows, pv, pq) -> None:
        """Analysis only (no GPU needed): fills plan_array() / info()."""
        ip, ix, pv, pq = _i32(indptr), _i32(indices), _i32(pv), _i32(pq)
        _check(self._lib, self._h, self._lib.pf_analyze_host(self._h, _ptr(ip), _ptr(ix), rows, ix.size, _ptr(pv),
                                                             pv.size, _ptr(pq), pq.size))

    # -- forward --
    def solve(self, indptr, indices, data, rows, cols, sbus, v0, pv, pq, config=None, solve_options=None) -> NRResult:
        sbus, v0 = _c128(sbus), _c128(v0)
        if sbus.ndim != 1 or v0.ndim != 1:
            raise ValueError("sbus and v0 must be 1D arrays for solve()")
        if sbus.size != rows or v0.size != rows:
            raise ValueError("sbus/v0 length must match Ybus rows")
        r = self.solve_batch(indptr, indices, data, rows, cols, sbus[None, :], v0[None, :], pv, pq, config,
                             solve_options)
        return NRResult(r.V_numpy[0], r.iterations_numpy[0], r.final_mismatch_numpy[0], r.converged_numpy[0])

    def solve_batch(self, indptr, indices, data, rows, cols, sbus, v0, pv, pq, config=None,
                    solve_options=None) -> NRBatchResult:
        sbus, v0 = _c128(sbus), _c128(v0)
        if sbus.ndim != 2 or v0.ndim != 2:
            raise ValueError("sbus and v0 must be 2D arrays [batch, n_bus] for solve_batch()")
        if sbus.shape[0] != v0.shape[0] or sbus.shape[1] != rows or v0.shape[1] != rows:
            raise ValueError("sbus/v0 shape must be [batch, rows]")
        ip, ix, dt, pv, pq = _i32(indptr), _i32(indices), _c128(data), _i32(pv), _i32(pq)
        B = sbus.shape[0]
        V = np.zeros((B, rows), dtype=np.complex128)
        its = np.zeros(B, dtype=np.int32)
        fm = np.zeros(B, dtype=np.float64)
        cv = np.zeros(B, dtype=np.uint8)
        cfg, so = _nr_config(config), _solve_options(solve_options)
        if dt.ndim == 2:
            # per-scenario Ybus values [batch, nnz] on the initialized pattern
            if dt.shape[0] != B or dt.shape[1] != ix.size:
                raise ValueError("per-scenario Ybus data must be [batch, nnz]")
            _check(self._lib, self._h, self._lib.pf_solve_batch_ybus(
                self._h, _ptr(dt), dt.shape[1], _ptr(sbus), rows, _ptr(v0), rows, B, C.byref(cfg), C.byref(so),
                _ptr(V), _ptr(its), _ptr(fm), _ptr(cv)))
            self._batch = B
            return NRBatchResult(V, rows, B, its, fm, cv)
        _check(self._lib, self._h, self._lib.pf_solve_batch(
            self._h, _ptr(ip), _ptr(ix), _ptr(dt), rows, cols, dt.size, _ptr(sbus), rows, _ptr(v0), rows, B,
            _ptr(pv), pv.size, _ptr(pq), pq.size, C.byref(cfg), C.byref(so), _ptr(V), _ptr(its), _ptr(fm), _ptr(cv)))
        self._batch = B
        return NRBatchResult(V, rows, B, its, fm, cv)

    # -- backward (host) --
    def solve_adjoint(self, grad_va, grad_vm, pv, pq, options=None) -> AdjointResult:
        ga = np.ascontiguousarray(grad_va, dtype=np.float64)
        gm = np.ascontiguousarray(grad_vm, dtype=np.float64)
        if ga.ndim != gm.ndim:
            raise ValueError("grad_va and grad_vm must have the same rank")
        if ga.ndim == 1:
            if ga.shape != gm.shape:
                raise ValueError("1D grad_va/grad_vm shapes must match")
            ga, gm = ga[None, :], gm[None, :]
        elif ga.ndim == 2:
            if ga.shape != gm.shape:
                raise ValueError("2D grad_va/grad_vm shapes must match")
        else:
            raise ValueError("grad_va and grad_vm must be 1D [n_bus] or 2D [batch, n_bus]")
        B, n = ga.shape
        pv, pq = _i32(pv), _i32(pq)
        dim = pv.size + 2 * pq.size
        lam = np.zeros((B, dim))
        gp = np.zeros((B, n))
        gq = np.zeros((B, n))
        raw = _capi.PfAdjointResult()
        ao = _adjoint_options(options)
        _check(self._lib, self._h, self._lib.pf_solve_adjoint(self._h, _ptr(ga), n, _ptr(gm), n, B, _ptr(pv), pv.size,
                                                              _ptr(pq), pq.size, C.byref(ao), _ptr(lam), _ptr(gp),
                                                              _ptr(gq), C.byref(raw)))
        return AdjointResult(raw, lam, gp, gq)

    # -- torch zero-copy entry points (torch_cupf_extension.cpp:81-173) --
    def _torch_checks(self, ref, *tensors):
        import torch

        if not ref.is_cuda:
            raise RuntimeError("tensors must be CUDA tensors")
        for name, t, shape in tensors:
            if not t.is_cuda or t.device != ref.device:
                raise RuntimeError(f"{name} must be on the same CUDA device")
            if t.dtype != ref.dtype:
                raise RuntimeError(f"{name} dtype must match")
            if not t.is_contiguous():
                raise RuntimeError(f"{name} must be contiguous")
            if tuple(t.shape) != tuple(shape):
                raise RuntimeError(f"{name} shape must be {tuple(shape)}")
        return torch.cuda.current_stream(ref.device).cuda_stream

    def solve_with_adjoint_cache_torch(self, sbus_base_re, sbus_base_im, load_p, load_q, v0_va, v0_vm, va_out,
                                       vm_out, config=None, solve_options=None) -> AdjointResult:
        if load_p.dim() != 2:
            raise RuntimeError("load_p must have shape [batch_size, n_bus]")
        B, n = load_p.shape
        batched_v0 = v0_va.dim() == 2
        v0_shape = (B, n) if batched_v0 else (n,)
        stream = self._torch_checks(load_p, ("load_p", load_p, (B, n)), ("load_q", load_q, (B, n)),
                                    ("va_out", va_out, (B, n)), ("vm_out", vm_out, (B, n)),
                                    ("sbus_base_re", sbus_base_re, (n,)), ("sbus_base_im", sbus_base_im, (n,)),
                                    ("v0_va", v0_va, v0_shape), ("v0_vm", v0_vm, v0_shape))
        dt = str(load_p.dtype).replace("torch.", "")
        raw = _capi.PfAdjointResult()
        cfg, so = _nr_config(config), _solve_options(solve_options)
        _check(self._lib, self._h, self._lib.pf_solve_forward_device(
            self._h, sbus_base_re.data_ptr(), sbus_base_im.data_ptr(), load_p.data_ptr(), load_q.data_ptr(),
            v0_va.data_ptr(), v0_vm.data_ptr(), int(batched_v0), va_out.data_ptr(), vm_out.data_ptr(), B, n,
            dt.encode(), C.byref(cfg), C.byref(so), C.c_void_p(stream), C.byref(raw)))
        self._batch = B
        return AdjointResult(raw, zero_copy=True)

    solve_torch = solve_with_adjoint_cache_torch

    def solve_adjoint_torch(self, grad_va, grad_vm, grad_load_p_out, grad_load_q_out, options=None) -> AdjointResult:
        if grad_va.dim() != 2:
            raise RuntimeError("grad_va must have shape [batch_size, n_bus]")
        B, n = grad_va.shape
        stream = self._torch_checks(grad_va, ("grad_vm", grad_vm, (B, n)), ("grad_load_p_out", grad_load_p_out, (B, n)),
                                    ("grad_load_q_out", grad_load_q_out, (B, n)), ("grad_va", grad_va, (B, n)))
        dt = str(grad_va.dtype).replace("torch.", "")
        raw = _capi.PfAdjointResult()
        ao = _adjoint_options(options)
        _check(self._lib, self._h, self._lib.pf_solve_backward_device(
            self._h, grad_va.data_ptr(), grad_vm.data_ptr(), grad_load_p_out.data_ptr(), grad_load_q_out.data_ptr(),
            B, n, dt.encode(), C.byref(ao), C.c_void_p(stream), C.byref(raw)))
        return AdjointResult(raw, zero_copy=True)

    # -- engine extras --
    def solve_batch_device(self, sbus, v0, v_out=None, config=None, solve_options=None, ybus=None):
        """Device-resident solve: sbus / v0 are complex128 CUDA tensors [batch, n_bus];
        ybus, when given, a complex128 CUDA tensor [batch, nnz] of per-scenario
        Ybus values on the initialized pattern."""
        import torch

        B, n = sbus.shape
        if v_out is None:
            v_out = torch.empty_like(sbus)
        fm = torch.empty(B, dtype=torch.float64, device=sbus.device)
        stream = torch.cuda.current_stream(sbus.device).cuda_stream
        raw = _capi.PfAdjointResult()
        cfg, so = _nr_config(config), _solve_options(solve_options)
        if ybus is not None:
            if ybus.dtype != torch.complex128 or ybus.dim() != 2 or ybus.shape[0] != B or ybus.stride(1) != 1:
                raise ValueError("ybus must be a complex128 tensor [batch, nnz] with contiguous rows")
            _check(self._lib, self._h, self._lib.pf_solve_batch_ybus_device(
                self._h, ybus.data_ptr(), ybus.stride(0), sbus.data_ptr(), n, v0.data_ptr(), n, B, C.byref(cfg),
                C.byref(so), v_out.data_ptr(), fm.data_ptr(), C.c_void_p(stream), C.byref(raw)))
            return v_out, fm, raw.iterations
        _check(self._lib, self._h, self._lib.pf_solve_batch_device(
            self._h, sbus.data_ptr(), n, v0.data_ptr(), n, B, C.byref(cfg), C.byref(so), v_out.data_ptr(),
            fm.data_ptr(), C.c_void_p(stream), C.byref(raw)))
        return v_out, fm, raw.iterations

    def solve_batch_warm_device(self, sbus, v0, pred, v_out=None, config=None, solve_options=None,
                                pred_scale=None, pred_shift=None):
        """Device-resident solve from a predicted state: pred is a float32 CUDA
        tensor [>= batch, >= dim_f] with unit column stride, in Jacobian-row
        order (Va at the PV and PQ angle rows, Vm at the PQ magnitude rows),
        mapped to the state by pred * pred_scale + pred_shift when those
        (float32 [dim_f]) are given; v0 complex128 [n_bus] (one row for every
        scenario) or [batch, n_bus] supplies the other buses.  Whether every
        scenario converged is kept in self.last_all_converged."""
        import torch

        B, n = sbus.shape
        if pred.dtype != torch.float32 or pred.dim() != 2 or pred.shape[0] < B or pred.stride(1) != 1:
            raise ValueError("pred must be a float32 tensor [>= batch, >= dim_f] with unit column stride")
        if (pred_scale is None) != (pred_shift is None):
            raise ValueError("pred_scale and pred_shift go together")
        v0_stride = 0 if v0.dim() == 1 else n
        if v_out is None:
            v_out = torch.empty_like(sbus)
        fm = torch.empty(B, dtype=torch.float64, device=sbus.device)
        stream = torch.cuda.current_stream(sbus.device).cuda_stream
        raw = _capi.PfAdjointResult()
        cfg, so = _nr_config(config), _solve_options(solve_options)
        sc = pred_scale.data_ptr() if pred_scale is not None else None
        sh = pred_shift.data_ptr() if pred_shift is not None else None
        _check(self._lib, self._h, self._lib.pf_solve_batch_warm_device(
            self._h, sbus.data_ptr(), n, v0.data_ptr(), v0_stride, pred.data_ptr(), pred.stride(0), sc, sh, B,
            C.byref(cfg), C.byref(so), v_out.data_ptr(), fm.data_ptr(), C.c_void_p(stream), C.byref(raw)))
        self.last_all_converged = bool(raw.all_converged)
        return v_out, fm, raw.iterations

    def info(self) -> dict:
        inf = _capi.PfInfo()
        _check(self._lib, self._h, self._lib.pf_info(self._h, C.byref(inf)))
        return {f[0]: getattr(inf, f[0]) for f in _capi.PfInfo._fields_}

    def dump_fronts_csv(self, path) -> None:
        """Per-front structure of the Jacobian's factor plan as CSV
        (q,p,fsz,nc,uc,level,parent,asm_len,extend_elems; the reference's
        front dump, custom_linear_solver/src/analyze/pipeline.cpp:162-193)."""
        _check(self._lib, self._h, self._lib.pf_dump_fronts_csv(self._h, str(path).encode()))

    def plan_array(self, name: str) -> np.ndarray:
        ln = C.c_int64(0)
        _check(self._lib, self._h, self._lib.pf_plan_array(self._h, name.encode(), None, 0, C.byref(ln)))
        out = np.zeros(ln.value, dtype=np.int32)
        _check(self._lib, self._h, self._lib.pf_plan_array(self._h, name.encode(), _ptr(out), out.size, C.byref(ln)))
        return out

    def plan_array64(self, name: str) -> np.ndarray:
        ln = C.c_int64(0)
        _check(self._lib, self._h, self._lib.pf_plan_array64(self._h, name.encode(), None, 0, C.byref(ln)))
        out = np.zeros(ln.value, dtype=np.int64)
        _check(self._lib, self._h, self._lib.pf_plan_array64(self._h, name.encode(), _ptr(out), out.size,
                                                             C.byref(ln)))
        return out

    def evaluate(self, V, sbus) -> tuple[np.ndarray, np.ndarray]:
        """Mismatch F [batch, dim_f] and Jacobian values [batch, nnz] at host states (verification)."""
        V, sbus = _c128(np.atleast_2d(V)), _c128(np.atleast_2d(sbus))
        B = V.shape[0]
        inf = self.info()
        F = np.zeros((B, inf["dim_f"]))
        J = np.zeros((B, inf["nnz_jacobian"]))
        _check(self._lib, self._h, self._lib.pf_evaluate(self._h, _ptr(V), _ptr(sbus), B, _ptr(F), _ptr(J)))
        return F, J

    STAGES = ("mismatch", "jacobian", "factorize", "solve", "voltage_update")

    def set_profiling(self, on: bool = True) -> None:
        _check(self._lib, self._h, self._lib.pf_set_profiling(self._h, int(bool(on))))

    def stage_times(self) -> dict:
        """{stage: (ms, launches)} of the last solve (profiling must be on)."""
        t = np.zeros(5)
        n = np.zeros(5, dtype=np.int64)
        _check(self._lib, self._h, self._lib.pf_stage_times(self._h, _ptr(t), _ptr(n)))
        return {k: (float(t[i]), int(n[i])) for i, k in enumerate(self.STAGES)}

    def singular_flags(self, batch: int) -> np.ndarray:
        out = np.zeros(batch, dtype=np.int32)
        _check(self._lib, self._h, self._lib.pf_singular_flags(self._h, _ptr(out), batch))
        return out


from .linear_solver import LinearSolver, SolverConfig  # noqa: E402

__all__ = [
    "BackendKind", "ComputePolicy", "CpuLinearSolverKind", "CudaJacobianKind", "CudaLinearSolverKind",
    "CustomPrecision", "CustomMatchingMode", "CustomPivotStrategy", "CustomSolverConfig",
    "AdjointCacheMode", "CuDSSAlgorithm", "CuDSSOptions", "AdjointOptions", "AdjointResult", "NRConfig",
    "SolveOptions", "NewtonOptions", "NRResult", "NRBatchResult", "NewtonSolver", "LinearSolver", "SolverConfig",
]

try:
    from .torch_autograd import CuPFFunction, solve  # noqa: E402
except Exception:  # torch missing
    CuPFFunction = None
    solve = None
else:
    __all__ += ["CuPFFunction", "solve"]
