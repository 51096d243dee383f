"""Differentiable batched power flow for torch.

The public surface is the reference's (cuPF/python/cupf/torch_autograd.py:28-103),
so code written against it runs unchanged: the class ``CuPFFunction`` with the
same ``forward`` arguments, the keyword interface of ``solve()``, and the
``RuntimeError`` (same text) raised when one solver serves a second forward
pass before the first graph's backward.

How it maps onto this engine:

* forward -- one batched Newton solve on torch's current stream
  (``pf_solve_forward_device``).  The engine then factors the Jacobian of the
  converged state once more with the L factors kept, so the adjoint needs no
  refactorization.
* backward -- the adjoint system J^T lambda = dL/d(Va, Vm) on those cached
  factors (U^T and L^T sweeps plus FP64 residual refinement inside the
  engine, ``pf_solve_backward_device``); the load gradients are
  dL/dP = -lambda_P and dL/dQ = -lambda_Q.
* reuse guard -- the cached factors belong to the last forward pass.  Each
  forward stamps the solver with a new epoch before it solves and keeps the
  stamp in its autograd context; a backward whose stamp is no longer the
  solver's would read another pass's factors and raises instead.
"""
from __future__ import annotations

import copy
from typing import Any

import torch

from . import AdjointOptions, NRConfig, SolveOptions

_REUSED = ("cuPF autograd detected that the same NewtonSolver was reused "
           "before this graph's backward pass. Use one solver per active "
           "autograd graph or run backward before issuing another forward.")

# keyword arguments of solve(), in CuPFFunction.forward's order after the solver
_REQUIRED = ("sbus_base_re", "sbus_base_im", "v0_va", "v0_vm")
_OPTIONAL = ("config", "solve_options")


class _FactorStamp:
    """The epoch a forward pass gave its solver's cached factors."""

    __slots__ = ("solver", "epoch")

    def __init__(self, solver: Any):
        self.solver = solver
        self.epoch = getattr(solver, "_cupf_factor_epoch", 0) + 1
        solver._cupf_factor_epoch = self.epoch

    def current(self) -> bool:
        return getattr(self.solver, "_cupf_factor_epoch", None) == self.epoch


def _forward_options(solve_options: Any | None) -> Any:
    """The caller's options (copied, not modified) with the adjoint cache on."""
    opts = SolveOptions() if solve_options is None else copy.copy(solve_options)
    opts.prepare_adjoint_cache = True
    return opts


def _backward_options() -> AdjointOptions:
    """Adjoint on the forward pass's own factors: no refactorization, and no
    residual readback (which would synchronize the stream)."""
    return AdjointOptions(require_cached_factorization=True, allow_refactorize=False,
                          allow_refactorize_for_backward=False, check_residual=False)


class CuPFFunction(torch.autograd.Function):
    """(load_p, load_q) -> (Va, Vm) through a converged Newton solve."""

    @staticmethod
    def forward(ctx: Any, load_p: torch.Tensor, load_q: torch.Tensor, solver: Any, sbus_base_re: torch.Tensor,
                sbus_base_im: torch.Tensor, v0_va: torch.Tensor, v0_vm: torch.Tensor, config: Any | None = None,
                solve_options: Any | None = None) -> tuple[torch.Tensor, torch.Tensor]:
        p = load_p.contiguous()
        q = load_q.contiguous()
        va = torch.empty_like(p)
        vm = torch.empty_like(q)
        # stamp first: the solve overwrites the factors an earlier graph relied on
        ctx.stamp = _FactorStamp(solver)
        solver.solve_with_adjoint_cache_torch(sbus_base_re, sbus_base_im, p, q, v0_va, v0_vm, va, vm,
                                              config if config is not None else NRConfig(),
                                              _forward_options(solve_options))
        return va, vm

    @staticmethod
    def backward(ctx: Any, grad_va: torch.Tensor, grad_vm: torch.Tensor) -> tuple[Any, ...]:
        stamp: _FactorStamp = ctx.stamp
        if not stamp.current():
            raise RuntimeError(_REUSED)
        gva = grad_va.contiguous()
        gvm = grad_vm.contiguous()
        grad_p = torch.empty_like(gva)
        grad_q = torch.empty_like(gvm)
        stamp.solver.solve_adjoint_torch(gva, gvm, grad_p, grad_q, _backward_options())
        # gradients for load_p and load_q; the solver, bases, start and options get none
        return (grad_p, grad_q) + (None,) * 7


def solve(load_p: torch.Tensor, load_q: torch.Tensor, solver: Any, **kwargs: Any) -> tuple[torch.Tensor, torch.Tensor]:
    """Differentiable solve: ``sbus_base_re``, ``sbus_base_im``, ``v0_va`` and
    ``v0_vm`` are required keywords, ``config`` and ``solve_options`` optional."""
    args = [kwargs[k] for k in _REQUIRED] + [kwargs.get(k) for k in _OPTIONAL]
    return CuPFFunction.apply(load_p, load_q, solver, *args)
