"""CuPFFunction's host logic on the CPU, with a stand-in solver.

The stand-in records the calls the wrapper makes and fills the outputs with
known values, so these tests check the wrapper itself: the forward asks for
the adjoint cache without touching the caller's options, the backward reads
the cached factors without refactoring, the load gradients reach the leaves,
and a second forward on the same solver before the first graph's backward
raises the reference's RuntimeError (cuPF/python/cupf/torch_autograd.py:61-66).
"""
import pytest
import torch

import cupf
from cupf import torch_autograd


class StandInSolver:
    def __init__(self):
        self.forward_options = []
        self.adjoint_options = []

    def solve_with_adjoint_cache_torch(self, base_re, base_im, p, q, va0, vm0, va, vm, config, solve_options):
        self.forward_options.append(solve_options)
        va.copy_(base_re - p)
        vm.copy_(base_im - q)

    def solve_adjoint_torch(self, gva, gvm, gp, gq, options):
        self.adjoint_options.append(options)
        gp.copy_(-gva)
        gq.copy_(-gvm)


def _inputs(B=3, n=4):
    p = torch.rand(B, n, dtype=torch.float64, requires_grad=True)
    q = torch.rand(B, n, dtype=torch.float64, requires_grad=True)
    kw = dict(sbus_base_re=torch.ones(n, dtype=torch.float64), sbus_base_im=torch.zeros(n, dtype=torch.float64),
              v0_va=torch.zeros(n, dtype=torch.float64), v0_vm=torch.ones(n, dtype=torch.float64))
    return p, q, kw


def test_forward_and_backward_route_through_the_solver():
    s = StandInSolver()
    p, q, kw = _inputs()
    caller_opts = cupf.SolveOptions()
    va, vm = torch_autograd.solve(p, q, s, solve_options=caller_opts, **kw)
    assert torch.equal(va, kw["sbus_base_re"] - p.detach())
    assert s.forward_options[0].prepare_adjoint_cache is True
    assert caller_opts.prepare_adjoint_cache is False  # the caller's object is not modified
    (2.0 * va.sum() + 3.0 * vm.sum()).backward()
    assert torch.equal(p.grad, torch.full_like(p, -2.0))
    assert torch.equal(q.grad, torch.full_like(q, -3.0))
    ao = s.adjoint_options[0]
    assert ao.require_cached_factorization and not ao.allow_refactorize and not ao.allow_refactorize_for_backward
    assert ao.check_residual is False


def test_reusing_a_solver_before_backward_raises():
    s = StandInSolver()
    p, q, kw = _inputs()
    va1, _ = torch_autograd.solve(p, q, s, **kw)
    va2, _ = torch_autograd.solve(p, q, s, **kw)  # overwrites the factors the first graph needs
    with pytest.raises(RuntimeError, match="reused before this graph's backward pass"):
        va1.sum().backward()
    va2.sum().backward()  # the latest graph still owns the factors
    assert len(s.adjoint_options) == 1


def test_separate_solvers_do_not_interfere():
    s1, s2 = StandInSolver(), StandInSolver()
    p, q, kw = _inputs()
    va1, _ = torch_autograd.solve(p, q, s1, **kw)
    va2, _ = torch_autograd.solve(p, q, s2, **kw)
    (va1.sum() + va2.sum()).backward()
    assert len(s1.adjoint_options) == 1 and len(s2.adjoint_options) == 1


def test_missing_required_keyword():
    s = StandInSolver()
    p, q, kw = _inputs()
    del kw["v0_vm"]
    with pytest.raises(KeyError):
        torch_autograd.solve(p, q, s, **kw)
