"""Thin torch.autograd binding of the hand-written adjoints (for gradcheck).

The reference has no derivatives; these functions expose the adjoint
kernels of this library to torch so that gradients through an SpMV and
through a full IC(0)-PCG solve can be checked against central finite
differences and an FP64 CPU gradient.  Forward and backward both run on the
GPU through liblab200.so:

* ``spmv(A_plan, values, x)``   y = A x;  dL/dx = A^T g (la_spmv_transpose),
  dL/dvalues = g_i x_j over the pattern (la_sddmm_pattern).
* ``SymmetricSolve``            u = A^-1 b for a symmetric A parameterised by
  its upper triangle (diagonal included): the stored full-matrix values are
  gathered from the upper values, so a perturbation keeps A symmetric and CG
  valid; backward runs the adjoint PCG (la_pcg_adjoint):
  lambda = A^-1 dL/du, dL/db = lambda, dL/dA_ij = -lambda_i u_j, and the
  gather's backward adds the mirrored entries.
"""
from __future__ import annotations

import numpy as np
import torch

from . import api


def upper_gather_index(n, ai, aj):
    """For every stored entry (i, j) of a structurally symmetric CSR, the index
    of entry (min(i,j), max(i,j)) in the upper-triangle list (row-major, the
    order of api.SplitTriangle('U')).  Returns (index, upper_mask)."""
    ai = np.asarray(ai, np.int64)
    aj = np.asarray(aj, np.int64)
    rows = np.repeat(np.arange(n), np.diff(ai))
    upper = aj >= rows
    up_pos = np.full(len(aj), -1, np.int64)
    up_pos[upper] = np.arange(int(upper.sum()))
    key_up = rows[upper] * n + aj[upper]
    lo, hi = np.minimum(rows, aj), np.maximum(rows, aj)
    key = lo * n + hi
    idx = np.searchsorted(key_up, key)
    if np.any(idx >= len(key_up)) or np.any(key_up[np.minimum(idx, len(key_up) - 1)] != key):
        raise ValueError("pattern is not structurally symmetric")
    return idx, upper


class _SpMVFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, x, plan):
        plan.A.update_values(values.detach().contiguous())
        y = torch.empty(plan.A.n, dtype=torch.float64, device=x.device)
        plan(x.detach().contiguous(), y)
        ctx.save_for_backward(x)
        ctx.plan = plan
        return y

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        plan = ctx.plan
        g = g.contiguous()
        dvals = dx = None
        if ctx.needs_input_grad[0]:
            dvals = torch.empty(plan.A.nnz, dtype=torch.float64, device=g.device)
            plan.sddmm(g, x.contiguous(), dvals)
        if ctx.needs_input_grad[1]:
            dx = torch.empty(plan.A.ncols, dtype=torch.float64, device=g.device)
            plan.transpose(g, dx)
        return dvals, dx, None


def spmv(plan: "api.SPMV", values: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    """y = A(values) x with hand-written adjoints (FP64, CUDA tensors)."""
    return _SpMVFn.apply(values, x, plan)


class _SolveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, b, solver, rtol, maxit):
        solver.A.update_values(values.detach().contiguous())
        u = torch.empty_like(b)
        solver.solve(b.detach().contiguous(), u, rtol=rtol, maxit=maxit)
        ctx.save_for_backward(u)
        ctx.solver, ctx.rtol, ctx.maxit = solver, rtol, maxit
        return u

    @staticmethod
    def backward(ctx, gu):
        (u,) = ctx.saved_tensors
        s = ctx.solver
        db = torch.empty_like(u)
        dv = torch.empty(s.A.nnz, dtype=torch.float64, device=u.device)
        s.adjoint(gu.contiguous(), u, db, dv, rtol=ctx.rtol, maxit=ctx.maxit)
        return dv, db, None, None, None


class SymmetricSolve:
    """u = A^-1 b for an SPD A given by its upper-triangle values.

    solver: an api.PCG built for A's pattern (its IC(0) factor only steers
    convergence; the solution is that of the current values)."""

    def __init__(self, solver: "api.PCG", n, ai, aj, rtol=1e-13, maxit=10000):
        idx, _ = upper_gather_index(n, ai, aj)
        self.solver = solver
        self.index = torch.as_tensor(idx, device="cuda")
        self.rtol, self.maxit = rtol, maxit

    def __call__(self, upper_values: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        full = upper_values[self.index]
        return _SolveFn.apply(full, b, self.solver, self.rtol, self.maxit)
