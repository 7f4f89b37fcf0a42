"""Differentiable mixed-precision solve X = A^-1 B (new; the reference's LU
has no derivative).

Forward: a column-major fp32 copy of A is factored without pivoting by
lu_nopiv_rl_c (trailing updates in the chosen precision), then every column
of B is solved and, by default, refined in FP64 to `tol` (lu_refine_ex_c).
Backward (lu_adjoint_c) reuses the same factors:

    dL/dB = A^-T G            (transposed triangular solves, refined in FP64)
    dL/dA = -(A^-T G) X^T     (FP64 outer product, stored fp32)

with G = dL/dX.  Nothing here computes on the host or through torch ops
beyond copies into column-major layout.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .api import TC32, _ptr, _stream, colmajor, ld, lu_nopiv_rl


def _colmajor64(t: torch.Tensor) -> torch.Tensor:
    """Column-major fp64 copy of a 2-D tensor (always a fresh buffer)."""
    out = torch.empty((t.shape[1], t.shape[0]), dtype=torch.float64,
                      device=t.device).t()
    out.copy_(t)
    return out


def refine_ex(a: torch.Tensor, lu: torch.Tensor, b: torch.Tensor, x: torch.Tensor,
              trans: bool = False, tol: float = 1e-14, max_iter: int = 30,
              stream=None, raise_on_stall: bool = False):
    """FP64 refinement of op(A) X = B for all columns of B (n x nrhs, fp64,
    column-major); X receives the solution.  Returns (iterations, berr), the
    largest over the columns."""
    n, k = b.shape
    it = ctypes.c_int(0)
    be = ctypes.c_double(0.0)
    st = _lib.lib().lu_refine_ex_c(_stream(stream), n, k, _ptr(a), ld(a), _ptr(lu),
                                   ld(lu), _ptr(b), ld(b), _ptr(x), ld(x),
                                   int(bool(trans)), float(tol), int(max_iter),
                                   ctypes.byref(it), ctypes.byref(be), None, 0)
    if not (st == _lib.ERR_NOT_CONVERGED and not raise_on_stall):
        _lib.check(st, "lu_refine_ex_c")
    return it.value, be.value


def adjoint(lu: torch.Tensor, x: torch.Tensor, g: torch.Tensor,
            da: torch.Tensor | None = None, a: torch.Tensor | None = None,
            tol: float = 1e-14, max_iter: int = 30, stream=None):
    """lu_adjoint_c: g (fp64, n x nrhs, column-major) is overwritten with
    A^-T g; da (fp32, column-major), when given, receives -(A^-T g) x^T.
    With `a` (the fp32 matrix) the transposed solve is refined in FP64."""
    n, k = g.shape
    it = ctypes.c_int(0)
    be = ctypes.c_double(0.0)
    st = _lib.lib().lu_adjoint_c(
        _stream(stream), n, k, _ptr(a), ld(a) if a is not None else 0, _ptr(lu),
        ld(lu), _ptr(x), ld(x), _ptr(g), ld(g), _ptr(da),
        ld(da) if da is not None else 0, float(tol), int(max_iter),
        ctypes.byref(it), ctypes.byref(be), None, 0)
    if st != _lib.ERR_NOT_CONVERGED:
        _lib.check(st, "lu_adjoint_c")
    return it.value, be.value


class LUSolve(torch.autograd.Function):
    """X = A^-1 B through the no-pivot LU of A (see module docstring)."""

    @staticmethod
    def forward(ctx, a, b, outer, nb, refine, tol, max_iter):
        if a.dim() != 2 or a.shape[0] != a.shape[1] or not a.is_cuda:
            raise ValueError("lu_solve: A must be a square CUDA matrix")
        if a.dtype != torch.float32:
            raise ValueError("lu_solve: A must be float32")
        vec = b.dim() == 1
        b2 = b.view(-1, 1) if vec else b
        if b2.shape[0] != a.shape[0]:
            raise ValueError("lu_solve: B has the wrong number of rows")
        a_cm = colmajor(a.detach())
        lu = colmajor(a.detach())
        info = lu_nopiv_rl(lu, nb=nb, outer=outer)
        bad = int(info.item())
        if bad != 0:
            raise RuntimeError(f"lu_solve: factorization failed, info = {bad}")
        b64 = _colmajor64(b2.detach())
        if refine:
            x = _colmajor64(b2.detach())
            refine_ex(a_cm, lu, b64, x, tol=tol, max_iter=max_iter)
        else:
            x = b64
            st = _lib.lib().lu_solve_c(_stream(), lu.shape[0], _ptr(lu), ld(lu),
                                       _ptr(x), ld(x), x.shape[1], 0)
            _lib.check(st, "lu_solve_c")
        ctx.save_for_backward(a_cm if refine else None, lu, x)
        ctx.vec, ctx.refine, ctx.tol, ctx.max_iter = vec, refine, tol, max_iter
        ctx.b_dtype = b.dtype
        out = x.view(-1) if vec else x
        return out.clone() if vec else out.clone(memory_format=torch.preserve_format)

    @staticmethod
    def backward(ctx, gx):
        a_cm, lu, x = ctx.saved_tensors
        g = _colmajor64(gx.view(-1, 1) if ctx.vec else gx)
        need_a = ctx.needs_input_grad[0]
        da = None
        if need_a:
            da = torch.empty((lu.shape[1], lu.shape[0]), dtype=torch.float32,
                             device=lu.device).t()
        adjoint(lu, x, g, da=da, a=a_cm if ctx.refine else None, tol=ctx.tol,
                max_iter=ctx.max_iter)
        db = None
        if ctx.needs_input_grad[1]:
            db = (g.view(-1) if ctx.vec else g).to(ctx.b_dtype)
        return da, db, None, None, None, None, None


def lu_solve_autograd(a: torch.Tensor, b: torch.Tensor, outer=TC32, nb: int = 256,
                      refine: bool = True, tol: float = 1e-14,
                      max_iter: int = 30) -> torch.Tensor:
    """Differentiable X = A^-1 B (A fp32 n x n, B n or n x nrhs); X is fp64.
    Gradients flow to A (fp32) and B (B's dtype)."""
    return LUSolve.apply(a, b, outer, nb, refine, tol, max_iter)
