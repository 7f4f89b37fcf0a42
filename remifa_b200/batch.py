"""Batched no-pivot LU of many uneven matrices (new; the reference factors
one matrix per call).

    sizes = batch_sizes(10_000)                 # n_i = floor(16 * 32**u_i)
    mats = MatrixBatch(sizes)                   # back to back in one buffer
    mats.generate(seed=11)                      # diagonally dominant, factor 1.5
    plan = BatchPlan(sizes, outer=TC32)         # sorts, buckets, uploads
    plan.autotune()                             # block width per size bucket
    info = plan(mats)                           # one persistent launch
    g = plan.graph(mats, info); g.launch()      # the same, as a CUDA graph

All work runs in liblu_b200.so (lu_batch_* of include/lu_b200.h).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .api import FP32, TC32, _stream, make_opts

MAX_N = _lib.BATCH_MAX_N
BUCKETS = _lib.BATCH_BUCKETS


def batch_sizes(count: int = 10_000, seed: int = 11, lo: int = 16,
                ratio: float = 32.0) -> np.ndarray:
    """Log-uniform sizes n_i = floor(lo * ratio**u_i), u_i ~ U[0, 1) from
    numpy's default generator seeded with `seed` (16 .. 511 by default)."""
    u = np.random.default_rng(seed).random(count)
    return np.floor(lo * ratio ** u).astype(np.int32)


def bucket_of(n: int) -> int:
    """Size bucket: n < 32, [32, 64), [64, 128), [128, 256), [256, 512), 512."""
    b = 0
    while (32 << b) <= n and b < BUCKETS - 1:
        b += 1
    return b


class MatrixBatch:
    """fp32 column-major matrices stored back to back in one device buffer
    (matrix i has leading dimension n_i rounded up to `align`), with the
    device arrays of pointers, sizes and leading dimensions."""

    def __init__(self, sizes, device="cuda", align: int = 1,
                 data: torch.Tensor | None = None):
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int32)
        if self.sizes.size and (self.sizes.min() < 1 or self.sizes.max() > MAX_N):
            raise ValueError(f"batch sizes must lie in [1, {MAX_N}]")
        self.align = int(align)
        self.lda = ((self.sizes + align - 1) // align * align).astype(np.int32)
        off = np.zeros(self.sizes.size + 1, dtype=np.int64)
        off[1:] = np.cumsum(self.lda.astype(np.int64) * self.sizes)
        self.offsets = off
        if data is None:
            data = torch.zeros(max(int(off[-1]), 1), dtype=torch.float32, device=device)
        elif (data.dtype != torch.float32 or data.dim() != 1 or not data.is_contiguous()
              or data.numel() < int(off[-1])):
            raise ValueError("MatrixBatch: data must be a contiguous flat float32 tensor "
                             "holding the whole batch")
        self.data = data
        device = data.device
        base = self.data.data_ptr()
        self.ptrs = torch.from_numpy(base + off[:-1] * 4).to(device)
        self.d_n = torch.from_numpy(self.sizes).to(device)
        self.d_lda = torch.from_numpy(self.lda).to(device)

    def __len__(self) -> int:
        return int(self.sizes.size)

    def like(self, data: torch.Tensor | None = None) -> "MatrixBatch":
        """Same sizes and layout over `data` (or fresh zeros)."""
        return MatrixBatch(self.sizes, device=self.data.device, align=self.align, data=data)

    @property
    def flops(self) -> float:
        """sum of 2 n^3 / 3 (the reference's LU flop count per matrix)."""
        n = self.sizes.astype(np.float64)
        return float((2.0 * n ** 3 / 3.0).sum())

    def matrix(self, i: int) -> torch.Tensor:
        """Column-major (n_i x n_i) view of matrix i."""
        n, ld = int(self.sizes[i]), int(self.lda[i])
        o = int(self.offsets[i])
        return self.data[o:o + ld * n].view(n, ld).t()[:n]

    def generate(self, seed: int = 11, kind: int = 0, alpha: float = 1.5,
                 stream=None) -> "MatrixBatch":
        """Matrix i = the seeded generator with seed + i (kind 0: U[-1,1)
        off-diagonal, row dominance alpha)."""
        st = _lib.lib().lu_gen_batch_c(_stream(stream), len(self), self.ptrs.data_ptr(),
                                       self.d_n.data_ptr(), self.d_lda.data_ptr(),
                                       int(seed), int(kind), float(alpha))
        _lib.check(st, "lu_gen_batch_c")
        return self


class RhsBatch:
    """fp64 right-hand sides / solutions of a batch: matrix i's block n_i x
    nrhs (column-major, ld n_i) stored back to back, with the device array
    of block pointers."""

    def __init__(self, sizes, nrhs: int = 1, device="cuda",
                 data: torch.Tensor | None = None):
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int32)
        self.nrhs = int(nrhs)
        off = np.zeros(self.sizes.size + 1, dtype=np.int64)
        off[1:] = np.cumsum(self.sizes.astype(np.int64) * self.nrhs)
        self.offsets = off
        if data is None:
            data = torch.zeros(max(int(off[-1]), 1), dtype=torch.float64, device=device)
        elif (data.dtype != torch.float64 or data.dim() != 1 or not data.is_contiguous()
              or data.numel() < int(off[-1])):
            raise ValueError("RhsBatch: data must be a contiguous flat float64 tensor")
        self.data = data
        self.ptrs = torch.from_numpy(data.data_ptr() + off[:-1] * 8).to(data.device)

    def block(self, i: int) -> torch.Tensor:
        n, o = int(self.sizes[i]), int(self.offsets[i])
        return self.data[o:o + n * self.nrhs].view(self.nrhs, n).t()

    def like(self, data: torch.Tensor | None = None) -> "RhsBatch":
        return RhsBatch(self.sizes, self.nrhs, device=self.data.device, data=data)


def _tuning_struct(t: dict) -> _lib.LuBatchTuning:
    s = _lib.LuBatchTuning()
    for b in range(BUCKETS):
        s.nb[b] = int(t["nb"][b])
        s.outer[b] = int(t["outer"][b])
    return s


def _tuning_dict(s: _lib.LuBatchTuning) -> dict:
    return {"nb": [int(s.nb[b]) for b in range(BUCKETS)],
            "outer": [int(s.outer[b]) for b in range(BUCKETS)]}


class BatchGraph:
    """lu_batch_c captured once into a CUDA graph."""

    def __init__(self, handle: ctypes.c_void_p, keep):
        self._g = handle
        self._keep = keep  # tensors the graph points at

    def launch(self, stream=None) -> None:
        _lib.check(_lib.lib().lu_batch_graph_launch(self._g, _stream(stream)),
                   "lu_batch_graph_launch")

    def close(self) -> None:
        if self._g:
            _lib.lib().lu_batch_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan:
    """lu_batch_plan: sizes, work order and per-bucket tuning on the device."""

    def __init__(self, sizes, outer=TC32, nb: int = 0, tuning: dict | None = None):
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int32)
        o = make_opts(nb=nb, outer=outer, inner=FP32)
        p = ctypes.c_void_p()
        ts = _tuning_struct(tuning) if tuning is not None else None
        st = _lib.lib().lu_batch_plan_create(
            ctypes.byref(o), int(self.sizes.size), self.sizes.ctypes.data_as(ctypes.c_void_p),
            ctypes.byref(ts) if ts is not None else None, ctypes.byref(p))
        _lib.check(st, "lu_batch_plan_create")
        self._p = p

    def close(self) -> None:
        if getattr(self, "_p", None):
            _lib.lib().lu_batch_plan_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tuning(self) -> dict:
        s = _lib.LuBatchTuning()
        _lib.check(_lib.lib().lu_batch_plan_tuning(self._p, ctypes.byref(s)),
                   "lu_batch_plan_tuning")
        return _tuning_dict(s)

    def set_tuning(self, t: dict) -> None:
        s = _tuning_struct(t)
        _lib.check(_lib.lib().lu_batch_plan_set_tuning(self._p, ctypes.byref(s)),
                   "lu_batch_plan_set_tuning")

    def autotune(self, reps: int = 3, stream=None) -> dict:
        s = _lib.LuBatchTuning()
        _lib.check(_lib.lib().lu_batch_autotune(self._p, _stream(stream), int(reps),
                                                ctypes.byref(s)), "lu_batch_autotune")
        return _tuning_dict(s)

    def __call__(self, mats: MatrixBatch, info: torch.Tensor | None = None,
                 stream=None) -> torch.Tensor:
        if info is None:
            info = torch.zeros(max(len(mats), 1), dtype=torch.int32, device=mats.data.device)
        st = _lib.lib().lu_batch_c(self._p, _stream(stream), mats.ptrs.data_ptr(),
                                   mats.d_lda.data_ptr(), info.data_ptr())
        _lib.check(st, "lu_batch_c")
        return info

    def solve(self, lu: MatrixBatch, x: RhsBatch, a: MatrixBatch | None = None,
              trans: bool = False, refine_iters: int = 0, stream=None) -> RhsBatch:
        """lu_batch_solve_c: x holds B on entry, op(A)^-1 B on exit; with the
        original matrices `a`, refine_iters rounds of FP64 refinement."""
        st = _lib.lib().lu_batch_solve_c(
            self._p, _stream(stream), lu.ptrs.data_ptr(), lu.d_lda.data_ptr(),
            a.ptrs.data_ptr() if a is not None else None,
            a.d_lda.data_ptr() if a is not None else None,
            x.ptrs.data_ptr(), x.nrhs, int(bool(trans)), int(refine_iters))
        _lib.check(st, "lu_batch_solve_c")
        return x

    def adjoint(self, lu: MatrixBatch, x: RhsBatch, g: RhsBatch,
                da: MatrixBatch | None = None, a: MatrixBatch | None = None,
                refine_iters: int = 0, stream=None) -> None:
        """lu_batch_adjoint_c: g <- A^-T g, da <- -(A^-T g) x^T."""
        st = _lib.lib().lu_batch_adjoint_c(
            self._p, _stream(stream), lu.ptrs.data_ptr(), lu.d_lda.data_ptr(),
            a.ptrs.data_ptr() if a is not None else None,
            a.d_lda.data_ptr() if a is not None else None,
            x.ptrs.data_ptr(), g.ptrs.data_ptr(),
            da.ptrs.data_ptr() if da is not None else None,
            da.d_lda.data_ptr() if da is not None else None, x.nrhs, int(refine_iters))
        _lib.check(st, "lu_batch_adjoint_c")

    def graph(self, mats: MatrixBatch, info: torch.Tensor, stream=None) -> BatchGraph:
        """Capture this plan on `mats` into a CUDA graph.  Capture needs a
        non-default stream; one is made when none is given."""
        s = stream if stream is not None else torch.cuda.Stream()
        g = ctypes.c_void_p()
        st = _lib.lib().lu_batch_graph_create(self._p, ctypes.c_void_p(s.cuda_stream),
                                              mats.ptrs.data_ptr(), mats.d_lda.data_ptr(),
                                              info.data_ptr(), ctypes.byref(g))
        _lib.check(st, "lu_batch_graph_create")
        return BatchGraph(g, (mats, info, self))


class BatchedLUSolve(torch.autograd.Function):
    """X_i = A_i^-1 B_i for a whole batch.  a_flat: the matrices in the
    layout of `layout` (a MatrixBatch), b_flat: an RhsBatch's flat data.
    Forward: one batched factorization of a copy, batched solves refined
    refine_iters times in FP64.  Backward: lu_batch_adjoint_c with the same
    factors (dB_i = A_i^-T G_i, dA_i = -dB_i X_i^T)."""

    @staticmethod
    def forward(ctx, a_flat, b_flat, layout, plan, nrhs, refine_iters):
        a = layout.like(a_flat.detach().contiguous())
        lu = layout.like(a.data.clone())
        info = plan(lu)
        bad = int((info[:len(lu)] != 0).sum())
        if bad:
            raise RuntimeError(f"batched_lu_solve: {bad} factorization(s) failed")
        x = RhsBatch(layout.sizes, nrhs, device=a_flat.device,
                     data=b_flat.detach().to(torch.float64).contiguous().clone())
        plan.solve(lu, x, a=a, refine_iters=refine_iters)
        ctx.save_for_backward(a.data, lu.data, x.data)
        ctx.layout, ctx.plan, ctx.nrhs, ctx.iters = layout, plan, nrhs, refine_iters
        ctx.b_dtype = b_flat.dtype
        return x.data.clone()

    @staticmethod
    def backward(ctx, gx):
        a_d, lu_d, x_d = ctx.saved_tensors
        lay = ctx.layout
        a, lu = lay.like(a_d), lay.like(lu_d)
        x = RhsBatch(lay.sizes, ctx.nrhs, device=x_d.device, data=x_d)
        g = x.like(gx.to(torch.float64).contiguous().clone())
        da = lay.like() if ctx.needs_input_grad[0] else None
        ctx.plan.adjoint(lu, x, g, da=da, a=a, refine_iters=ctx.iters)
        db = g.data.to(ctx.b_dtype) if ctx.needs_input_grad[1] else None
        return (da.data if da is not None else None), db, None, None, None, None


def batched_lu_solve(a_flat: torch.Tensor, b_flat: torch.Tensor, layout: MatrixBatch,
                     plan: BatchPlan, nrhs: int = 1, refine_iters: int = 2) -> torch.Tensor:
    """Differentiable batched solve (see BatchedLUSolve); returns the flat
    fp64 solutions in RhsBatch layout."""
    return BatchedLUSolve.apply(a_flat, b_flat, layout, plan, nrhs, refine_iters)
