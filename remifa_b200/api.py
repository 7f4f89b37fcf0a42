"""Host-side mirror of the reference's lu_nopiv interface over the C ABI.

The reference (flipflapflop/remifa) exposes C++ templates; this module keeps
their names and argument meaning for Python callers, on column-major torch
CUDA tensors (a 2-D tensor with stride(0) == 1; its leading dimension is
stride(1)).  PyTorch only supplies device memory and the current stream; all
work runs in liblu_b200.so.

    remifa::lu_nopiv_rl       (src/lu_nopiv.hxx:44-63)     -> lu_nopiv_rl
    remifa::lu_nopiv_ll       (src/lu_nopiv_ll.hxx:41-66)  -> lu_nopiv_ll
    remifa::lu_nopiv_panel    (src/lu_nopiv.cuh:12-19)     -> lu_nopiv_panel
    remifa::convert           (src/convert.cuh:17-18)      -> convert
    remifa::gemmex            (src/gemm.cuh:24-40)         -> gemmex
    remifa::align_lda         (src/utils.hxx:48-62)        -> align_lda
    remifa::compute_type      (src/utils.hxx:18-24)        -> compute_type
"""
from __future__ import annotations

import ctypes
import enum

import torch

from . import _lib


class compute_type(enum.IntEnum):
    """Update compute types; FP32..TC16 keep the reference's values."""
    FP32 = _lib.COMPUTE_FP32
    FP16 = _lib.COMPUTE_FP16
    TC32 = _lib.COMPUTE_TC32
    TC16 = _lib.COMPUTE_TC16
    TC32_BF16 = _lib.COMPUTE_TC32_BF16
    TC32_E4M3 = _lib.COMPUTE_TC32_E4M3
    TC32_SPLIT = _lib.COMPUTE_TC32_SPLIT


FP32, FP16, TC32, TC16 = (compute_type.FP32, compute_type.FP16,
                          compute_type.TC32, compute_type.TC16)

_DTYPES = {
    torch.float32: _lib.F32,
    torch.float16: _lib.F16,
    torch.bfloat16: _lib.BF16,
    torch.float8_e4m3fn: _lib.E4M3,
    torch.float64: _lib.F64,
}


def align_lda(m: int, itemsize: int = 4) -> int:
    """Smallest multiple of 64 bytes (in elements) >= m, as the reference's
    align_lda (src/utils.hxx:48-62)."""
    t = 64 // itemsize
    return t * ((m - 1) // t + 1) if m > 0 else t


def colmajor_empty(m: int, n: int, lda: int | None = None,
                   dtype=torch.float32, device="cuda") -> torch.Tensor:
    """An m x n column-major tensor with leading dimension lda."""
    lda = m if lda is None else lda
    if lda < max(1, m):
        raise ValueError("lda < m")
    buf = torch.empty((max(n, 1), lda), dtype=dtype, device=device)
    return buf.t()[:m, :n]


def colmajor(t: torch.Tensor, lda: int | None = None) -> torch.Tensor:
    """Column-major copy of a 2-D tensor (same device and dtype)."""
    m, n = t.shape
    out = colmajor_empty(m, n, lda, t.dtype, t.device)
    out.copy_(t)
    return out


def ld(t: torch.Tensor) -> int:
    """Leading dimension of a column-major 2-D tensor."""
    if t.dim() != 2 or (t.stride(0) != 1 and t.shape[0] > 1):
        raise ValueError("expected a column-major 2-D tensor (stride(0) == 1)")
    return max(t.stride(1), t.shape[0], 1)


def _ptr(t: torch.Tensor | None):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)


def make_opts(nb: int = 256, inner=FP32, outer=FP32, lookahead: bool = True,
              diag_width: int = 0, variant: int = _lib.RIGHT_LOOKING,
              panel_fp32: bool = False, bulk_steps: int = 0) -> _lib.LuOpts:
    o = _lib.LuOpts()
    _lib.lib().lu_opts_default(ctypes.byref(o))
    o.nb = int(nb)
    o.inner_update = int(inner)
    o.outer_update = int(outer)
    o.lookahead = int(bool(lookahead))
    o.diag_width = int(diag_width)
    o.variant = int(variant)
    o.panel_fp32 = int(bool(panel_fp32))
    o.bulk_steps = int(bulk_steps)
    return o


def workspace_size(n: int, nb: int = 256, inner=FP32, outer=FP32,
                   variant: int = _lib.RIGHT_LOOKING, dtype=torch.float32,
                   lookahead: bool = True, bulk_steps: int = 0) -> int:
    o = make_opts(nb, inner, outer, lookahead, variant=variant, bulk_steps=bulk_steps)
    sz = ctypes.c_size_t(0)
    _lib.check(_lib.lib().lu_workspace_size(ctypes.byref(o), n, n, _DTYPES[dtype],
                                            ctypes.byref(sz)), "lu_workspace_size")
    return sz.value


def _factor(fn_name: str, variant: int, a: torch.Tensor, nb: int, inner, outer,
            a_cpy, info, lookahead, diag_width, workspace, stream, panel_fp32=False,
            bulk_steps=0):
    if not a.is_cuda:
        raise ValueError(f"{fn_name}: the matrix must be a CUDA tensor")
    m, n = a.shape
    lda = ld(a)
    if info is None:
        info = torch.zeros(1, dtype=torch.int32, device=a.device)
    o = make_opts(nb, inner, outer, lookahead, diag_width, variant, panel_fp32, bulk_steps)
    ws_ptr, ws_bytes = None, 0
    if workspace is not None:
        ws_ptr, ws_bytes = _ptr(workspace), workspace.numel() * workspace.element_size()
    st = getattr(_lib.lib(), fn_name)(
        ctypes.byref(o), _stream(stream), m, n, _ptr(a), _DTYPES[a.dtype], lda,
        _ptr(info), _ptr(a_cpy), ld(a_cpy) if a_cpy is not None else 0,
        ws_ptr, ws_bytes)
    _lib.check(st, fn_name)
    return info


def lu_nopiv_rl(a: torch.Tensor, nb: int = 256, inner=FP32, outer=FP32,
                a_cpy: torch.Tensor | None = None, info: torch.Tensor | None = None,
                lookahead: bool = True, diag_width: int = 0,
                workspace: torch.Tensor | None = None, stream=None,
                bulk_steps: int = 0) -> torch.Tensor:
    """In-place right-looking no-pivot LU of the column-major CUDA matrix `a`
    (remifa::lu_nopiv_rl).  Returns the device info tensor (0 = success,
    k > 0 = first bad pivot, 1-based).  Asynchronous on `stream`.
    bulk_steps: q = 2 .. 8 lets q consecutive outer steps share one pass
    over the bulk of the trailing matrix (fp16 / bf16 updates with
    look-ahead; 0 = the default, 4), 1 applies every step separately (the
    reference's rounding order)."""
    return _factor("lu_nopiv_rl_c", _lib.RIGHT_LOOKING, a, nb, inner, outer,
                   a_cpy, info, lookahead, diag_width, workspace, stream,
                   bulk_steps=bulk_steps)


def lu_nopiv_rl_host(h_a: torch.Tensor, d_a: torch.Tensor, nb: int = 256, inner=FP32,
                     outer=FP32, info: torch.Tensor | None = None, lookahead: bool = True,
                     diag_width: int = 0, workspace: torch.Tensor | None = None,
                     stream=None, bulk_steps: int = 0) -> torch.Tensor:
    """Factor the column-major fp32 matrix in (pinned) host memory `h_a` in
    place, using the device matrix `d_a` (same shape) as the working copy.
    The matrix goes in by column chunks while the device works on the chunks
    already in, and each chunk's factors go back as soon as they are final
    (lu_nopiv_rl_host_c); with bulk_steps = 1 the factors equal
    lu_nopiv_rl's (bulk_steps = 1) bit for bit.  Returns the device info
    tensor."""
    if h_a.is_cuda or not d_a.is_cuda:
        raise ValueError("lu_nopiv_rl_host: h_a must be a host tensor, d_a a CUDA tensor")
    if h_a.dtype != torch.float32 or d_a.dtype != torch.float32 or h_a.shape != d_a.shape:
        raise ValueError("lu_nopiv_rl_host: float32 matrices of the same shape expected")
    n = h_a.shape[0]
    if info is None:
        info = torch.zeros(1, dtype=torch.int32, device=d_a.device)
    o = make_opts(nb, inner, outer, lookahead, diag_width, _lib.RIGHT_LOOKING,
                  bulk_steps=bulk_steps)
    ws_ptr, ws_bytes = None, 0
    if workspace is not None:
        ws_ptr, ws_bytes = _ptr(workspace), workspace.numel() * workspace.element_size()
    st = _lib.lib().lu_nopiv_rl_host_c(ctypes.byref(o), _stream(stream), n, _ptr(h_a),
                                       ld(h_a), _ptr(d_a), ld(d_a), _ptr(info), ws_ptr,
                                       ws_bytes)
    _lib.check(st, "lu_nopiv_rl_host_c")
    return info


def lu_nopiv_ll(a: torch.Tensor, nb: int = 256, inner=FP32, outer=FP32,
                a_cpy: torch.Tensor | None = None, info: torch.Tensor | None = None,
                lookahead: bool = True, diag_width: int = 0,
                workspace: torch.Tensor | None = None, stream=None,
                panel_fp32: bool = False) -> torch.Tensor:
    """In-place left-looking (Crout) no-pivot LU (remifa::lu_nopiv_ll).
    panel_fp32 (fp16 matrices): keep each block column / row update in fp32
    until its panel is factored (the reference's OP = OF = fp32 wrappers)."""
    return _factor("lu_nopiv_ll_c", _lib.LEFT_LOOKING, a, nb, inner, outer,
                   a_cpy, info, lookahead, diag_width, workspace, stream, panel_fp32)


def lu_nopiv_panel(m: int, n: int, d: torch.Tensor, l: torch.Tensor,
                   u: torch.Tensor, stat: torch.Tensor | None = None,
                   stream=None) -> None:
    """remifa::lu_nopiv_panel<float,8>: factor the n x n tile copy `d`, apply
    it to the L rows (in `l`) and U columns (in `u`) of an m-row panel."""
    if stat is None:
        stat = torch.zeros(1, dtype=torch.int32, device=l.device)
    st = _lib.lib().lu_panel_c(_stream(stream), _DTYPES[l.dtype], m, n, _ptr(d),
                               ld(d), _ptr(l), ld(l), _ptr(u), ld(u), _ptr(stat))
    _lib.check(st, "lu_panel_c")


def convert(a: torch.Tensor, out: torch.Tensor, scale_log2: int = 0,
            stream=None) -> torch.Tensor:
    """remifa::convert: out = round(a * 2^scale_log2) (column-major)."""
    m, n = a.shape
    if tuple(out.shape) != (m, n):
        raise ValueError("convert: shape mismatch")
    st = _lib.lib().lu_convert_c(_stream(stream), m, n, _ptr(a), _DTYPES[a.dtype],
                                 ld(a), _ptr(out), _DTYPES[out.dtype], ld(out),
                                 int(scale_log2))
    _lib.check(st, "lu_convert_c")
    return out


def gemmex(compute, alpha: float, a: torch.Tensor, b: torch.Tensor, beta: float,
           c: torch.Tensor, workspace: torch.Tensor | None = None,
           stream=None) -> torch.Tensor:
    """remifa::gemmex: c = alpha * a @ b + beta * c (column-major; a and b
    both float32 or both float16, c float32 or float16)."""
    m, k = a.shape
    k2, n = b.shape
    if k != k2 or tuple(c.shape) != (m, n):
        raise ValueError("gemmex: shape mismatch")
    for name, t in (("a", a), ("b", b), ("c", c)):
        if t.dtype not in (torch.float32, torch.float16) or not t.is_cuda:
            raise ValueError(f"gemmex: {name} must be a float32 / float16 CUDA tensor")
    ws_ptr, ws_bytes = None, 0
    if workspace is not None:
        ws_ptr, ws_bytes = _ptr(workspace), workspace.numel() * workspace.element_size()
    st = _lib.lib().lu_gemm_update_ex_c(_stream(stream), int(compute), m, n, k,
                                        float(alpha), _ptr(a), _DTYPES[a.dtype], ld(a),
                                        _ptr(b), _DTYPES[b.dtype], ld(b), float(beta),
                                        _ptr(c), _DTYPES[c.dtype], ld(c), ws_ptr, ws_bytes)
    _lib.check(st, "lu_gemm_update_ex_c")
    return c


def gen_matrix(n: int, seed: int, kind: int = 0, alpha: float = 2.0,
               kscale: int = 0, gamma_bits: float = 0.0, lda: int | None = None,
               device="cuda", stream=None) -> torch.Tensor:
    """Seeded diagonally dominant test matrix generated on the device
    (identical to the CPU generator of the tests)."""
    a = colmajor_empty(n, n, lda, torch.float32, device)
    st = _lib.lib().lu_gen_matrix_c(_stream(stream), n, _ptr(a), ld(a), seed, kind,
                                    float(alpha), int(kscale), float(gamma_bits))
    _lib.check(st, "lu_gen_matrix_c")
    return a


class profile:
    """Context manager recording per-kernel-class CUDA-event times inside
    the library (on the stream each kernel is launched on).

        with rb.profile() as prof:
            rb.lu_nopiv_rl(a, outer=rb.TC32)
        prof.entries["tc_update"]  -> dict(launches, total_ms, bytes, flops)
    """

    def __enter__(self):
        self.entries = {}
        self.launches0 = _lib.lib().lu_launch_count()
        _lib.lib().lu_profile_begin()
        return self

    def __exit__(self, *exc):
        L = _lib.lib()
        buf = (_lib.LuProfileEntry * 64)()
        k = L.lu_profile_end(buf, 64)
        for i in range(min(k, 64)):
            e = buf[i]
            self.entries[e.name.decode()] = dict(launches=int(e.launches),
                                                 total_ms=float(e.total_ms),
                                                 bytes=float(e.bytes),
                                                 flops=float(e.flops))
        self.launches = L.lu_launch_count() - self.launches0
        return False

    def trace(self) -> list:
        """Per-launch timeline: dicts (name, stream, start_ms, end_ms)."""
        L = _lib.lib()
        k = L.lu_profile_trace(None, 0)
        buf = (_lib.LuTraceEntry * max(k, 1))()
        k = L.lu_profile_trace(buf, k)
        return [dict(name=buf[i].name.decode(), stream=int(buf[i].stream),
                     start_ms=float(buf[i].start_ms), end_ms=float(buf[i].end_ms))
                for i in range(k)]


def launch_count() -> int:
    """Kernels launched by liblu_b200.so in this process so far."""
    return int(_lib.lib().lu_launch_count())


def trim_memory() -> None:
    """Return the unused memory of the library's stream-ordered pool on the
    current device to the driver (lu_trim_memory_c); calls that leave their
    workspace to the library keep it pooled in between."""
    _lib.check(_lib.lib().lu_trim_memory_c(), "lu_trim_memory_c")


def lu_solve(lu: torch.Tensor, b: torch.Tensor, trans: bool = False,
             stream=None) -> torch.Tensor:
    """Solve op(A) X = B with the in-place factors `lu` (fp32, column-major)
    of A; B is fp64 (n or n x nrhs, column-major) and is overwritten with X
    (returned).  trans=True solves A^T X = B."""
    n = lu.shape[0]
    x = b if b.dim() == 2 else b.view(-1, 1)
    if x.dtype != torch.float64:
        raise ValueError("lu_solve: right-hand sides must be float64")
    ldx = ld(x) if x.shape[1] > 1 else max(n, 1)
    st = _lib.lib().lu_solve_c(_stream(stream), n, _ptr(lu), ld(lu), _ptr(x), ldx,
                               x.shape[1], int(bool(trans)))
    _lib.check(st, "lu_solve_c")
    return b


def _check_refine_args(fn: str, a: torch.Tensor, lu: torch.Tensor, b: torch.Tensor,
                       x: torch.Tensor | None) -> int:
    """The checks the C ABI cannot make on raw pointers: a and lu float32
    n x n column-major, b and x float64 vectors of n contiguous elements, all
    CUDA tensors on one device.  Returns n; raises ValueError otherwise."""
    if a.dim() != 2 or a.shape[0] != a.shape[1]:
        raise ValueError(f"{fn}: a must be a square matrix")
    n = a.shape[0]
    for name, t in (("a", a), ("lu", lu)):
        if t.dtype != torch.float32 or t.dim() != 2 or tuple(t.shape) != (n, n):
            raise ValueError(f"{fn}: {name} must be a float32 {n} x {n} matrix")
        ld(t)  # column-major
    vecs = [("b", b)] + ([("x", x)] if x is not None else [])
    for name, t in vecs:
        if t.dtype != torch.float64 or t.dim() != 1 or t.numel() != n or \
                not t.is_contiguous():
            raise ValueError(f"{fn}: {name} must be a contiguous float64 vector of {n} "
                             "elements")
    for name, t in [("a", a), ("lu", lu)] + vecs:
        if not t.is_cuda or t.device != a.device:
            raise ValueError(f"{fn}: {name} must be a CUDA tensor on a's device")
    return n


def refine(a: torch.Tensor, lu: torch.Tensor, b: torch.Tensor,
           x: torch.Tensor | None = None, tol: float = 1e-14, max_iter: int = 30,
           stream=None, raise_on_stall: bool = False):
    """FP64 iterative refinement of A x = b with (possibly low-precision)
    factors `lu` of the fp32 matrix `a`.  Returns (x, iterations, berr)
    where berr = ||b - Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf)."""
    n = _check_refine_args("refine", a, lu, b, x)
    if x is None:
        x = torch.empty(n, dtype=torch.float64, device=a.device)
    it = ctypes.c_int(0)
    be = ctypes.c_double(0.0)
    st = _lib.lib().lu_refine_c(_stream(stream), n, _ptr(a), ld(a), _ptr(lu), ld(lu),
                                _ptr(b), _ptr(x), float(tol), int(max_iter),
                                ctypes.byref(it), ctypes.byref(be), None, 0)
    if st == _lib.ERR_NOT_CONVERGED and not raise_on_stall:
        return x, it.value, be.value
    _lib.check(st, "lu_refine_c")
    return x, it.value, be.value


def gmres_ir(a: torch.Tensor, lu: torch.Tensor, b: torch.Tensor,
             x: torch.Tensor | None = None, tol: float = 1e-14, max_outer: int = 20,
             restart: int = 40, inner_tol: float = 1e-6, stream=None,
             raise_on_stall: bool = False):
    """GMRES-based FP64 refinement of A x = b (lu_gmres_ir_c): the
    corrections are solved by GMRES preconditioned with the (possibly
    low-precision) factors `lu`, which converges where classic refinement
    stalls.  Returns (x, outer iterations, Arnoldi steps, berr)."""
    n = _check_refine_args("gmres_ir", a, lu, b, x)
    if x is None:
        x = torch.empty(n, dtype=torch.float64, device=a.device)
    it = ctypes.c_int(0)
    inner = ctypes.c_int(0)
    be = ctypes.c_double(0.0)
    st = _lib.lib().lu_gmres_ir_c(_stream(stream), n, _ptr(a), ld(a), _ptr(lu), ld(lu),
                                  _ptr(b), _ptr(x), float(tol), int(max_outer), int(restart),
                                  float(inner_tol), ctypes.byref(it), ctypes.byref(inner),
                                  ctypes.byref(be), None, 0)
    if not (st == _lib.ERR_NOT_CONVERGED and not raise_on_stall):
        _lib.check(st, "lu_gmres_ir_c")
    return x, it.value, inner.value, be.value


def equilibrate(a: torch.Tensor, force: bool = False, stream=None):
    """Scale the column-major fp32 CUDA matrix `a` in place by powers of two
    (LAPACK geequb + laqge, lu_equilibrate_c; force: scale rows and columns
    whatever laqge decides).  Returns (r, c, equed, rowcnd, colcnd, amax): a
    became diag(r) a diag(c)."""
    if a.dtype != torch.float32 or not a.is_cuda or a.dim() != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("equilibrate: a must be a square float32 CUDA matrix")
    n = a.shape[0]
    r = torch.empty(n, dtype=torch.float32, device=a.device)
    c = torch.empty(n, dtype=torch.float32, device=a.device)
    eq = ctypes.create_string_buffer(1)
    rc, cc, am = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
    st = _lib.lib().lu_equilibrate_c(_stream(stream), n, _ptr(a), ld(a), _ptr(r), _ptr(c),
                                     int(bool(force)), eq,
                                     ctypes.byref(rc), ctypes.byref(cc), ctypes.byref(am))
    _lib.check(st, "lu_equilibrate_c")
    return r, c, eq.raw.decode(), rc.value, cc.value, am.value


def gesv_mixed(a: torch.Tensor, b: torch.Tensor, outer=TC32, nb: int = 256,
               tol: float = 1e-14, max_iter: int = 30, lookahead: bool = True,
               stream=None, equilibrate_first: bool = False, solver: str = "classic"):
    """Solve A x = b to an fp64-level backward error: factor a copy of the
    fp32 matrix with the `outer` trailing-update precision, then refine in
    fp64 (solver "classic": lu_refine_c, "gmres": lu_gmres_ir_c).  With
    equilibrate_first the copy is scaled to R A C by powers of two first
    (geequb / laqge), the scaled system R A C y = R b is refined, and x = C y.
    Returns (x, info, iterations, berr), berr that of the system solved."""
    lu = colmajor(a)
    if equilibrate_first:
        r, c, _, _, _, _ = equilibrate(lu, force=True, stream=stream)
        a_s = colmajor(lu)
        b_s = b * r.double()
    else:
        a_s, b_s = a, b
    info = lu_nopiv_rl(lu, nb=nb, outer=outer, lookahead=lookahead, stream=stream)
    if solver == "gmres":
        x, it, _, be = gmres_ir(a_s, lu, b_s, tol=tol, max_outer=max_iter, stream=stream)
    else:
        x, it, be = refine(a_s, lu, b_s, tol=tol, max_iter=max_iter, stream=stream)
    if equilibrate_first:
        x = x * c.double()
    return x, info, it, be


def refine_static(a: torch.Tensor, lu: torch.Tensor, b: torch.Tensor,
                  x: torch.Tensor, tol: float = 1e-14, max_iter: int = 30,
                  stream=None):
    """refine() without any device allocation (lu_refine_static_c): the
    scratch is compiled into the library, so n <= 4096 and calls must not
    overlap in time on one device.  x (fp64, n) receives the solution.
    Returns (iterations, berr)."""
    n = _check_refine_args("refine_static", a, lu, b, x)
    it = ctypes.c_int(0)
    be = ctypes.c_double(0.0)
    st = _lib.lib().lu_refine_static_c(_stream(stream), n, _ptr(a), ld(a), _ptr(lu),
                                       ld(lu), _ptr(b), _ptr(x), float(tol),
                                       int(max_iter), ctypes.byref(it),
                                       ctypes.byref(be))
    if st != _lib.ERR_NOT_CONVERGED:
        _lib.check(st, "lu_refine_static_c")
    return it.value, be.value
