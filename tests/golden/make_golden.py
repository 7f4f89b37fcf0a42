"""Generate golden vectors from the REFERENCE's own compiled code (GPU).

    python tests/golden/make_golden.py [outdir]   (default: this folder)

Runs oracle/_ref/libremifa_ref.so (the reference's src/lu_nopiv.cu,
src/convert.cu, src/gemm.cu, src/lu_nopiv_ll.cxx compiled unmodified) on a
CUDA device and stores its inputs and outputs as .npz fixtures.  The CPU
tests then pin the oracle against them without a GPU.  Inputs come from the
reference's own generators (gen_diagdom / gen_randmat, restated bit-exactly
by the oracle with std::default_random_engine).

Sizes are multiples of 8: the reference's U-part panel kernel indexes rows
beyond a partial tile (src/lu_nopiv.cu:241-248, 304-316 with ld = n < 8), so
only full tiles have well-defined reference output.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "libremifa_ref.so")


def ref_lib():
    L = ctypes.CDLL(REF)
    vp, i64, i = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    L.ref_panel_f32.argtypes = [vp, i, i, vp, i, vp, i, vp, i, vp]
    L.ref_convert_f32_f16.argtypes = [vp, i, i, vp, i, vp, i]
    L.ref_lu_nopiv_rl_f32.argtypes = [vp, i64, i64, i64, vp, i64, vp, i, i, vp, i64]
    L.ref_lu_nopiv_ll_f32.argtypes = [vp, i, i, i, vp, i, vp]
    L.ref_lu_nopiv_ll_f16_tc32.argtypes = [vp, i, i, i, vp, i, vp]
    L.ref_lu_nopiv_ll_f16_variant.argtypes = [vp, i, i, i, i, vp, i, vp]
    L.ref_panel_f16.argtypes = [vp, i, i, vp, i, vp, i, vp, i, vp]
    return L


def to_dev(a: np.ndarray) -> torch.Tensor:
    """Column-major numpy (Fortran view) -> column-major CUDA tensor."""
    lda = oracle.ld(a)
    n = a.shape[1]
    buf = np.zeros((n, lda), dtype=a.dtype)
    buf.T[: a.shape[0], :] = a
    return torch.from_numpy(buf).cuda()


def from_dev(t: torch.Tensor, m: int) -> np.ndarray:
    buf = t.cpu().numpy()
    return np.asfortranarray(buf.T[:m, :])


def main(outdir: str) -> None:
    os.makedirs(outdir, exist_ok=True)
    L = ref_lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")

    # 1. panel kernel (lu_nopiv_panel<float,8>) on a 48-row panel of a
    #    gen_diagdom matrix: the tile is rows/cols 0..7, L rows 8..47,
    #    U columns 8..47.
    a = oracle.gen_diagdom(48, lda=48)
    d = np.asfortranarray(a[:8, :8].copy())
    da, dd = to_dev(a), to_dev(d)
    L.ref_panel_f32(st, 48, 8, ctypes.c_void_p(dd.data_ptr()), 8,
                    ctypes.c_void_p(da.data_ptr()), 48,
                    ctypes.c_void_p(da.data_ptr()), 48,
                    ctypes.c_void_p(info.data_ptr()))
    torch.cuda.synchronize()
    np.savez_compressed(os.path.join(outdir, "ref_panel_48x8.npz"),
                        a_in=np.array(a), out=np.array(from_dev(da, 48)),
                        stat=info.cpu().numpy())

    # 2. convert<float,half>: values covering ties, overflow, subnormals.
    rng = np.random.default_rng(5)
    vals = np.concatenate([
        rng.uniform(-1, 1, 2000), rng.uniform(-7e4, 7e4, 500),
        rng.uniform(-1e-6, 1e-6, 500), np.array([65504, 65519, 65520, 1e5, -65520,
                                                 2.0 ** -24, 3 * 2.0 ** -25,
                                                 1 + 2.0 ** -11, 1 + 3 * 2.0 ** -11]),
    ]).astype(np.float32)
    m = 64
    n = (len(vals) + m - 1) // m
    x = np.zeros((m * n,), np.float32)
    x[: len(vals)] = vals
    xa = np.asfortranarray(x.reshape(n, m).T)
    dx = to_dev(xa)
    dh = torch.zeros((n, m), dtype=torch.float16, device="cuda")
    L.ref_convert_f32_f16(st, m, n, ctypes.c_void_p(dx.data_ptr()), m,
                          ctypes.c_void_p(dh.data_ptr()), m)
    torch.cuda.synchronize()
    np.savez_compressed(os.path.join(outdir, "ref_convert_f32_f16.npz"),
                        a_in=np.array(xa), out=dh.cpu().numpy().T.astype(np.float32))

    # 3. lu_nopiv_rl<float,FP32,FP32,8> on gen_diagdom matrices.
    for nn, nb in ((64, 64), (256, 64), (256, 256), (512, 256)):
        a = oracle.gen_diagdom(nn, lda=nn)
        da = to_dev(a)
        L.ref_lu_nopiv_rl_f32(st, nn, nn, nb, ctypes.c_void_p(da.data_ptr()), nn,
                              ctypes.c_void_p(info.data_ptr()), 0, 0, None, 0)
        torch.cuda.synchronize()
        np.savez_compressed(os.path.join(outdir, f"ref_rl_f32_n{nn}_nb{nb}.npz"),
                            a_in=np.array(a), lu=np.array(from_dev(da, nn)))

    # 4. lu_nopiv_rl<float,FP32,TC32,8> (fp16 outer update) on gen_randmat +
    #    diagonal shift (dominant), n = 512, nb = 128.
    nn, nb = 512, 128
    a = oracle.gen_diagdom(nn, lda=nn)
    da = to_dev(a)
    cpy = torch.zeros((nn, nn), dtype=torch.float16, device="cuda")
    L.ref_lu_nopiv_rl_f32(st, nn, nn, nb, ctypes.c_void_p(da.data_ptr()), nn,
                          ctypes.c_void_p(info.data_ptr()), 0, 1,
                          ctypes.c_void_p(cpy.data_ptr()), nn)
    torch.cuda.synchronize()
    np.savez_compressed(os.path.join(outdir, f"ref_rl_tc32_n{nn}_nb{nb}.npz"),
                        a_in=np.array(a), lu=np.array(from_dev(da, nn)))

    # 5. left-looking fp32 (lu_nopiv_ll_f32), n = 256, nb = 64.
    nn, nb = 256, 64
    a = oracle.gen_diagdom(nn, lda=nn)
    da = to_dev(a)
    L.ref_lu_nopiv_ll_f32(st, nn, nn, nb, ctypes.c_void_p(da.data_ptr()), nn,
                          ctypes.c_void_p(info.data_ptr()))
    torch.cuda.synchronize()
    np.savez_compressed(os.path.join(outdir, f"ref_ll_f32_n{nn}_nb{nb}.npz"),
                        a_in=np.array(a), lu=np.array(from_dev(da, nn)))

    # 6. left-looking on an fp16 matrix (W = fp16), n = 256, nb = 64, input
    #    gen_diagdom rounded to fp16: the wrappers lu_nopiv_ll_f16_tc32xtc32
    #    (variant 2, src/lu_nopiv_ll.cxx:282), lu_nopiv_ll_f16_tc16xtc16
    #    (variant 1, :246) and lu_nopiv_ll_f16_tc32xtc32_fp32xfp32_fp32xfp32
    #    (variant 7, :618).
    nn, nb = 256, 64
    a16 = oracle.gen_diagdom(nn, lda=nn).astype(np.float16)
    for variant, tag in ((2, "tc32"), (1, "tc16"), (7, "tc32_fp32panel")):
        dh = to_dev(np.asfortranarray(a16))
        rc = L.ref_lu_nopiv_ll_f16_variant(st, variant, nn, nn, nb,
                                           ctypes.c_void_p(dh.data_ptr()), nn,
                                           ctypes.c_void_p(info.data_ptr()))
        torch.cuda.synchronize()
        if rc != 0:
            print(f"variant {variant} ({tag}) returned {rc}; skipped")
            continue
        np.savez_compressed(os.path.join(outdir, f"ref_ll_f16_{tag}_n{nn}_nb{nb}.npz"),
                            a_in=np.asfortranarray(a16), lu=np.array(from_dev(dh, nn)))
    # 7. lu_nopiv_panel<half,8> (fp16 arithmetic) on the fp16 rounding of a
    #    64-row gen_diagdom panel
    a16 = np.asfortranarray(oracle.gen_diagdom(64, lda=64).astype(np.float16))
    d16 = np.asfortranarray(a16[:8, :8].copy())
    da, dd = to_dev(a16), to_dev(d16)
    L.ref_panel_f16(st, 64, 8, ctypes.c_void_p(dd.data_ptr()), 8,
                    ctypes.c_void_p(da.data_ptr()), 64, ctypes.c_void_p(da.data_ptr()), 64,
                    ctypes.c_void_p(info.data_ptr()))
    torch.cuda.synchronize()
    np.savez_compressed(os.path.join(outdir, "ref_panel_f16_64x8.npz"),
                        a_in=np.array(a16), out=np.array(from_dev(da, 64)))
    print("golden vectors written to", outdir)


if __name__ == "__main__":
    # default: next to this script (the committed fixtures)
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
