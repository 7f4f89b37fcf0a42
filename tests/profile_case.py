"""Small, fixed cases to put under a profiler.

    python tests/profile_case.py [n] [compute] [reps]
    python tests/profile_case.py update M K [compute] [reps]
    python tests/profile_case.py ll16 [n] [nb] [reps]
    python tests/profile_case.py rowstep [nc] [reps]

The first form factors the seeded matrix A = R + D (R ~ N(0,1)/sqrt(n), row
dominance 1.5, the generator of the benchmarks) `reps` times on cuda:0 with
the right-looking driver (nb = 256), each time from a fresh copy, and prints
the largest factor entry as a check.  Defaults: n = 4096, compute TC32,
reps 2.  Every kernel of the factorization runs with the shapes it has
inside larger factorizations (the diagonal blocks are always 128 x 128, the
sub-panels 128 wide), while the device holds only a few hundred MB, so a
profiler capture of one launch ends quickly.

The second form runs the trailing (Schur) update alone: C (M x M, fp32) -=
A (M x K) B (K x M) through the library's update entry (operands packed, then
one persistent tensor-core launch over all SMs: CTA pairs from K = 512 up)
`reps` times -- the shape class of the factorization's largest launches
(K = 6 nb = 1536 when six outer steps share a pass) at a size whose C
(M = 8192: 256 MB) is larger than L2 and small enough for a full capture.

The third form factors an fp16 matrix with the left-looking driver and fp16
tensor-core updates (fp16 storage, nb = 256 by default): its block-column
updates have K up to n and N = nb, the shapes of the fp16-storage workload.

The fourth form runs one block-row step of the host entry's left-looking
chunk catch-up (lu_catchup_row_step_c, fused: the K = 256 fp16 product with
the previous block row, then the 256-row unit-lower solve) on a 256 x nc
block row (nc = 4096 by default, the columns of one chunk at n = 16384 with
four chunks) `reps` times, in place.
"""
import os
import sys

import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from remifa_b200 import api  # noqa: E402


def factor(argv) -> None:
    n = int(argv[0]) if len(argv) > 0 else 4096
    outer = getattr(api, argv[1]) if len(argv) > 1 else api.TC32
    reps = int(argv[2]) if len(argv) > 2 else 2
    a = api.gen_matrix(n, seed=1, kind=1, alpha=1.5)
    lu = api.colmajor_empty(n, n, n, torch.float32)
    for _ in range(reps):
        lu.copy_(a)
        api.lu_nopiv_rl(lu, nb=256, outer=outer)
    torch.cuda.synchronize()
    print("ok", float(lu.abs().max()))


def update(argv) -> None:
    m = int(argv[0]) if len(argv) > 0 else 8192
    k = int(argv[1]) if len(argv) > 1 else 512
    compute = getattr(api.compute_type, argv[2]) if len(argv) > 2 else api.TC32
    reps = int(argv[3]) if len(argv) > 3 else 2
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    a = api.colmajor(torch.randn(m, k, device="cuda", generator=g))
    b = api.colmajor(torch.randn(k, m, device="cuda", generator=g))
    c = api.colmajor(torch.randn(m, m, device="cuda", generator=g))
    for _ in range(reps):
        api.gemmex(compute, -1.0, a, b, 1.0, c)
    torch.cuda.synchronize()
    print("ok", float(c.abs().max()))


def factor_f16(argv) -> None:
    n = int(argv[0]) if len(argv) > 0 else 4096
    nb = int(argv[1]) if len(argv) > 1 else 256
    reps = int(argv[2]) if len(argv) > 2 else 2
    a32 = api.gen_matrix(n, seed=1, kind=1, alpha=1.5)
    a = api.colmajor_empty(n, n, n, torch.float16)
    api.convert(a32, a)
    lu = api.colmajor_empty(n, n, n, torch.float16)
    for _ in range(reps):
        lu.copy_(a)
        api.lu_nopiv_ll(lu, nb=nb, outer=api.TC32)
    torch.cuda.synchronize()
    print("ok", float(lu.float().abs().max()))


def rowstep(argv) -> None:
    import ctypes
    from remifa_b200 import _lib
    nc = int(argv[0]) if len(argv) > 0 else 4096
    reps = int(argv[1]) if len(argv) > 1 else 2
    inn = kl = 256
    ldx = inn + 8
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    d = api.colmajor(torch.randn(inn, inn + nc, device="cuda", generator=g))
    d[:, :inn] = torch.tril(d[:, :inn], -1) * 0.01 + torch.eye(inn, device="cuda")
    la = (torch.rand(inn, ldx, device="cuda", generator=g) * 0.1).half()
    xb = torch.rand(nc * ldx, device="cuda", generator=g).half()
    xo = torch.zeros(nc * ldx, device="cuda", dtype=torch.float16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    for _ in range(reps):
        s = _lib.lib().lu_catchup_row_step_c(st, 1, 0, inn, nc, inn, kl, p(d), inn, p(la), ldx,
                                             p(xb), p(xo), ldx, None, 0, 0, 0, p(err))
        assert s == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    print("ok", float(d[:, inn:].abs().max()))


def main(argv=None) -> None:
    argv = list(sys.argv[1:] if argv is None else argv)
    if argv and argv[0] == "update":
        update(argv[1:])
    elif argv and argv[0] == "ll16":
        factor_f16(argv[1:])
    elif argv and argv[0] == "rowstep":
        rowstep(argv[1:])
    else:
        factor(argv)


if __name__ == "__main__":
    main()
