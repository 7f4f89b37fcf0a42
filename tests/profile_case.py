"""A small, fixed factorization to put under a profiler.

    python tests/profile_case.py [n] [compute] [reps]

factors the seeded matrix A = R + D (R ~ N(0,1)/sqrt(n), row dominance 1.5,
the generator of the benchmarks) `reps` times on cuda:0 with the
right-looking driver (nb = 256), each time from a fresh copy, and prints the
largest factor entry as a check.  Defaults: n = 4096, compute TC32, reps 2.
Every kernel of the factorization runs with the shapes it has inside larger
factorizations (the diagonal blocks are always 128 x 128, the sub-panels 128
wide), while the device holds only a few hundred MB, so a profiler capture
of one launch ends quickly.
"""
import os
import sys

import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from remifa_b200 import api  # noqa: E402


def main(argv=None) -> None:
    argv = list(sys.argv[1:] if argv is None else argv)
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


if __name__ == "__main__":
    main()
