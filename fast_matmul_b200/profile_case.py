"""One product configuration run a few times, for profiler captures.

    python -m fast_matmul_b200.profile_case ALG N STEPS PRECISION SLICES [--calls C]

ALG is an algorithm name or "classical"; PRECISION is fp64, split_bf16 or
split_int8; the operands are seeded uniform [0, 1) N x N matrices in device
memory.  Each call launches the same kernels, so a capture can skip the
first call's launches (ncu -s) and record the second's.
"""

import argparse
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("alg")
    ap.add_argument("n", type=int)
    ap.add_argument("steps", type=int)
    ap.add_argument("precision", choices=["fp64", "split_bf16", "split_int8"])
    ap.add_argument("slices", type=int)
    ap.add_argument("--calls", type=int, default=2)
    a = ap.parse_args(argv)

    import fast_matmul_b200 as fmm

    A = fmm.random_matrix(a.n, a.n, 1, 1)
    B = fmm.random_matrix(a.n, a.n, 1, 2)
    C = fmm.colmajor_empty(a.n, a.n, A.device)
    for _ in range(a.calls):
        if a.alg == "classical":
            if a.precision == "split_int8":
                fmm.matmul_split_int8(A, B, C, slices=a.slices)
            elif a.precision == "split_bf16":
                fmm.matmul_split_bf16(A, B, C, slices=a.slices)
            else:
                fmm.matmul(A, B, C)
        else:
            fmm.fast_matmul(a.alg, A, B, C, a.steps, precision=a.precision, split_slices=a.slices)
    fmm.synchronize()
    print("ok", a.alg, a.n, a.steps, a.precision, a.slices, float(C[0, 0]))
    return 0


if __name__ == "__main__":
    sys.exit(main())
