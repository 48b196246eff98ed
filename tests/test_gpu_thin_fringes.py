"""The fringe products of dynamic peeling on the thin kernel (csrc/thin_gemm.cu).

Dynamic peeling (linalg/linalg.hpp:201-244) leaves, at each level, a row
fringe C(mx, :) = A(mx, :) B and a column fringe C(:, nx) = A B(:, nx) of
1..2 m0 - 1 rows (blocks of 256 or more rows are made even) and 1..n0 - 1
columns against the level's whole inner dimension; these run on the thin
kernel, whose sums are sized for 4, 8 or 16 rows or columns, and the k
fringe C_core += A(:, kx) B(kx, :) of 1..2 k0 - 1 inner indices runs on its
block kernel (16-byte C accesses where C allows them).  The shapes
below reach each of those paths (with alpha / beta, odd leading
dimensions' views, and depth-first levels whose sibling fringes share one
launch), and the result must match the CPU oracle's FastMatmul within the
parity tolerance, 1e-13 max relative difference, with every schedule and
both GEMM tile configurations giving the same bits.
"""

import numpy as np
import pytest

import oracle
from helpers import gpu_available, to_device, to_host

pytestmark = pytest.mark.gpu

if gpu_available():
    import fast_matmul_b200 as fmm

# (algorithm, m, k, n, steps): the fringe widths each shape produces
CASES = [
    ("grey424_26_206", 4 * 300 + 7, 2 * 290 + 1, 4 * 260 + 3, 1),    # 7 rows (8-wide), 3 columns (4-wide)
    ("smirnov633_40_960", 6 * 258 + 11, 3 * 200 + 2, 3 * 150 + 2, 1),  # 11 rows (16-wide), 2 columns
    ("smirnov336_40_960", 3 * 270 + 2, 3 * 100 + 1, 6 * 60 + 5, 1),   # 2 rows, 5 columns (8-wide)
    ("grey333_23_125", 3 * (3 * 90 + 2) + 2, 3 * (3 * 60 + 1) + 1, 3 * (3 * 70 + 2) + 2, 2),  # both levels
    ("strassen", 2 * 255 + 1, 2 * 254 + 1, 2 * 253 + 1, 2),  # 1 row and column at both levels
    ("smirnov363_40_960", 3 * 200 + 1, 6 * 258 + 11, 3 * 150 + 2, 1),  # 11 inner indices (the k fringe)
]


def case_id(c):
    return "%s-%dx%dx%d-s%d" % c


@pytest.mark.parametrize("case", CASES, ids=[case_id(c) for c in CASES])
def test_thin_fringes_match_the_oracle_under_every_schedule(case):
    alg, m, k, n, steps = case
    A = oracle.uniform(m, k, 31, 1)
    B = oracle.uniform(k, n, 31, 2)
    C0 = oracle.uniform(m, n, 31, 3)
    alpha, beta = 1.5, -0.75
    want = C0.copy(order="F")
    oracle.fast_matmul(alg, A, B, want, steps, 1e-8, alpha, beta)
    results = {}
    for sched in ("bfs", "dfs"):
        for tile in ("large", "small"):
            Cd = to_device(C0)
            fmm.fast_matmul(alg, to_device(A), to_device(B), Cd, steps, 1e-8, alpha, beta, schedule=sched,
                            gemm_tile=tile)
            results[(sched, tile)] = to_host(Cd)
    first = results[("bfs", "large")]
    for key, got in results.items():
        assert np.array_equal(got, first), key
    rel = float(np.abs(first - want).max() / np.abs(want).max())
    assert rel <= 1e-13, rel
