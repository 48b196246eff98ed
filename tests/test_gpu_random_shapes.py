"""Seeded random products against the CPU oracle.

Shapes, algorithms, recursion depths, schedules, alpha and beta drawn from a
fixed seed, so that the planner's less common paths meet in combinations no
hand-written case picks: block dimensions that become even (256 or more),
fringes of every kind at several levels (rows, columns and inner indices;
the thin kernels), depth-first siblings whose fringes share one launch,
blocks of size zero.  Each result must be within the parity tolerance of the
oracle's FastMatmul -- 1e-13 max relative difference for exact algorithms,
2x the oracle's own error against the classical product (plus 1e-13) for
approximate ones -- and the depth-first and breadth-first programs must give
the same bits.
"""

import numpy as np
import pytest

import oracle
from helpers import gpu_available, to_device, to_host

pytestmark = pytest.mark.gpu

if gpu_available():
    import fast_matmul_b200 as fmm

ALGS = ["strassen", "grey424_26_206", "grey333_23_125", "smirnov333_23_128", "grey522_18_99",
        "smirnov363_40_960", "grey323_15_89", "bini322_10_52_approx", "schonhage333_21_117_approx"]
APPROX = {"bini322_10_52_approx", "schonhage333_21_117_approx"}


def draw_cases(count=40, seed=2024):
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(count):
        alg = ALGS[i % len(ALGS)]
        steps = int(rng.integers(1, 4))
        base = float(np.exp(rng.uniform(np.log(20), np.log(1100))))  # a common size, each dimension jittered
        dims = [max(1, int(base * f)) for f in rng.uniform(0.5, 1.5, 3)]
        alpha = float(rng.choice([1.0, -0.5, 2.25]))
        beta = float(rng.choice([0.0, 1.0, -1.5]))
        cases.append((alg, dims[0], dims[1], dims[2], steps, alpha, beta, 100 + i))
    return cases


CASES = draw_cases()


@pytest.mark.parametrize("case", CASES, ids=["%s-%dx%dx%d-s%d" % c[:5] for c in CASES])
def test_random_product_matches_the_oracle(case):
    alg, m, k, n, steps, alpha, beta, seed = case
    A = oracle.uniform(m, k, seed, 1)
    B = oracle.uniform(k, n, seed, 2)
    C0 = oracle.uniform(m, n, seed, 3)
    x = 1e-4 if alg in APPROX else 1e-8
    want = C0.copy(order="F")
    oracle.fast_matmul(alg, A, B, want, steps, x, alpha, beta)
    got = {}
    for sched in ("dfs", "bfs"):
        Cd = to_device(C0)
        fmm.fast_matmul(alg, to_device(A), to_device(B), Cd, steps, x, alpha, beta, schedule=sched)
        got[sched] = to_host(Cd)
    assert np.array_equal(got["dfs"], got["bfs"])
    scale = float(np.abs(want).max())
    rel = float(np.abs(got["bfs"] - want).max()) / scale
    if alg in APPROX:
        cls = C0.copy(order="F")
        oracle.matmul(A, B, cls, alpha, beta)
        ref_err = float(np.abs(want - cls).max()) / scale
        assert rel <= 2.0 * ref_err + 1e-13, (rel, ref_err)
    else:
        assert rel <= 1e-13, rel
