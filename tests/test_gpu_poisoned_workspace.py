"""Read-before-write check of the device workspace (a sanitizer substitute).

Before each product the handle's whole workspace -- every S, T and M
temporary of every level, and the slice buffers of the split forms -- is
filled with 0xFF bytes, so every double in it is a NaN.  A kernel that read
a temporary it had not written (a planner layout overlap, a missing
formation, an uncovered fringe) would carry a NaN into C.  On the odd shapes
that exercise dynamic peeling at every level (tests/matmul_tests.cpp:140-145)
and on every schedule, the result must be bit-identical to the same call on a
zero-filled workspace, and, in FP64 for the exact algorithms, within 1e-13
max relative difference of the oracle (the parity bar).
"""

import numpy as np
import pytest

import oracle
from helpers import gpu_available, to_device, to_host

pytestmark = pytest.mark.gpu

if gpu_available():
    import fast_matmul_b200 as fmm

SHAPES = [(257, 500, 55), (1001, 200, 309), (402, 500, 562)]
ALGS = [("strassen", 1), ("strassen", 3), ("grey424_26_206", 2), ("grey333_23_125", 2),
        ("smirnov333_23_128", 2), ("bini322_10_52_approx", 2)]
PRECISIONS = [("fp64", 0), ("split_bf16", 5), ("split_int8", 6)]


@pytest.mark.parametrize("shape", SHAPES, ids=["%dx%dx%d" % s for s in SHAPES])
@pytest.mark.parametrize("alg,steps", ALGS, ids=["%s-s%d" % a for a in ALGS])
@pytest.mark.parametrize("precision,slices", PRECISIONS, ids=[p[0] for p in PRECISIONS])
def test_nan_poisoned_workspace_changes_nothing(shape, alg, steps, precision, slices):
    m, k, n = shape
    x = 1e-4 if "approx" in alg else 1e-8
    A = oracle.uniform(m, k, 61, 1)
    B = oracle.uniform(k, n, 61, 2)
    C0 = oracle.uniform(m, n, 61, 3)
    want = C0.copy(order="F")
    oracle.fast_matmul(alg, A, B, want, steps, x, 1.5, 0.5)
    h = fmm.Handle(0)
    h.bind_current_stream()
    try:
        for sched in ("bfs", "dfs", "hybrid"):
            need = fmm.workspace_bytes(alg, m, k, n, steps, sched, precision=precision, split_slices=slices,
                                       handle=h)
            got = {}
            for pattern in (0x00, 0xFF):
                h.debug_fill_workspace(need, pattern)
                Cd = to_device(C0)
                fmm.fast_matmul(alg, to_device(A), to_device(B), Cd, steps, x, 1.5, 0.5, schedule=sched,
                                precision=precision, split_slices=slices, handle=h)
                h.synchronize()
                got[pattern] = to_host(Cd)
            assert np.isfinite(got[0xFF]).all(), (sched, "NaN from the poisoned workspace")
            assert np.array_equal(got[0xFF], got[0x00]), sched
            if precision == "fp64" and "approx" not in alg:
                assert oracle.max_relative_diff(want, got[0xFF]) <= 1e-13, sched
    finally:
        h.close()
