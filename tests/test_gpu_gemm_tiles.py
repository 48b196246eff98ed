"""The FP64 GEMM's two tile configurations (128 x 64 and 64 x 64).

Both sum every output element over the same k blocks in the same order, so
the configuration may change speed but never a bit of the result: checked on
classical products and FastMatmul (leaf and fringe products) with odd
shapes, alpha/beta, and on a batch whose items mix configurations.  The
autotuner's table carries the configuration as its sixth column.
"""

import pytest

from helpers import colmajor_copy, gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm

CASES = [("strassen", (517, 389, 461), 2), ("grey333_23_125", (401, 403, 399), 2), ("grey424_26_206", (130, 70, 66), 1),
         ("strassen", (67, 1001, 65), 1), ("smirnov333_23_128", (1000, 200, 309), 1)]


@pytest.mark.parametrize("alg,shape,steps", CASES, ids=["%s-%dx%dx%d" % ((c[0],) + c[1]) for c in CASES])
def test_tile_configurations_give_identical_results(alg, shape, steps):
    m, k, n = shape
    A = fmm.random_matrix(m, k, 11, 1)
    B = fmm.random_matrix(k, n, 11, 2)
    C0 = fmm.random_matrix(m, n, 11, 3)
    out = {}
    for tile in ("large", "small", "auto"):
        C = colmajor_copy(C0)
        fmm.fast_matmul(alg, A, B, C, steps, 1e-8, 1.5, 0.5, gemm_tile=tile)
        out[tile] = C
    torch.cuda.synchronize()
    assert torch.equal(out["large"], out["small"])
    assert torch.equal(out["large"], out["auto"])


def test_batch_items_mixing_tiles_equal_single_calls():
    shapes = [(100, 300, 90), (257, 64, 129), (64, 64, 64), (700, 130, 500)]
    probs, want = [], []
    for i, (m, k, n) in enumerate(shapes):
        A = fmm.random_matrix(m, k, 20 + i, 1)
        B = fmm.random_matrix(k, n, 20 + i, 2)
        C0 = fmm.random_matrix(m, n, 20 + i, 3)
        C = colmajor_copy(C0)
        fmm.matmul(A, B, C, 1.0, 0.5)
        want.append(C)
        probs.append({"A": A, "B": B, "C": colmajor_copy(C0), "alg": fmm.CLASSICAL, "beta": 0.5,
                      "gemm_tile": ("large", "small")[i % 2]})
    fmm.fast_matmul_batched(probs)
    torch.cuda.synchronize()
    for p, w in zip(probs, want):
        assert torch.equal(p["C"], w)


def test_autotune_table_has_a_tile_column():
    h = fmm.Handle(0)
    h.bind_current_stream()
    try:
        fmm.autotune([(96, 96, 96), (300, 300, 300)], max_steps=1, handle=h)
        lines = [ln.split() for ln in fmm.autotune_table(handle=h).strip().splitlines()]
        assert lines and all(len(ln) == 6 for ln in lines)
        assert all(int(ln[5]) in (1, 2) for ln in lines)
        assert fmm.autotune_tile(96, 96, 96, handle=h) in ("large", "small")
        assert fmm.autotune_tile(5000, 5000, 5000, handle=h) == "auto"  # bucket not measured
        # a table without the tile column still loads
        fmm.autotune_load("7 7 7 -2 0\n", handle=h)
        assert fmm.autotune_tile(100, 100, 100, handle=h) == "auto"
    finally:
        h.close()
