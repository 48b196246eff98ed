"""GPU parity of the split-INT8 leaf products (tcgen05 kind::i8).

The device result equals the CPU model of the split-INT8 arithmetic
(tests/native/plan_emulator.cpp: 7-bit signed digits, exact integer sums per
diagonal over groups of up to 32768 k, FP64 recombination in diagonal
order) bit for bit: the int32 accumulation is exact and the FP64 order is
fixed, so nothing may differ.  FastMatmul with split-INT8 leaves equals the
model's planner run bit for bit on every schedule, batches give each item
its alone result, and the error against the FP64 product stays within the
bound.

Tolerances: bit-exact against the model; against the FP64 result
max_ij |C - D| / max |D| <= 1e-11 at 6 slices and <= 1e-12 at 7 for exact
algorithms on uniform [0, 1) inputs.
"""

import ctypes

import numpy as np
import pytest

import oracle
from helpers import emulator, gpu_available, to_device, to_host

pytestmark = pytest.mark.gpu

if gpu_available():
    import fast_matmul_b200 as fmm

P = ctypes.POINTER(ctypes.c_double)
I8 = 16  # the planner's split code of INT8 digits: 16 + slices


def model_gemm(A, B, C0, alpha, beta, slices):
    E = emulator()
    m, k = A.shape
    n = B.shape[1]
    C = C0.copy(order="F")
    E.emu_split_gemm(m, k, n, A.ctypes.data_as(P), max(m, 1), B.ctypes.data_as(P), max(k, 1), C.ctypes.data_as(P),
                     max(m, 1), alpha, beta, I8 + slices)
    return C


def model_fast(alg, A, B, C0, steps, x, alpha, beta, d, slices):
    E = emulator()
    idx = fmm.algorithm_index(alg)
    m, k = A.shape
    n = B.shape[1]
    C = C0.copy(order="F")
    stats = (ctypes.c_int64 * 5)()
    rc = E.emu_fast_matmul_split(idx, A.ctypes.data_as(P), m, B.ctypes.data_as(P), k, C.ctypes.data_as(P), m, m, k,
                                 n, steps, x, alpha, beta, d, I8 + slices, stats)
    assert rc == 0
    return C


def test_int8_small_product_equals_model():
    A = oracle.uniform(256, 256, 1, 1)
    B = oracle.uniform(256, 128, 1, 2)
    Cd = to_device(np.zeros((256, 128), order="F"))
    fmm.matmul_split_int8(to_device(A), to_device(B), Cd, slices=6)
    fmm.synchronize()
    assert np.array_equal(to_host(Cd), model_gemm(A, B, np.zeros((256, 128), order="F"), 1.0, 0.0, 6))


SHAPES = [(1, 1, 1), (128, 128, 128), (130, 257, 129), (3, 0, 2), (200, 1000, 70), (520, 390, 300), (64, 64, 700),
          (40, 33000, 24)]


@pytest.mark.parametrize("shape", SHAPES, ids=["%dx%dx%d" % s for s in SHAPES])
def test_int8_gemm_equals_model_bit_exact(shape):
    m, k, n = shape
    A = oracle.uniform(m, k, 5, 1) if k else np.zeros((m, 0), order="F")
    B = oracle.uniform(k, n, 5, 2) if k else np.zeros((0, n), order="F")
    C0 = oracle.uniform(m, n, 5, 3)
    cases = [(6, 1.0, 0.0), (8, -0.75, 1.5), (2, 2.0, 0.0), (4, 1.0, -1.0)]
    if k > 30000:
        cases = cases[:2]  # two int32 groups per diagonal; the model is slow at this depth
    for slices, alpha, beta in cases:
        Cd = to_device(C0)
        fmm.matmul_split_int8(to_device(A), to_device(B), Cd, alpha, beta, slices)
        fmm.synchronize()
        got = to_host(Cd)
        want = model_gemm(A, B, C0, alpha, beta, slices)
        assert np.array_equal(got, want), (shape, slices, float(np.abs(got - want).max()))


def test_int8_gemm_scaled_normal_inputs():
    rng = np.random.default_rng(9)
    m, k, n = 300, 640, 260
    A = np.asfortranarray(rng.standard_normal((m, k)) * np.exp2(rng.integers(-16, 17, (m, 1))))
    B = np.asfortranarray(rng.standard_normal((k, n)) * np.exp2(rng.integers(-16, 17, (1, n))))
    C0 = np.zeros((m, n), order="F")
    Cd = to_device(C0)
    fmm.matmul_split_int8(to_device(A), to_device(B), Cd, slices=7)
    fmm.synchronize()
    got = to_host(Cd)
    assert np.array_equal(got, model_gemm(A, B, C0, 1.0, 0.0, 7))
    den = k * np.outer(np.abs(A).max(axis=1), np.abs(B).max(axis=0))
    assert float((np.abs(got - A @ B) / den).max()) <= 9.0 * 2.0 ** -49 + 1e-15


CASES = [("strassen", 2, (300, 520, 276)), ("grey424_26_206", 1, (256, 512, 256)), ("grey333_23_125", 2, (189, 198, 171))]


@pytest.mark.parametrize("case", CASES, ids=["%s-s%d-%dx%dx%d" % ((c[0], c[1]) + c[2]) for c in CASES])
def test_int8_fast_matmul_equals_model_every_schedule(case):
    alg, steps, (m, k, n) = case
    A = oracle.uniform(m, k, 6, 1)
    B = oracle.uniform(k, n, 6, 2)
    C0 = oracle.uniform(m, n, 6, 3)
    want = model_fast(alg, A, B, C0, steps, 1e-8, 1.0, 0.5, 0, 6)
    for sched in ("dfs", "bfs", "hybrid"):
        Cd = to_device(C0)
        fmm.fast_matmul(alg, to_device(A), to_device(B), Cd, steps, 1e-8, 1.0, 0.5, schedule=sched,
                        precision="split_int8", split_slices=6)
        fmm.synchronize()
        assert np.array_equal(to_host(Cd), want), sched
    exact = C0.copy(order="F")
    oracle.fast_matmul(alg, A, B, exact, steps, 1e-8, 1.0, 0.5)
    assert float(np.abs(want - exact).max() / np.abs(exact).max()) <= 1e-11


def test_int8_strassen_error_at_size():
    n = 2048
    A = fmm.random_matrix(n, n, 17, 1)
    B = fmm.random_matrix(n, n, 17, 2)
    ref = fmm.colmajor_empty(n, n)
    fmm.matmul(A, B, ref)
    for slices, tol in [(6, 1e-11), (7, 1e-12)]:
        C = fmm.colmajor_empty(n, n)
        fmm.fast_matmul("strassen", A, B, C, 2, precision="split_int8", split_slices=slices)
        fmm.synchronize()
        rel, _ = fmm.max_relative_diff(ref, C)
        assert rel <= tol, (slices, rel)


def test_int8_batch_items_equal_their_single_calls():
    import torch

    dims = [(90, 300, 80), (257, 129, 130), (64, 700, 33)]
    ops = []
    for i, (m, k, n) in enumerate(dims):
        ops.append((to_device(oracle.uniform(m, k, 8, 3 * i)), to_device(oracle.uniform(k, n, 8, 3 * i + 1)),
                    oracle.uniform(m, n, 8, 3 * i + 2)))
    singles = []
    for A, B, C0 in ops:
        Cd = to_device(C0)
        fmm.fast_matmul("strassen", A, B, Cd, 1, 1e-8, 1.0, 0.25, precision="split_int8", split_slices=6)
        singles.append(Cd)
    batch = [{"alg": "strassen", "num_steps": 1, "A": A, "B": B, "C": to_device(C0), "alpha": 1.0, "beta": 0.25,
              "precision": "split_int8", "split_slices": 6} for A, B, C0 in ops]
    fmm.fast_matmul_batched(batch)
    torch.cuda.synchronize()
    for item, single in zip(batch, singles):
        assert torch.equal(item["C"], single)


def test_int8_slice_count_out_of_range_is_rejected():
    A = to_device(oracle.uniform(8, 8, 1, 1))
    B = to_device(oracle.uniform(8, 8, 1, 2))
    C = to_device(np.zeros((8, 8), order="F"))
    with pytest.raises(fmm.FmmError):
        fmm.matmul_split_int8(A, B, C, slices=9)
    with pytest.raises(fmm.FmmError):
        fmm.fast_matmul("strassen", A, B, C, 1, precision="split_int8", split_slices=1)


def test_int8_requests_in_the_server_equal_alone():
    """Split-INT8, split-BF16 and FP64 requests mixed in one server: each
    result equals the same product computed alone."""
    import torch

    rng = np.random.default_rng(5)
    reqs = []
    for i in range(12):
        m, k, n = (int(v) for v in rng.integers(100, 700, 3))
        A = fmm.random_matrix(m, k, 23, 3 * i)
        B = fmm.random_matrix(k, n, 23, 3 * i + 1)
        prec, sl = [("split_int8", 6), ("split_bf16", 5), ("fp64", 0)][i % 3]
        reqs.append((A, B, prec, sl))
    alone = []
    for A, B, prec, sl in reqs:
        C = fmm.colmajor_empty(A.shape[0], B.shape[1], A.device)
        fmm.fast_matmul("strassen", A, B, C, 1, precision=prec, split_slices=sl)
        alone.append(C)
    fmm.synchronize()
    srv = fmm.Server(workspace_bytes=4 << 30, max_inflight=3)
    try:
        outs, tickets = [], []
        for A, B, prec, sl in reqs:
            C = fmm.colmajor_empty(A.shape[0], B.shape[1], A.device)
            tickets.append(srv.submit(A, B, C, alg="strassen", num_steps=1, precision=prec, split_slices=sl))
            outs.append(C)
        for t in tickets:
            assert srv.wait(t, 60000.0)["status"] == 0
    finally:
        srv.close()
    for a, o in zip(alone, outs):
        assert torch.equal(a, o)
