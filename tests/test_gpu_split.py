"""GPU parity of the split-BF16 leaf products (tcgen05 tensor cores).

* the device result equals the CPU model of the split arithmetic
  (tests/native/plan_emulator.cpp) bit for bit: the FP32 accumulation of
  every diagonal and k-chunk is exact and the FP64 recombination runs in a
  fixed order, so nothing may differ -- deep k and Inf / NaN inputs (NaN in
  every entry they reach) included;
* FastMatmul with split leaves equals the model's planner run bit for bit
  (every schedule), and stays within the stated error of the FP64 oracle;
* batches and the request server give every split item the result it gets
  alone;
* the bounded waits give up and report instead of hanging.

Tolerances: bit-exact against the model; against the FP64 result
max_ij |C - D| / max |D| <= 1e-12 at 6 slices and <= 1e-11 at 5 slices for
exact algorithms on uniform [0, 1) inputs (approximate algorithms: divided
by their lambda).
"""

import ctypes

import numpy as np
import pytest

import oracle
from helpers import emulator, gpu_available, to_device, to_host

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm

P = ctypes.POINTER(ctypes.c_double)


def model_gemm(A, B, C0, alpha, beta, slices):
    E = emulator()
    m, k = A.shape
    n = B.shape[1]
    C = C0.copy(order="F")
    E.emu_split_gemm(m, k, n, A.ctypes.data_as(P), max(m, 1), B.ctypes.data_as(P), max(k, 1), C.ctypes.data_as(P),
                     max(m, 1), alpha, beta, slices)
    return C


def model_fast(alg, A, B, C0, steps, x, alpha, beta, d, slices):
    E = emulator()
    idx = fmm.algorithm_index(alg)
    m, k = A.shape
    n = B.shape[1]
    C = C0.copy(order="F")
    stats = (ctypes.c_int64 * 5)()
    rc = E.emu_fast_matmul_split(idx, A.ctypes.data_as(P), m, B.ctypes.data_as(P), k, C.ctypes.data_as(P), m, m, k,
                                 n, steps, x, alpha, beta, d, slices, stats)
    assert rc == 0
    return C


def test_bounded_wait_gives_up_and_the_context_stays_usable():
    h = fmm.default_handle()
    code = ctypes.c_int(0)
    fmm.lib().fmm_selftest_wait_timeout(h.ptr, 20.0, ctypes.byref(code))
    assert code.value == 99
    # the device keeps working afterwards
    A = oracle.uniform(40, 50, 1, 1)
    B = oracle.uniform(50, 30, 1, 2)
    Cd = to_device(np.zeros((40, 30), order="F"))
    fmm.matmul_split_bf16(to_device(A), to_device(B), Cd, slices=4)
    fmm.synchronize()
    assert np.array_equal(to_host(Cd), model_gemm(A, B, np.zeros((40, 30), order="F"), 1.0, 0.0, 4))


SHAPES = [(1, 1, 1), (128, 128, 128), (130, 257, 129), (3, 0, 2), (200, 1000, 70), (520, 390, 300), (64, 64, 700)]


@pytest.mark.parametrize("shape", SHAPES, ids=["%dx%dx%d" % s for s in SHAPES])
def test_split_gemm_equals_model_bit_exact(shape):
    m, k, n = shape
    A = oracle.uniform(m, k, 3, 1) if k else np.zeros((m, 0), order="F")
    B = oracle.uniform(k, n, 3, 2) if k else np.zeros((0, n), order="F")
    C0 = oracle.uniform(m, n, 3, 3)
    for slices, alpha, beta in [(5, 1.0, 0.0), (6, -0.75, 1.5), (2, 2.0, 0.0), (3, 1.0, -1.0)]:
        Cd = to_device(C0)
        fmm.matmul_split_bf16(to_device(A), to_device(B), Cd, alpha, beta, slices)
        fmm.synchronize()
        got = to_host(Cd)
        want = model_gemm(A, B, C0, alpha, beta, slices)
        assert np.array_equal(got, want), (shape, slices, float(np.abs(got - want).max()))


@pytest.mark.parametrize("slices", [3, 5])
def test_split_gemm_deep_k_equals_model(slices):
    # k = 33000: 258 chunks (3 slices: 129 chunk pairs)
    m, k, n = 40, 33000, 36
    A = oracle.uniform(m, k, 12, 1)
    B = oracle.uniform(k, n, 12, 2)
    C0 = oracle.uniform(m, n, 12, 3)
    Cd = to_device(C0)
    fmm.matmul_split_bf16(to_device(A), to_device(B), Cd, 1.25, -0.5, slices)
    fmm.synchronize()
    got = to_host(Cd)
    assert np.array_equal(got, model_gemm(A, B, C0, 1.25, -0.5, slices))
    want = 1.25 * (A @ B) - 0.5 * C0
    assert float(np.abs(got - want).max() / np.abs(want).max()) <= 3.0 * k * 2.0 ** (-8 * slices)


@pytest.mark.parametrize("code", [5, 6, 16 + 6], ids=["bf16-s5", "bf16-s6", "int8-s6"])
def test_split_gemm_non_finite_inputs_give_nan_where_they_reach(code):
    m, k, n = 300, 500, 260
    A = oracle.uniform(m, k, 13, 1)
    B = oracle.uniform(k, n, 13, 2)
    A[7, 33] = np.nan
    A[150, 0] = np.inf
    B[499, 5] = -np.inf
    B[250, 259] = np.nan
    C0 = oracle.uniform(m, n, 13, 3)
    Cd = to_device(C0)
    if code >= 16:
        fmm.matmul_split_int8(to_device(A), to_device(B), Cd, 1.0, 0.5, code - 16)
    else:
        fmm.matmul_split_bf16(to_device(A), to_device(B), Cd, 1.0, 0.5, code)
    fmm.synchronize()
    got = to_host(Cd)
    bad = np.zeros((m, n), bool)
    bad[[7, 150], :] = True
    bad[:, [5, 259]] = True
    assert np.array_equal(np.isnan(got), bad)
    assert np.array_equal(got, model_gemm(A, B, C0, 1.0, 0.5, code), equal_nan=True)
    # the other entries are those of the inputs with the bad rows and columns cleared
    A2, B2 = A.copy(order="F"), B.copy(order="F")
    A2[[7, 150], :] = 0.0
    B2[:, [5, 259]] = 0.0
    clean = model_gemm(A2, B2, C0, 1.0, 0.5, code)
    assert np.array_equal(got[~bad], clean[~bad])


def test_split_gemm_scaled_normal_inputs():
    rng = np.random.default_rng(7)
    m, k, n = 300, 640, 260
    A = np.asfortranarray(rng.standard_normal((m, k)) * np.exp2(rng.integers(-16, 17, (m, 1))))
    B = np.asfortranarray(rng.standard_normal((k, n)) * np.exp2(rng.integers(-16, 17, (1, n))))
    C0 = np.zeros((m, n), order="F")
    Cd = to_device(C0)
    fmm.matmul_split_bf16(to_device(A), to_device(B), Cd, slices=6)
    fmm.synchronize()
    got = to_host(Cd)
    assert np.array_equal(got, model_gemm(A, B, C0, 1.0, 0.0, 6))
    den = k * np.outer(np.abs(A).max(axis=1), np.abs(B).max(axis=0))
    assert float((np.abs(got - A @ B) / den).max()) <= 3.0 * 2.0 ** -48 + 1e-15


# Dimensions divisible by the algorithm's blocks at every level: no dynamic
# peeling, so every product is a split product and the result is bit-exact.
# With peeling, the FP64 fringe products (device DMMA against the model's
# loop) differ in summation order, so those cases compare within 1e-14.
CASES = [("strassen", 2, 1e-8, (300, 260, 276), True), ("grey424_26_206", 1, 1e-8, (256, 256, 256), True),
         ("grey333_23_125", 2, 1e-8, (189, 198, 171), True),
         ("bini322_10_52_approx", 1, 2.0 ** -13, (150, 120, 140), True),
         ("strassen", 2, 1e-8, (301, 259, 277), False), ("grey333_23_125", 2, 1e-8, (190, 200, 170), False),
         ("strassen", 2, 1e-8, (7, 5, 3), False)]


@pytest.mark.parametrize("case", CASES, ids=["%s-s%d-%dx%dx%d" % ((c[0], c[1]) + c[3]) for c in CASES])
def test_split_fast_matmul_equals_model_every_schedule(case):
    alg, steps, x, (m, k, n), exact = case
    A = oracle.uniform(m, k, 5, 1)
    B = oracle.uniform(k, n, 5, 2)
    C0 = oracle.uniform(m, n, 5, 3)
    want = model_fast(alg, A, B, C0, steps, x, 1.0, 0.5, 0, 5)
    results = []
    for sched in ("bfs", "dfs", "hybrid"):
        Cd = to_device(C0)
        fmm.fast_matmul(alg, to_device(A), to_device(B), Cd, steps, x, 1.0, 0.5, schedule=sched,
                        precision="split_bf16", split_slices=5)
        fmm.synchronize()
        got = to_host(Cd)
        if exact:
            assert np.array_equal(got, want), sched
        else:
            assert float(np.abs(got - want).max() / np.abs(want).max()) <= 1e-14, sched
        results.append(got)
    for r in results[1:]:
        assert np.array_equal(results[0], r)  # every schedule runs the same products


def test_split_strassen_error_against_fp64_at_2048():
    n = 2048
    torch.manual_seed(0)
    A = fmm.random_matrix(n, n, 11, 1)
    B = fmm.random_matrix(n, n, 11, 2)
    ref = fmm.colmajor_empty(n, n, A.device)
    fmm.matmul(A, B, ref)
    for slices, tol in [(6, 1e-12), (5, 1e-11)]:
        for steps in (1, 2):
            C = fmm.colmajor_empty(n, n, A.device)
            fmm.fast_matmul("strassen", A, B, C, steps, precision="split_bf16", split_slices=slices)
            fmm.synchronize()
            rel, _ = fmm.max_relative_diff(ref, C)
            assert rel <= tol, (slices, steps, rel)


def test_split_batch_items_equal_their_single_calls():
    shapes = [(100, 80, 90), (257, 64, 33), (64, 300, 128), (20, 20, 20)]
    problems, singles = [], []
    for i, (m, k, n) in enumerate(shapes):
        A = to_device(oracle.uniform(m, k, 9, 3 * i))
        B = to_device(oracle.uniform(k, n, 9, 3 * i + 1))
        C0 = oracle.uniform(m, n, 9, 3 * i + 2)
        prec = "split_bf16" if i % 2 == 0 else "fp64"
        alg = "strassen" if i < 2 else fmm.CLASSICAL
        problems.append(dict(A=A, B=B, C=to_device(C0), alg=alg, num_steps=1, beta=0.5, precision=prec,
                             split_slices=6))
        Cs = to_device(C0)
        if alg == fmm.CLASSICAL:
            if prec == "fp64":
                fmm.matmul(A, B, Cs, 1.0, 0.5)
            else:
                fmm.matmul_split_bf16(A, B, Cs, 1.0, 0.5, 6)
        else:
            fmm.fast_matmul(alg, A, B, Cs, 1, beta=0.5, precision=prec, split_slices=6)
        singles.append(Cs)
    fmm.fast_matmul_batched(problems)
    fmm.synchronize()
    for p, s in zip(problems, singles):
        assert torch.equal(p["C"], s)


def test_split_requests_in_the_server_equal_alone():
    rng = np.random.default_rng(3)
    reqs = []
    for i in range(12):
        m, k, n = (int(v) for v in rng.integers(100, 700, 3))
        A = fmm.random_matrix(m, k, 21, 3 * i)
        B = fmm.random_matrix(k, n, 21, 3 * i + 1)
        prec = "split_bf16" if i % 3 == 0 else "fp64"
        reqs.append((A, B, prec))
    alone = []
    for A, B, prec in reqs:
        C = fmm.colmajor_empty(A.shape[0], B.shape[1], A.device)
        fmm.fast_matmul("strassen", A, B, C, 1, precision=prec, split_slices=5)
        alone.append(C)
    fmm.synchronize()
    srv = fmm.Server(workspace_bytes=4 << 30, max_inflight=3)
    try:
        outs, tickets = [], []
        for A, B, prec in reqs:
            C = fmm.colmajor_empty(A.shape[0], B.shape[1], A.device)
            tickets.append(srv.submit(A, B, C, alg="strassen", num_steps=1, precision=prec, split_slices=5))
            outs.append(C)
        for t in tickets:
            assert srv.wait(t, 60000.0)["status"] == 0
    finally:
        srv.close()
    for a, o in zip(alone, outs):
        assert torch.equal(a, o)


def test_split_cuda_graph_plan_equals_direct_call():
    m, k, n = 384, 320, 352
    A = fmm.random_matrix(m, k, 4, 1)
    B = fmm.random_matrix(k, n, 4, 2)
    direct = fmm.colmajor_empty(m, n, A.device)
    fmm.fast_matmul("strassen", A, B, direct, 2, precision="split_bf16", split_slices=5)
    C = fmm.colmajor_empty(m, n, A.device)
    plan = fmm.Plan.for_product("strassen", A, B, C, 2, precision="split_bf16", split_slices=5)
    try:
        plan.execute()
        plan.execute()
        fmm.synchronize()
    finally:
        plan.close()
    assert torch.equal(direct, C)
