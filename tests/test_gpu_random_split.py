"""Seeded random split products against the CPU model of the split arithmetic.

Shapes, digit kinds (BF16 with 2-6 slices, INT8 with 2-8), alpha and beta
drawn from a fixed seed.  A classical split product must equal the model
(tests/native/plan_emulator.cpp) bit for bit: exact integer sums per group,
the recombination in a fixed order.  A FastMatmul with split leaves must stay
within 1e-14 of the model's run of the same program -- its fringe products
are FP64 and summed in another order than the model's loops -- with every
schedule giving the same bits.
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
INT8 = 16  # split code offset of INT8 digits


def draw(count, seed, fast):
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(count):
        base = float(np.exp(rng.uniform(np.log(8), np.log(340))))
        m, k, n = (max(1, int(base * f)) for f in rng.uniform(0.5, 1.5, 3))
        code = int(rng.integers(2, 7)) if i % 2 == 0 else INT8 + int(rng.integers(2, 9))
        alpha = float(rng.choice([1.0, -0.75, 3.0]))
        beta = float(rng.choice([0.0, 1.0, 0.5]))
        alg = ["strassen", "grey333_23_125", "grey424_26_206"][i % 3] if fast else None
        steps = int(rng.integers(1, 3)) if fast else 0
        cases.append((alg, m, k, n, steps, code, alpha, beta, 300 + i))
    return cases


GEMM_CASES = draw(16, 77, False)
FAST_CASES = draw(9, 78, True)


def cid(c):
    kind = "i8s%d" % (c[5] - INT8) if c[5] >= INT8 else "bf16s%d" % c[5]
    return "%s-%dx%dx%d-%s" % ((c[0] or "classical"), c[1], c[2], c[3], kind)


def run_gpu(alg, A, B, C0, steps, code, alpha, beta, schedule="auto"):
    Cd = to_device(C0)
    dA, dB = to_device(A), to_device(B)
    slices = code - INT8 if code >= INT8 else code
    prec = "split_int8" if code >= INT8 else "split_bf16"
    if alg is None:
        (fmm.matmul_split_int8 if code >= INT8 else fmm.matmul_split_bf16)(dA, dB, Cd, alpha, beta, slices)
    else:
        fmm.fast_matmul(alg, dA, dB, Cd, steps, 1e-8, alpha, beta, schedule=schedule, precision=prec,
                        split_slices=slices)
    fmm.synchronize()
    return to_host(Cd)


@pytest.mark.parametrize("case", GEMM_CASES, ids=[cid(c) for c in GEMM_CASES])
def test_random_split_gemm_equals_the_model(case):
    _, m, k, n, _, code, alpha, beta, seed = case
    A = oracle.uniform(m, k, seed, 1, -1.0, 1.0)
    B = oracle.uniform(k, n, seed, 2, -1.0, 1.0)
    C0 = oracle.uniform(m, n, seed, 3)
    want = C0.copy(order="F")
    emulator().emu_split_gemm(m, k, n, A.ctypes.data_as(P), m, B.ctypes.data_as(P), k, want.ctypes.data_as(P), m,
                              alpha, beta, code)
    got = run_gpu(None, A, B, C0, 0, code, alpha, beta)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("case", FAST_CASES, ids=[cid(c) for c in FAST_CASES])
def test_random_split_fast_matmul_stays_with_the_model(case):
    alg, m, k, n, steps, code, alpha, beta, seed = case
    A = oracle.uniform(m, k, seed, 1)
    B = oracle.uniform(k, n, seed, 2)
    C0 = oracle.uniform(m, n, seed, 3)
    want = C0.copy(order="F")
    stats = (ctypes.c_int64 * 5)()
    rc = emulator().emu_fast_matmul_split(fmm.algorithm_index(alg), A.ctypes.data_as(P), m, B.ctypes.data_as(P), k,
                                          want.ctypes.data_as(P), m, m, k, n, steps, 1e-8, alpha, beta, 0, code,
                                          stats)
    assert rc == 0
    got = {s: run_gpu(alg, A, B, C0, steps, code, alpha, beta, s) for s in ("bfs", "dfs")}
    assert np.array_equal(got["bfs"], got["dfs"])
    assert float(np.abs(got["bfs"] - want).max() / np.abs(want).max()) <= 1e-14
