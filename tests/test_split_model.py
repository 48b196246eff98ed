"""Split-BF16 leaf products, planned and executed on the CPU.

The test interpreter (tests/native/plan_emulator.cpp) models the device
arithmetic of the split-BF16 products exactly: power-of-two row / column
scaling, 8-bit digit slices, exact integer sums per diagonal and 128-deep
k-chunk, FP64 recombination in the device's order, NaN from Inf / NaN
inputs.  These tests check that
model against the FP64 oracle (error bound per slice count), that the
planner gives every schedule and batch the same split products, and that the
workspace query covers the split scratch.  The GPU tests compare the device
against the same model bit for bit.
"""

import ctypes

import numpy as np
import pytest

import oracle
from helpers import emulator

P = ctypes.POINTER(ctypes.c_double)
L_ORACLE = oracle.oracle_lib()
NAMES = [L_ORACLE.oracle_algorithm_name(i).decode() for i in range(L_ORACLE.oracle_num_algorithms())]


def split_gemm(E, A, B, C, alpha, beta, slices):
    m, k = A.shape
    n = B.shape[1]
    E.emu_split_gemm(m, k, n, A.ctypes.data_as(P), max(m, 1), B.ctypes.data_as(P), max(k, 1), C.ctypes.data_as(P),
                     max(m, 1), alpha, beta, slices)


def split_fast(E, alg, A, B, C, steps, x, alpha, beta, d, slices):
    m, k = A.shape
    n = B.shape[1]
    stats = (ctypes.c_int64 * 5)()
    rc = E.emu_fast_matmul_split(NAMES.index(alg), A.ctypes.data_as(P), m, B.ctypes.data_as(P), k,
                                 C.ctypes.data_as(P), m, m, k, n, steps, x, alpha, beta, d, slices, stats)
    assert rc == 0, rc
    return list(stats)


def scaled_error(A, B, got, want):
    """max_ij |got - want| / (k max_p |a_ip| max_p |b_pj|)."""
    k = A.shape[1]
    ra = np.abs(A).max(axis=1)
    cb = np.abs(B).max(axis=0)
    den = k * np.outer(ra, cb)
    return float((np.abs(got - want) / np.where(den > 0, den, 1.0)).max())


@pytest.mark.parametrize("slices", [2, 3, 4, 5, 6])
def test_split_product_within_its_error_bound(slices):
    E = emulator()
    rng = np.random.default_rng(slices)
    m, k, n = 70, 300, 45
    # N(0, 1) entries with per-row / per-column scales 2^U(-16, 16)
    A = np.asfortranarray(rng.standard_normal((m, k)) * np.exp2(rng.uniform(-16, 16, (m, 1))))
    B = np.asfortranarray(rng.standard_normal((k, n)) * np.exp2(rng.uniform(-16, 16, (1, n))))
    got = np.zeros((m, n), order="F")
    split_gemm(E, A, B, got, 1.0, 0.0, slices)
    want = A @ B
    err = scaled_error(A, B, got, want)
    # representation error 2^-(8S+1) per operand (relative to the row / column
    # maximum) on both sides plus the dropped diagonals, and the FP64 rounding
    assert err <= 3.0 * 2.0 ** (-8 * slices) + 1e-15, (slices, err)
    if slices >= 3:
        assert err <= 1e-5 * 2.0 ** (-8 * (slices - 3))


@pytest.mark.parametrize("code", [3, 5, 6, 16 + 6])
def test_non_finite_rows_and_columns_give_nan(code):
    E = emulator()
    m, k, n = 20, 300, 15
    A = oracle.uniform(m, k, 6, 1)
    B = oracle.uniform(k, n, 6, 2)
    A[3, 10] = np.nan
    B[0, 4] = np.inf
    got = np.zeros((m, n), order="F")
    split_gemm(E, A, B, got, 1.0, 0.0, code)
    bad = np.zeros((m, n), bool)
    bad[3, :] = True
    bad[:, 4] = True
    assert np.array_equal(np.isnan(got), bad)
    A[3, :] = 0.0
    B[:, 4] = 0.0
    clean = np.zeros((m, n), order="F")
    split_gemm(E, A, B, clean, 1.0, 0.0, code)
    assert np.array_equal(got[~bad], clean[~bad])


def test_more_slices_are_more_accurate():
    E = emulator()
    A = oracle.uniform(64, 256, 5, 1)
    B = oracle.uniform(256, 48, 5, 2)
    want = A @ B
    errs = []
    for s in range(2, 7):
        got = np.zeros((64, 48), order="F")
        split_gemm(E, A, B, got, 1.0, 0.0, s)
        errs.append(float(np.abs(got - want).max() / np.abs(want).max()))
    assert all(a > b for a, b in zip(errs[:3], errs[1:4])), errs
    # about 256x per slice: S = 5 near 1e-13, S = 6 near 1e-15 at k = 256
    assert errs[3] < 1e-12 and errs[4] < 1e-14, errs


def test_split_alpha_beta_and_ragged_shapes():
    E = emulator()
    for (m, k, n) in [(1, 1, 1), (3, 0, 2), (129, 131, 130), (5, 257, 1)]:
        A = oracle.uniform(m, k, 7, 1) if k else np.zeros((m, 0), order="F")
        B = oracle.uniform(k, n, 7, 2) if k else np.zeros((0, n), order="F")
        C0 = oracle.uniform(m, n, 7, 3)
        got = C0.copy(order="F")
        split_gemm(E, A, B, got, -1.5, 0.25, 6)
        want = -1.5 * (A @ B) + 0.25 * C0
        assert np.allclose(got, want, rtol=1e-13, atol=1e-13 * max(k, 1)), (m, k, n)


@pytest.mark.parametrize("alg,steps,x", [("strassen", 2, 1e-8), ("grey424_26_206", 1, 1e-8),
                                         ("grey333_23_125", 2, 1e-8), ("bini322_10_52_approx", 1, 2.0 ** -13)])
def test_split_fast_matmul_every_schedule_identical_and_close_to_oracle(alg, steps, x):
    E = emulator()
    m, k, n = 133, 150, 97
    A = oracle.uniform(m, k, 3, 1)
    B = oracle.uniform(k, n, 3, 2)
    C0 = oracle.uniform(m, n, 3, 3)
    want = C0.copy(order="F")
    oracle.fast_matmul(alg, A, B, want, steps, x, 1.0, 0.5)
    for slices, tol in [(5, 1e-11), (6, 1e-12)]:
        results = []
        for d in range(steps + 1):
            got = C0.copy(order="F")
            split_fast(E, alg, A, B, got, steps, x, 1.0, 0.5, d, slices)
            assert not np.isnan(got).any()
            results.append(got)
        for r in results[1:]:
            assert np.array_equal(results[0], r)
        rel = float(np.abs(results[0] - want).max() / np.abs(want).max())
        # approximate algorithms amplify leaf errors by their 1/x coefficients
        if "approx" in alg:
            tol /= x
        assert rel <= tol, (slices, rel)


def test_split_workspace_query_covers_the_program():
    E = emulator()
    for alg, steps in [("strassen", 3), ("grey424_26_206", 2), ("smirnov333_23_128", 1)]:
        idx = NAMES.index(alg)
        for d in range(steps + 1):
            q = E.emu_workspace_bytes_split(idx, 300, 260, 280, steps, d, 4)
            A = oracle.uniform(300, 260, 1, 1)
            B = oracle.uniform(260, 280, 1, 2)
            C = np.zeros((300, 280), order="F")
            st = split_fast(E, alg, A, B, C, steps, 1e-8, 1.0, 0.0, d, 4)
            assert st[4] == q, (alg, steps, d, st[4], q)
            assert q > E.emu_workspace_bytes(idx, 300, 260, 280, steps, d)


def test_split_batch_items_equal_their_single_calls():
    E = emulator()
    items = [("strassen", 2, (90, 70, 80), 5), (None, 0, (33, 40, 21), 6), ("grey424_26_206", 1, (64, 64, 64), 0),
             ("strassen", 1, (50, 44, 61), 5)]
    algs = (ctypes.c_int * len(items))(*[NAMES.index(a) if a else -1 for a, _, _, _ in items])
    steps = (ctypes.c_int * len(items))(*[s for _, s, _, _ in items])
    dims = (ctypes.c_int64 * (3 * len(items)))(*[v for _, _, d, _ in items for v in d])
    slices = (ctypes.c_int * len(items))(*[s for _, _, _, s in items])
    As, Bs, Cs = [], [], []
    for i, (_, _, (m, k, n), _) in enumerate(items):
        As.append(oracle.uniform(m, k, 11, 3 * i))
        Bs.append(oracle.uniform(k, n, 11, 3 * i + 1))
        Cs.append(oracle.uniform(m, n, 11, 3 * i + 2))
    Acat = np.concatenate([a.ravel(order="F") for a in As])
    Bcat = np.concatenate([b.ravel(order="F") for b in Bs])
    Ccat = np.concatenate([c.ravel(order="F") for c in Cs])
    off = lambda arrs: (ctypes.c_int64 * len(arrs))(*np.cumsum([0] + [a.size for a in arrs[:-1]]).tolist())
    stats = (ctypes.c_int64 * 5)()
    rc = E.emu_fast_matmul_batch_split(len(items), algs, steps, dims, Acat.ctypes.data_as(P), off(As),
                                       Bcat.ctypes.data_as(P), off(Bs), Ccat.ctypes.data_as(P), off(Cs), 1e-8, 1.0,
                                       0.75, slices, stats)
    assert rc == 0
    # FP64 leaves in one grouped GEMM, split leaves in one launch per slice count
    assert stats[1] == 3
    pos = 0
    for i, (alg, s, (m, k, n), sl) in enumerate(items):
        got = Ccat[pos:pos + m * n].reshape((m, n), order="F")
        pos += m * n
        want = Cs[i].copy(order="F")
        if alg is None:
            if sl:
                split_gemm(E, As[i], Bs[i], want, 1.0, 0.75, sl)
            else:
                want = As[i] @ Bs[i] + 0.75 * Cs[i]
        else:
            split_fast(E, alg, As[i], Bs[i], want, s, 1e-8, 1.0, 0.75, 0, sl)
        assert np.array_equal(got, want), i


# ---------------------------------------------------------------------------
# Split-INT8: the same scaling, 7-bit signed digits, exact int32 sums per
# diagonal over up to 32768 k, FP64 recombination.  The model passes the
# planner's split code (16 + slices) through every entry point.

I8 = 16


@pytest.mark.parametrize("slices", [2, 3, 4, 5, 6, 7, 8])
def test_int8_product_within_its_error_bound(slices):
    E = emulator()
    rng = np.random.default_rng(100 + slices)
    m, k, n = 70, 300, 45
    A = np.asfortranarray(rng.standard_normal((m, k)) * np.exp2(rng.uniform(-16, 16, (m, 1))))
    B = np.asfortranarray(rng.standard_normal((k, n)) * np.exp2(rng.uniform(-16, 16, (1, n))))
    got = np.zeros((m, n), order="F")
    split_gemm(E, A, B, got, 1.0, 0.0, I8 + slices)
    err = scaled_error(A, B, got, A @ B)
    # representation error 2^-7S per operand (relative to the row / column
    # maximum) on both sides, the dropped diagonals (S - 1 terms of at most
    # 2^-7S), and the FP64 rounding
    assert err <= (slices + 2) * 2.0 ** (-7 * slices) + 1e-15, (slices, err)


def test_int8_six_slices_match_five_bf16_slices():
    E = emulator()
    A = oracle.uniform(64, 512, 21, 1)
    B = oracle.uniform(512, 48, 21, 2)
    want = A @ B
    errs = {}
    for code in (5, I8 + 6, I8 + 7):
        got = np.zeros((64, 48), order="F")
        split_gemm(E, A, B, got, 1.0, 0.0, code)
        errs[code] = float(np.abs(got - want).max() / np.abs(want).max())
    assert errs[I8 + 6] < 2.0 * errs[5] and errs[I8 + 6] < 1e-12, errs
    assert errs[I8 + 7] < errs[I8 + 6] / 16, errs


def test_int8_sum_groups_past_32768_k():
    """k beyond one int32 group (128 chunks of 256): the second group is summed
    separately, and the result stays within the bound."""
    E = emulator()
    m, k, n = 6, 32768 + 300, 5
    A = oracle.uniform(m, k, 4, 1)
    B = oracle.uniform(k, n, 4, 2)
    got = np.zeros((m, n), order="F")
    split_gemm(E, A, B, got, 1.0, 0.0, I8 + 6)
    assert scaled_error(A, B, got, A @ B) <= 8 * 2.0 ** -42 + 1e-15


def test_int8_alpha_beta_and_ragged_shapes():
    E = emulator()
    for (m, k, n) in [(1, 1, 1), (3, 0, 2), (129, 257, 130), (5, 513, 1)]:
        A = oracle.uniform(m, k, 8, 1) if k else np.zeros((m, 0), order="F")
        B = oracle.uniform(k, n, 8, 2) if k else np.zeros((0, n), order="F")
        C0 = oracle.uniform(m, n, 8, 3)
        got = C0.copy(order="F")
        split_gemm(E, A, B, got, -1.5, 0.25, I8 + 8)
        want = -1.5 * (A @ B) + 0.25 * C0
        assert np.allclose(got, want, rtol=1e-13, atol=1e-13 * max(k, 1)), (m, k, n)


@pytest.mark.parametrize("alg,steps", [("strassen", 2), ("grey424_26_206", 1)])
def test_int8_fast_matmul_every_schedule_identical_and_close_to_oracle(alg, steps):
    E = emulator()
    m, k, n = 133, 150, 97
    A = oracle.uniform(m, k, 13, 1)
    B = oracle.uniform(k, n, 13, 2)
    C0 = oracle.uniform(m, n, 13, 3)
    want = C0.copy(order="F")
    oracle.fast_matmul(alg, A, B, want, steps, 1e-8, 1.0, 0.5)
    # 6 INT8 slices are about as accurate as 5 BF16 ones, 7 as 6
    for slices, tol in [(6, 1e-11), (7, 1e-12)]:
        results = []
        for d in range(steps + 1):
            got = C0.copy(order="F")
            split_fast(E, alg, A, B, got, steps, 1e-8, 1.0, 0.5, d, I8 + slices)
            results.append(got)
        for r in results[1:]:
            assert np.array_equal(results[0], r)
        assert float(np.abs(results[0] - want).max() / np.abs(want).max()) <= tol, slices


def test_int8_workspace_query_covers_the_program():
    E = emulator()
    idx = NAMES.index("strassen")
    for d in range(3):
        q = E.emu_workspace_bytes_split(idx, 300, 600, 280, 2, d, I8 + 6)
        A = oracle.uniform(300, 600, 2, 1)
        B = oracle.uniform(600, 280, 2, 2)
        C = np.zeros((300, 280), order="F")
        st = split_fast(E, "strassen", A, B, C, 2, 1e-8, 1.0, 0.0, d, I8 + 6)
        assert st[4] == q, (d, st[4], q)
        # six one-byte slices take less scratch than five two-byte ones
        assert q < E.emu_workspace_bytes_split(idx, 300, 600, 280, 2, d, 5)


def test_batch_mixing_int8_bf16_and_fp64_items_equals_single_calls():
    """One batch with INT8, BF16 and FP64 leaf products: one split launch per
    split code, each item equal to its own planner run."""
    E = emulator()
    items = [("strassen", 1, (90, 300, 80), I8 + 6), ("strassen", 1, (70, 260, 66), 5), (None, 0, (40, 520, 30), I8 + 7),
             ("grey424_26_206", 1, (64, 64, 64), 0)]
    algs = (ctypes.c_int * len(items))(*[NAMES.index(a) if a else -1 for a, _, _, _ in items])
    steps = (ctypes.c_int * len(items))(*[s for _, s, _, _ in items])
    dims = (ctypes.c_int64 * (3 * len(items)))(*[v for _, _, d, _ in items for v in d])
    codes = (ctypes.c_int * len(items))(*[c for _, _, _, c in items])
    As, Bs, Cs = [], [], []
    for i, (_, _, (m, k, n), _) in enumerate(items):
        As.append(oracle.uniform(m, k, 12, 3 * i))
        Bs.append(oracle.uniform(k, n, 12, 3 * i + 1))
        Cs.append(oracle.uniform(m, n, 12, 3 * i + 2))
    Acat = np.concatenate([a.ravel(order="F") for a in As])
    Bcat = np.concatenate([b.ravel(order="F") for b in Bs])
    Ccat = np.concatenate([c.ravel(order="F") for c in Cs])
    off = lambda arrs: (ctypes.c_int64 * len(arrs))(*np.cumsum([0] + [a.size for a in arrs[:-1]]).tolist())
    stats = (ctypes.c_int64 * 5)()
    rc = E.emu_fast_matmul_batch_split(len(items), algs, steps, dims, Acat.ctypes.data_as(P), off(As),
                                       Bcat.ctypes.data_as(P), off(Bs), Ccat.ctypes.data_as(P), off(Cs), 1e-8, 1.0,
                                       0.5, codes, stats)
    assert rc == 0
    # one FP64 grouped GEMM and one split launch per split code (three codes)
    assert stats[1] == 4
    pos = 0
    for i, (alg, s, (m, k, n), code) in enumerate(items):
        got = Ccat[pos:pos + m * n].reshape((m, n), order="F")
        pos += m * n
        want = Cs[i].copy(order="F")
        if alg is None:
            split_gemm(E, As[i], Bs[i], want, 1.0, 0.5, code)
        else:
            split_fast(E, alg, As[i], Bs[i], want, s, 1e-8, 1.0, 0.5, 0, code)
        assert np.array_equal(got, want), i
