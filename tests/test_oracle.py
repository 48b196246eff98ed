"""Pins the CPU oracle to the reference.

* the seeded generator against its known answer;
* the C restatement against the golden vectors that the reference itself
  produced (tests/golden/make_golden.py);
* where the reference build oracle/_ref is present: the restatement with the
  reference's own leaf BLAS is bit-identical to the reference for every
  algorithm, and the reference reproduces the golden vectors bit for bit.
"""

import numpy as np
import pytest

import oracle
from helpers import decode_matrix, load_golden

G = load_golden()
FULL = [c for c in G["cases"] if c["kind"] == "full"]
DIGEST = [c for c in G["cases"] if c["kind"] == "digest"]
APPROX = {"bini322_10_52_approx", "schonhage333_21_117_approx", "smirnov333_20_182_approx"}


def inputs(c):
    A = oracle.uniform(c["m"], c["k"], c["seed"], 1)
    B = oracle.uniform(c["k"], c["n"], c["seed"], 2)
    C0 = oracle.uniform(c["m"], c["n"], c["seed"], 3)
    return A, B, C0


def classical(A, B, C0, alpha, beta):
    C = C0.copy(order="F")
    oracle.matmul(A, B, C, alpha, beta)
    return C


def test_generator_known_answer():
    ka = G["uniform_known_answer"]
    got = oracle.uniform(ka["rows"], ka["cols"], ka["seed"], ka["stream"])
    assert [float(v).hex() for v in got.T.ravel()] == ka["values"]


def test_generator_matches_c_implementation():
    import ctypes
    a = oracle.uniform(7, 5, 11, 2, -1.0, 1.0)
    b = np.zeros((7, 5), order="F")
    oracle.oracle_lib().oracle_fill_uniform(b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 35, 11, 2, -1.0, 1.0)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("c", FULL, ids=["%s-%dx%dx%d-s%d" % (c["alg"], c["m"], c["k"], c["n"], c["steps"]) for c in FULL])
def test_restatement_matches_reference_golden(c):
    A, B, C0 = inputs(c)
    C = C0.copy(order="F")
    oracle.fast_matmul(c["alg"], A, B, C, c["steps"], c["x"], c["alpha"], c["beta"])
    ref = decode_matrix(c["C"], c["m"], c["n"])
    if c["alg"] in APPROX:
        err = oracle.max_relative_diff(classical(A, B, C0, c["alpha"], c["beta"] if c["steps"] else 0.0), C)
        assert err <= 2.0 * c["ref_err"] + 1e-15
    else:
        assert oracle.max_relative_diff(ref, C) <= 1e-13


@pytest.mark.parametrize("c", DIGEST, ids=["%s-%dx%dx%d-s%d" % (c["alg"], c["m"], c["k"], c["n"], c["steps"]) for c in DIGEST])
def test_restatement_matches_reference_digests(c):
    A, B, C0 = inputs(c)
    C = C0.copy(order="F")
    oracle.fast_matmul(c["alg"], A, B, C, c["steps"], c["x"], c["alpha"], c["beta"])
    if c["alg"] in APPROX:
        err = oracle.max_relative_diff(classical(A, B, C0, 1.0, 0.0), C)
        assert err <= 2.0 * c["ref_err"] + 1e-15
        return
    colsum = np.array([float.fromhex(v) for v in c["colsum"]])
    assert np.max(np.abs(C.sum(axis=0)[: len(colsum)] - colsum) / np.abs(colsum)) <= 1e-13
    for i, j, v in c["samples"]:
        want = float.fromhex(v)
        assert abs(C[i, j] - want) <= 1e-13 * abs(want)


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
def test_reference_build_reproduces_golden():
    oracle.ref_lib().fmmref_set_threads(1)
    for c in FULL:
        A, B, C0 = inputs(c)
        C = C0.copy(order="F")
        oracle.ref_fast_matmul(c["alg"], A, B, C, c["steps"], c["x"], c["alpha"], c["beta"])
        assert np.array_equal(C, decode_matrix(c["C"], c["m"], c["n"])), c["alg"]


@needs_ref
def test_restatement_is_bit_exact_with_reference_leaves():
    """Same leaf BLAS => every addition, multiplier and fringe identical."""
    L = oracle.oracle_lib()
    oracle.ref_lib().fmmref_set_threads(1)
    oracle.use_reference_leaf(True)
    try:
        for i in range(L.oracle_num_algorithms()):
            alg = L.oracle_algorithm_name(i).decode()
            for (m, k, n, steps, alpha, beta) in [(57, 40, 35, 2, 1.0, 0.0), (30, 33, 29, 3, -1.2, 2.5),
                                                  (67, 91, 55, 1, 7.0, -1.3)]:
                A = oracle.uniform(m, k, 3, 1)
                B = oracle.uniform(k, n, 3, 2)
                C0 = oracle.uniform(m, n, 3, 3)
                x = 1e-4 if alg in APPROX else 1e-8
                C1 = C0.copy(order="F")
                C2 = C0.copy(order="F")
                oracle.ref_fast_matmul(alg, A, B, C1, steps, x, alpha, beta)
                oracle.fast_matmul(alg, A, B, C2, steps, x, alpha, beta)
                assert np.array_equal(C1, C2, equal_nan=True), (alg, m, k, n, steps)
    finally:
        oracle.use_reference_leaf(False)


def test_quad_oracle_is_exact_on_integer_products_and_sees_fp64_rounding():
    """The quad-precision sampled-entry check (linalg/quadmatmul.hpp restated):
    zero error on integer matrices (every product and sum exact), a small
    nonzero error for an FP64 product, a planted 1e-10 error found as such,
    and agreement with exact rational sums (fractions) on a few entries."""
    from fractions import Fraction

    rng = np.random.default_rng(5)
    m, k, n = 40, 300, 30
    Ai = np.asfortranarray(rng.integers(-1000, 1000, (m, k)).astype(np.float64))
    Bi = np.asfortranarray(rng.integers(-1000, 1000, (k, n)).astype(np.float64))
    exact = (Ai.astype(np.int64) @ Bi.astype(np.int64)).astype(np.float64)
    rows = rng.integers(0, m, 50)
    cols = rng.integers(0, n, 50)
    rel, scaled = oracle.quad_errors(Ai, Bi, rows, cols, exact[rows, cols])
    assert rel == 0.0 and scaled == 0.0

    A = oracle.uniform(m, k, 9, 1)
    B = oracle.uniform(k, n, 9, 2)
    C = np.zeros((m, n), order="F")
    oracle.matmul(A, B, C)
    rel, scaled = oracle.quad_errors(A, B, rows, cols, C[rows, cols])
    assert 0.0 < rel <= k * 2.0 ** -53 and scaled <= rel
    bad = C[rows, cols].copy()
    bad[7] *= 1.0 + 1e-10
    rel_bad, _ = oracle.quad_errors(A, B, rows, cols, bad)
    assert 0.5e-10 < rel_bad < 2e-10

    # exactly rounded rational sums measure within one rounding of the quad result
    ex = [float(sum(Fraction(A[i, l]) * Fraction(B[l, j]) for l in range(k))) for i, j in zip(rows[:8], cols[:8])]
    rel_ex, _ = oracle.quad_errors(A, B, rows[:8], cols[:8], ex)
    assert rel_ex <= 2.0 ** -53


def scaled_normal(m, n, seed, per):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((m, n))
    e = rng.integers(-16, 17, m if per == "row" else n)
    X *= np.exp2(e)[:, None] if per == "row" else np.exp2(e)[None, :]
    return np.asfortranarray(X)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build not present")
@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_scaling_restatement_equals_reference_bit_for_bit(kind):
    """oracle_scaling / oracle_scaling_postprocess against the reference's
    Scaling<double> / PostProcessScaling (scaling/scaling.hpp)."""
    for steps in (1, 2, 3):
        A = scaled_normal(37, 53, kind + 10 * steps, "row")
        B = scaled_normal(53, 29, kind + 10 * steps + 1, "col")
        A1, B1 = A.copy(order="F"), B.copy(order="F")
        A2, B2 = A.copy(order="F"), B.copy(order="F")
        r1, s1 = oracle.scaling(A1, B1, steps, kind)
        r2, s2 = oracle.scaling(A2, B2, steps, kind, ref=True)
        for x, y in [(A1, A2), (B1, B2), (r1, r2), (s1, s2)]:
            assert np.array_equal(x, y), (kind, steps)
        C1 = A1 @ B1
        C2 = np.asfortranarray(C1.copy())
        C1 = np.asfortranarray(C1)
        oracle.scaling_postprocess(C1, r1, s1)
        oracle.scaling_postprocess(C2, r2, s2, ref=True)
        assert np.array_equal(C1, C2)
        # the unscaled product is recovered (up to rounding)
        assert np.abs(C1 - A @ B).max() <= 1e-13 * np.abs(A @ B).max()


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build not present")
def test_scaling_multiplies_into_vectors_that_arrive_sized():
    """Scaling's r_vals.resize(m, 1.0) keeps the entries of vectors that
    arrive sized; the outer maxima are multiplied into them."""
    A = scaled_normal(20, 30, 1, "row")
    B = scaled_normal(30, 25, 2, "col")
    r0 = np.linspace(0.5, 3.0, 20)
    s0 = np.linspace(1.5, 0.25, 25)
    A1, B1, A2, B2 = A.copy(order="F"), B.copy(order="F"), A.copy(order="F"), B.copy(order="F")
    r1, s1 = oracle.scaling(A1, B1, 2, 0, r=r0, s=s0)
    r2, s2 = oracle.scaling(A2, B2, 2, 0, ref=True, r=r0, s=s0)
    assert np.array_equal(r1, r2) and np.array_equal(s1, s2)
    assert not np.array_equal(r1, oracle.scaling(A.copy(order="F"), B.copy(order="F"), 2, 0)[0])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build not present")
def test_reference_fp32_build_rounds_in_fp32():
    """The reference's FastMatmul<float> / MatMul<float> (sgemm) built here:
    errors of FP32 arithmetic against the exact product of the FP32 inputs."""
    n = 256
    A = np.asfortranarray(oracle.uniform(n, n, 1, 1).astype(np.float32))
    B = np.asfortranarray(oracle.uniform(n, n, 1, 2).astype(np.float32))
    want = A.astype(np.float64) @ B.astype(np.float64)
    C = np.zeros((n, n), dtype=np.float32, order="F")
    oracle.ref_fast_matmul_f32("strassen", A, B, C, 2)
    e = float((np.abs(C - want) / want).max())
    assert 1e-8 < e < 1e-4, e
    C[:] = 0
    oracle.ref_matmul_f32(A, B, C)
    e = float((np.abs(C - want) / want).max())
    assert 1e-9 < e < 1e-5, e
