"""GPU parity of the diagonal scaling (scaling/scaling.hpp).

* fmm_diagonal_scaling leaves A, B, r and s bit for bit as the oracle's C
  restatement does (itself pinned bit for bit against the reference's
  Scaling<double> in tests/test_oracle.py), for every scaling type, several
  step counts and ragged / empty shapes, NaN and infinite entries included;
* fmm_scaling_postprocess equals PostProcessScaling bit for bit;
* on operands whose rows, columns and inner dimension are skewed by powers
  of two, scaling first brings Strassen's error (FP64 and split-BF16 leaves)
  back to the classical product's, as the reference's scaling_stability
  experiment measures; on the quadrant case of scaling/strassen_bad_case.cpp
  it changes nothing.
"""

import numpy as np
import pytest

import oracle
from helpers import gpu_available, to_device, to_host

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm


def skewed(m, n, seed, per):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((m, n))
    if m and n:
        e = rng.integers(-20, 21, m if per == "row" else n)
        X *= np.exp2(e)[:, None] if per == "row" else np.exp2(e)[None, :]
    return np.asfortranarray(X)


def device_scaling(A, B, steps, kind):
    Ad, Bd = to_device(A), to_device(B)
    r, s = fmm.diagonal_scaling(Ad, Bd, steps, kind)
    fmm.synchronize()
    return to_host(Ad), to_host(Bd), r.cpu().numpy(), s.cpu().numpy()


SHAPES = [(37, 53, 29), (300, 1000, 257), (1, 1, 1), (5, 0, 3), (0, 4, 3), (513, 65, 700)]


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
@pytest.mark.parametrize("shape", SHAPES, ids=["%dx%dx%d" % s for s in SHAPES])
def test_scaling_equals_oracle_bit_for_bit(kind, shape):
    m, k, n = shape
    for steps in (0, 1, 2, 5):
        A = skewed(m, k, 3 * steps + kind, "row")
        B = skewed(k, n, 3 * steps + kind + 1, "col")
        got = device_scaling(A, B, steps, kind)
        Ao, Bo = A.copy(order="F"), B.copy(order="F")
        ro, so = oracle.scaling(Ao, Bo, steps, kind)
        for name, g, w in zip("ABrs", got, (Ao, Bo, ro, so)):
            assert np.array_equal(g, w, equal_nan=True), (kind, shape, steps, name)


def test_scaling_with_nan_inf_and_zero_rows_equals_oracle():
    m, k, n = 70, 90, 60
    A = skewed(m, k, 5, "row")
    B = skewed(k, n, 6, "col")
    A[3, 7] = np.nan      # skipped by the maxima, like the reference's `v > max`
    A[10, :] = 0.0        # zero row: its factor is 1/0
    B[:, 4] = 0.0
    B[2, 9] = np.inf
    A[:, 11] = -0.0
    for kind in range(4):
        got = device_scaling(A, B, 2, kind)
        Ao, Bo = A.copy(order="F"), B.copy(order="F")
        ro, so = oracle.scaling(Ao, Bo, 2, kind)
        for name, g, w in zip("ABrs", got, (Ao, Bo, ro, so)):
            assert np.array_equal(g, w, equal_nan=True), (kind, name)


def test_factors_multiply_into_given_vectors():
    A = skewed(60, 80, 1, "row")
    B = skewed(80, 50, 2, "col")
    r0 = np.linspace(0.5, 3.0, 60)
    s0 = np.linspace(1.5, 0.25, 50)
    Ad, Bd = to_device(A), to_device(B)
    rd, sd = torch.from_numpy(r0).cuda(), torch.from_numpy(s0).cuda()
    r, s = fmm.diagonal_scaling(Ad, Bd, 3, fmm.INSIDE_OUTSIDE, r_vals=rd, s_vals=sd)
    fmm.synchronize()
    assert r is rd and s is sd
    Ao, Bo = A.copy(order="F"), B.copy(order="F")
    ro, so = oracle.scaling(Ao, Bo, 3, 1, r=r0, s=s0)
    assert np.array_equal(rd.cpu().numpy(), ro) and np.array_equal(sd.cpu().numpy(), so)
    assert np.array_equal(to_host(Ad), Ao) and np.array_equal(to_host(Bd), Bo)


def test_host_entry_points_equal_oracle():
    """fmm_diagonal_scaling_host / fmm_scaling_postprocess_host (the C++
    adapter's Scaling / PostProcessScaling) on strided host buffers."""
    import ctypes

    from fast_matmul_b200._lib import check

    m, k, n = 90, 70, 110
    A = skewed(m + 5, k, 11, "row")
    B = skewed(k + 3, n, 12, "col")
    r = np.ones(m)
    s = np.ones(n)
    Ao, Bo = A[:m].copy(order="F"), B[:k].copy(order="F")
    ro, so = oracle.scaling(Ao, Bo, 2, 0)
    P = ctypes.c_void_p
    h = fmm.default_handle()
    check(fmm.lib().fmm_diagonal_scaling_host(h.ptr, P(A.ctypes.data), m + 5, P(B.ctypes.data), k + 3, m, k, n,
                                                  2, 0, P(r.ctypes.data), P(s.ctypes.data)))
    assert np.array_equal(A[:m], Ao) and np.array_equal(B[:k], Bo)
    assert np.array_equal(r, ro) and np.array_equal(s, so)
    C = skewed(m + 2, n, 13, "row")
    want = C[:m].copy(order="F")
    oracle.scaling_postprocess(want, r, s)
    check(fmm.lib().fmm_scaling_postprocess_host(h.ptr, P(C.ctypes.data), m + 2, m, n, P(r.ctypes.data),
                                                     P(s.ctypes.data)))
    assert np.array_equal(C[:m], want)


def test_postprocess_equals_oracle_bit_for_bit():
    for (m, n) in [(1, 1), (300, 257), (513, 70)]:
        C = skewed(m, n, m, "row")
        rng = np.random.default_rng(n)
        r = np.exp2(rng.uniform(-30, 30, m))
        s = np.exp2(rng.uniform(-30, 30, n)) * rng.uniform(0.5, 1.0, n)
        Cd = to_device(C)
        fmm.scaling_postprocess(Cd, torch.from_numpy(r).cuda(), torch.from_numpy(s).cuda())
        fmm.synchronize()
        want = C.copy(order="F")
        oracle.scaling_postprocess(want, r, s)
        assert np.array_equal(to_host(Cd), want), (m, n)


def test_bad_arguments_fail_loudly():
    A = fmm.colmajor_empty(4, 5, "cuda")
    B = fmm.colmajor_empty(5, 6, "cuda")
    with pytest.raises(fmm.FmmError, match="Unknown iteration type"):
        fmm.diagonal_scaling(A, B, 1, 7)
    with pytest.raises(ValueError):
        fmm.diagonal_scaling(A, B, 1, "outer_inner")
    with pytest.raises(fmm.FmmError):
        fmm.diagonal_scaling(A, B, -1, 0)


def skewed_pair(n, seed, inner_range=20):
    """Uniform [0, 1) operands with rows of A, columns of B and the inner
    dimension scaled by powers of two 2^U{-20..20}: A = D_r U_A D_t,
    B = D_t^-1 U_B D_c.  The product is as well conditioned as U_A U_B, but
    Strassen's sums mix rows (columns) of very different sizes."""
    rng = np.random.default_rng(seed)
    er = np.ldexp(1.0, rng.integers(-20, 21, n))
    ec = np.ldexp(1.0, rng.integers(-20, 21, n))
    et = rng.integers(-inner_range, inner_range + 1, n)
    A = fmm.random_matrix(n, n, 41, 1)
    B = fmm.random_matrix(n, n, 41, 2)
    A.mul_(torch.from_numpy(er).cuda()[:, None]).mul_(torch.from_numpy(np.ldexp(1.0, et)).cuda()[None, :])
    B.mul_(torch.from_numpy(np.ldexp(1.0, -et)).cuda()[:, None]).mul_(torch.from_numpy(ec).cuda()[None, :])
    return A, B


def scaled_product(A, B, steps, scaling_steps, kind, **kw):
    n = A.shape[0]
    As = fmm.colmajor_empty(n, n, A.device).copy_(A)
    Bs = fmm.colmajor_empty(n, n, A.device).copy_(B)
    C = fmm.colmajor_empty(n, n, A.device)
    r, s = fmm.diagonal_scaling(As, Bs, scaling_steps, kind)
    fmm.fast_matmul("strassen", As, Bs, C, steps, **kw)
    fmm.scaling_postprocess(C, r, s)
    return C


def test_scaling_repairs_strassen_on_skewed_operands():
    """Errors against the classical FP64 product (MaxRelativeDiff), the
    measurement of benchmarks/scaling_stability.cpp.  The reference build
    gives 3e18 unscaled and 2.1e-14..2.6e-14 with outside-inside or
    inside-outside scaling on this input at n = 1024, 4 steps."""
    n, steps = 1024, 4
    A, B = skewed_pair(n, 5)
    C1 = fmm.colmajor_empty(n, n, A.device)
    fmm.matmul(A, B, C1)
    C2 = fmm.colmajor_empty(n, n, A.device)
    fmm.fast_matmul("strassen", A, B, C2, steps)
    e_plain, _ = fmm.max_relative_diff(C1, C2)
    assert e_plain > 1e-3, e_plain
    for kind, sc in [(fmm.OUTSIDE_INSIDE, 1), (fmm.OUTSIDE_INSIDE, 5), (fmm.INSIDE_OUTSIDE, 1)]:
        e, _ = fmm.max_relative_diff(C1, scaled_product(A, B, steps, sc, kind))
        assert e < 1e-12, (kind, sc, e)


def test_scaling_repairs_split_bf16_strassen_on_skewed_operands():
    """The split-BF16 leaves scale rows of A and columns of B by powers of
    two themselves, but Strassen's additions mix rows of different sizes
    before the leaves see them, and a skewed inner dimension defeats the
    per-row scale; outside-inside scaling first repairs both (CPU model of
    the split arithmetic at n = 256: 2e19 -> 1.1e-12 at 5 slices, 4.5e-15 at
    6 slices; inside scaling alone leaves 1e9)."""
    n = 512
    A, B = skewed_pair(n, 7)
    C1 = fmm.colmajor_empty(n, n, A.device)
    fmm.matmul(A, B, C1)
    C2 = fmm.colmajor_empty(n, n, A.device)
    fmm.fast_matmul("strassen", A, B, C2, 1, precision="split_bf16", split_slices=5)
    e_plain, _ = fmm.max_relative_diff(C1, C2)
    assert e_plain > 1e-3, e_plain
    for slices, tol in [(5, 1e-11), (6, 1e-13)]:
        C3 = scaled_product(A, B, 1, 5, fmm.OUTSIDE_INSIDE, precision="split_bf16", split_slices=slices)
        e, _ = fmm.max_relative_diff(C1, C3)
        assert e < tol, (slices, e)


def test_scaling_on_the_quadrant_case_costs_nothing():
    """scaling/strassen_bad_case.cpp (top-left quadrant of A times 1e-8) at
    n = 1024, 4 steps: the reference build's MaxRelativeDiff is 2.1e-14
    unscaled and 2.2e-14 after 50 inside-outside steps -- here every entry of
    C is dominated by the unscaled blocks, so scaling neither helps nor hurts."""
    n, steps = 1024, 4
    A = fmm.random_matrix(n, n, 41, 1)
    B = fmm.random_matrix(n, n, 41, 2)
    A[: n // 2, : n // 2] *= 1e-8
    C1 = fmm.colmajor_empty(n, n, A.device)
    fmm.matmul(A, B, C1)
    e, _ = fmm.max_relative_diff(C1, scaled_product(A, B, steps, 50, fmm.INSIDE_OUTSIDE))
    assert e < 1e-13, e


# ---------------------------------------------------------------------------
# Scalar = float: against the reference's own Scaling<float> (oracle/_ref)


def skewed32(m, n, seed, per):
    return np.asfortranarray(skewed(m, n, seed, per).astype(np.float32))


def dev32(a):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


SHAPES32 = [(37, 53, 29), (300, 1000, 257), (1, 1, 1), (5, 0, 3), (513, 65, 700)]


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
@pytest.mark.parametrize("shape", SHAPES32, ids=["%dx%dx%d" % s for s in SHAPES32])
def test_scaling_f32_equals_the_references_bit_for_bit(kind, shape):
    if not oracle.ref_available():
        pytest.skip("reference build oracle/_ref not present")
    m, k, n = shape
    for steps in (0, 1, 2, 5):
        A = skewed32(m, k, 3 * steps + kind, "row")
        B = skewed32(k, n, 3 * steps + kind + 1, "col")
        Ad, Bd = dev32(A), dev32(B)
        r, s = fmm.diagonal_scaling(Ad, Bd, steps, kind)
        fmm.synchronize()
        Ar, Br = A.copy(order="F"), B.copy(order="F")
        rr, sr = oracle.ref_scaling_f32(Ar, Br, steps, kind)
        got = (np.asfortranarray(Ad.cpu().numpy()), np.asfortranarray(Bd.cpu().numpy()), r.cpu().numpy(),
               s.cpu().numpy())
        for name, g, w in zip("ABrs", got, (Ar, Br, rr, sr)):
            assert g.dtype == np.float32 and np.array_equal(g, w, equal_nan=True), (kind, shape, steps, name)


def test_postprocess_f32_and_host_entry_points_equal_the_references():
    if not oracle.ref_available():
        pytest.skip("reference build oracle/_ref not present")
    import ctypes

    from fast_matmul_b200._lib import check

    m, k, n = 90, 70, 110
    A = skewed32(m + 5, k, 11, "row")
    B = skewed32(k + 3, n, 12, "col")
    r = np.ones(m, dtype=np.float32)
    s = np.ones(n, dtype=np.float32)
    Ar, Br = A[:m].copy(order="F"), B[:k].copy(order="F")
    rr, sr = oracle.ref_scaling_f32(Ar, Br, 3, 0)
    P = ctypes.c_void_p
    h = fmm.default_handle()
    check(fmm.lib().fmm_diagonal_scaling_f32_host(h.ptr, P(A.ctypes.data), m + 5, P(B.ctypes.data), k + 3, m, k, n,
                                                  3, 0, P(r.ctypes.data), P(s.ctypes.data)))
    assert np.array_equal(A[:m], Ar) and np.array_equal(B[:k], Br)
    assert np.array_equal(r, rr) and np.array_equal(s, sr)
    C = skewed32(m + 2, n, 13, "row")
    want = C[:m].copy(order="F")
    oracle.ref_scaling_postprocess_f32(want, r, s)
    check(fmm.lib().fmm_scaling_postprocess_f32_host(h.ptr, P(C.ctypes.data), m + 2, m, n, P(r.ctypes.data),
                                                     P(s.ctypes.data)))
    assert np.array_equal(C[:m], want)
    Cd = dev32(C[:m].copy(order="F"))
    fmm.scaling_postprocess(Cd, torch.from_numpy(r).cuda(), torch.from_numpy(s).cuda())
    fmm.synchronize()
    want2 = C[:m].copy(order="F")
    oracle.ref_scaling_postprocess_f32(want2, r, s)
    assert np.array_equal(np.asfortranarray(Cd.cpu().numpy()), want2)
