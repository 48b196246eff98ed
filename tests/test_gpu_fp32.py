"""FP32 operands: FastMatmul<float> and MatMul<float> (fmm_fast_matmul_f32,
fmm_sgemm and their host forms).

The reference computes these in FP32 throughout (Scalar = float, sgemm
leaves); the engine widens the operands to FP64, multiplies there (by
default with split-INT8 leaves of 5 slices) and rounds once.  Each case
runs the reference itself (oracle/_ref, the reference's headers with
Scalar = float) on the same FP32 inputs and checks, against the exact
product of those inputs:

* the engine's error is within 2x the reference's (the bar for every
  algorithm, exact or approximate);
* for exact algorithms it is about one FP32 rounding (<= 2^-23 elementwise
  on uniform [0, 1) inputs), far below the reference's.
"""

import ctypes

import numpy as np
import pytest

import oracle
from helpers import gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm


def f32(m, n, seed, stream):
    return np.asfortranarray(oracle.uniform(m, n, seed, stream).astype(np.float32))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def host(t):
    return np.asfortranarray(t.cpu().numpy())


def exact(A, B, C0=None, alpha=1.0, beta=0.0):
    P = A.astype(np.float64) @ B.astype(np.float64)
    return alpha * P + (beta * C0.astype(np.float64) if C0 is not None and beta else 0.0)


def rel_err(got, want):
    return float((np.abs(got.astype(np.float64) - want) / np.abs(want)).max())


def skip_without_reference():
    if not oracle.ref_available():
        pytest.skip("reference build oracle/_ref not present")


CASES = [("strassen", 1, 1e-8, (512, 512, 512)), ("strassen", 2, 1e-8, (600, 520, 560)),
         ("grey424_26_206", 2, 1e-8, (512, 256, 512)), ("grey333_23_125", 1, 1e-8, (301, 299, 302)),
         ("bini322_10_52_approx", 1, 1e-4, (300, 200, 250)), ("smirnov333_23_128", 2, 1e-8, (243, 270, 251))]


@pytest.mark.parametrize("case", CASES, ids=["%s-s%d" % (c[0], c[1]) for c in CASES])
def test_fast_matmul_f32_within_the_references_error(case):
    skip_without_reference()
    alg, steps, x, (m, k, n) = case
    A, B = f32(m, k, 3, 1), f32(k, n, 3, 2)
    want = exact(A, B)
    Cr = np.zeros((m, n), dtype=np.float32, order="F")
    oracle.ref_fast_matmul_f32(alg, A, B, Cr, steps, x)
    e_ref = rel_err(Cr, want)
    Cd = dev(np.zeros((m, n), dtype=np.float32, order="F"))
    fmm.fast_matmul(alg, dev(A), dev(B), Cd, steps, x)
    fmm.synchronize()
    e = rel_err(host(Cd), want)
    assert e <= 2.0 * e_ref, (e, e_ref)
    if "approx" not in alg:
        assert e <= 2.0 ** -23, (e, e_ref)


def test_alpha_beta_and_fp64_leaves():
    skip_without_reference()
    m, k, n = 400, 330, 350
    A, B, C0 = f32(m, k, 5, 1), f32(k, n, 5, 2), f32(m, n, 5, 3)
    want = exact(A, B, C0, 1.5, -0.75)
    Cr = C0.copy(order="F")
    oracle.ref_fast_matmul_f32("strassen", A, B, Cr, 2, 1e-8, 1.5, -0.75)
    e_ref = rel_err(Cr, want)
    for prec, sl in ((None, 0), ("fp64", 0), ("split_bf16", 5), ("split_int8", 4)):
        Cd = dev(C0)
        fmm.fast_matmul("strassen", dev(A), dev(B), Cd, 2, alpha=1.5, beta=-0.75, precision=prec, split_slices=sl)
        fmm.synchronize()
        e = rel_err(host(Cd), want)
        assert e <= min(2.0 * e_ref, 2.0 ** -22), (prec, e, e_ref)
    # num_steps == 0 is one classical product that ignores beta, as in FastMatmul
    Cd = dev(C0)
    fmm.fast_matmul("strassen", dev(A), dev(B), Cd, 0, alpha=1.5, beta=-0.75)
    fmm.synchronize()
    assert rel_err(host(Cd), exact(A, B, alpha=1.5)) <= 2.0 ** -23


def test_sgemm_within_the_references_error():
    skip_without_reference()
    m, k, n = 700, 900, 650
    A, B, C0 = f32(m, k, 7, 1), f32(k, n, 7, 2), f32(m, n, 7, 3)
    want = exact(A, B, C0, 2.0, 0.5)
    Cr = C0.copy(order="F")
    oracle.ref_matmul_f32(A, B, Cr, 2.0, 0.5)
    e_ref = rel_err(Cr, want)
    Cd = dev(C0)
    fmm.matmul(dev(A), dev(B), Cd, 2.0, 0.5)
    fmm.synchronize()
    e = rel_err(host(Cd), want)
    assert e <= 2.0 * e_ref and e <= 2.0 ** -23, (e, e_ref)


def test_host_entry_points_equal_the_device_ones():
    m, k, n = 257, 190, 301
    A, B, C0 = f32(m + 3, k, 9, 1), f32(k, n, 9, 2), f32(m, n, 9, 3)
    Cd = dev(C0)
    fmm.fast_matmul("grey333_23_125", dev(np.asfortranarray(A[:m])), dev(B), Cd, 1, beta=0.25)
    fmm.synchronize()
    Ch = C0.copy(order="F")
    P = ctypes.c_void_p
    h = fmm.default_handle()
    ms = ctypes.c_double()
    from fast_matmul_b200._lib import check

    check(fmm.lib().fmm_fast_matmul_f32_host(h.ptr, fmm.algorithm_index("grey333_23_125"), P(A.ctypes.data), m + 3,
                                             P(B.ctypes.data), k, P(Ch.ctypes.data), m, m, k, n, 1, 1e-8, 1.0, 0.25,
                                             None, ctypes.byref(ms)))
    assert np.array_equal(Ch, host(Cd))
    Cg = dev(C0)
    fmm.matmul(dev(np.asfortranarray(A[:m])), dev(B), Cg, 1.0, 0.25)
    fmm.synchronize()
    Cs = C0.copy(order="F")
    check(fmm.lib().fmm_sgemm_host(h.ptr, P(A.ctypes.data), m + 3, P(B.ctypes.data), k, P(Cs.ctypes.data), m, m, k,
                                   n, 1.0, 0.25, None))
    assert np.array_equal(Cs, host(Cg))


def test_mixed_dtypes_are_rejected():
    A = dev(f32(8, 8, 1, 1))
    B = fmm.colmajor_empty(8, 8, "cuda")
    C = dev(f32(8, 8, 1, 2))
    with pytest.raises(TypeError):
        fmm.fast_matmul("strassen", A, B, C, 1)
