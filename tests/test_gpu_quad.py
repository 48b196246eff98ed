"""Device results against quad-precision products on sampled entries.

The correctness oracle of the benchmark definition is the relative error
against the classical product backed by quad-precision products on sampled
entries (the reference's linalg/quadmatmul.hpp, restated in the oracle as
oracle_quad_errors).  Here 128 sampled entries of device results are checked
against their __float128 values:

* FP64 exact algorithms (Strassen 2 steps, fast424_26_206 2 steps, grey333 1
  step) and the engine's classical GEMM: max relative error <= 1e-13;
* split-BF16 leaf products: <= 1e-12 at 6 slices, <= 1e-11 at 5 slices
  (uniform [0, 1) inputs, where elementwise relative errors are meaningful);
  split-INT8: <= 1e-12 at 7 slices, <= 1e-11 at 6;
* Bini's approximate <3,2,2;10> at lambda = 2^-13: the same error in FP64 and
  split-BF16 (6 slices), within a factor 2.
"""

import numpy as np
import pytest

import oracle
from helpers import gpu_available, to_device, to_host

pytestmark = pytest.mark.gpu

if gpu_available():
    import fast_matmul_b200 as fmm

N = 1536


@pytest.fixture(scope="module")
def operands():
    A = oracle.uniform(N, N, 17, 1)
    B = oracle.uniform(N, N, 17, 2)
    rng = np.random.default_rng(1)
    return A, B, rng.integers(0, N, 128), rng.integers(0, N, 128)


def run(A, B, fn):
    Cd = to_device(np.zeros((N, N), order="F"))
    fn(to_device(A), to_device(B), Cd)
    fmm.synchronize()
    return to_host(Cd)


CASES = [
    ("classical fp64", lambda A, B, C: fmm.matmul(A, B, C), 1e-13),
    ("strassen s2 fp64", lambda A, B, C: fmm.fast_matmul("strassen", A, B, C, 2), 1e-13),
    ("fast424 s2 fp64", lambda A, B, C: fmm.fast_matmul("grey424_26_206", A, B, C, 2), 1e-13),
    ("grey333 s1 fp64", lambda A, B, C: fmm.fast_matmul("grey333_23_125", A, B, C, 1), 1e-13),
    ("classical split x6", lambda A, B, C: fmm.matmul_split_bf16(A, B, C, slices=6), 1e-12),
    ("strassen s2 split x6",
     lambda A, B, C: fmm.fast_matmul("strassen", A, B, C, 2, precision="split_bf16", split_slices=6), 1e-12),
    ("strassen s2 split x5",
     lambda A, B, C: fmm.fast_matmul("strassen", A, B, C, 2, precision="split_bf16", split_slices=5), 1e-11),
    ("classical int8 x7", lambda A, B, C: fmm.matmul_split_int8(A, B, C, slices=7), 1e-12),
    ("strassen s2 int8 x7",
     lambda A, B, C: fmm.fast_matmul("strassen", A, B, C, 2, precision="split_int8", split_slices=7), 1e-12),
    ("strassen s2 int8 x6",
     lambda A, B, C: fmm.fast_matmul("strassen", A, B, C, 2, precision="split_int8", split_slices=6), 1e-11),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_sampled_entries_against_quad(operands, case):
    A, B, rows, cols = operands
    name, fn, tol = case
    C = run(A, B, fn)
    rel, scaled = oracle.quad_errors(A, B, rows, cols, C[rows, cols])
    assert rel <= tol, (name, rel)
    assert scaled <= rel


def test_approximate_algorithm_same_error_in_fp64_and_split(operands):
    A, B, rows, cols = operands
    x = 2.0 ** -13
    C64 = run(A, B, lambda a, b, c: fmm.fast_matmul("bini322_10_52_approx", a, b, c, 1, x))
    Cs = run(A, B, lambda a, b, c: fmm.fast_matmul("bini322_10_52_approx", a, b, c, 1, x, precision="split_bf16",
                                                   split_slices=6))
    Ci = run(A, B, lambda a, b, c: fmm.fast_matmul("bini322_10_52_approx", a, b, c, 1, x, precision="split_int8",
                                                   split_slices=7))
    e64, _ = oracle.quad_errors(A, B, rows, cols, C64[rows, cols])
    es, _ = oracle.quad_errors(A, B, rows, cols, Cs[rows, cols])
    ei, _ = oracle.quad_errors(A, B, rows, cols, Ci[rows, cols])
    assert 1e-8 < e64 < 1e-2  # lambda dominates the error
    assert es <= 2.0 * e64 and e64 <= 2.0 * es
    assert ei <= 2.0 * e64 and e64 <= 2.0 * ei
