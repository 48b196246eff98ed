"""The engine's FP64 tensor-core GEMM (the leaf kernel) against cuBLAS FP64
and the CPU oracle: odd shapes, strided and misaligned views, alpha/beta."""

import numpy as np
import pytest

import oracle
from helpers import colmajor_copy, gpu_available, to_device, to_host

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm

# Uniform [0, 1) data: no cancellation, so the relative error of any
# summation order is bounded by about k * 2^-53.
TOL = 1e-12


def cm(t):
    """Column-major copy of a torch matrix."""
    return colmajor_copy(t)


def view(m, n, seed, stream, offset=0, pad=0):
    """m x n column-major view at `offset` elements into a (m + pad + offset)-row buffer."""
    base = fmm.random_matrix(m + pad + offset, n, seed, stream)
    return base[offset:offset + m, :]


@pytest.mark.parametrize("m,k,n", [(1, 1, 1), (5, 3, 7), (128, 16, 128), (129, 257, 131), (256, 64, 300),
                                   (1000, 200, 309), (63, 1001, 65)])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.2, 0.0), (7.0, -1.3)])
def test_dgemm_matches_cublas(m, k, n, alpha, beta):
    A = view(m, k, 1, 1)
    B = view(k, n, 1, 2)
    C0 = view(m, n, 1, 3)
    C = cm(C0)
    fmm.matmul(A, B, C, alpha, beta)
    ref = cm(alpha * (A @ B) + (beta * C0 if beta != 0 else 0))
    rel, _ = fmm.max_relative_diff(ref, C)
    assert rel <= TOL


@pytest.mark.parametrize("offset,pad", [(1, 0), (1, 1), (0, 3), (3, 2)])
def test_dgemm_strided_and_misaligned_views(offset, pad):
    m, k, n = 131, 77, 95
    A = view(m, k, 2, 1, offset, pad)
    B = view(k, n, 2, 2, offset, pad)
    Cbuf = view(m, n, 2, 3, offset, pad)
    C0 = cm(Cbuf)
    fmm.matmul(A, B, Cbuf, 2.0, 0.5)
    ref = cm(2.0 * (A @ B) + 0.5 * C0)
    assert fmm.max_relative_diff(ref, Cbuf)[0] <= TOL


def test_dgemm_zero_inner_dimension_scales_c():
    C = fmm.random_matrix(5, 4, 3, 3)
    C0 = cm(C)
    A = fmm.colmajor_empty(5, 0, "cuda")
    B = fmm.colmajor_empty(0, 4, "cuda")
    fmm.matmul(A, B, C, 1.0, 2.0)
    torch.cuda.synchronize()
    assert torch.equal(C, 2.0 * C0)


def test_dgemm_beta_zero_ignores_nan_in_c():
    A = fmm.random_matrix(70, 33, 4, 1)
    B = fmm.random_matrix(33, 50, 4, 2)
    C = fmm.colmajor_empty(70, 50, "cuda")
    C.fill_(float("nan"))
    fmm.matmul(A, B, C, 1.0, 0.0)
    assert not torch.isnan(C).any()
    assert fmm.max_relative_diff(cm(A @ B), C)[0] <= TOL


def test_dgemm_matches_cpu_oracle():
    m, k, n = 203, 190, 177
    A = oracle.uniform(m, k, 9, 1)
    B = oracle.uniform(k, n, 9, 2)
    want = np.zeros((m, n), order="F")
    oracle.matmul(A, B, want, 1.0, 0.0)
    Cd = fmm.colmajor_empty(m, n, "cuda")
    fmm.matmul(to_device(A), to_device(B), Cd)
    got = to_host(Cd)
    assert oracle.max_relative_diff(want, got) <= TOL


def test_device_generator_matches_host_generator():
    d = to_host(fmm.random_matrix(37, 23, 5, 7, -1.0, 1.0))
    h = oracle.uniform(37, 23, 5, 7, -1.0, 1.0)
    assert np.array_equal(d, h)
