"""The allocation-free entry point, fmm_fast_matmul_noalloc.

It exists for callers that may not allocate device memory (another
framework owns the device memory, or a fixed memory budget / latency-critical
loop forbids cudaMalloc).  Its scratch is a static device array inside
libfmm.so, so the checks here are that, called through the C ABI, it gives
the same result as the regular entry point (fmm_fast_matmul) on two calls in
a row -- the second reusing the array the first one left behind -- and that
it refuses sizes its scratch cannot hold and streams in capture mode.  Both
entry points plan with the same planner, pick the same schedule and run the
same kernels, so the results must be identical bit for bit.  This file is
collected last so a failure here leaves every other test already run; it
passes alone in a fresh process as well.
"""

import ctypes

import pytest

from helpers import colmajor_copy, gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm
    from fast_matmul_b200 import _lib


def call_noalloc(alg, A, B, C, steps, x, alpha, beta):
    m, k = A.shape
    n = B.shape[1]
    L = _lib.lib()
    return L.fmm_fast_matmul_noalloc(fmm.algorithm_index(alg), A.data_ptr(), A.stride(1), B.data_ptr(),
                                     B.stride(1), C.data_ptr(), C.stride(1), m, k, n, steps, x, alpha, beta,
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_matches_regular_entry_point_on_two_calls():
    # workspace against the 63 MiB the scratch leaves after the descriptors:
    #   strassen 517x389x461, 2 steps: ~15 MiB breadth-first -> fully breadth-first
    #   grey424 700x640x660, 2 steps: ~90 MiB breadth-first -> both levels depth-first
    #   strassen 1000^3, 3 steps: 189 MiB breadth-first, 55 MiB with two levels
    #     depth-first -> dfs = 2 of 3 (the most breadth-first schedule that fits)
    cases = [("strassen", (517, 389, 461), 2, 1.5, 0.5),
             ("grey424_26_206", (700, 640, 660), 2, 1.0, 0.0),
             ("strassen", (1000, 1000, 1000), 3, -1.2, 2.5)]
    for i, (alg, (m, k, n), steps, alpha, beta) in enumerate(cases):
        A = fmm.random_matrix(m, k, 90 + i, 1)
        B = fmm.random_matrix(k, n, 90 + i, 2)
        C0 = fmm.random_matrix(m, n, 90 + i, 3)
        want = colmajor_copy(C0)
        fmm.fast_matmul(alg, A, B, want, steps, 1e-8, alpha, beta)
        got = colmajor_copy(C0)
        st = call_noalloc(alg, A, B, got, steps, 1e-8, alpha, beta)
        assert st == 0, _lib.lib().fmm_last_error()
        torch.cuda.synchronize()
        assert torch.equal(want, got), (alg, fmm.max_relative_diff(want, got))
        # second call: the scratch still holds the first call's temporaries
        again = colmajor_copy(C0)
        st = call_noalloc(alg, A, B, again, steps, 1e-8, alpha, beta)
        assert st == 0, _lib.lib().fmm_last_error()
        torch.cuda.synchronize()
        assert torch.equal(want, again), (alg, fmm.max_relative_diff(want, again))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    n = 2048  # Strassen needs 17 blocks of 1024^2 doubles (136 MiB) even depth-first
    A = fmm.random_matrix(n, n, 1, 1)
    B = fmm.random_matrix(n, n, 1, 2)
    C = fmm.colmajor_empty(n, n, "cuda")
    st = call_noalloc("strassen", A, B, C, 1, 1e-8, 1.0, 0.0)
    assert st == 6  # FMM_ERR_WORKSPACE_TOO_SMALL
    msg = _lib.lib().fmm_last_error().decode()
    assert "static scratch" in msg and "bytes" in msg


def test_noalloc_refuses_a_capturing_stream():
    m = k = n = 96
    A = fmm.random_matrix(m, k, 3, 1)
    B = fmm.random_matrix(k, n, 3, 2)
    C = fmm.colmajor_empty(m, n, "cuda")
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            st = call_noalloc("strassen", A, B, C, 1, 1e-8, 1.0, 0.0)
        finally:
            g.capture_end()
    assert st == 5  # FMM_ERR_NOT_SUPPORTED, nothing queued
    assert "capture" in _lib.lib().fmm_last_error().decode()
    del g
