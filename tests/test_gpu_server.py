"""The continuous-batching request loop (fmm_server_*).

Requests submitted while others run are admitted as slots and workspace free
up; each result must equal the one the request gives alone (bit for bit);
requests that can never fit the workspace pool fail with a status instead of
blocking the queue; waits time out with a status."""

import numpy as np
import pytest

from helpers import colmajor_copy, gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm


def alone(A, B, C0, alg, steps, alpha, beta):
    C = colmajor_copy(C0)
    if alg == fmm.AUTO:
        alg, steps = fmm.autotune_choice(A.shape[0], A.shape[1], B.shape[1])
    if alg == fmm.CLASSICAL:
        fmm.matmul(A, B, C, alpha, beta)
    else:
        fmm.fast_matmul(alg, A, B, C, steps, 1e-8, alpha, beta)
    return C


def test_server_results_equal_alone_and_in_the_mix():
    rng = np.random.default_rng(11)
    srv = fmm.Server(0, workspace_bytes=4 << 30, max_inflight=3, max_batch=8)
    kinds = [("strassen", 1), ("strassen", 2), ("grey424_26_206", 1), (fmm.CLASSICAL, 0), (fmm.AUTO, 0),
             ("grey333_23_125", 1)]
    reqs = []
    for i in range(36):
        m, k, n = (int(v) for v in rng.integers(96, 1600, size=3))
        A = fmm.random_matrix(m, k, 500 + i, 1, -1.0, 1.0)
        B = fmm.random_matrix(k, n, 500 + i, 2, -1.0, 1.0)
        C0 = fmm.random_matrix(m, n, 500 + i, 3, -1.0, 1.0)
        alg, steps = kinds[i % len(kinds)]
        beta = 0.5 if i % 3 == 0 else 0.0
        C = colmajor_copy(C0)
        torch.cuda.synchronize()
        t = srv.submit(A, B, C, alg, steps, alpha=1.25, beta=beta)
        reqs.append((t, A, B, C0, C, alg, steps, beta))
    srv.drain()
    st = srv.stats()
    assert st["completed"] == st["submitted"] == 36
    assert st["batches"] >= 2
    for t, A, B, C0, C, alg, steps, beta in reqs:
        info = srv.wait(t)
        assert info["done"] and info["status"] == 0
        assert info["submit_ms"] <= info["launch_ms"] <= info["done_ms"]
        assert torch.equal(alone(A, B, C0, alg, steps, 1.25, beta), C)
    srv.close()


def test_server_fails_requests_larger_than_its_pool_and_keeps_serving():
    srv = fmm.Server(0, workspace_bytes=16 << 20, max_inflight=2)
    A = fmm.random_matrix(2048, 2048, 1, 1)
    B = fmm.random_matrix(2048, 2048, 1, 2)
    C = fmm.colmajor_empty(2048, 2048)
    big = srv.submit(A, B, C, "strassen", 1)  # needs 136 MiB of S/T/M
    small_C = fmm.colmajor_empty(2048, 2048)
    small = srv.submit(A, B, small_C, fmm.CLASSICAL)  # no workspace
    assert srv.wait(big)["status"] == 3  # FMM_ERR_OUT_OF_MEMORY
    assert srv.wait(small)["status"] == 0
    want = fmm.colmajor_empty(2048, 2048)
    fmm.matmul(A, B, want)
    torch.cuda.synchronize()
    assert torch.equal(want, small_C)
    srv.close()


def test_server_wait_reports_timeout_then_completes():
    srv = fmm.Server(0, workspace_bytes=8 << 30)  # 2 Strassen steps at 6144^3 need 3.5 GB breadth-first
    A = fmm.random_matrix(6144, 6144, 2, 1)
    B = fmm.random_matrix(6144, 6144, 2, 2)
    C = fmm.colmajor_empty(6144, 6144)
    t = srv.submit(A, B, C, "strassen", 2)
    try:
        info = srv.wait(t, timeout_ms=0.001)
        assert info["done"]
    except fmm.FmmError as ex:
        assert ex.status == 7  # FMM_ERR_TIMEOUT
    assert srv.wait(t)["status"] == 0
    srv.close()
