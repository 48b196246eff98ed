"""Pipelined host-memory calls (fmm_fast_matmul_host_async / fmm_host_sync).

Each queued call must give exactly what the synchronous host call
(fmm_fast_matmul_host) gives for the same operands: the same planner and
kernels run, only the copies move to their own streams.  Checked bit for bit
over a sequence of calls that
  * alternates the two staging slots with different shapes (slot buffers grow
    while the other slot's call is still in flight),
  * accumulates into one host C with beta != 0 (each call reads the C the
    previous call wrote back),
  * mixes a synchronous call in (it waits for the queued ones first),
and with pageable as well as pinned host buffers.
"""

import numpy as np
import pytest

import oracle
from helpers import gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm


def host(a, pinned):
    """Column-major float64 host tensor holding a (pinned or pageable)."""
    t = torch.from_numpy(np.ascontiguousarray(a.T)).t()
    p = torch.empty((a.shape[1], a.shape[0]), dtype=torch.float64, pin_memory=pinned).t()
    p.copy_(t)
    return p


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_queued_host_calls_equal_synchronous_ones(pinned):
    shapes = [("strassen", (517, 389, 461), 2), ("grey424_26_206", (640, 512, 700), 2),
              ("grey333_23_125", (301, 290, 333), 2), ("strassen", (1031, 1030, 1029), 1)]
    ops = []
    for i, (alg, (m, k, n), steps) in enumerate(shapes):
        ops.append((alg, steps, host(oracle.uniform(m, k, 40 + i, 1), pinned), host(oracle.uniform(k, n, 40 + i, 2),
                                                                                   pinned),
                    host(oracle.uniform(m, n, 40 + i, 3), pinned)))
    want = []
    for alg, steps, A, B, C0 in ops:
        C = C0.clone()
        fmm.fast_matmul_host(alg, A, B, C, steps, 1e-8, 1.5, 0.5)
        want.append(C)
    got = [host(C0.numpy(), pinned) for (_, _, _, _, C0) in ops]
    for (alg, steps, A, B, _), C in zip(ops, got):
        fmm.fast_matmul_host_async(alg, A, B, C, steps, 1e-8, 1.5, 0.5)
    fmm.host_sync()
    for w, g in zip(want, got):
        assert torch.equal(w, g)


def test_queued_calls_accumulating_into_one_host_c():
    m, k, n = 700, 600, 650
    A = host(oracle.uniform(m, k, 7, 1), True)
    B = host(oracle.uniform(k, n, 7, 2), True)
    want = host(oracle.uniform(m, n, 7, 3), True)
    got = host(want.numpy(), True)
    for _ in range(5):
        fmm.fast_matmul_host("strassen", A, B, want, 2, 1e-8, 1.0, 1.0)
    for _ in range(5):
        fmm.fast_matmul_host_async("strassen", A, B, got, 2, 1e-8, 1.0, 1.0)
    fmm.host_sync()
    assert torch.equal(want, got)
    # a synchronous call after queued ones sees their results
    fmm.fast_matmul_host_async("strassen", A, B, got, 2, 1e-8, 1.0, 1.0)
    fmm.fast_matmul_host("strassen", A, B, got, 2, 1e-8, 1.0, 1.0)
    fmm.fast_matmul_host("strassen", A, B, want, 2, 1e-8, 1.0, 1.0)
    fmm.fast_matmul_host("strassen", A, B, want, 2, 1e-8, 1.0, 1.0)
    assert torch.equal(want, got)
