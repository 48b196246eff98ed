"""Device-side bounds checks of the descriptor walks (a sanitizer substitute).

libfmm_checked.so is the engine built with -DFMM_DEVICE_CHECKS: its grouped
GEMM checks the problem and tile every CTA decodes from its descriptors, and
its formation and combination kernels check that every S/T block they write
and every product block they read lies inside the running program's
workspace; a failed check skips the access and sets a bit that
fmm_debug_check_flags returns.  A child process runs a set of products on
the checked library (FMM_LIBRARY selects it); the parent runs the same ones
on the regular library.  No bit may be set, and the results must be
identical bit for bit: the checks observe, they change nothing.

Cases: the reference's odd peeling shapes, exact and approximate algorithms,
every schedule, beta != 0, a batch of mixed items, split-BF16 leaves (whose
formations, combinations and fringe products go through the checked
kernels).
"""

import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import REPO, gpu_available

pytestmark = pytest.mark.gpu

CHECKED = os.path.join(REPO, "fast_matmul_b200", "libfmm_checked.so")

CASES = [("strassen", (257, 500, 55), 2, "bfs", "fp64"), ("strassen", (1001, 200, 309), 3, "dfs", "fp64"),
         ("grey333_23_125", (402, 500, 562), 2, "hybrid", "fp64"), ("grey424_26_206", (600, 500, 671), 1, "bfs", "fp64"),
         ("bini322_10_52_approx", (366, 500, 200), 2, "bfs", "fp64"), ("smirnov333_23_128", (634, 700, 1000), 1, "dfs",
                                                                         "fp64"),
         ("strassen", (301, 259, 277), 2, "bfs", "split_bf16"), ("grey333_23_125", (190, 200, 170), 2, "dfs",
                                                                  "split_int8")]


def run_cases(out_path):
    """Runs CASES and a batch on the library FMM_LIBRARY names (or the
    regular one), saving the results and the check word to out_path."""
    import torch

    import fast_matmul_b200 as fmm
    from fast_matmul_b200 import _lib

    res = {}
    for i, (alg, (m, k, n), steps, sched, prec) in enumerate(CASES):
        A = fmm.random_matrix(m, k, 70 + i, 1)
        B = fmm.random_matrix(k, n, 70 + i, 2)
        C = fmm.random_matrix(m, n, 70 + i, 3)
        x = 1e-4 if "approx" in alg else 1e-8
        fmm.fast_matmul(alg, A, B, C, steps, x, 1.5, 0.5, schedule=sched, precision=prec)
        res["case%d" % i] = C.t().contiguous().cpu().numpy()
    probs = []
    for i, (m, k, n, alg) in enumerate([(300, 280, 260, "strassen"), (97, 300, 65, fmm.CLASSICAL),
                                        (400, 401, 399, "grey333_23_125")]):
        probs.append({"A": fmm.random_matrix(m, k, 90 + i, 1), "B": fmm.random_matrix(k, n, 90 + i, 2),
                      "C": fmm.random_matrix(m, n, 90 + i, 3), "alg": alg, "num_steps": 2, "beta": 0.25})
    fmm.fast_matmul_batched(probs)
    for i, p in enumerate(probs):
        res["batch%d" % i] = p["C"].t().contiguous().cpu().numpy()
    torch.cuda.synchronize()
    flags = ctypes.c_uint(0)
    st = _lib.lib().fmm_debug_check_flags(ctypes.byref(flags))
    res["status"] = np.array([st])
    res["flags"] = np.array([flags.value])
    np.savez(out_path, **res)


@pytest.mark.skipif(not os.path.exists(CHECKED), reason="libfmm_checked.so not built")
def test_checked_kernels_flag_nothing_and_change_nothing(tmp_path):
    assert gpu_available()
    checked_out = str(tmp_path / "checked.npz")
    env = dict(os.environ, FMM_LIBRARY=CHECKED)
    code = ("import sys; sys.path.insert(0, %r); sys.path.insert(0, %r); import test_gpu_device_checks as t; "
            "t.run_cases(sys.argv[1])" % (os.path.join(REPO, "tests"), REPO))
    proc = subprocess.run([sys.executable, "-c", code, checked_out], env=env, capture_output=True, text=True,
                          timeout=600)
    assert proc.returncode == 0, proc.stderr[-4000:]
    regular_out = str(tmp_path / "regular.npz")
    run_cases(regular_out)
    got = np.load(checked_out)
    want = np.load(regular_out)
    assert int(got["status"][0]) == 0  # the checked build answers
    assert int(got["flags"][0]) == 0, "device checks failed: bits %#x" % int(got["flags"][0])
    assert int(want["status"][0]) == 5  # the regular build has no checks (FMM_ERR_NOT_SUPPORTED)
    for key in want.files:
        if key in ("status", "flags"):
            continue
        assert np.array_equal(got[key], want[key]), key
