"""GPU parity against the reference's own results at large sizes.

The fixtures (tests/golden/reference_{baseline,matrix,lambda}.json, written by
tests/golden/make_reference_digests.py) hold digests of the results of the
reference's FastMatmul itself -- its headers compiled unchanged with host BLAS
leaves -- on seeded inputs: sampled entries (fringe rows and columns of the
dynamic peeling included) and row/column band sums, plus the reference's
error against its own classical product.  Here the same inputs are generated
on the device (fmm.random_matrix is the generator of oracle.uniform), the
engine's FastMatmul runs in FP64, and its digest is compared:

  * exact algorithms: max relative difference of every sampled entry and
    every band sum <= 1e-13 (the plain form's parity bar against the
    reference's result for the same algorithm and recursion depth);
  * approximate algorithms (Bini, Schonhage, Smirnov's 20-term <3,3,3>): the
    engine's max relative difference against the classical product
    (MaxRelativeDiff, linalg/linalg.hpp:280-295) <= 2x the reference's own,
    at the reference's lambda for the step count (all_algorithms.hpp:102-141)
    or at every lambda of the sweeps (tests/bini_stability.cpp:17-38 and its
    Schonhage and Smirnov twins; the benchmark's 2^-10..2^-26 at 8192^3).

Sets: the benchmark configurations (Strassen 4096^3 with 1 and 2 steps, the
headline grey424_26_206 16384^3 with 2 steps, and the three algorithms of
the FP64 study on its three shapes at 1-3 steps), the reference's test
matrix (tests/matmul_tests.cpp:137-173: 27 algorithms x 17 shapes x steps
1-3) and the lambda sweeps.
"""

import json
import os
import sys

import pytest

from helpers import REPO, gpu_available

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(REPO, "tests", "golden")
EXACT_TOL = 1e-13
APPROX_FACTOR = 2.0

sys.path.insert(0, GOLDEN)
import digest as dg  # noqa: E402

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm

ALGS = {a["name"]: a for a in json.load(open(os.path.join(REPO, "fast_matmul_b200", "generated",
                                                           "algorithms.json")))["algorithms"]}


def load(name):
    path = os.path.join(GOLDEN, "reference_%s.json" % name)
    if not os.path.exists(path):
        return []
    with open(path) as fh:
        return json.load(fh)["cases"]


def case_id(c):
    lam = "" if not c.get("sweep") else "-x%.3g" % c["x"]
    enum = "-%s" % c["enum"] if c.get("enum") else ""
    return "%s%s-s%d-%dx%dx%d%s" % (c["alg"], enum, c["steps"], c["m"], c["k"], c["n"], lam)


class Operands:
    """Device operands (and the engine's classical product) of the last shape."""

    key = None
    A = B = Cc = None

    @classmethod
    def get(cls, m, k, n, seed, classical=False):
        if cls.key != (m, k, n, seed):
            cls.A = cls.B = cls.Cc = None
            torch.cuda.empty_cache()
            cls.A = fmm.random_matrix(m, k, seed, 1)
            cls.B = fmm.random_matrix(k, n, seed, 2)
            cls.key = (m, k, n, seed)
        if classical and cls.Cc is None:
            cls.Cc = fmm.colmajor_empty(m, n, cls.A.device)
            fmm.matmul(cls.A, cls.B, cls.Cc)
        return cls.A, cls.B, cls.Cc


def run_case(c):
    alg, m, k, n, steps = c["alg"], c["m"], c["k"], c["n"], c["steps"]
    approx = ALGS[alg]["approximate"]
    A, B, Cc = Operands.get(m, k, n, c["seed"], classical=approx)
    C = fmm.colmajor_empty(m, n, A.device)
    fmm.fast_matmul(alg, A, B, C, steps, c["x"], c["alpha"], c["beta"])
    info = ALGS[alg]
    rows, cols = dg.positions(m, n, info["m0"], info["n0"], steps, c["samples_count"], c["seed"])
    got = dg.digest_torch(C, rows, cols, c["groups"])
    want = {key: dg.dec(c[key]) for key in ("samples", "rowsum", "colsum")}
    diff = dg.rel_diffs(want, got)
    err = None
    if approx:
        err, _ = fmm.max_relative_diff(Cc, C)
    del C
    return approx, diff, err


RESULTS = []


@pytest.fixture(scope="module", autouse=True)
def parity_report():
    """With FMM_PARITY_REPORT=<path>, writes every case's measured differences
    there as JSON lines when the module finishes."""
    yield
    path = os.environ.get("FMM_PARITY_REPORT")
    if path and RESULTS:
        with open(path, "w") as fh:
            for r in RESULTS:
                fh.write(json.dumps(r) + "\n")


def check(c):
    approx, diff, err = run_case(c)
    RESULTS.append({"id": case_id(c), "approx": approx, "vs_reference": diff, "err_vs_classical": err,
                    "ref_err": c["ref_err"]})
    if approx:
        assert err <= APPROX_FACTOR * c["ref_err"], (case_id(c), err, c["ref_err"])
    else:
        assert diff["max"] <= EXACT_TOL, (case_id(c), diff)


BASELINE = load("baseline")
MATRIX = load("matrix")
LAMBDA = load("lambda")


@pytest.mark.parametrize("c", BASELINE, ids=[case_id(c) for c in BASELINE])
def test_benchmark_configurations_match_the_reference(c):
    check(c)


@pytest.mark.parametrize("c", MATRIX, ids=[case_id(c) for c in MATRIX])
def test_reference_test_matrix(c):
    check(c)


@pytest.mark.parametrize("c", LAMBDA, ids=[case_id(c) for c in LAMBDA])
def test_lambda_sweeps_within_twice_the_reference_error(c):
    check(c)

