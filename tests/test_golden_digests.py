"""The reference-digest fixtures and their helper, checked on the CPU.

* completeness: every set holds the cases its generator promises;
* the digest helper: fringe indices follow the floor sub-blocking of
  linalg/linalg.hpp:179-184 and 201-244, positions are in range and
  deterministic;
* pinning: the oracle's C restatement of the recursion, with its leaf
  products routed through the reference build's BLAS, reproduces the
  fixtures' digests bit for bit on a selection of the small cases (the
  restatement equals the reference bit for bit with that leaf, so this ties
  the fixtures, the restatement and the reference together).
"""

import json
import os
import sys

import numpy as np
import pytest

import oracle
from helpers import REPO

GOLDEN = os.path.join(REPO, "tests", "golden")
sys.path.insert(0, GOLDEN)
import digest as dg  # noqa: E402

ALGS = {a["name"]: a for a in json.load(open(os.path.join(REPO, "fast_matmul_b200", "generated",
                                                           "algorithms.json")))["algorithms"]}


def load(name):
    with open(os.path.join(GOLDEN, "reference_%s.json" % name)) as fh:
        return json.load(fh)["cases"]


def test_fixture_sets_are_complete():
    base, matrix, lam = load("baseline"), load("matrix"), load("lambda")
    assert len(base) == 41
    assert {(c["alg"], c["m"], c["k"], c["n"], c["steps"]) for c in base} >= {
        ("strassen", 4096, 4096, 4096, 1), ("strassen", 4096, 4096, 4096, 2),
        ("grey424_26_206", 16384, 16384, 16384, 2)}
    assert len(matrix) == 28 * 17 * 3
    assert len({c["enum"] for c in matrix}) == 28  # 27 enum values of the reference's test + grey323_15_89
    assert len([c for c in lam if c["sweep"] == "stability"]) == 3 * 2 * 52
    assert len([c for c in lam if c["sweep"] == "benchmark"]) == 2 * 17
    for c in base + matrix + lam:
        assert np.isfinite(c["ref_err"])
        assert dg.dec(c["samples"]).size == c["samples_count"]
    exact_errs = [c["ref_err"] for c in base + matrix if not ALGS[c["alg"]]["approximate"]]
    assert max(exact_errs) < 1e-12  # the reference's own error for exact algorithms


def test_fringe_indices_follow_floor_subblocking():
    # 4001 rows, 3 blocks per level: level 0 keeps 3 x 1333, peels row 3999-4000;
    # each 1333 block keeps 3 x 444 and peels its last row; 444 = 3 x 148 peels none
    assert dg.fringe(4001, 3, 1) == [3999, 4000]
    assert dg.fringe(4001, 3, 2) == [1332, 2665, 3998, 3999, 4000]
    assert dg.fringe(4001, 3, 3) == dg.fringe(4001, 3, 2)
    assert dg.fringe(16384, 4, 3) == []
    assert dg.fringe(7, 2, 2) == [2, 5, 6]


def test_positions_are_in_range_and_deterministic():
    r1, c1 = dg.positions(4001, 1200, 3, 3, 2, 48, 507)
    r2, c2 = dg.positions(4001, 1200, 3, 3, 2, 48, 507)
    assert np.array_equal(r1, r2) and np.array_equal(c1, c2)
    assert r1.min() >= 0 and r1.max() < 4001 and c1.min() >= 0 and c1.max() < 1200
    fr = set(dg.fringe(4001, 3, 2))
    assert all(int(r) in fr for r in r1[:12])


PIN = [c for c in load("matrix") if c["m"] <= 402 and c["enum"] in (
    "STRASSEN", "FAST424_26_206", "FAST333_23_125", "SMIRNOV333_23_128", "BINI322_10_52_APPROX",
    "SCHONHAGE333_21_117_APPROX", "FAST522_18_99", "CLASSICAL333")]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build oracle/_ref not present")
@pytest.mark.parametrize("c", PIN, ids=["%s-s%d-%dx%dx%d" % (c["alg"], c["steps"], c["m"], c["k"], c["n"])
                                       for c in PIN])
def test_restatement_reproduces_the_reference_digests(c):
    m, k, n = c["m"], c["k"], c["n"]
    A = oracle.uniform(m, k, c["seed"], 1)
    B = oracle.uniform(k, n, c["seed"], 2)
    C = np.zeros((m, n), order="F")
    oracle.use_reference_leaf(True)
    try:
        oracle.fast_matmul(c["alg"], A, B, C, c["steps"], c["x"], c["alpha"], c["beta"])
    finally:
        oracle.use_reference_leaf(False)
    info = ALGS[c["alg"]]
    rows, cols = dg.positions(m, n, info["m0"], info["n0"], c["steps"], c["samples_count"], c["seed"])
    got = dg.digest_np(C, rows, cols, c["groups"])
    for key in ("samples", "rowsum", "colsum"):
        assert np.array_equal(got[key], dg.dec(c[key])), key
