"""Generates tests/golden/reference_cases.json from the reference itself.

Runs the reference's own FastMatmul (its headers compiled unchanged by
oracle/Makefile into oracle/_ref/libfmm_ref.so, leaf products on the host
BLAS) on seeded inputs and records the results:

  * "full" cases (small shapes): the whole result matrix, bit-exact;
  * "digest" cases (the peeling shapes of tests/matmul_tests.cpp:140-145):
    the sums of the first 32 columns and 64 sampled entries;
  * for every case, the reference's error against its own classical product
    (max relative difference, linalg/linalg.hpp:280-295), which bounds the
    approximate algorithms' error ("within 2x of the reference's").

Inputs: A = uniform(m, k, seed, 1), B = uniform(k, n, seed, 2),
C0 = uniform(m, n, seed, 3), all in [0, 1) (oracle.uniform).

Usage: python tests/golden/make_golden.py   (needs oracle/_ref built)
"""

from __future__ import annotations

import base64
import json
import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import oracle  # noqa: E402

# lambda per step count, as the reference's RunAlgorithm chooses it
# (algorithms/all_algorithms.hpp:102-141)
def default_x(alg: str, steps: int) -> float:
    if alg == "bini322_10_52_approx":
        return {2: 1e-4, 3: 1e-2, 4: 1e-1}.get(steps, 1e-8)
    if alg == "schonhage333_21_117_approx":
        return {1: 1e-4, 2: 1e-2, 3: 1e-1, 4: 1e-1}.get(steps, 1e-4)
    return 1e-8


FULL_ALGS = ["strassen", "grey424_26_206", "grey333_23_125", "smirnov333_23_128", "bini322_10_52_approx",
             "schonhage333_21_117_approx", "grey522_18_99", "grey323_15_89"]
FULL_SHAPES = [  # m, k, n, steps, alpha, beta
    (24, 20, 18, 2, 1.0, 0.0),
    (19, 15, 21, 1, 7.0, -1.3),
    (28, 27, 26, 3, -1.2, 2.5),
    (9, 7, 5, 2, 1.0, 0.5),
    (13, 11, 9, 0, 2.0, 3.0),
]
DIGEST_ALGS = ["strassen", "grey424_26_206", "grey333_23_125", "smirnov333_23_128", "bini322_10_52_approx"]
DIGEST_SHAPES = [(257, 500, 55), (101, 500, 340), (402, 500, 562)]


def enc(a: np.ndarray) -> str:
    return base64.b64encode(zlib.compress(np.asfortranarray(a).T.tobytes(), 9)).decode()


def dec(s: str, m: int, n: int) -> np.ndarray:
    raw = np.frombuffer(zlib.decompress(base64.b64decode(s)), dtype=np.float64)
    return np.asfortranarray(raw.reshape(n, m).T)


def sample_positions(m: int, n: int, count: int = 64):
    rng = np.random.default_rng(m * 1000003 + n)
    return [(int(rng.integers(0, m)), int(rng.integers(0, n))) for _ in range(count)]


def run_case(alg, m, k, n, steps, alpha, beta, seed):
    A = oracle.uniform(m, k, seed, 1)
    B = oracle.uniform(k, n, seed, 2)
    C0 = oracle.uniform(m, n, seed, 3)
    x = default_x(alg, steps)
    C = C0.copy(order="F")
    oracle.ref_fast_matmul(alg, A, B, C, steps, x, alpha, beta)
    Cc = C0.copy(order="F")
    oracle.ref_matmul(A, B, Cc, alpha, beta)
    return x, C, oracle.max_relative_diff(Cc, C)


def main():
    if not oracle.ref_available():
        print("oracle/_ref is not built")
        return 1
    oracle.ref_lib().fmmref_set_threads(1)
    cases = []
    seed = 100
    for alg in FULL_ALGS:
        for (m, k, n, steps, alpha, beta) in FULL_SHAPES:
            seed += 1
            x, C, err = run_case(alg, m, k, n, steps, alpha, beta, seed)
            cases.append({"kind": "full", "alg": alg, "m": m, "k": k, "n": n, "steps": steps, "x": x,
                          "alpha": alpha, "beta": beta, "seed": seed, "ref_err": err, "C": enc(C)})
    for alg in DIGEST_ALGS:
        for (m, k, n) in DIGEST_SHAPES:
            for steps in (1, 2):
                seed += 1
                x, C, err = run_case(alg, m, k, n, steps, 1.0, 0.0, seed)
                pos = sample_positions(m, n)
                cases.append({"kind": "digest", "alg": alg, "m": m, "k": k, "n": n, "steps": steps, "x": x,
                              "alpha": 1.0, "beta": 0.0, "seed": seed, "ref_err": err,
                              "colsum": [float(v).hex() for v in C.sum(axis=0)[:32]],
                              "samples": [[i, j, float(C[i, j]).hex()] for (i, j) in pos]})
    gen = oracle.uniform(4, 4, 1, 1)
    out = {
        "generator": "tests/golden/make_golden.py",
        "source": "reference headers compiled by oracle/Makefile, host BLAS leaves (1 thread)",
        "uniform_known_answer": {"rows": 4, "cols": 4, "seed": 1, "stream": 1,
                                 "values": [float(v).hex() for v in gen.T.ravel()]},
        "cases": cases,
    }
    path = os.path.join(HERE, "reference_cases.json")
    with open(path, "w") as fh:
        json.dump(out, fh, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes,", len(cases), "cases")
    return 0


if __name__ == "__main__":
    sys.exit(main())
