"""Generates digest fixtures of the reference's own results at large sizes.

The reference's FastMatmul (its headers compiled unchanged by oracle/Makefile
into oracle/_ref/libfmm_ref.so, leaf products on the host BLAS) runs here on
seeded inputs; each result is stored as a digest (tests/golden/digest.py:
sampled entries, fringe rows and columns included, and row/column band sums)
together with the reference's own error against its classical product
(MaxRelativeDiff, linalg/linalg.hpp:280-295).  The GPU tests recompute the
same inputs on the device (fmm.random_matrix is the same generator as
oracle.uniform) and compare.

Sets (each written to its own JSON file beside this script):

  baseline   the benchmark configurations: Strassen 4096^3 with 1 and 2
             steps; grey424_26_206, grey333_23_125 and smirnov333_23_128 at
             4096^3 with 1-3 steps; the same three at 1-3 steps on 16384^3,
             16384 x 1600 x 16384 and 65536 x 2400 x 2400 (fast424_26_206
             at 16384^3 with 2 steps is the headline product, seed 1234 as
             the benchmark uses); Strassen 16384^3 with 1-3 steps.
  matrix     tests/matmul_tests.cpp:137-173: the 27 algorithms of
             FastMatmulTests x its 17 shapes x steps 1-3 (TestSet, :30-41),
             plus grey323_15_89 itself (the reference's dispatcher runs
             grey323_15_103 for FAST323_15_89, all_algorithms.hpp:159-160).
  lambda     tests/bini_stability.cpp:17-38, schonhage_stability.cpp and
             smirnov333_stability.cpp: lambda = DBL_EPSILON doubling while
             below 1, steps 1-2, 90 x 80 x 80 (Bini) or 90^3; and Bini at
             8192^3 with lambda = 2^-10 .. 2^-26, steps 1-2.

Usage:  python tests/golden/make_reference_digests.py [baseline|matrix|lambda ...]
        (needs oracle/_ref built; uses every host thread for the BLAS)
"""

from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, HERE)

import digest as dg  # noqa: E402
import oracle  # noqa: E402

ALGS = {a["name"]: a for a in json.load(open(os.path.join(REPO, "fast_matmul_b200", "generated",
                                                           "algorithms.json")))["algorithms"]}

# tests/matmul_tests.cpp:147-173, as (enum name, namespace the dispatcher runs)
MATRIX_ALGS = [
    ("STRASSEN", "strassen"), ("FAST333_23_125", "grey333_23_125"), ("FAST322_11_50", "grey322_11_50"),
    ("FAST332_15_103", "grey332_15_103"), ("FAST323_15_103", "grey323_15_103"),
    ("FAST323_15_89", "grey323_15_103"), ("FAST333_23_152", "grey333_23_152"),
    ("FAST333_23_221", "grey333_23_221"), ("FAST432_20_144", "grey432_20_144"),
    ("FAST423_20_144", "grey423_20_144"), ("FAST324_20_144", "grey324_20_144"),
    ("FAST342_20_144", "grey342_20_144"), ("FAST234_20_144", "grey234_20_144"),
    ("FAST243_20_144", "grey243_20_144"), ("FAST422_14_84", "grey422_14_84"),
    ("FAST424_26_257", "grey424_26_257"), ("FAST424_26_206", "grey424_26_206"),
    ("FAST433_29_234", "grey433_29_234"), ("FAST522_18_99", "grey522_18_99"),
    ("SMIRNOV333_23_128", "smirnov333_23_128"), ("SMIRNOV333_23_139", "smirnov333_23_139"),
    ("HK332_15_94", "hk332_15_94"), ("HK323_15_84", "hk323_15_84"),
    ("BINI322_10_52_APPROX", "bini322_10_52_approx"),
    ("SCHONHAGE333_21_117_APPROX", "schonhage333_21_117_approx"),
    ("CLASSICAL222", "classical222_8_24"), ("CLASSICAL333", "classical333_27_81"),
    (None, "grey323_15_89"),
]
# tests/matmul_tests.cpp:138-143
MATRIX_SHAPES = list(zip([257, 300, 366, 101, 402, 600, 634, 4001, 4002, 4003, 4004, 4005, 4006, 4007, 4008, 4009,
                          4010],
                         [500, 500, 500, 500, 500, 500, 700, 1000, 1200, 1301, 1400, 1477, 1514, 2020, 2100, 2800,
                          2900],
                         [55, 100, 200, 340, 562, 671, 1000, 1200, 1201, 1201, 1300, 1400, 1500, 2000, 2003, 2489,
                          2765]))
MATRIX_SAMPLES, MATRIX_GROUPS = 48, 16
BASE_SAMPLES, BASE_GROUPS = 256, 64


def default_x(alg: str, steps: int) -> float:
    """lambda per step count as the reference's RunAlgorithm picks it
    (algorithms/all_algorithms.hpp:102-141); 1e-8 (FastMatmul's default x)
    for the exact algorithms."""
    if alg == "bini322_10_52_approx":
        return {2: 1e-4, 3: 1e-2, 4: 1e-1}.get(steps, 1e-8)
    if alg == "schonhage333_21_117_approx":
        return {1: 1e-4, 2: 1e-2, 3: 1e-1, 4: 1e-1}.get(steps, 1e-4)
    return 1e-8


class Inputs:
    """Seeded operands and the reference's classical product, kept per shape."""

    def __init__(self):
        self.key = None

    def get(self, m, k, n, seed):
        if self.key != (m, k, n, seed):
            self.A = oracle.uniform(m, k, seed, 1)
            self.B = oracle.uniform(k, n, seed, 2)
            self.Cc = np.zeros((m, n), order="F")
            oracle.ref_matmul(self.A, self.B, self.Cc)
            self.key = (m, k, n, seed)
        return self.A, self.B, self.Cc


def run(inputs, alg, m, k, n, steps, seed, x, samples, groups):
    A, B, Cc = inputs.get(m, k, n, seed)
    C = np.zeros((m, n), order="F")
    t0 = time.perf_counter()
    oracle.ref_fast_matmul(alg, A, B, C, steps, x, 1.0, 0.0)
    dt = time.perf_counter() - t0
    info = ALGS[alg]
    rows, cols = dg.positions(m, n, info["m0"], info["n0"], steps, samples, seed)
    d = dg.digest_np(C, rows, cols, groups)
    rec = {"alg": alg, "m": m, "k": k, "n": n, "steps": steps, "seed": seed, "x": x, "alpha": 1.0, "beta": 0.0,
           "samples_count": samples, "groups": groups, "ref_err": oracle.max_relative_diff(Cc, C),
           "ref_s": round(dt, 3), "samples": dg.enc(d["samples"]), "rowsum": dg.enc(d["rowsum"]),
           "colsum": dg.enc(d["colsum"])}
    return rec


def write(name, cases, note):
    out = {"generator": "tests/golden/make_reference_digests.py " + name,
           "source": "reference headers compiled by oracle/Makefile, host BLAS leaves",
           "inputs": "A = uniform(m, k, seed, 1), B = uniform(k, n, seed, 2) in [0, 1) (oracle.uniform), "
                     "alpha 1, beta 0",
           "note": note, "cases": cases}
    path = os.path.join(HERE, "reference_%s.json" % name)
    with open(path, "w") as fh:
        json.dump(out, fh, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes,", len(cases), "cases", flush=True)


def make_baseline():
    cases = []
    inp = Inputs()
    plan = [((4096, 4096, 4096), [("strassen", (1, 2)), ("grey424_26_206", (1, 2, 3)), ("grey333_23_125", (1, 2, 3)),
                                  ("smirnov333_23_128", (1, 2, 3))]),
            ((16384, 16384, 16384), [("grey424_26_206", (2, 1, 3)), ("strassen", (1, 2, 3)),
                                     ("grey333_23_125", (1, 2, 3)), ("smirnov333_23_128", (1, 2, 3))]),
            ((16384, 1600, 16384), [("grey424_26_206", (1, 2, 3)), ("grey333_23_125", (1, 2, 3)),
                                    ("smirnov333_23_128", (1, 2, 3))]),
            ((65536, 2400, 2400), [("grey424_26_206", (1, 2, 3)), ("grey333_23_125", (1, 2, 3)),
                                   ("smirnov333_23_128", (1, 2, 3))])]
    for (m, k, n), algs in plan:
        for alg, steps_list in algs:
            for steps in steps_list:
                rec = run(inp, alg, m, k, n, steps, 1234, default_x(alg, steps), BASE_SAMPLES, BASE_GROUPS)
                cases.append(rec)
                print("%s %dx%dx%d s%d: ref_err %.3e, %.1f s" % (alg, m, k, n, steps, rec["ref_err"], rec["ref_s"]),
                      flush=True)
                write("baseline", cases, "benchmark configurations; seed 1234 for every shape")


def make_matrix():
    cases = []
    inp = Inputs()
    done = {}
    for si, (m, k, n) in enumerate(MATRIX_SHAPES):
        seed = 500 + si
        for enum, alg in MATRIX_ALGS:
            for steps in (1, 2, 3):
                key = (alg, steps)
                if key in done:  # FAST323_15_89 runs grey323_15_103 (same inputs, same result)
                    rec = dict(done[key])
                else:
                    rec = run(inp, alg, m, k, n, steps, seed, default_x(alg, steps), MATRIX_SAMPLES,
                              MATRIX_GROUPS)
                    done[key] = rec
                rec = dict(rec)
                rec["enum"] = enum
                cases.append(rec)
        done.clear()
        print("shape %dx%dx%d done (%d cases)" % (m, k, n, len(cases)), flush=True)
    write("matrix", cases, "tests/matmul_tests.cpp FastMatmulTests: 27 algorithms x 17 shapes x steps 1-3, "
                           "plus grey323_15_89 (enum null)")


def make_lambda():
    cases = []
    inp = Inputs()
    eps = float(np.finfo(np.float64).eps)
    for alg, (m, k, n) in (("bini322_10_52_approx", (90, 80, 80)), ("schonhage333_21_117_approx", (90, 90, 90)),
                           ("smirnov333_20_182_approx", (90, 90, 90))):
        for steps in (1, 2):
            lam = eps
            while lam < 1:
                rec = run(inp, alg, m, k, n, steps, 900, lam, 64, 16)
                rec["sweep"] = "stability"
                cases.append(rec)
                lam *= 2
    for steps in (1, 2):
        for e in range(10, 27):
            rec = run(inp, "bini322_10_52_approx", 8192, 8192, 8192, steps, 901, 2.0 ** -e, 256, 64)
            rec["sweep"] = "benchmark"
            cases.append(rec)
            print("bini 8192^3 s%d lambda 2^-%d: ref_err %.3e" % (steps, e, rec["ref_err"]), flush=True)
    write("lambda", cases, "lambda sweeps: tests/*_stability.cpp (DBL_EPSILON doubling below 1) and the benchmark's "
                           "2^-10..2^-26 at 8192^3")


def main(argv):
    if not oracle.ref_available():
        print("oracle/_ref is not built (make -C oracle ref)")
        return 1
    oracle.ref_lib().fmmref_set_threads(os.cpu_count() or 1)
    todo = argv or ["lambda", "matrix", "baseline"]
    for name in todo:
        {"baseline": make_baseline, "matrix": make_matrix, "lambda": make_lambda}[name]()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
