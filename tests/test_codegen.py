"""Coefficient parsing, algorithm validity (Brent equations) and generated tables.

Known-answer checks for the coefficient files: an exact algorithm must
satisfy the Brent equations over the rationals (the reference's
codegen/verify.py:108-130 and verify2.py:163-319 check the same), an
approximate one must satisfy them up to O(x).
"""

import json
import os
import subprocess
import sys
import tempfile
from fractions import Fraction

import numpy as np
import pytest

from helpers import REPO

sys.path.insert(0, os.path.join(REPO, "fast_matmul_b200", "codegen"))
import coeffs  # noqa: E402
import oracle  # noqa: E402

JSON = os.path.join(REPO, "fast_matmul_b200", "generated", "algorithms.json")


def algorithms():
    with open(JSON) as fh:
        return json.load(fh)["algorithms"]


ALGS = algorithms()


@pytest.mark.parametrize("text,expr", [
    ("1", "1.0"), ("-1", "-1.0"), (".5", "0.5"), ("-1/8", "-0.125"), ("x", "x"), ("-x", "-(x)"),
    ("xi", "1.0 / (x)"), ("-x2i", "-(1.0 / (x * x))"), ("x3", "x * x * x"), ("2x3", "2.0 * (x * x * x)"),
    ("-2x2", "-(2.0 * (x * x))"), ("(1+-x3)", "(1.0 + -(x * x * x))"), ("(-x+x2)", "(-(x) + x * x)"),
])
def test_parse_coeff_grammar(text, expr):
    assert coeffs.parse_coeff(text) == expr


def test_parse_coeff_rejects_garbage():
    with pytest.raises(coeffs.CoeffParseError):
        coeffs.parse_coeff("3x3x3")


brent_residual = coeffs.brent_residual


EXACT = [a for a in ALGS if not a["approximate"]]
APPROX = [a for a in ALGS if a["approximate"]]


@pytest.mark.parametrize("alg", EXACT, ids=[a["name"] for a in EXACT])
def test_exact_algorithms_satisfy_brent_equations(alg):
    assert brent_residual(alg) == 0


# smirnov333_20_182_approx: its coefficient file does not reduce to the
# product as x -> 0 (the reference's own header gives errors of 1e15 and
# more); it is generated and run like the others but not held to validity.
BROKEN_APPROX = {"smirnov333_20_182_approx"}


@pytest.mark.parametrize("alg", APPROX, ids=[a["name"] for a in APPROX])
def test_approximate_algorithms_converge(alg):
    r1 = brent_residual(alg, 1e-3)
    r2 = brent_residual(alg, 1e-5)
    if alg["name"] in BROKEN_APPROX:
        assert r2 > 1e-2
        return
    assert r2 < r1 and r2 < 1e-3


def test_tables_encode_raw_coefficients():
    for a in ALGS:
        slots = a["slots"]
        for key in ("U", "V", "W", "SX", "TX", "MX"):
            for row_raw, row_enc in zip(a["raw"][key], a[key]):
                for t, e in zip(row_raw, row_enc):
                    if coeffs.is_zero_text(t):
                        assert e == 0
                    else:
                        assert slots[e - 1] == coeffs.parse_coeff(t)


def test_operand_sources_match_column_structure():
    for a in ALGS:
        R = a["rank"]
        nA = a["m0"] * a["k0"]
        for r in range(R):
            nz = [i for i in range(len(a["U"])) if a["U"][i][r]]
            kind, idx, mult = a["a_src"][r]
            if len(nz) >= 2:
                assert kind == 1 and mult == 0 and a["a_out"][idx] == ["S", r]
            elif nz[0] < nA:
                assert kind == 0 and idx == nz[0] and mult == a["U"][nz[0]][r]
            else:
                assert kind == 1 and a["a_out"][idx] == ["X", nz[0] - nA]


def test_slot_expressions_evaluate_like_c():
    """The header eval functions and Python agree on every coefficient."""
    for a in ALGS:
        for e in a["slots"]:
            v = eval(e, {"__builtins__": {}}, {"x": 1e-4})
            assert np.isfinite(v)


@pytest.mark.skipif(oracle.reference_tree() is None, reason="reference tree not present")
def test_generated_files_are_current():
    gen = os.path.join(REPO, "fast_matmul_b200", "codegen", "gen_cuda.py")
    coeff_dir = os.path.join(oracle.reference_tree(), "codegen", "algorithms")
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([sys.executable, gen, coeff_dir, tmp], check=True, capture_output=True)
        for rel in ("fast_matmul_b200/csrc/generated/fmm_algorithms.h",
                    "fast_matmul_b200/csrc/generated/fmm_alg_kernels.cuh",
                    "include/fmm/algorithms.hpp",
                    "fast_matmul_b200/generated/algorithms.json"):
            with open(os.path.join(tmp, rel)) as a, open(os.path.join(REPO, rel)) as b:
                assert a.read() == b.read(), rel


def test_operation_counts_of_grey333_23_125_match_the_reference_example():
    """The example output in the docstring of the reference's
    codegen/counts.py:15-28 for algorithms/eliminated/grey333-23-125."""
    alg = next(a for a in ALGS if a["name"] == "grey333_23_125")
    c = coeffs.operation_counts(alg)
    assert c["A"] == (12, 35, 10) and c["B"] == (11, 34, 10) and c["C"] == (29, 38, 9)
    assert c["AX"] == (6, 12, 6) and c["BX"] == (7, 14, 7) and c["CX"] == (5, 10, 5)
    assert c["tot"] == (70, 143, 47)


def test_strassen_has_eighteen_additions():
    c = coeffs.operation_counts(next(a for a in ALGS if a["name"] == "strassen"))
    assert c["A"] == (5, 12, 5) and c["B"] == (5, 12, 5) and c["C"] == (8, 12, 4)
    assert c["tot"][0] == 18 and c["xtot"] == (0, 0, 0)


def test_counts_and_verify_command_line(tmp_path):
    """python coeffs.py counts|verify FILE M0,K0,N0 on a coefficient file
    written from the generated tables (the reference tree is not needed)."""
    script = os.path.join(REPO, "fast_matmul_b200", "codegen", "coeffs.py")
    for name in ("strassen", "grey333_23_125", "bini322_10_52_approx"):
        alg = next(a for a in ALGS if a["name"] == name)
        raw = alg["raw"]
        path = tmp_path / name
        secs = [raw["U"], raw["V"], raw["W"]] + ([raw["SX"], raw["TX"], raw["MX"]] if raw["SX"] else [])
        path.write_text("\n#\n".join("\n".join(" ".join(r) for r in sec) for sec in secs) + "\n")
        dims = "%d,%d,%d" % (alg["m0"], alg["k0"], alg["n0"])
        out = subprocess.run([sys.executable, script, "counts", str(path), dims], capture_output=True, text=True)
        assert out.returncode == 0, out.stderr
        tot = coeffs.operation_counts(alg)["tot"]
        assert out.stdout.strip().splitlines()[-1].split()[1:] == [str(v) for v in tot]
        out = subprocess.run([sys.executable, script, "verify", str(path), dims], capture_output=True, text=True)
        assert out.returncode == 0, out.stdout + out.stderr
    # a broken algorithm fails verification
    alg = next(a for a in ALGS if a["name"] == "strassen")
    U = [row[:] for row in alg["raw"]["U"]]
    U[0][0] = "-1"
    path = tmp_path / "broken"
    path.write_text("\n#\n".join("\n".join(" ".join(r) for r in sec) for sec in (U, alg["raw"]["V"], alg["raw"]["W"])) + "\n")
    out = subprocess.run([sys.executable, script, "verify", str(path), "2,2,2"], capture_output=True, text=True)
    assert out.returncode == 1, out.stdout
