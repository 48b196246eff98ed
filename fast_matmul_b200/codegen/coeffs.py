"""Coefficient files of fast matrix-multiplication algorithms.

A fast algorithm <M0,K0,N0;R> is three coefficient matrices U, V, W stored as
text, one row per sub-block (row-major block order), one column per product,
sections separated by lines starting with '#' (format described in
codegen/gen.py:26-50 of the reference).  Files produced by the reference's
common-subexpression elimination (codegen/subexpr_elim.py) append rows to U
and V that reference temporaries X_i, columns to W for output temporaries,
and, after a '# Substitution information' line, three more sections that
define the temporaries: A_X_i = sum_j SX[i][j] A_j, B_X_i = sum_j TX[i][j] B_j,
M_X_i = sum_r MX[i][r] M_r (consumed by codegen/gen.py:401-414,685-692,742-781).

This module parses that format into plain Python data and turns every
nonzero coefficient into a C expression in the algorithm parameter ``x``
(lambda for approximate algorithms).  The expression grammar follows
codegen/gen.py:101-147 (parse_coeff):

    c  -> c 'i'        1.0 / (c)
        | '-' c        -(c)
        | c DIGIT      (c) * (c) * ...   (DIGIT factors)
        | NUM 'x' ...  NUM * (rest)
        | '(' c '+' c ... ')'
        | letter       x
        | rational     its double value

and the emitted C text keeps the same association, so the value computed in
double precision is bit-identical to the reference's ``Scalar(<expr>)``.
"""

from __future__ import annotations

import dataclasses
import os
from fractions import Fraction
from typing import Dict, List, Optional, Tuple


class CoeffParseError(ValueError):
    pass


def _is_rational(text: str) -> Optional[Fraction]:
    try:
        return Fraction(text)
    except (ValueError, ZeroDivisionError):
        return None


def _double_literal(value: float) -> str:
    """C literal that round-trips to exactly ``value``."""
    text = repr(float(value))
    if "e" not in text and "." not in text and "inf" not in text and "nan" not in text:
        text += ".0"
    return text


def parse_coeff(text: str) -> str:
    """Return the C expression for one coefficient string.

    Mirrors codegen/gen.py:101-147: a rational becomes its double value; the
    parameterised forms become an expression in ``x`` with the same
    operator association as the reference's generated ``Scalar(...)``.
    """
    coeff = text.strip()
    if not coeff:
        raise CoeffParseError("empty coefficient")
    frac = _is_rational(coeff)
    if frac is not None:
        return _double_literal(float(frac))
    if len(coeff) == 1:
        # any single letter is the algorithm parameter
        return "x"
    if coeff[0] == "(":
        if coeff[-1] != ")":
            raise CoeffParseError("unbalanced parenthesis in %r" % text)
        parts = coeff[1:-1].split("+")
        return "(" + " + ".join(parse_coeff(p) for p in parts) + ")"
    if coeff[0] == "-":
        return "-(%s)" % parse_coeff(coeff[1:])
    xpos = coeff.find("x")
    if xpos > 0:
        mult = _is_rational(coeff[:xpos])
        if mult is not None:
            return "%s * (%s)" % (_double_literal(float(mult)), parse_coeff(coeff[xpos:]))
    if coeff[-1] == "i":
        return "1.0 / (%s)" % parse_coeff(coeff[:-1])
    if coeff[-1].isdigit():
        inner = parse_coeff(coeff[:-1])
        return " * ".join([inner] * int(coeff[-1]))
    raise CoeffParseError("cannot parse coefficient %r" % text)


def is_zero_text(text: str) -> bool:
    frac = _is_rational(text.strip())
    return frac is not None and frac == 0


def rational_value(text: str) -> Optional[Fraction]:
    """Exact value of a constant coefficient, or None if it depends on x."""
    return _is_rational(text.strip())


@dataclasses.dataclass
class AlgorithmSpec:
    """One fast algorithm, exactly as its coefficient file defines it.

    ``U`` has M0*K0 (+ number of A temporaries) rows and R columns,
    ``V`` has K0*N0 (+ B temporaries) rows and R columns,
    ``W`` has M0*N0 rows and R (+ M temporaries) columns,
    ``SX``/``TX``/``MX`` define the temporaries (empty when there is no CSE).
    Entries are the raw coefficient strings ("0", "1", "-.5", "x2i", ...).
    """

    name: str            # C++ namespace of the reference header, e.g. grey424_26_206
    header: str          # reference header file name, e.g. fast424_26_206.hpp
    source: str          # coefficient file, relative to codegen/algorithms
    m0: int
    k0: int
    n0: int
    U: List[List[str]]
    V: List[List[str]]
    W: List[List[str]]
    SX: List[List[str]]
    TX: List[List[str]]
    MX: List[List[str]]

    @property
    def rank(self) -> int:
        return len(self.U[0])

    @property
    def n_ax(self) -> int:
        return len(self.SX)

    @property
    def n_bx(self) -> int:
        return len(self.TX)

    @property
    def n_mx(self) -> int:
        return len(self.MX)

    @property
    def approximate(self) -> bool:
        for mat in (self.U, self.V, self.W, self.SX, self.TX, self.MX):
            for row in mat:
                for c in row:
                    if rational_value(c) is None:
                        return True
        return False

    def validate(self) -> None:
        m0, k0, n0, r = self.m0, self.k0, self.n0, self.rank
        if len(self.U) != m0 * k0 + self.n_ax:
            raise CoeffParseError("%s: U has %d rows, expected %d" % (self.name, len(self.U), m0 * k0 + self.n_ax))
        if len(self.V) != k0 * n0 + self.n_bx:
            raise CoeffParseError("%s: V has %d rows, expected %d" % (self.name, len(self.V), k0 * n0 + self.n_bx))
        if len(self.W) != m0 * n0:
            raise CoeffParseError("%s: W has %d rows, expected %d" % (self.name, len(self.W), m0 * n0))
        for row in self.U + self.V:
            if len(row) != r:
                raise CoeffParseError("%s: ragged U/V row" % self.name)
        for row in self.W:
            if len(row) != r + self.n_mx:
                raise CoeffParseError("%s: W row has %d entries, expected %d" % (self.name, len(row), r + self.n_mx))
        for row in self.SX:
            if len(row) != m0 * k0:
                raise CoeffParseError("%s: SX row length" % self.name)
        for row in self.TX:
            if len(row) != k0 * n0:
                raise CoeffParseError("%s: TX row length" % self.name)
        for row in self.MX:
            if len(row) != r:
                raise CoeffParseError("%s: MX row length" % self.name)
        for mat in (self.U, self.V, self.W, self.SX, self.TX, self.MX):
            for row in mat:
                for c in row:
                    if not is_zero_text(c):
                        parse_coeff(c)


def read_sections(path: str) -> List[List[List[str]]]:
    """Split a coefficient file into its '#'-separated sections
    (codegen/gen.py:150-170, read_coeffs)."""
    sections: List[List[List[str]]] = []
    current: List[List[str]] = []
    with open(path, "r") as fh:
        for line in fh:
            if line.startswith("#"):
                if current:
                    sections.append(current)
                    current = []
                continue
            toks = line.split()
            if toks:
                current.append(toks)
    sections.append(current)
    if len(sections) < 3:
        raise CoeffParseError("%s: expected at least three coefficient sections" % path)
    return sections


def load_algorithm(path: str, name: str, header: str, source: str,
                   dims: Tuple[int, int, int]) -> AlgorithmSpec:
    secs = read_sections(path)
    while len(secs) < 6:
        secs.append([])
    spec = AlgorithmSpec(name=name, header=header, source=source,
                         m0=dims[0], k0=dims[1], n0=dims[2],
                         U=secs[0], V=secs[1], W=secs[2],
                         SX=secs[3], TX=secs[4], MX=secs[5])
    spec.validate()
    return spec


# (namespace, reference header, coefficient file under codegen/algorithms, <M0,K0,N0>)
# The pairing of coefficient file, dimensions and namespace follows
# codegen/gen_all_algorithms.sh:31-86 and the namespaces declared at line 7 of
# each algorithms/*.hpp header.
ALGORITHM_TABLE: List[Tuple[str, str, str, Tuple[int, int, int]]] = [
    ("strassen", "strassen.hpp", "strassen", (2, 2, 2)),
    ("classical222_8_24", "classical222.hpp", "classical222-8-24", (2, 2, 2)),
    ("grey322_11_50", "fast322_11_50.hpp", "grey322-11-50", (3, 2, 2)),
    ("bini322_10_52_approx", "bini322_10_52_approx.hpp", "bini322-10-52-approx", (3, 2, 2)),
    ("grey332_15_103", "fast332_15_103.hpp", "grey332-15-103", (3, 3, 2)),
    ("grey323_15_103", "fast323_15_103.hpp", "grey323-15-103", (3, 2, 3)),
    ("hk332_15_94", "hk332_15_94.hpp", "hk332-15-94", (3, 3, 2)),
    ("hk323_15_94", "hk323_15_94.hpp", "hk323-15-94", (3, 2, 3)),
    ("hk323_15_84", "hk323_15_84.hpp", "eliminated/hk323-15-84", (3, 2, 3)),
    ("grey323_15_89", "fast323_15_89.hpp", "eliminated/grey323-15-89", (3, 2, 3)),
    ("grey333_23_152", "fast333_23_152.hpp", "grey333-23-152", (3, 3, 3)),
    ("grey333_23_221", "fast333_23_221.hpp", "grey333-23-221", (3, 3, 3)),
    ("grey333_23_125", "fast333_23_125.hpp", "eliminated/grey333-23-125", (3, 3, 3)),
    ("smirnov333_23_139", "smirnov333_23_139.hpp", "smirnov333-23-139", (3, 3, 3)),
    ("smirnov333_23_128", "smirnov333_23_128.hpp", "eliminated/smirnov333-23-128", (3, 3, 3)),
    ("classical333_27_81", "classical333.hpp", "classical333-27-81", (3, 3, 3)),
    ("schonhage333_21_117_approx", "schonhage333_21_117_approx.hpp", "schonhage333-21-117-approx", (3, 3, 3)),
    ("smirnov333_20_182_approx", "smirnov333_20_182_approx.hpp", "smirnov333-20-182-approx", (3, 3, 3)),
    ("grey422_14_84", "fast422_14_84.hpp", "grey422-14-84", (4, 2, 2)),
    ("grey432_20_144", "fast432_20_144.hpp", "grey432-20-144", (4, 3, 2)),
    ("grey423_20_144", "fast423_20_144.hpp", "grey423-20-144", (4, 2, 3)),
    ("grey324_20_144", "fast324_20_144.hpp", "grey324-20-144", (3, 2, 4)),
    ("grey342_20_144", "fast342_20_144.hpp", "grey342-20-144", (3, 4, 2)),
    ("grey234_20_144", "fast234_20_144.hpp", "grey234-20-144", (2, 3, 4)),
    ("grey243_20_144", "fast243_20_144.hpp", "grey243-20-144", (2, 4, 3)),
    ("classical423_24_72", "classical423.hpp", "classical423-24-72", (4, 2, 3)),
    ("fast423_130", "fast423_20_130.hpp", "fast423-130", (4, 2, 3)),
    ("fast423_134", "fast423_20_134.hpp", "fast423-134", (4, 2, 3)),
    ("fast423_138", "fast423_20_138.hpp", "fast423-138", (4, 2, 3)),
    ("fast423_156", "fast423_20_156.hpp", "fast423-156", (4, 2, 3)),
    ("grey433_29_234", "fast433_29_234.hpp", "grey433-29-234", (4, 3, 3)),
    ("grey343_29_234", "fast343_29_234.hpp", "grey343-29-234", (3, 4, 3)),
    ("grey442_26_257", "fast442_26_257.hpp", "grey442-26-257", (4, 4, 2)),
    ("grey424_26_257", "fast424_26_257.hpp", "grey424-26-257", (4, 2, 4)),
    ("grey424_26_206", "fast424_26_206.hpp", "eliminated/grey424-26-206", (4, 2, 4)),
    ("grey522_18_99", "fast522_18_99.hpp", "grey522-18-99", (5, 2, 2)),
    ("grey252_18_99", "fast252_18_99.hpp", "grey252-18-99", (2, 5, 2)),
    ("smirnov336_40_960", "smirnov336_40_960.hpp", "smirnov336-40-960", (3, 3, 6)),
    ("smirnov363_40_960", "smirnov363_40_960.hpp", "smirnov363-40-960", (3, 6, 3)),
    ("smirnov633_40_960", "smirnov633_40_960.hpp", "smirnov633-40-960", (6, 3, 3)),
    ("tichavsky_kovac336_40_960", "tichavsky_kovac336_40_960.hpp", "tichavsky_kovac336-40-960", (3, 3, 6)),
    ("tichavsky_kovac363_40_960", "tichavsky_kovac363_40_960.hpp", "tichavsky_kovac363-40-960", (3, 6, 3)),
]


def load_all(coeff_root: str) -> Dict[str, AlgorithmSpec]:
    out: Dict[str, AlgorithmSpec] = {}
    for name, header, source, dims in ALGORITHM_TABLE:
        out[name] = load_algorithm(os.path.join(coeff_root, source), name, header, source, dims)
    return out


# ---------------------------------------------------------------------------
# Checks and counts for coefficient files (CI tooling for new algorithms)


def as_record(spec: AlgorithmSpec) -> dict:
    """The fields of an algorithm record in generated/algorithms.json that
    the checks below read."""
    return {"name": spec.name, "m0": spec.m0, "k0": spec.k0, "n0": spec.n0, "rank": spec.rank,
            "raw": {"U": spec.U, "V": spec.V, "W": spec.W, "SX": spec.SX, "TX": spec.TX, "MX": spec.MX}}


def coefficient_value(text: str, x=None):
    """Exact rational value of a coefficient, or its value at x for one that
    depends on the algorithm parameter (the generated C expression, which
    only uses + - * / on x and double literals, evaluated in Python)."""
    if is_zero_text(text):
        return 0
    frac = rational_value(text)
    if frac is not None:
        return frac
    if x is None:
        raise ValueError("coefficient %r depends on x" % text)
    return eval(parse_coeff(text), {"__builtins__": {}}, {"x": x})


def effective_uvw(rec: dict, x=None):
    """U, V, W over the plain blocks with the common-subexpression
    temporaries substituted (A_X, B_X, M_X rows folded into the products)."""
    raw = rec["raw"]
    m0, k0, n0, R = rec["m0"], rec["k0"], rec["n0"], rec["rank"]
    nA, nB, nC = m0 * k0, k0 * n0, m0 * n0
    val = lambda t: coefficient_value(t, x)  # noqa: E731
    U = [[val(raw["U"][i][r]) for r in range(R)] for i in range(nA)]
    V = [[val(raw["V"][i][r]) for r in range(R)] for i in range(nB)]
    W = [[val(raw["W"][c][r]) for r in range(R)] for c in range(nC)]
    for xi, row in enumerate(raw["SX"]):
        for r in range(R):
            u = val(raw["U"][nA + xi][r])
            if u:
                for i in range(nA):
                    U[i][r] += u * val(row[i])
    for xi, row in enumerate(raw["TX"]):
        for r in range(R):
            v = val(raw["V"][nB + xi][r])
            if v:
                for i in range(nB):
                    V[i][r] += v * val(row[i])
    for xi, row in enumerate(raw["MX"]):
        for c in range(nC):
            w = val(raw["W"][c][R + xi])
            if w:
                for r in range(R):
                    W[c][r] += w * val(row[r])
    return U, V, W


def brent_residual(rec: dict, x=None):
    """max over the Brent equations sum_r U[ik][r] V[k'j][r] W[i'j'][r] =
    d(i,i') d(k,k') d(j,j') of |lhs - rhs|: exactly 0 (rationals) for an exact
    algorithm, O(x) for an approximate one evaluated at x (the check of the
    reference's codegen/verify.py:108-130 and verify2.py:163-319)."""
    U, V, W = effective_uvw(rec, x)
    m0, k0, n0, R = rec["m0"], rec["k0"], rec["n0"], rec["rank"]
    worst = 0
    for i in range(m0):
        for k in range(k0):
            for k2 in range(k0):
                for j in range(n0):
                    for i2 in range(m0):
                        for j2 in range(n0):
                            s = sum(U[i * k0 + k][r] * V[k2 * n0 + j][r] * W[i2 * n0 + j2][r] for r in range(R))
                            want = 1 if (i == i2 and k == k2 and j == j2) else 0
                            worst = max(worst, abs(s - want))
    return worst


def _nonzero(text: str) -> bool:
    # codegen/gen.py:61-62 of the reference compares the text with '0' and '0.0'
    return text not in ("0", "0.0")


def operation_counts(rec: dict) -> Dict[str, Tuple[int, int, int]]:
    """Additions, reads and writes of one recursion level, with the
    definitions of the reference's codegen/counts.py:36-58: per product, its
    S (T) operand costs nnz - 1 additions, nnz reads and one write when nnz >
    1 (columns of U, V); per C block the same over its row of W; per
    common-subexpression temporary nnz - 1 additions, nnz reads, one write.
    Returns rows A, B, C, AX, BX, CX, xtot, tot."""
    raw = rec["raw"]

    def base(cols):
        nnz = [sum(1 for t in col if _nonzero(t)) for col in cols]
        return (sum(c - 1 for c in nnz), sum(nnz), sum(1 for c in nnz if c > 1))

    def elim(rows):
        if not rows or any(len(r) == 0 for r in rows):
            return (0, 0, 0)
        nnz = [sum(1 for t in row if _nonzero(t)) for row in rows]
        return (sum(c - 1 for c in nnz), sum(nnz), len(rows))

    transpose = lambda m: [list(c) for c in zip(*m)] if m else []  # noqa: E731
    out = {"A": base(transpose(raw["U"])), "B": base(transpose(raw["V"])), "C": base(raw["W"]),
           "AX": elim(raw["SX"]), "BX": elim(raw["TX"]), "CX": elim(raw["MX"])}
    out["xtot"] = tuple(sum(v) for v in zip(out["AX"], out["BX"], out["CX"]))
    out["tot"] = tuple(sum(v) for v in zip(*(out[k] for k in ("A", "B", "C", "AX", "BX", "CX"))))
    return out


def format_counts(counts: Dict[str, Tuple[int, int, int]]) -> str:
    lines = ["      +   r   w"]
    for key in ("A", "B", "C", "AX", "BX", "CX", "xtot", "tot"):
        lines.append("%-4s %4d %3d %3d" % ((key,) + tuple(counts[key])))
    return "\n".join(lines)


def main(argv=None) -> int:
    """python coeffs.py counts|verify COEFF_FILE M0,K0,N0

    counts  additions / reads / writes of one level (A, B, C, temporaries)
    verify  Brent equations: exit 0 when an exact algorithm satisfies them
            exactly, or an approximate one converges as x -> 0"""
    import sys

    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 3 or argv[0] not in ("counts", "verify"):
        print(main.__doc__)
        return 2
    dims = tuple(int(d) for d in argv[2].split(","))
    spec = load_algorithm(argv[1], os.path.basename(argv[1]), "", argv[1], dims)
    rec = as_record(spec)
    if argv[0] == "counts":
        print(format_counts(operation_counts(rec)))
        return 0
    if not spec.approximate:
        res = brent_residual(rec)
        print("exact algorithm: max Brent residual %s" % res)
        return 0 if res == 0 else 1
    r1, r2 = brent_residual(rec, 1e-3), brent_residual(rec, 1e-5)
    print("approximate algorithm: residual %.3e at x = 1e-3, %.3e at x = 1e-5" % (r1, r2))
    return 0 if r2 < r1 and r2 < 1e-3 else 1


if __name__ == "__main__":
    raise SystemExit(main())
