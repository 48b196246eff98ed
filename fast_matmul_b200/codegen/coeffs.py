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
