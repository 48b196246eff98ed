"""CUDA backend of the fast-matmul code generator.

The reference's generator (codegen/gen.py:880-1016) turns one coefficient
file into one C++ header with per-product addition loops.  This backend reads
the same coefficient files and emits, for every algorithm at once:

  csrc/generated/fmm_algorithms.h    C tables: dimensions, rank, U/V/W/SX/TX/MX
                                     as coefficient-slot indices, the
                                     source of every product's operands, and
                                     a host function that evaluates the
                                     coefficient slots for a given x.
  csrc/generated/fmm_alg_kernels.cuh device functions that form all S (or T)
                                     operands of one algorithm level from the
                                     M0*K0 (K0*N0) input blocks in one pass,
                                     and combine the R products into the
                                     M0*N0 output blocks (+ beta*C).
  include/fmm/algorithms.hpp         the C++ drop-in surface: one namespace per
                                     algorithm with the reference's
                                     FastMatmul(A, B, C, num_steps, x, alpha, beta).
  generated/algorithms.json          the same tables for Python tooling/tests.

Arithmetic order.  Every addition is emitted in the order the reference's
write-once adds evaluate it (codegen/gen.py:444-523 via arith_expression
:216-235): terms in increasing sub-block / product index, temporaries after
the plain blocks, a coefficient of 1 as a plain add, -1 as a subtract (a
leading -1 as a negation), anything else as a rounded product then a rounded
add, and ``+ beta * C`` last.  The device helpers use __dadd_rn/__dmul_rn so
no multiply-add contraction changes the rounding.

Operand sourcing follows codegen/gen.py:574-657 (write_multiply): a product
whose U (V) column has two or more nonzeros gets a materialised S (T)
operand; a single nonzero makes the operand a view of that block (or of a
materialised temporary) and folds the coefficient into the product's
multiplier.  Temporaries that some product uses alone must be materialised
(codegen/gen.py:237-265, need_streaming_cse_tmp); the rest live in registers.

Usage:  python gen_cuda.py <reference codegen/algorithms dir> [repo root]
"""

from __future__ import annotations

import json
import os
import sys
from typing import Dict, List, Tuple

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import coeffs as C  # noqa: E402

BANNER = ("Generated by fast_matmul_b200/codegen/gen_cuda.py from the fast-matmul "
          "coefficient files. Do not edit.")


class AlgTables:
    """Derived per-algorithm data shared by every emitted artefact."""

    def __init__(self, spec: C.AlgorithmSpec):
        self.spec = spec
        s = spec
        self.nA = s.m0 * s.k0
        self.nB = s.k0 * s.n0
        self.nC = s.m0 * s.n0
        self.R = s.rank
        # coefficient slots: every distinct nonzero coefficient string
        self.slot_of: Dict[str, int] = {}
        self.slot_expr: List[str] = []
        self.slot_const: List[bool] = []
        for mat in (s.U, s.V, s.W, s.SX, s.TX, s.MX):
            for row in mat:
                for c in row:
                    if C.is_zero_text(c):
                        continue
                    expr = C.parse_coeff(c)
                    if expr not in self.slot_of:
                        self.slot_of[expr] = len(self.slot_expr)
                        self.slot_expr.append(expr)
                        self.slot_const.append(C.rational_value(c) is not None)

        def enc(mat):
            return [[0 if C.is_zero_text(c) else self.slot_of[C.parse_coeff(c)] + 1 for c in row]
                    for row in mat]

        self.U = enc(s.U)
        self.V = enc(s.V)
        self.W = enc(s.W)
        self.SX = enc(s.SX)
        self.TX = enc(s.TX)
        self.MX = enc(s.MX)
        self.a_out, self.a_src = self._operands(self.U, self.nA, s.n_ax)
        self.b_out, self.b_src = self._operands(self.V, self.nB, s.n_bx)

    def _operands(self, mat, nplain, nx):
        """Materialised outputs and per-product operand source.

        Returns (outputs, sources).  outputs: list of ('X', x) / ('S', r) in
        the order the forming kernel writes them.  sources[r] =
        (kind, index, mult_slot): kind 0 = view of input block ``index``,
        kind 1 = materialised output ``index``; mult_slot = coefficient slot
        + 1 of a single nonzero (0 when the operand is a sum).
        """
        R = self.R
        cols = [[mat[i][r] for i in range(len(mat))] for r in range(R)]
        single_x = []
        for r in range(R):
            nz = [i for i, v in enumerate(cols[r]) if v]
            if len(nz) == 1 and nz[0] >= nplain and (nz[0] - nplain) not in single_x:
                single_x.append(nz[0] - nplain)
        single_x.sort()
        outputs = [("X", x) for x in single_x]
        sources = []
        for r in range(R):
            nz = [i for i, v in enumerate(cols[r]) if v]
            if len(nz) == 0:
                raise C.CoeffParseError("%s: product %d has an empty operand" % (self.spec.name, r + 1))
            if len(nz) >= 2:
                outputs.append(("S", r))
                sources.append((1, len(outputs) - 1, 0))
            elif nz[0] < nplain:
                sources.append((0, nz[0], cols[r][nz[0]]))
            else:
                sources.append((1, single_x.index(nz[0] - nplain), cols[r][nz[0]]))
        return outputs, sources


# ----------------------------------------------------------------------------
# expression emission


def _coef_text(t: AlgTables, slot1: int) -> str:
    slot = slot1 - 1
    if t.slot_const[slot]:
        return t.slot_expr[slot]
    return "cf[%d]" % slot


def _is_pm_one(t: AlgTables, slot1: int) -> int:
    slot = slot1 - 1
    if not t.slot_const[slot]:
        return 0
    v = float(t.slot_expr[slot])
    if v == 1.0:
        return 1
    if v == -1.0:
        return -1
    return 0


def _sum_expr(t: AlgTables, terms: List[Tuple[int, str]]) -> str:
    """terms: (coef slot+1, operand) in evaluation order."""
    acc = None
    for slot1, val in terms:
        pm = _is_pm_one(t, slot1)
        if acc is None:
            if pm == 1:
                acc = val
            elif pm == -1:
                acc = "fmm_neg(%s)" % val
            else:
                acc = "fmm_mul(%s, %s)" % (_coef_text(t, slot1), val)
        else:
            if pm == 1:
                acc = "fmm_add(%s, %s)" % (acc, val)
            elif pm == -1:
                acc = "fmm_sub(%s, %s)" % (acc, val)
            else:
                acc = "fmm_add(%s, fmm_mul(%s, %s))" % (acc, _coef_text(t, slot1), val)
    assert acc is not None
    return acc


def _emit_form(t: AlgTables, mat, xmat, nplain, outputs, in_prefix, fn) -> List[str]:
    lines = []
    lines.append("  template <class T, class Ld, class St>")
    lines.append("  __device__ __forceinline__ static void %s(const double* __restrict__ cf, Ld&& ld, St&& st) {" % fn)
    lines.append("    (void)cf;")
    for i in range(nplain):
        lines.append("    const T %s%d = ld(%d);" % (in_prefix, i, i))
    for x, row in enumerate(xmat):
        terms = [(row[i], "%s%d" % (in_prefix, i)) for i in range(nplain) if row[i]]
        lines.append("    const T %sx%d = %s;" % (in_prefix, x, _sum_expr(t, terms)))
    for o, (kind, idx) in enumerate(outputs):
        if kind == "X":
            lines.append("    st(%d, %sx%d);" % (o, in_prefix, idx))
        else:
            r = idx
            terms = []
            for i in range(len(mat)):
                if mat[i][r]:
                    name = ("%s%d" % (in_prefix, i)) if i < nplain else ("%sx%d" % (in_prefix, i - nplain))
                    terms.append((mat[i][r], name))
            lines.append("    st(%d, %s);  // operand of M%d" % (o, _sum_expr(t, terms), r + 1))
    lines.append("  }")
    return lines


def _emit_combine(t: AlgTables) -> List[str]:
    R = t.R
    lines = []
    lines.append("  template <class T, bool kBeta, class Ld, class LdC, class St>")
    lines.append("  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {")
    lines.append("    (void)cf; (void)beta;")
    for r in range(R):
        lines.append("    const T m%d = ld(%d);" % (r, r))
    for x, row in enumerate(t.MX):
        terms = [(row[r], "m%d" % r) for r in range(R) if row[r]]
        if not terms:
            continue
        lines.append("    const T mx%d = %s;" % (x, _sum_expr(t, terms)))
    for c, row in enumerate(t.W):
        terms = []
        for j, v in enumerate(row):
            if v:
                terms.append((v, ("m%d" % j) if j < R else ("mx%d" % (j - R))))
        expr = _sum_expr(t, terms)
        lines.append("    if (kBeta) st(%d, fmm_add(%s, fmm_mul(beta, ldc(%d)))); else st(%d, %s);"
                     % (c, expr, c, c, expr))
    lines.append("  }")
    return lines


def emit_kernels(tabs: List[AlgTables]) -> str:
    out = ["// " + BANNER,
           "// One struct per algorithm; FMM_FOR_EACH_ALGORITHM(X) expands X(index, struct).",
           "#pragma once",
           ""]
    for idx, t in enumerate(tabs):
        s = t.spec
        out.append("// %s  <%d,%d,%d; %d>  (reference header algorithms/%s, coefficients codegen/algorithms/%s)"
                   % (s.name, s.m0, s.k0, s.n0, t.R, s.header, s.source))
        out.append("struct FmmAlg_%s {" % s.name)
        out.append("  static constexpr int kM0 = %d, kK0 = %d, kN0 = %d, kR = %d;" % (s.m0, s.k0, s.n0, t.R))
        out.append("  static constexpr int kNumAOut = %d, kNumBOut = %d;" % (len(t.a_out), len(t.b_out)))
        out += _emit_form(t, t.U, t.SX, t.nA, t.a_out, "a", "form_s")
        out += _emit_form(t, t.V, t.TX, t.nB, t.b_out, "b", "form_t")
        out += _emit_combine(t)
        out.append("};")
        out.append("")
    out.append("#define FMM_FOR_EACH_ALGORITHM(X) \\")
    for idx, t in enumerate(tabs):
        out.append("  X(%d, FmmAlg_%s)%s" % (idx, t.spec.name, " \\" if idx + 1 < len(tabs) else ""))
    out.append("")
    return "\n".join(out)


def _c_array(name: str, rows: List[List[int]], ctype="short") -> str:
    flat = [v for row in rows for v in row]
    if not flat:
        return "static const %s %s[1] = {0};" % (ctype, name)
    body = ", ".join(str(v) for v in flat)
    return "static const %s %s[%d] = {%s};" % (ctype, name, len(flat), body)


def emit_tables(tabs: List[AlgTables]) -> str:
    out = ["/* " + BANNER + " */",
           "#ifndef FMM_ALGORITHMS_GENERATED_H_",
           "#define FMM_ALGORITHMS_GENERATED_H_",
           "",
           "/* Coefficient matrices are stored row-major with entries = coefficient slot + 1",
           " * (0 = zero coefficient). Slot values come from the eval function, which",
           " * computes each coefficient with the same double-precision expression the",
           " * reference header uses. Operand sources: kind 0 = view of input block",
           " * `index`, kind 1 = materialised output `index` of the forming kernel;",
           " * mult = slot + 1 of the single coefficient folded into the product's",
           " * multiplier (0 = none). */",
           "",
           "typedef struct fmm_alg_table {",
           "  const char* name;        /* namespace of the reference header */",
           "  const char* header;      /* reference header file name */",
           "  int m0, k0, n0, rank;",
           "  int n_ax, n_bx, n_mx;    /* common-subexpression temporaries */",
           "  int n_slots;",
           "  int approximate;         /* coefficients depend on x */",
           "  void (*eval)(double x, double* slots);",
           "  const short* U;          /* (m0*k0 + n_ax) x rank */",
           "  const short* V;          /* (k0*n0 + n_bx) x rank */",
           "  const short* W;          /* (m0*n0) x (rank + n_mx) */",
           "  const short* SX;         /* n_ax x (m0*k0) */",
           "  const short* TX;         /* n_bx x (k0*n0) */",
           "  const short* MX;         /* n_mx x rank */",
           "  int n_a_out, n_b_out;    /* materialised S-side / T-side outputs */",
           "  const short* a_src;      /* rank x 3: kind, index, mult */",
           "  const short* b_src;      /* rank x 3 */",
           "} fmm_alg_table;",
           ""]
    for t in tabs:
        s = t.spec
        n = s.name
        out.append("/* %s <%d,%d,%d;%d> */" % (n, s.m0, s.k0, s.n0, t.R))
        out.append("static void fmm_eval_%s(double x, double* slots) {" % n)
        out.append("  (void)x;")
        for i, e in enumerate(t.slot_expr):
            out.append("  slots[%d] = %s;" % (i, e))
        out.append("}")
        out.append(_c_array("fmm_U_%s" % n, t.U))
        out.append(_c_array("fmm_V_%s" % n, t.V))
        out.append(_c_array("fmm_W_%s" % n, t.W))
        out.append(_c_array("fmm_SX_%s" % n, t.SX))
        out.append(_c_array("fmm_TX_%s" % n, t.TX))
        out.append(_c_array("fmm_MX_%s" % n, t.MX))
        out.append(_c_array("fmm_asrc_%s" % n, [list(x) for x in t.a_src]))
        out.append(_c_array("fmm_bsrc_%s" % n, [list(x) for x in t.b_src]))
        out.append("")
    out.append("#define FMM_NUM_ALGORITHMS %d" % len(tabs))
    out.append("#define FMM_MAX_SLOTS %d" % max(len(t.slot_expr) for t in tabs))
    out.append("#define FMM_MAX_RANK %d" % max(t.R for t in tabs))
    out.append("static const fmm_alg_table fmm_algorithms[FMM_NUM_ALGORITHMS] = {")
    for t in tabs:
        s = t.spec
        n = s.name
        out.append('  {"%s", "%s", %d, %d, %d, %d, %d, %d, %d, %d, %d, fmm_eval_%s, fmm_U_%s, fmm_V_%s, fmm_W_%s, '
                   'fmm_SX_%s, fmm_TX_%s, fmm_MX_%s, %d, %d, fmm_asrc_%s, fmm_bsrc_%s},'
                   % (n, s.header, s.m0, s.k0, s.n0, t.R, s.n_ax, s.n_bx, s.n_mx, len(t.slot_expr),
                      1 if s.approximate else 0, n, n, n, n, n, n, n, len(t.a_out), len(t.b_out), n, n))
    out.append("};")
    out.append("")
    out.append("#endif /* FMM_ALGORITHMS_GENERATED_H_ */")
    out.append("")
    return "\n".join(out)


def emit_adapter(tabs: List[AlgTables]) -> str:
    out = ["// " + BANNER,
           "// The reference's per-algorithm entry points (one namespace per generated",
           "// header, e.g. algorithms/strassen.hpp:661-722), routed to the B200 engine.",
           "#pragma once",
           '#include "fmm/matrix.hpp"',
           "",
           "namespace fmm {",
           "enum AlgorithmId {"]
    for i, t in enumerate(tabs):
        out.append("  kAlg_%s = %d," % (t.spec.name, i))
    out.append("};")
    out.append("}  // namespace fmm")
    out.append("")
    for i, t in enumerate(tabs):
        s = t.spec
        out.append("namespace %s {" % s.name)
        out.append("// C := alpha * A * B + beta * C with <%d,%d,%d;%d>, num_steps recursive levels." % (s.m0, s.k0, s.n0, t.R))
        out.append("template <typename Scalar>")
        out.append("double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,")
        out.append("                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {")
        out.append("  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_%s, A, B, C, num_steps, x, alpha, beta);" % s.name)
        out.append("}")
        out.append("}  // namespace %s" % s.name)
        out.append("")
    return "\n".join(out)


def emit_json(tabs: List[AlgTables]) -> str:
    algs = []
    for t in tabs:
        s = t.spec
        algs.append({
            "name": s.name, "header": s.header, "source": s.source,
            "m0": s.m0, "k0": s.k0, "n0": s.n0, "rank": t.R,
            "n_ax": s.n_ax, "n_bx": s.n_bx, "n_mx": s.n_mx,
            "approximate": s.approximate,
            "raw": {"U": s.U, "V": s.V, "W": s.W, "SX": s.SX, "TX": s.TX, "MX": s.MX},
            "slots": t.slot_expr,
            "U": t.U, "V": t.V, "W": t.W, "SX": t.SX, "TX": t.TX, "MX": t.MX,
            "a_out": t.a_out, "b_out": t.b_out,
            "a_src": t.a_src, "b_src": t.b_src,
        })
    return json.dumps({"generator": BANNER, "algorithms": algs}, indent=None, separators=(",", ":"))


def main(argv):
    if len(argv) < 2:
        print(__doc__)
        return 2
    coeff_root = argv[1]
    repo = argv[2] if len(argv) > 2 else os.path.abspath(os.path.join(HERE, "..", ".."))
    specs = C.load_all(coeff_root)
    tabs = [AlgTables(specs[name]) for name, _, _, _ in C.ALGORITHM_TABLE]
    pkg = os.path.join(repo, "fast_matmul_b200")
    files = {
        os.path.join(pkg, "csrc", "generated", "fmm_algorithms.h"): emit_tables(tabs),
        os.path.join(pkg, "csrc", "generated", "fmm_alg_kernels.cuh"): emit_kernels(tabs),
        os.path.join(repo, "include", "fmm", "algorithms.hpp"): emit_adapter(tabs),
        os.path.join(pkg, "generated", "algorithms.json"): emit_json(tabs),
    }
    for path, text in files.items():
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as fh:
            fh.write(text)
        print("wrote", os.path.relpath(path, repo))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
