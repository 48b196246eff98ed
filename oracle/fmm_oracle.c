/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle.  Never linked into, called by,
 * or shipped with the product library; only tests/, the smoke check and the
 * benchmark's CPU-baseline leg load it, and only to check results.
 *
 * A plain-C restatement of the reference's recursive fast matrix multiply as
 * its generated headers perform it in the sequential configuration:
 *
 *   Matrix view + multiplier      linalg/linalg.hpp:41-192
 *   floor sub-blocking            linalg/linalg.hpp:97-102,179-184
 *   MatMul (alpha = C.multiplier) linalg/linalg.hpp:261-269
 *   DynamicPeeling                linalg/linalg.hpp:201-244
 *   FastMatmulRecursive           algorithms/strassen.hpp:377-659 (emitted by
 *                                 codegen/gen.py:880-1016 for every algorithm)
 *   write-once additions          codegen/gen.py:444-523, arith_expression :216-235
 *   CSE temporaries (write-once)  algorithms/fast424_26_206.hpp:2107-2131,2893-2934
 *   FastMatmul wrapper            algorithms/strassen.hpp:661-722
 *   MaxRelativeDiff               linalg/linalg.hpp:280-295
 *
 * Coefficients come from the generated tables (fmm_algorithms.h), which hold
 * the coefficient files' values; every addition is evaluated term by term in
 * the reference's order with separate multiply and add roundings, so the
 * addition phases are bit-identical to the reference.  The leaf product is a
 * straightforward triple loop (the reference calls the host BLAS dgemm there;
 * no reference test pins bits at that boundary).
 *
 * Pinned against the reference itself: tests compare this oracle with the
 * reference headers compiled by oracle/Makefile (oracle/_ref) and with the
 * golden vectors under tests/golden, which that build produced.
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../fast_matmul_b200/csrc/generated/fmm_algorithms.h"

typedef struct {
  double* data;
  long stride;
  int m, n;
  double mult;
} omat;

static omat omat_view(double* data, long stride, int m, int n) {
  omat a;
  a.data = data;
  a.stride = stride;
  a.m = m;
  a.n = n;
  a.mult = 1.0;
  return a;
}

static omat omat_alloc(int m, int n, double mult) {
  omat a;
  size_t cnt = (size_t)(m > 0 ? m : 0) * (size_t)(n > 0 ? n : 0);
  a.data = (double*)malloc((cnt ? cnt : 1) * sizeof(double));
  a.stride = m > 0 ? m : 1;
  a.m = m;
  a.n = n;
  a.mult = mult;
  return a;
}

static void omat_free(omat* a) {
  free(a->data);
  a->data = NULL;
}

#define AT(a, i, j) ((a).data[(long)(i) + (long)(j) * (a).stride])

/* linalg/linalg.hpp:106-108 Submatrix (keeps the parent's multiplier) */
static omat submatrix(omat a, int r0, int c0, int nr, int nc) {
  omat s = a;
  s.data = a.data + r0 + (long)c0 * a.stride;
  s.m = nr;
  s.n = nc;
  return s;
}

/* linalg/linalg.hpp:97-102 + 179-184: block (bi, bj), 0-based here, of an
 * nbr x nbc floor split. */
static omat subblock(omat a, int nbr, int nbc, int bi, int bj) {
  int rs = a.m / nbr, cs = a.n / nbc;
  return submatrix(a, rs * bi, cs * bj, rs, cs);
}

/* Optional leaf-product hook: when set, every MatMul goes to it (the tests
 * install the reference's own BLAS here to pin the additions bit for bit). */
typedef void (*oracle_gemm_fn)(double* a, int lda, double* b, int ldb, double* c, int ldc, int m, int k, int n,
                               double alpha, double beta);
static oracle_gemm_fn g_leaf_gemm = NULL;

void oracle_set_leaf_gemm(oracle_gemm_fn fn) { g_leaf_gemm = fn; }

/* MatMul: C <- C.mult * A * B + beta * C (linalg/linalg.hpp:261-269); a
 * dgemm with beta == 0 overwrites C without reading it. */
static void omatmul(omat A, omat B, omat C, double beta) {
  int i, j, p;
  double alpha = C.mult;
  double* col;
  if (C.m <= 0 || C.n <= 0) return;
  if (g_leaf_gemm) {
    g_leaf_gemm(A.data, (int)A.stride, B.data, (int)B.stride, C.data, (int)C.stride, C.m, A.n, C.n, alpha, beta);
    return;
  }
  col = (double*)malloc(sizeof(double) * (size_t)C.m);
  for (j = 0; j < C.n; ++j) {
    for (i = 0; i < C.m; ++i) col[i] = 0.0;
    for (p = 0; p < A.n; ++p) {
      double b = AT(B, p, j);
      const double* acol = &AT(A, 0, p);
      for (i = 0; i < C.m; ++i) col[i] += acol[i] * b;
    }
    for (i = 0; i < C.m; ++i) {
      double v = alpha * col[i];
      if (beta != 0.0) v = v + beta * AT(C, i, j);
      AT(C, i, j) = v;
    }
  }
  free(col);
}

/* linalg/linalg.hpp:201-244 */
static void dynamic_peeling(omat A, omat B, omat C, int d1, int d2, int d3, double beta) {
  int extra_rows_A = A.m - (A.m / d1) * d1;
  int extra_cols_A = A.n - (A.n / d2) * d2;
  int extra_cols_B = B.n - (B.n / d3) * d3;
  if (extra_cols_A > 0) {
    int row_dim = A.m - extra_rows_A;
    int col_dim = B.n - extra_cols_B;
    int inner = A.n - extra_cols_A;
    omat Ax = submatrix(A, 0, inner, row_dim, extra_cols_A);
    omat Bx = submatrix(B, inner, 0, extra_cols_A, col_dim);
    omat Cx = submatrix(C, 0, 0, row_dim, col_dim);
    omatmul(Ax, Bx, Cx, 1.0);
  }
  if (extra_cols_B > 0) {
    int s = B.n - extra_cols_B;
    omat Bx = submatrix(B, 0, s, B.m, extra_cols_B);
    omat Cx = submatrix(C, 0, s, C.m, extra_cols_B);
    omatmul(A, Bx, Cx, beta);
  }
  if (extra_rows_A > 0) {
    int s = A.m - extra_rows_A;
    int nc = B.n - extra_cols_B;
    omat Ax = submatrix(A, s, 0, extra_rows_A, A.n);
    omat Bx = submatrix(B, 0, 0, B.m, nc);
    omat Cx = submatrix(C, s, 0, extra_rows_A, nc);
    omatmul(Ax, Bx, Cx, beta);
  }
}

/* One write-once addition: dst = sum_t coef_t * src_t (+ beta * dst), terms
 * in the given order, a coefficient of +-1 as a plain add / subtract
 * (codegen/gen.py:216-235, 444-523). */
static void add_terms(int nterm, const omat* src, const double* coef, omat dst, int with_beta, double beta) {
  int i, j, t;
  for (j = 0; j < dst.n; ++j) {
    for (i = 0; i < dst.m; ++i) {
      double acc = 0.0;
      for (t = 0; t < nterm; ++t) {
        double v = AT(src[t], i, j);
        double c = coef[t];
        double term;
        if (c == 1.0) term = v;
        else if (c == -1.0) term = -v;
        else term = c * v;
        if (t == 0) acc = term;
        else if (c == -1.0) acc = acc - v;
        else acc = acc + term;
      }
      if (with_beta) acc = acc + beta * AT(dst, i, j);
      AT(dst, i, j) = acc;
    }
  }
}

typedef struct {
  const fmm_alg_table* t;
  double slots[FMM_MAX_SLOTS > 0 ? FMM_MAX_SLOTS : 1];
} ctx_t;

static double coef_of(const ctx_t* cx, int slot1) { return cx->slots[slot1 - 1]; }

/* FastMatmulRecursive (algorithms/strassen.hpp:377-659; gen.py:880-1016). */
static void recurse(const ctx_t* cx, omat* A, omat* B, omat* C, int steps_left, double beta) {
  const fmm_alg_table* t = cx->t;
  int m0 = t->m0, k0 = t->k0, n0 = t->n0, R = t->rank;
  int nA = m0 * k0, nB = k0 * n0, nC = m0 * n0;
  int i, r, x;
  omat *Ab, *Bb, *Cb, *AX, *BX, *M, *MXm;
  omat srcs[64 + FMM_MAX_RANK];
  double cs[64 + FMM_MAX_RANK];

  C->mult *= A->mult;  /* :380-383 */
  C->mult *= B->mult;
  A->mult = 1.0;
  B->mult = 1.0;
  if (steps_left == 0) { /* :385-388 -- MatMul with its default beta of 0 */
    omatmul(*A, *B, *C, 0.0);
    return;
  }
  Ab = (omat*)malloc(sizeof(omat) * (size_t)(nA + t->n_ax));
  Bb = (omat*)malloc(sizeof(omat) * (size_t)(nB + t->n_bx));
  Cb = (omat*)malloc(sizeof(omat) * (size_t)nC);
  M = (omat*)malloc(sizeof(omat) * (size_t)(R + t->n_mx));
  for (i = 0; i < nA; ++i) Ab[i] = subblock(*A, m0, k0, i / k0, i % k0);
  for (i = 0; i < nB; ++i) Bb[i] = subblock(*B, k0, n0, i / n0, i % n0);
  for (i = 0; i < nC; ++i) Cb[i] = subblock(*C, m0, n0, i / n0, i % n0);
  AX = Ab + nA;
  BX = Bb + nB;
  MXm = M + R;
  /* M_r carry C's multiplier (:405-421) */
  for (r = 0; r < R; ++r) M[r] = omat_alloc(Cb[0].m, Cb[0].n, C->mult);
  /* CSE input temporaries, write-once (fast424_26_206.hpp:2107-2131) */
  for (x = 0; x < t->n_ax; ++x) {
    int nt = 0;
    AX[x] = omat_alloc(Ab[0].m, Ab[0].n, 1.0);
    for (i = 0; i < nA; ++i) {
      int s = t->SX[x * nA + i];
      if (s) { srcs[nt] = Ab[i]; cs[nt] = coef_of(cx, s); ++nt; }
    }
    add_terms(nt, srcs, cs, AX[x], 0, 0.0);
  }
  for (x = 0; x < t->n_bx; ++x) {
    int nt = 0;
    BX[x] = omat_alloc(Bb[0].m, Bb[0].n, 1.0);
    for (i = 0; i < nB; ++i) {
      int s = t->TX[x * nB + i];
      if (s) { srcs[nt] = Bb[i]; cs[nt] = coef_of(cx, s); ++nt; }
    }
    add_terms(nt, srcs, cs, BX[x], 0, 0.0);
  }
  /* the R products (codegen/gen.py:574-657) */
  for (r = 0; r < R; ++r) {
    omat S, T;
    int sa = 0, sb = 0, nt;
    nt = 0;
    for (i = 0; i < nA + t->n_ax; ++i) {
      int s = t->U[i * R + r];
      if (s) { srcs[nt] = Ab[i]; cs[nt] = coef_of(cx, s); ++nt; }
    }
    if (nt >= 2) {
      S = omat_alloc(Ab[0].m, Ab[0].n, 1.0);
      add_terms(nt, srcs, cs, S, 0, 0.0);
      sa = 1;
    } else {
      S = srcs[0];
      M[r].mult *= cs[0]; /* UpdateMultiplier, gen.py:611-621 */
    }
    nt = 0;
    for (i = 0; i < nB + t->n_bx; ++i) {
      int s = t->V[i * R + r];
      if (s) { srcs[nt] = Bb[i]; cs[nt] = coef_of(cx, s); ++nt; }
    }
    if (nt >= 2) {
      T = omat_alloc(Bb[0].m, Bb[0].n, 1.0);
      add_terms(nt, srcs, cs, T, 0, 0.0);
      sb = 1;
    } else {
      T = srcs[0];
      M[r].mult *= cs[0];
    }
    recurse(cx, &S, &T, &M[r], steps_left - 1, 0.0);
    if (sa) omat_free(&S);
    if (sb) omat_free(&T);
  }
  /* CSE output temporaries (fast424_26_206.hpp:2893-2918) */
  for (x = 0; x < t->n_mx; ++x) {
    int nt = 0;
    for (r = 0; r < R; ++r) {
      int s = t->MX[x * R + r];
      if (s) { srcs[nt] = M[r]; cs[nt] = coef_of(cx, s); ++nt; }
    }
    MXm[x] = omat_alloc(Cb[0].m, Cb[0].n, 1.0);
    if (nt) add_terms(nt, srcs, cs, MXm[x], 0, 0.0);
  }
  /* M_Add: C_ij = sum gamma * M (+ beta C_ij) (strassen.hpp:646-649) */
  for (i = 0; i < nC; ++i) {
    int nt = 0;
    for (r = 0; r < R + t->n_mx; ++r) {
      int s = t->W[i * (R + t->n_mx) + r];
      if (s) { srcs[nt] = M[r]; cs[nt] = coef_of(cx, s); ++nt; }
    }
    add_terms(nt, srcs, cs, Cb[i], beta != 0.0, beta);
  }
  dynamic_peeling(*A, *B, *C, m0, k0, n0, beta); /* :658 */
  for (r = 0; r < R + t->n_mx; ++r) omat_free(&M[r]);
  for (x = 0; x < t->n_ax; ++x) omat_free(&AX[x]);
  for (x = 0; x < t->n_bx; ++x) omat_free(&BX[x]);
  free(Ab);
  free(Bb);
  free(Cb);
  free(M);
}

int oracle_num_algorithms(void) { return FMM_NUM_ALGORITHMS; }

const char* oracle_algorithm_name(int i) {
  if (i < 0 || i >= FMM_NUM_ALGORITHMS) return NULL;
  return fmm_algorithms[i].name;
}

int oracle_algorithm_index(const char* name) {
  int i;
  for (i = 0; i < FMM_NUM_ALGORITHMS; ++i)
    if (strcmp(fmm_algorithms[i].name, name) == 0) return i;
  return -1;
}

/* <alg>::FastMatmul(A, B, C, num_steps, x, alpha, beta) on caller buffers
 * (algorithms/strassen.hpp:661-722): A's multiplier is set to alpha, then the
 * recursion runs.  Returns 0, or -1 for a bad algorithm index. */
int oracle_fast_matmul(int alg, double* a, long lda, double* b, long ldb, double* c, long ldc, int m, int k,
                       int n, int num_steps, double x, double alpha, double beta) {
  ctx_t cx;
  omat A, B, C;
  if (alg < 0 || alg >= FMM_NUM_ALGORITHMS) return -1;
  cx.t = &fmm_algorithms[alg];
  cx.t->eval(x, cx.slots);
  A = omat_view(a, lda, m, k);
  B = omat_view(b, ldb, k, n);
  C = omat_view(c, ldc, m, n);
  A.mult = alpha;
  recurse(&cx, &A, &B, &C, num_steps, beta);
  return 0;
}

/* MatMul with an explicit alpha (linalg/linalg.hpp:261-269). */
void oracle_matmul(double* a, long lda, double* b, long ldb, double* c, long ldc, int m, int k, int n,
                   double alpha, double beta) {
  omat A = omat_view(a, lda, m, k), B = omat_view(b, ldb, k, n), C = omat_view(c, ldc, m, n);
  C.mult = alpha;
  omatmul(A, B, C, beta);
}

/* linalg/linalg.hpp:280-295: max_ij |a_ij - b_ij| / |a_ij| */
double oracle_max_relative_diff(const double* a, long lda, const double* b, long ldb, int m, int n) {
  double mx = 0.0;
  int i, j;
  for (j = 0; j < n; ++j)
    for (i = 0; i < m; ++i) {
      double x = a[i + (long)j * lda], y = b[i + (long)j * ldb];
      double d = fabs(x - y) / fabs(x);
      if (d > mx) mx = d;
    }
  return mx;
}

/* The seeded input generator shared by tests and benchmarks: a
 * counter-based splitmix64 stream, element e of stream `stream` under `seed`
 * mapped to [0, 1) with 53 random bits. */
static uint64_t fmm_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

void oracle_fill_uniform(double* out, long count, uint64_t seed, uint64_t stream, double lo, double hi) {
  uint64_t key = seed * 0xD1B54A32D192ED03ULL + stream * 0x8CB92BA72F3D8DD7ULL;
  long e;
  for (e = 0; e < count; ++e) {
    uint64_t z = fmm_mix(key + (uint64_t)(e + 1) * 0x9E3779B97F4A7C15ULL);
    double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    out[e] = lo + (hi - lo) * u;
  }
}

/* Quad-precision check of sampled entries: the reference's QuadMatmul
 * (linalg/quadmatmul.hpp:8-28, C(i,j) += (__float128)A(i,l) * (__float128)B(l,j))
 * restricted to `count` (row, column) samples.  arows holds the sampled rows
 * of A (count x k, row s contiguous), bcols the sampled columns of B (count x
 * k, column s contiguous), values the computed C entries.  In __float128, q_s
 * = sum_l a_l b_l and aq_s = sum_l |a_l| |b_l|; *max_rel receives
 * max_s |values[s] - q_s| / |q_s| (q_s == 0 skipped) and *max_scaled
 * max_s |values[s] - q_s| / aq_s (aq_s == 0 skipped). */
void oracle_quad_errors(const double* arows, const double* bcols, long k, long count, const double* values,
                        double* max_rel, double* max_scaled) {
  double mr = 0.0, ms = 0.0;
  long s, l;
  for (s = 0; s < count; ++s) {
    const double* a = arows + s * k;
    const double* b = bcols + s * k;
    __float128 q = 0, aq = 0, d;
    for (l = 0; l < k; ++l) {
      const __float128 p = (__float128)a[l] * (__float128)b[l];
      q += p;
      aq += p < 0 ? -p : p;
    }
    d = (__float128)values[s] - q;
    if (d < 0) d = -d;
    if (q != 0) {
      const double r = (double)(d / (q < 0 ? -q : q));
      if (r > mr) mr = r;
    }
    if (aq != 0) {
      const double r = (double)(d / aq);
      if (r > ms) ms = r;
    }
  }
  *max_rel = mr;
  *max_scaled = ms;
}

/* ---- diagonal scaling (scaling/scaling.hpp) ---- */

/* MaxAbsRow (scaling.hpp:63-73) / MaxAbsCol (:78-88): the largest |entry|,
 * starting from 0 with a strict > (NaN entries never win). */
static double o_max_abs_row(const double* a, long lda, int row, int cols) {
  double mx = 0.0;
  int c;
  for (c = 0; c < cols; ++c) {
    const double v = fabs(a[row + (long)c * lda]);
    if (v > mx) mx = v;
  }
  return mx;
}

static double o_max_abs_col(const double* a, long lda, int col, int rows) {
  double mx = 0.0;
  int r;
  for (r = 0; r < rows; ++r) {
    const double v = fabs(a[r + (long)col * lda]);
    if (v > mx) mx = v;
  }
  return mx;
}

/* RowScale (:28-35) and ColScale (:40-47): one multiplication per entry. */
static void o_row_scale(double* a, long lda, int rows, int cols, const double* v) {
  int i, j;
  for (j = 0; j < cols; ++j)
    for (i = 0; i < rows; ++i) a[i + (long)j * lda] *= v[i];
}

static void o_col_scale(double* a, long lda, int rows, int cols, const double* v) {
  int i, j;
  for (j = 0; j < cols; ++j)
    for (i = 0; i < rows; ++i) a[i + (long)j * lda] *= v[j];
}

/* OuterScaling (:105-124): rows of A by 1 / max|row|, columns of B by
 * 1 / max|column| (InverseVector, :52-58), maxima returned in x and y. */
static void o_outer(double* a, long lda, double* b, long ldb, int m, int k, int n, double* x, double* y, double* tmp) {
  int i;
  for (i = 0; i < m; ++i) x[i] = o_max_abs_row(a, lda, i, k);
  for (i = 0; i < m; ++i) tmp[i] = 1.0 / x[i];
  o_row_scale(a, lda, m, k, tmp);
  for (i = 0; i < n; ++i) y[i] = o_max_abs_col(b, ldb, i, k);
  for (i = 0; i < n; ++i) tmp[i] = 1.0 / y[i];
  o_col_scale(b, ldb, k, n, tmp);
}

/* InnerScaling (:129-138): z_k = sqrt(max|A(:,k)| / max|B(k,:)|); columns
 * of A by 1 / z_k, rows of B by z_k. */
static void o_inner(double* a, long lda, double* b, long ldb, int m, int k, int n, double* z, double* zinv) {
  int l;
  for (l = 0; l < k; ++l) z[l] = sqrt(o_max_abs_col(a, lda, l, m) / o_max_abs_row(b, ldb, l, n));
  for (l = 0; l < k; ++l) zinv[l] = 1.0 / z[l];
  o_col_scale(a, lda, m, k, zinv);
  o_row_scale(b, ldb, k, n, z);
}

/* Scaling (:153-196) with type 0 OUTSIDE_INSIDE, 1 INSIDE_OUTSIDE, 2 INSIDE,
 * 3 OUTSIDE.  r (m) and s (n) hold their starting values (resize(m, 1.0) at
 * :158-159 keeps the entries of vectors that arrive sized; fresh vectors are
 * all 1) and collect the outer maxima (UpdateVals, :93-98).  Returns -1 for
 * an unknown type. */
int oracle_scaling(double* a, long lda, double* b, long ldb, int m, int k, int n, int num_steps, int type, double* r,
                   double* s) {
  const int big = (m > n ? m : n) > k ? (m > n ? m : n) : k;
  double* x = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  double* y = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double* t1 = (double*)malloc(sizeof(double) * (size_t)(big > 0 ? big : 1));
  double* t2 = (double*)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1));
  int step, i, rc = 0;
  if (type < 0 || type > 3) rc = -1;
  for (step = 0; rc == 0 && step < num_steps; ++step) {
    if (type == 1 || type == 2) o_inner(a, lda, b, ldb, m, k, n, t1, t2);
    if (type != 2) {
      o_outer(a, lda, b, ldb, m, k, n, x, y, t1);
      for (i = 0; i < m; ++i) r[i] *= x[i];
      for (i = 0; i < n; ++i) s[i] *= y[i];
    }
    if (type == 0) o_inner(a, lda, b, ldb, m, k, n, t1, t2);
  }
  free(x);
  free(y);
  free(t1);
  free(t2);
  return rc;
}

/* PostProcessScaling (:144-149): rows of C by r, then columns by s. */
void oracle_scaling_postprocess(double* c, long ldc, int m, int n, const double* r, const double* s) {
  o_row_scale(c, ldc, m, n, r);
  o_col_scale(c, ldc, m, n, s);
}
