// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// C-ABI shim over the reference implementation itself: the reference's own
// generated headers (algorithms/*.hpp), compiled unchanged in their
// sequential configuration and linked against a host BLAS, so that the
// parity tests and the CPU baseline can call the reference's
// <namespace>::FastMatmul(A, B, C, num_steps, x, alpha, beta)
// (e.g. algorithms/strassen.hpp:661-722) and MatMul (linalg/linalg.hpp:261-269)
// on caller-owned column-major buffers.  Built by oracle/Makefile into
// oracle/_ref/libfmm_ref.so; the headers are read from the reference tree at
// build time, nothing of them is copied here.

#include <cstring>
#include <string>
#include <vector>

#include "linalg.hpp"
#include "scaling.hpp"

#include "bini322_10_52_approx.hpp"
#include "classical222.hpp"
#include "classical333.hpp"
#include "classical423.hpp"
#include "fast234_20_144.hpp"
#include "fast243_20_144.hpp"
#include "fast252_18_99.hpp"
#include "fast322_11_50.hpp"
#include "fast323_15_103.hpp"
#include "fast323_15_89.hpp"
#include "fast324_20_144.hpp"
#include "fast332_15_103.hpp"
#include "fast333_23_125.hpp"
#include "fast333_23_152.hpp"
#include "fast333_23_221.hpp"
#include "fast342_20_144.hpp"
#include "fast343_29_234.hpp"
#include "fast422_14_84.hpp"
#include "fast423_20_130.hpp"
#include "fast423_20_134.hpp"
#include "fast423_20_138.hpp"
#include "fast423_20_144.hpp"
#include "fast423_20_156.hpp"
#include "fast424_26_206.hpp"
#include "fast424_26_257.hpp"
#include "fast432_20_144.hpp"
#include "fast433_29_234.hpp"
#include "fast442_26_257.hpp"
#include "fast522_18_99.hpp"
#include "hk323_15_84.hpp"
#include "hk323_15_94.hpp"
#include "hk332_15_94.hpp"
#include "schonhage333_21_117_approx.hpp"
#include "smirnov333_20_182_approx.hpp"
#include "smirnov333_23_128.hpp"
#include "smirnov333_23_139.hpp"
#include "smirnov336_40_960.hpp"
#include "smirnov363_40_960.hpp"
#include "smirnov633_40_960.hpp"
#include "strassen.hpp"
#include "tichavsky_kovac336_40_960.hpp"
#include "tichavsky_kovac363_40_960.hpp"

extern "C" void openblas_set_num_threads(int);

namespace {

typedef double (*FastFn)(Matrix<double>&, Matrix<double>&, Matrix<double>&, int, double, double, double);

struct Entry {
  const char* name;
  FastFn fn;
};

#define FMMREF_ENTRY(ns) {#ns, &ns::FastMatmul<double>}

const Entry kEntries[] = {
    FMMREF_ENTRY(strassen),
    FMMREF_ENTRY(classical222_8_24),
    FMMREF_ENTRY(grey322_11_50),
    FMMREF_ENTRY(bini322_10_52_approx),
    FMMREF_ENTRY(grey332_15_103),
    FMMREF_ENTRY(grey323_15_103),
    FMMREF_ENTRY(hk332_15_94),
    FMMREF_ENTRY(hk323_15_94),
    FMMREF_ENTRY(hk323_15_84),
    FMMREF_ENTRY(grey323_15_89),
    FMMREF_ENTRY(grey333_23_152),
    FMMREF_ENTRY(grey333_23_221),
    FMMREF_ENTRY(grey333_23_125),
    FMMREF_ENTRY(smirnov333_23_139),
    FMMREF_ENTRY(smirnov333_23_128),
    FMMREF_ENTRY(classical333_27_81),
    FMMREF_ENTRY(schonhage333_21_117_approx),
    FMMREF_ENTRY(smirnov333_20_182_approx),
    FMMREF_ENTRY(grey422_14_84),
    FMMREF_ENTRY(grey432_20_144),
    FMMREF_ENTRY(grey423_20_144),
    FMMREF_ENTRY(grey324_20_144),
    FMMREF_ENTRY(grey342_20_144),
    FMMREF_ENTRY(grey234_20_144),
    FMMREF_ENTRY(grey243_20_144),
    FMMREF_ENTRY(classical423_24_72),
    FMMREF_ENTRY(fast423_130),
    FMMREF_ENTRY(fast423_134),
    FMMREF_ENTRY(fast423_138),
    FMMREF_ENTRY(fast423_156),
    FMMREF_ENTRY(grey433_29_234),
    FMMREF_ENTRY(grey343_29_234),
    FMMREF_ENTRY(grey442_26_257),
    FMMREF_ENTRY(grey424_26_257),
    FMMREF_ENTRY(grey424_26_206),
    FMMREF_ENTRY(grey522_18_99),
    FMMREF_ENTRY(grey252_18_99),
    FMMREF_ENTRY(smirnov336_40_960),
    FMMREF_ENTRY(smirnov363_40_960),
    FMMREF_ENTRY(smirnov633_40_960),
    FMMREF_ENTRY(tichavsky_kovac336_40_960),
    FMMREF_ENTRY(tichavsky_kovac363_40_960),
};

// The same headers with Scalar = float (leaf products through sgemm).
typedef double (*FastFnF)(Matrix<float>&, Matrix<float>&, Matrix<float>&, int, double, float, float);

struct EntryF {
  const char* name;
  FastFnF fn;
};

#define FMMREF_ENTRY_F(ns) {#ns, &ns::FastMatmul<float>}

const EntryF kEntriesF[] = {
    FMMREF_ENTRY_F(strassen),
    FMMREF_ENTRY_F(classical222_8_24),
    FMMREF_ENTRY_F(grey322_11_50),
    FMMREF_ENTRY_F(bini322_10_52_approx),
    FMMREF_ENTRY_F(grey332_15_103),
    FMMREF_ENTRY_F(grey323_15_103),
    FMMREF_ENTRY_F(hk332_15_94),
    FMMREF_ENTRY_F(hk323_15_94),
    FMMREF_ENTRY_F(hk323_15_84),
    FMMREF_ENTRY_F(grey323_15_89),
    FMMREF_ENTRY_F(grey333_23_152),
    FMMREF_ENTRY_F(grey333_23_221),
    FMMREF_ENTRY_F(grey333_23_125),
    FMMREF_ENTRY_F(smirnov333_23_139),
    FMMREF_ENTRY_F(smirnov333_23_128),
    FMMREF_ENTRY_F(classical333_27_81),
    FMMREF_ENTRY_F(schonhage333_21_117_approx),
    FMMREF_ENTRY_F(smirnov333_20_182_approx),
    FMMREF_ENTRY_F(grey422_14_84),
    FMMREF_ENTRY_F(grey432_20_144),
    FMMREF_ENTRY_F(grey423_20_144),
    FMMREF_ENTRY_F(grey324_20_144),
    FMMREF_ENTRY_F(grey342_20_144),
    FMMREF_ENTRY_F(grey234_20_144),
    FMMREF_ENTRY_F(grey243_20_144),
    FMMREF_ENTRY_F(classical423_24_72),
    FMMREF_ENTRY_F(fast423_130),
    FMMREF_ENTRY_F(fast423_134),
    FMMREF_ENTRY_F(fast423_138),
    FMMREF_ENTRY_F(fast423_156),
    FMMREF_ENTRY_F(grey433_29_234),
    FMMREF_ENTRY_F(grey343_29_234),
    FMMREF_ENTRY_F(grey442_26_257),
    FMMREF_ENTRY_F(grey424_26_257),
    FMMREF_ENTRY_F(grey424_26_206),
    FMMREF_ENTRY_F(grey522_18_99),
    FMMREF_ENTRY_F(grey252_18_99),
    FMMREF_ENTRY_F(smirnov336_40_960),
    FMMREF_ENTRY_F(smirnov363_40_960),
    FMMREF_ENTRY_F(smirnov633_40_960),
    FMMREF_ENTRY_F(tichavsky_kovac336_40_960),
    FMMREF_ENTRY_F(tichavsky_kovac363_40_960),
};

}  // namespace

extern "C" {

int fmmref_num_algorithms(void) { return (int)(sizeof(kEntries) / sizeof(kEntries[0])); }

const char* fmmref_algorithm_name(int i) {
  if (i < 0 || i >= fmmref_num_algorithms()) return nullptr;
  return kEntries[i].name;
}

void fmmref_set_threads(int n) { openblas_set_num_threads(n); }

// <name>::FastMatmul on caller buffers.  Returns the reference's own
// elapsed-milliseconds value, or -1 for an unknown algorithm name.
double fmmref_fast_matmul(const char* name, double* a, int lda, double* b, int ldb, double* c, int ldc,
                          int m, int k, int n, int num_steps, double x, double alpha, double beta) {
  for (const Entry& e : kEntries) {
    if (std::strcmp(e.name, name) == 0) {
      Matrix<double> A(a, lda, m, k);
      Matrix<double> B(b, ldb, k, n);
      Matrix<double> C(c, ldc, m, n);
      return e.fn(A, B, C, num_steps, x, alpha, beta);
    }
  }
  return -1.0;
}

// MatMul: C <- alpha * A * B + beta * C through the host BLAS.
void fmmref_matmul(double* a, int lda, double* b, int ldb, double* c, int ldc, int m, int k, int n,
                   double alpha, double beta) {
  Matrix<double> A(a, lda, m, k);
  Matrix<double> B(b, ldb, k, n);
  Matrix<double> C(c, ldc, m, n, alpha);
  MatMul(A, B, C, beta);
}

// <name>::FastMatmul<float> on caller buffers; -1 for an unknown name.
double fmmref_fast_matmul_f32(const char* name, float* a, int lda, float* b, int ldb, float* c, int ldc, int m, int k,
                              int n, int num_steps, double x, float alpha, float beta) {
  for (const EntryF& e : kEntriesF) {
    if (std::strcmp(e.name, name) == 0) {
      Matrix<float> A(a, lda, m, k);
      Matrix<float> B(b, ldb, k, n);
      Matrix<float> C(c, ldc, m, n);
      return e.fn(A, B, C, num_steps, x, alpha, beta);
    }
  }
  return -1.0;
}

// MatMul<float>: C <- alpha * A * B + beta * C through the host sgemm.
void fmmref_matmul_f32(float* a, int lda, float* b, int ldb, float* c, int ldc, int m, int k, int n, float alpha,
                       float beta) {
  Matrix<float> A(a, lda, m, k);
  Matrix<float> B(b, ldb, k, n);
  Matrix<float> C(c, ldc, m, n, alpha);
  MatMul(A, B, C, beta);
}

// Scaling<double>(A, B, num_steps, r_vals, s_vals, type) from
// scaling/scaling.hpp on caller buffers (A m x k, B k x n scaled in place);
// r (m) and s (n) are in/out: they arrive as vectors of the right size, which
// Scaling's resize(m, 1.0) keeps, and receive the factors multiplied in.
void fmmref_scaling(double* a, int lda, double* b, int ldb, int m, int k, int n, int num_steps, int type, double* r,
                    double* s) {
  Matrix<double> A(a, lda, m, k);
  Matrix<double> B(b, ldb, k, n);
  std::vector<double> rv(r, r + m), sv(s, s + n);
  Scaling<double>(A, B, num_steps, rv, sv, type);
  for (int i = 0; i < m; ++i) r[i] = rv[i];
  for (int j = 0; j < n; ++j) s[j] = sv[j];
}

// Scaling<float> / PostProcessScaling on float buffers (the same contract).
void fmmref_scaling_f32(float* a, int lda, float* b, int ldb, int m, int k, int n, int num_steps, int type, float* r,
                        float* s) {
  Matrix<float> A(a, lda, m, k);
  Matrix<float> B(b, ldb, k, n);
  std::vector<float> rv(r, r + m), sv(s, s + n);
  Scaling<float>(A, B, num_steps, rv, sv, type);
  for (int i = 0; i < m; ++i) r[i] = rv[i];
  for (int j = 0; j < n; ++j) s[j] = sv[j];
}

void fmmref_scaling_postprocess_f32(float* c, int ldc, int m, int n, const float* r, const float* s) {
  Matrix<float> C(c, ldc, m, n);
  std::vector<float> rv(r, r + m), sv(s, s + n);
  PostProcessScaling(C, rv, sv);
}

// PostProcessScaling(C, r_vals, s_vals) from scaling/scaling.hpp.
void fmmref_scaling_postprocess(double* c, int ldc, int m, int n, const double* r, const double* s) {
  Matrix<double> C(c, ldc, m, n);
  std::vector<double> rv(r, r + m), sv(s, s + n);
  PostProcessScaling(C, rv, sv);
}

}  // extern "C"
