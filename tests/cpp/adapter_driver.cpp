// Drop-in check of the C++ surface: a driver written against the
// reference's API (RunAlgorithm, <ns>::FastMatmul, MatMul, MaxRelativeDiff,
// RandomMatrix, Scaling / PostProcessScaling) built unchanged against
// include/fmm and libfmm.so.
// Exit status 0 when every error is within its bound.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "fmm/all_algorithms.hpp"
#include "fmm/scaling.hpp"

static int failures = 0;

static void expect(bool ok, const char* what, double val) {
  std::printf("%-56s %.3e %s\n", what, val, ok ? "ok" : "FAIL");
  if (!ok) ++failures;
}

int main() {
  std::srand(7);
  // RunAlgorithm against classical MatMul (tests/matmul_tests.cpp:19-27 pattern)
  const int algs[] = {STRASSEN, FAST424_26_206, FAST333_23_125, SMIRNOV333_23_128, FAST323_15_89, MKL};
  for (int alg : algs) {
    for (int steps = 1; steps <= 2; ++steps) {
      Matrix<double> A = RandomMatrix<double>(402, 500);
      Matrix<double> B = RandomMatrix<double>(500, 562);
      Matrix<double> C1(402, 562), C2(402, 562);
      RunAlgorithm(alg, A, B, C1, steps);
      MatMul(A, B, C2);
      char name[96];
      std::snprintf(name, sizeof name, "%s steps=%d max rel diff", Alg2Str(alg).c_str(), steps);
      expect(MaxRelativeDiff(C1, C2) <= 1e-13, name, MaxRelativeDiff(C1, C2));
    }
  }
  // approximate algorithm: error of the reference's order of magnitude
  {
    Matrix<double> A = RandomMatrix<double>(300, 200);
    Matrix<double> B = RandomMatrix<double>(200, 250);
    Matrix<double> C1(300, 250), C2(300, 250);
    RunAlgorithm(BINI322_10_52_APPROX, A, B, C1, 1);
    MatMul(A, B, C2);
    expect(MaxRelativeDiff(C1, C2) <= 1e-3, "BINI322_10_52_APPROX steps=1 max rel diff", MaxRelativeDiff(C1, C2));
  }
  // C := alpha * A * B + beta * C (tests/matmul_tests.cpp:47-135 pattern)
  {
    const double alpha = 7.0, beta = -1.3;
    Matrix<double> A = RandomMatrix<double>(1001, 200);
    Matrix<double> B = RandomMatrix<double>(200, 309);
    Matrix<double> C1 = RandomMatrix<double>(1001, 309);
    Matrix<double> C2 = C1;
    C2.set_multiplier(alpha);
    MatMul(A, B, C2, beta);
    smirnov333_23_128::FastMatmul(A, B, C1, 2, 0, alpha, beta);
    expect(MaxRelativeDiff(C1, C2) <= 1e-12, "smirnov333_23_128 alpha=7 beta=-1.3 max rel diff", MaxRelativeDiff(C1, C2));
    // multiplier side effect of the reference: C keeps alpha, A and B are reset
    expect(C1.multiplier() == alpha && A.multiplier() == 1.0 && B.multiplier() == 1.0, "multiplier side effects",
           C1.multiplier());
  }
  // views: a sub-block product written into a sub-block of a larger C
  {
    Matrix<double> A = RandomMatrix<double>(600, 600);
    Matrix<double> B = RandomMatrix<double>(600, 600);
    Matrix<double> C1(600, 600), C2(600, 600);
    Matrix<double> A11 = A.Subblock(2, 2, 1, 1), B12 = B.Subblock(2, 2, 1, 2);
    Matrix<double> C1v = C1.Subblock(2, 2, 2, 2), C2v = C2.Subblock(2, 2, 2, 2);
    strassen::FastMatmul(A11, B12, C1v, 2);
    MatMul(A11, B12, C2v);
    expect(MaxRelativeDiff(C1v, C2v) <= 1e-13, "strassen on strided views max rel diff", MaxRelativeDiff(C1v, C2v));
  }
  // Scalar = float (scaling/fast_scaling.cpp runs strassen::FastMatmul on
  // Matrix<float>): FP32 results of the fast and the classical product agree
  // to about one FP32 rounding
  {
    Matrix<float> A = RandomMatrix<float>(300, 260);
    Matrix<float> B = RandomMatrix<float>(260, 280);
    Matrix<float> C1(300, 280), C2(300, 280);
    strassen::FastMatmul(A, B, C1, 2);
    MatMul(A, B, C2);
    expect(MaxRelativeDiff(C1, C2) <= 1e-6, "float strassen steps=2 vs MatMul<float>", MaxRelativeDiff(C1, C2));
    Matrix<float> C3 = RandomMatrix<float>(300, 280);
    Matrix<float> C4 = C3;
    grey424_26_206::FastMatmul(A, B, C3, 1, 1e-8, 2.0f, 0.5f);
    C4.set_multiplier(2.0f);
    MatMul(A, B, C4, 0.5f);
    expect(MaxRelativeDiff(C3, C4) <= 1e-6, "float grey424 alpha=2 beta=0.5 vs MatMul<float>",
           MaxRelativeDiff(C3, C4));
    // scaling/fast_scaling.cpp's pattern: Scaling<float> + FastMatmul<float>
    // + PostProcessScaling back to the unscaled product
    Matrix<float> As = A, Bs = B, C5(300, 280);
    std::vector<float> r_vals, s_vals;
    Scaling<float>(As, Bs, 10, r_vals, s_vals, OUTSIDE);
    strassen::FastMatmul(As, Bs, C5, 2);
    PostProcessScaling(C5, r_vals, s_vals);
    expect(MaxRelativeDiff(C2, C5) <= 1e-5, "float Scaling + strassen + PostProcessScaling", MaxRelativeDiff(C2, C5));
  }
  // diagonal scaling (benchmarks/scaling_stability.cpp pattern): rows of A
  // and columns of B skewed by 2^-30..2^30; scaled Strassen back within the
  // classical product's error
  {
    Matrix<double> A = RandomMatrix<double>(512, 384);
    Matrix<double> B = RandomMatrix<double>(384, 448);
    for (int j = 0; j < A.n(); ++j)
      for (int i = 0; i < A.m(); ++i) A(i, j) = std::ldexp(A(i, j), i % 3 == 0 ? 30 : (i % 3 == 1 ? -30 : 0));
    for (int j = 0; j < B.n(); ++j)
      for (int i = 0; i < B.m(); ++i) B(i, j) = std::ldexp(B(i, j), j % 2 == 0 ? -30 : 30);
    Matrix<double> C1(512, 448), C2(512, 448);
    MatMul(A, B, C1);
    Matrix<double> As = A, Bs = B;
    std::vector<double> r_vals, s_vals;
    Scaling(As, Bs, 5, r_vals, s_vals, OUTSIDE_INSIDE);
    strassen::FastMatmul(As, Bs, C2, 2);
    PostProcessScaling(C2, r_vals, s_vals);
    expect(r_vals.size() == 512 && s_vals.size() == 448, "Scaling factor vector sizes", (double)r_vals.size());
    expect(MaxRelativeDiff(C1, C2) <= 1e-13, "Scaling + strassen + PostProcessScaling", MaxRelativeDiff(C1, C2));
    bool threw = false;
    try {
      Scaling(As, Bs, 1, r_vals, s_vals, 9);
    } catch (const std::runtime_error&) {
      threw = true;
    }
    expect(threw, "unknown scaling type throws", 0.0);
  }
  std::printf("%s\n", failures ? "FAILED" : "PASSED");
  return failures ? 1 : 0;
}
