// Generated by fast_matmul_b200/codegen/gen_cuda.py from the fast-matmul coefficient files. Do not edit.
// One struct per algorithm; FMM_FOR_EACH_ALGORITHM(X) expands X(index, struct).
#pragma once

// strassen  <2,2,2; 7>  (reference header algorithms/strassen.hpp, coefficients codegen/algorithms/strassen)
struct FmmAlg_strassen {
  static constexpr int kM0 = 2, kK0 = 2, kN0 = 2, kR = 7;
  static constexpr int kNumAOut = 5, kNumBOut = 5;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    st(0, fmm_add(a0, a3));  // operand of M1
    st(1, fmm_add(a2, a3));  // operand of M2
    st(2, fmm_add(a0, a1));  // operand of M5
    st(3, fmm_add(fmm_neg(a0), a2));  // operand of M6
    st(4, fmm_sub(a1, a3));  // operand of M7
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    st(0, fmm_add(b0, b3));  // operand of M1
    st(1, fmm_sub(b1, b3));  // operand of M3
    st(2, fmm_add(fmm_neg(b0), b2));  // operand of M4
    st(3, fmm_add(b0, b1));  // operand of M6
    st(4, fmm_add(b2, b3));  // operand of M7
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_sub(fmm_add(m0, m3), m4), m6), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_sub(fmm_add(m0, m3), m4), m6));
    if (kBeta) st(1, fmm_add(fmm_add(m2, m4), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(m2, m4));
    if (kBeta) st(2, fmm_add(fmm_add(m1, m3), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(m1, m3));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_sub(m0, m1), m2), m5), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_sub(m0, m1), m2), m5));
  }
};

// classical222_8_24  <2,2,2; 8>  (reference header algorithms/classical222.hpp, coefficients codegen/algorithms/classical222-8-24)
struct FmmAlg_classical222_8_24 {
  static constexpr int kM0 = 2, kK0 = 2, kN0 = 2, kR = 8;
  static constexpr int kNumAOut = 0, kNumBOut = 0;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    if (kBeta) st(0, fmm_add(fmm_add(m0, m1), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(m0, m1));
    if (kBeta) st(1, fmm_add(fmm_add(m2, m3), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(m2, m3));
    if (kBeta) st(2, fmm_add(fmm_add(m4, m5), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(m4, m5));
    if (kBeta) st(3, fmm_add(fmm_add(m6, m7), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(m6, m7));
  }
};

// grey322_11_50  <3,2,2; 11>  (reference header algorithms/fast322_11_50.hpp, coefficients codegen/algorithms/grey322-11-50)
struct FmmAlg_grey322_11_50 {
  static constexpr int kM0 = 3, kK0 = 2, kN0 = 2, kR = 11;
  static constexpr int kNumAOut = 5, kNumBOut = 6;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    st(0, fmm_add(a0, a4));  // operand of M2
    st(1, fmm_add(fmm_neg(a0), a1));  // operand of M4
    st(2, fmm_add(a0, a5));  // operand of M5
    st(3, fmm_add(a1, a5));  // operand of M7
    st(4, fmm_add(fmm_neg(a4), a5));  // operand of M10
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    st(0, fmm_add(b1, b3));  // operand of M1
    st(1, fmm_add(b0, b1));  // operand of M2
    st(2, fmm_add(b2, b3));  // operand of M3
    st(3, fmm_add(fmm_neg(b0), b3));  // operand of M5
    st(4, fmm_add(b2, b3));  // operand of M7
    st(5, fmm_add(b0, b2));  // operand of M9
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m4), m6), m8), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m4), m6), m8));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_neg(m0), m3), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_neg(m0), m3));
    if (kBeta) st(2, fmm_add(fmm_add(m5, m10), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(m5, m10));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(m2, m5), m7), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(m2, m5), m7));
    if (kBeta) st(4, fmm_add(fmm_sub(m8, m9), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(m8, m9));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(m0, m1), m4), m9), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(m0, m1), m4), m9));
  }
};

// bini322_10_52_approx  <3,2,2; 10>  (reference header algorithms/bini322_10_52_approx.hpp, coefficients codegen/algorithms/bini322-10-52-approx)
struct FmmAlg_bini322_10_52_approx {
  static constexpr int kM0 = 3, kK0 = 2, kN0 = 2, kR = 10;
  static constexpr int kNumAOut = 6, kNumBOut = 8;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    st(0, fmm_add(a0, a3));  // operand of M1
    st(1, fmm_add(fmm_mul(cf[1], a1), a3));  // operand of M4
    st(2, fmm_add(a0, fmm_mul(cf[1], a1)));  // operand of M5
    st(3, fmm_add(a2, a5));  // operand of M6
    st(4, fmm_add(fmm_mul(cf[1], a4), a5));  // operand of M9
    st(5, fmm_add(a2, fmm_mul(cf[1], a4)));  // operand of M10
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    st(0, fmm_add(fmm_mul(cf[1], b0), b3));  // operand of M1
    st(1, fmm_sub(fmm_neg(b2), b3));  // operand of M2
    st(2, fmm_add(fmm_mul(cf[2], b0), b2));  // operand of M4
    st(3, fmm_add(fmm_mul(cf[1], b1), b3));  // operand of M5
    st(4, fmm_add(b0, fmm_mul(cf[1], b3)));  // operand of M6
    st(5, fmm_sub(fmm_neg(b0), b1));  // operand of M8
    st(6, fmm_add(b0, fmm_mul(cf[1], b2)));  // operand of M9
    st(7, fmm_add(b1, fmm_mul(cf[2], b3)));  // operand of M10
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m0), fmm_mul(cf[4], m1)), fmm_mul(cf[5], m2)), fmm_mul(cf[4], m3)), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m0), fmm_mul(cf[4], m1)), fmm_mul(cf[5], m2)), fmm_mul(cf[4], m3)));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_mul(cf[5], m2), fmm_mul(cf[4], m4)), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_mul(cf[5], m2), fmm_mul(cf[4], m4)));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_add(m3, m5), m8), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_add(m3, m5), m8));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(m0, m4), m9), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(m0, m4), m9));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_mul(cf[5], m6), fmm_mul(cf[4], m8)), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_mul(cf[5], m6), fmm_mul(cf[4], m8)));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m5), fmm_mul(cf[5], m6)), fmm_mul(cf[4], m7)), fmm_mul(cf[4], m9)), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m5), fmm_mul(cf[5], m6)), fmm_mul(cf[4], m7)), fmm_mul(cf[4], m9)));
  }
};

// grey332_15_103  <3,3,2; 15>  (reference header algorithms/fast332_15_103.hpp, coefficients codegen/algorithms/grey332-15-103)
struct FmmAlg_grey332_15_103 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 2, kR = 15;
  static constexpr int kNumAOut = 11, kNumBOut = 11;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_sub(fmm_neg(a2), a7));  // operand of M2
    st(1, fmm_add(fmm_add(fmm_neg(a0), a1), a7));  // operand of M3
    st(2, fmm_sub(fmm_add(a2, a5), a6));  // operand of M4
    st(3, fmm_add(fmm_add(fmm_neg(a0), a1), a4));  // operand of M5
    st(4, fmm_add(fmm_sub(fmm_add(fmm_sub(a0, a1), a3), a4), a6));  // operand of M6
    st(5, fmm_sub(fmm_neg(a2), a5));  // operand of M7
    st(6, fmm_add(fmm_add(a2, a3), a5));  // operand of M8
    st(7, fmm_add(a1, a4));  // operand of M10
    st(8, fmm_add(fmm_add(a2, a6), a8));  // operand of M11
    st(9, fmm_add(fmm_sub(fmm_add(a2, a5), a7), a8));  // operand of M12
    st(10, fmm_sub(fmm_neg(a2), a4));  // operand of M15
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_add(b3, b5));  // operand of M1
    st(1, fmm_add(fmm_neg(b3), b4));  // operand of M2
    st(2, fmm_sub(fmm_neg(b2), b3));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_neg(b1), b4), b5));  // operand of M4
    st(4, fmm_add(fmm_add(b0, b2), b3));  // operand of M5
    st(5, fmm_sub(b1, b5));  // operand of M7
    st(6, fmm_add(b2, b4));  // operand of M9
    st(7, fmm_sub(fmm_neg(b0), b2));  // operand of M10
    st(8, fmm_add(b4, b5));  // operand of M11
    st(9, fmm_add(fmm_add(fmm_add(b0, b1), b2), b3));  // operand of M13
    st(10, fmm_sub(fmm_sub(fmm_add(b0, b1), b4), b5));  // operand of M14
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m1), m2), m4), m8), m9), m14), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m1), m2), m4), m8), m9), m14));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m0), m4), m9), m12), m14), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m0), m4), m9), m12), m14));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m1, m2), m3), m4), m5), m6), m8), m13), m14), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m1, m2), m3), m4), m5), m6), m8), m13), m14));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_add(m0, m6), m7), m14), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_add(m0, m6), m7), m14));
    if (kBeta) st(4, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m3), m6), m8), m11), m13), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m3), m6), m8), m11), m13));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(m0, m1), m3), m6), m10), m11), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(m0, m1), m3), m6), m10), m11));
  }
};

// grey323_15_103  <3,2,3; 15>  (reference header algorithms/fast323_15_103.hpp, coefficients codegen/algorithms/grey323-15-103)
struct FmmAlg_grey323_15_103 {
  static constexpr int kM0 = 3, kK0 = 2, kN0 = 3, kR = 15;
  static constexpr int kNumAOut = 11, kNumBOut = 11;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    st(0, fmm_add(fmm_add(fmm_neg(a1), a3), a5));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_neg(a0), a2), a5));  // operand of M2
    st(2, fmm_add(fmm_neg(a0), a2));  // operand of M3
    st(3, fmm_add(fmm_sub(a2, a4), a5));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_neg(a0), a1), a2));  // operand of M5
    st(5, fmm_sub(fmm_add(fmm_add(fmm_neg(a2), a3), a4), a5));  // operand of M7
    st(6, fmm_add(fmm_add(fmm_neg(a0), a2), a4));  // operand of M9
    st(7, fmm_add(fmm_neg(a0), a1));  // operand of M10
    st(8, fmm_sub(a4, a5));  // operand of M12
    st(9, fmm_sub(a2, a4));  // operand of M14
    st(10, fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a1), a2), a3));  // operand of M15
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_add(b4, b5));  // operand of M1
    st(1, fmm_sub(b2, b4));  // operand of M2
    st(2, fmm_sub(fmm_neg(b1), b4));  // operand of M3
    st(3, fmm_add(fmm_sub(b2, b3), b5));  // operand of M4
    st(4, fmm_add(fmm_add(b0, b1), b4));  // operand of M5
    st(5, fmm_sub(b3, b5));  // operand of M7
    st(6, fmm_add(b1, b2));  // operand of M9
    st(7, fmm_sub(fmm_neg(b0), b1));  // operand of M10
    st(8, fmm_add(b2, b5));  // operand of M11
    st(9, fmm_add(fmm_add(fmm_add(b0, b1), b3), b4));  // operand of M13
    st(10, fmm_sub(fmm_add(fmm_sub(b0, b2), b3), b5));  // operand of M14
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m2), m4), m5), m12), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_sub(fmm_neg(m2), m4), m5), m12));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_sub(fmm_add(m2, m4), m5), m9), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_sub(fmm_add(m2, m4), m5), m9));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m0), m1), m3), m6), m7), m10), m11), m14), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m0), m1), m3), m6), m7), m10), m11), m14));
    if (kBeta) st(3, fmm_add(fmm_add(m5, m7), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(m5, m7));
    if (kBeta) st(4, fmm_add(fmm_sub(fmm_add(fmm_sub(m4, m5), m9), m14), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(fmm_add(fmm_sub(m4, m5), m9), m14));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_sub(m3, m6), m7), m11), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_sub(m3, m6), m7), m11));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m3), m5), m10), m13), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_add(fmm_add(fmm_neg(m3), m5), m10), m13));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m2), m8), m11), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m2), m8), m11));
    if (kBeta) st(8, fmm_add(fmm_add(m10, m11), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(m10, m11));
  }
};

// hk332_15_94  <3,3,2; 15>  (reference header algorithms/hk332_15_94.hpp, coefficients codegen/algorithms/hk332-15-94)
struct FmmAlg_hk332_15_94 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 2, kR = 15;
  static constexpr int kNumAOut = 9, kNumBOut = 11;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_add(fmm_sub(a0, a1), a6));  // operand of M1
    st(1, fmm_sub(fmm_add(a0, a2), a3));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_neg(a3), a4), a7));  // operand of M3
    st(3, fmm_sub(a1, a3));  // operand of M5
    st(4, fmm_add(fmm_add(a5, a6), a8));  // operand of M7
    st(5, fmm_sub(a2, a6));  // operand of M8
    st(6, fmm_sub(fmm_sub(a1, a4), a5));  // operand of M9
    st(7, fmm_add(fmm_add(a2, a7), a8));  // operand of M12
    st(8, fmm_add(fmm_neg(a5), a7));  // operand of M14
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_sub(b0, b1));  // operand of M2
    st(1, fmm_add(b0, b2));  // operand of M4
    st(2, fmm_add(b1, b2));  // operand of M5
    st(3, fmm_add(fmm_neg(b0), b4));  // operand of M6
    st(4, fmm_add(fmm_add(fmm_neg(b0), b1), b4));  // operand of M8
    st(5, fmm_sub(b2, b3));  // operand of M9
    st(6, fmm_add(b1, b3));  // operand of M10
    st(7, fmm_add(fmm_neg(b3), b5));  // operand of M11
    st(8, fmm_sub(fmm_add(fmm_add(fmm_neg(b2), b3), b4), b5));  // operand of M13
    st(9, fmm_add(fmm_sub(b2, b3), b5));  // operand of M14
    st(10, fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b1), b4), b5));  // operand of M15
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m0, m1), m3), m4), m5), m7), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m0, m1), m3), m4), m5), m7));
    if (kBeta) st(1, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m0, m5), m7), m9), m14), fmm_mul(beta, ldc(1)))); else st(1, fmm_sub(fmm_add(fmm_add(fmm_sub(m0, m5), m7), m9), m14));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m2, m3), m10), m12), m13), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_sub(fmm_sub(fmm_add(m2, m3), m10), m12), m13));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(m2, m4), m8), m9), m10), m13), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(m2, m4), m8), m9), m10), m13));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m5, m6), m10), m12), m13), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_add(m5, m6), m10), m12), m13));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m5, m7), m10), m11), m14), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(fmm_sub(m5, m7), m10), m11), m14));
  }
};

// hk323_15_94  <3,2,3; 15>  (reference header algorithms/hk323_15_94.hpp, coefficients codegen/algorithms/hk323-15-94)
struct FmmAlg_hk323_15_94 {
  static constexpr int kM0 = 3, kK0 = 2, kN0 = 3, kR = 15;
  static constexpr int kNumAOut = 11, kNumBOut = 11;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    st(0, fmm_add(a0, a1));  // operand of M1
    st(1, fmm_add(a2, a3));  // operand of M3
    st(2, fmm_add(a0, a2));  // operand of M4
    st(3, fmm_sub(a0, a3));  // operand of M5
    st(4, fmm_add(fmm_add(fmm_sub(fmm_neg(a0), a1), a4), a5));  // operand of M6
    st(5, fmm_sub(fmm_add(a0, a1), a5));  // operand of M8
    st(6, fmm_add(a1, a3));  // operand of M10
    st(7, fmm_add(fmm_add(fmm_sub(fmm_neg(a2), a3), a4), a5));  // operand of M11
    st(8, fmm_add(fmm_neg(a2), a4));  // operand of M13
    st(9, fmm_add(fmm_sub(fmm_neg(a2), a3), a4));  // operand of M14
    st(10, fmm_add(fmm_neg(a1), a5));  // operand of M15
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_sub(b0, b3));  // operand of M2
    st(1, fmm_add(b0, b1));  // operand of M4
    st(2, fmm_add(b1, b3));  // operand of M5
    st(3, fmm_add(fmm_neg(b0), b2));  // operand of M6
    st(4, fmm_add(fmm_add(fmm_neg(b0), b2), b3));  // operand of M8
    st(5, fmm_sub(b1, b4));  // operand of M9
    st(6, fmm_add(b3, b4));  // operand of M10
    st(7, fmm_add(fmm_neg(b4), b5));  // operand of M11
    st(8, fmm_sub(fmm_add(fmm_add(fmm_neg(b1), b2), b4), b5));  // operand of M13
    st(9, fmm_add(fmm_sub(b1, b4), b5));  // operand of M14
    st(10, fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b2), b3), b5));  // operand of M15
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    if (kBeta) st(0, fmm_add(fmm_add(m0, m1), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(m0, m1));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m0), m4), m8), m9), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_neg(m0), m4), m8), m9));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(m1, m7), m11), m14), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(m1, m7), m11), m14));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m1), m2), m3), m4), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_sub(fmm_neg(m1), m2), m3), m4));
    if (kBeta) st(4, fmm_add(fmm_sub(m2, m8), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(m2, m8));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_sub(fmm_sub(m6, m8), m12), m13), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_sub(fmm_sub(m6, m8), m12), m13));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_add(fmm_sub(m0, m5), m6), m7), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_add(fmm_sub(m0, m5), m6), m7));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_sub(m2, m10), m11), m13), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_sub(m2, m10), m11), m13));
    if (kBeta) st(8, fmm_add(fmm_add(m6, m11), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(m6, m11));
  }
};

// hk323_15_84  <3,2,3; 15>  (reference header algorithms/hk323_15_84.hpp, coefficients codegen/algorithms/eliminated/hk323-15-84)
struct FmmAlg_hk323_15_84 {
  static constexpr int kM0 = 3, kK0 = 2, kN0 = 3, kR = 15;
  static constexpr int kNumAOut = 11, kNumBOut = 11;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T ax0 = fmm_add(a0, a1);
    const T ax1 = fmm_add(a2, a3);
    const T ax2 = fmm_add(a4, a5);
    st(0, ax0);
    st(1, ax1);
    st(2, fmm_add(a0, a2));  // operand of M4
    st(3, fmm_sub(a0, a3));  // operand of M5
    st(4, fmm_add(fmm_neg(ax0), ax2));  // operand of M6
    st(5, fmm_add(fmm_neg(a5), ax0));  // operand of M8
    st(6, fmm_add(a1, a3));  // operand of M10
    st(7, fmm_add(fmm_neg(ax1), ax2));  // operand of M11
    st(8, fmm_add(fmm_neg(a2), a4));  // operand of M13
    st(9, fmm_sub(a4, ax1));  // operand of M14
    st(10, fmm_add(fmm_neg(a1), a5));  // operand of M15
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T bx0 = fmm_sub(b0, b3);
    const T bx1 = fmm_sub(b1, b4);
    const T bx2 = fmm_sub(b2, b5);
    st(0, bx0);
    st(1, bx1);
    st(2, fmm_add(b0, b1));  // operand of M4
    st(3, fmm_add(b1, b3));  // operand of M5
    st(4, fmm_add(fmm_neg(b0), b2));  // operand of M6
    st(5, fmm_sub(b2, bx0));  // operand of M8
    st(6, fmm_add(b3, b4));  // operand of M10
    st(7, fmm_add(fmm_neg(b4), b5));  // operand of M11
    st(8, fmm_add(fmm_neg(bx1), bx2));  // operand of M13
    st(9, fmm_add(b5, bx1));  // operand of M14
    st(10, fmm_add(fmm_neg(bx0), bx2));  // operand of M15
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    if (kBeta) st(0, fmm_add(fmm_add(m0, m1), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(m0, m1));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m0), m4), m8), m9), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_neg(m0), m4), m8), m9));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(m1, m7), m11), m14), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(m1, m7), m11), m14));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m1), m2), m3), m4), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_sub(fmm_neg(m1), m2), m3), m4));
    if (kBeta) st(4, fmm_add(fmm_sub(m2, m8), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(m2, m8));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_sub(fmm_sub(m6, m8), m12), m13), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_sub(fmm_sub(m6, m8), m12), m13));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_add(fmm_sub(m0, m5), m6), m7), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_add(fmm_sub(m0, m5), m6), m7));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_sub(m2, m10), m11), m13), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_sub(m2, m10), m11), m13));
    if (kBeta) st(8, fmm_add(fmm_add(m6, m11), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(m6, m11));
  }
};

// grey323_15_89  <3,2,3; 15>  (reference header algorithms/fast323_15_89.hpp, coefficients codegen/algorithms/eliminated/grey323-15-89)
struct FmmAlg_grey323_15_89 {
  static constexpr int kM0 = 3, kK0 = 2, kN0 = 3, kR = 15;
  static constexpr int kNumAOut = 11, kNumBOut = 11;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T ax0 = fmm_add(fmm_neg(a1), a3);
    const T ax1 = fmm_add(fmm_neg(a0), a2);
    const T ax2 = fmm_sub(a2, a4);
    st(0, ax1);
    st(1, ax2);
    st(2, fmm_add(a5, ax0));  // operand of M1
    st(3, fmm_add(a5, ax1));  // operand of M2
    st(4, fmm_add(a5, ax2));  // operand of M4
    st(5, fmm_add(a1, ax1));  // operand of M5
    st(6, fmm_sub(fmm_sub(a3, a5), ax2));  // operand of M7
    st(7, fmm_add(a4, ax1));  // operand of M9
    st(8, fmm_add(fmm_neg(a0), a1));  // operand of M10
    st(9, fmm_sub(a4, a5));  // operand of M12
    st(10, fmm_add(fmm_neg(ax0), ax1));  // operand of M15
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T bx0 = fmm_sub(fmm_neg(b1), b4);
    const T bx1 = fmm_sub(b2, b3);
    st(0, bx0);
    st(1, fmm_add(b4, b5));  // operand of M1
    st(2, fmm_sub(b2, b4));  // operand of M2
    st(3, fmm_add(b5, bx1));  // operand of M4
    st(4, fmm_sub(b0, bx0));  // operand of M5
    st(5, fmm_sub(b3, b5));  // operand of M7
    st(6, fmm_add(b1, b2));  // operand of M9
    st(7, fmm_sub(fmm_neg(b0), b1));  // operand of M10
    st(8, fmm_add(b2, b5));  // operand of M11
    st(9, fmm_sub(fmm_add(b0, b3), bx0));  // operand of M13
    st(10, fmm_sub(fmm_sub(b0, b5), bx1));  // operand of M14
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T mx0 = fmm_sub(fmm_neg(m2), m4);
    const T mx1 = fmm_add(fmm_neg(m5), m9);
    const T mx2 = fmm_sub(m3, m6);
    const T mx3 = fmm_add(m7, m11);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(m5, m12), mx0), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(m5, m12), mx0));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_neg(mx0), mx1), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_neg(mx0), mx1));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m0), m1), m10), m14), mx2), mx3), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m0), m1), m10), m14), mx2), mx3));
    if (kBeta) st(3, fmm_add(fmm_add(m5, m7), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(m5, m7));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_sub(m4, m14), mx1), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_sub(m4, m14), mx1));
    if (kBeta) st(5, fmm_add(fmm_add(mx2, mx3), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(mx2, mx3));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m3), m5), m10), m13), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_add(fmm_add(fmm_neg(m3), m5), m10), m13));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m2), m8), m11), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m2), m8), m11));
    if (kBeta) st(8, fmm_add(fmm_add(m10, m11), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(m10, m11));
  }
};

// grey333_23_152  <3,3,3; 23>  (reference header algorithms/fast333_23_152.hpp, coefficients codegen/algorithms/grey333-23-152)
struct FmmAlg_grey333_23_152 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 3, kR = 23;
  static constexpr int kNumAOut = 15, kNumBOut = 17;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_add(a2, a3));  // operand of M3
    st(1, fmm_sub(fmm_add(fmm_sub(a3, a4), a6), a7));  // operand of M4
    st(2, fmm_sub(fmm_sub(fmm_neg(a0), a2), a6));  // operand of M5
    st(3, fmm_add(fmm_sub(a3, a4), a8));  // operand of M6
    st(4, fmm_add(fmm_neg(a0), a1));  // operand of M9
    st(5, fmm_add(fmm_add(fmm_sub(fmm_neg(a2), a3), a4), a5));  // operand of M10
    st(6, fmm_sub(a1, a3));  // operand of M12
    st(7, fmm_sub(fmm_sub(fmm_neg(a3), a5), a8));  // operand of M13
    st(8, fmm_sub(fmm_sub(a3, a4), a7));  // operand of M14
    st(9, fmm_sub(fmm_neg(a5), a8));  // operand of M15
    st(10, fmm_sub(a0, a1));  // operand of M16
    st(11, fmm_add(fmm_sub(a0, a1), a6));  // operand of M19
    st(12, fmm_sub(a3, a4));  // operand of M20
    st(13, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(a0), a1), a6), a7), a8));  // operand of M21
    st(14, fmm_add(a4, a7));  // operand of M22
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    st(0, fmm_sub(fmm_neg(b0), b3));  // operand of M1
    st(1, fmm_sub(fmm_add(fmm_add(b2, b5), b7), b8));  // operand of M3
    st(2, fmm_add(b2, b5));  // operand of M5
    st(3, fmm_add(fmm_neg(b5), b7));  // operand of M6
    st(4, fmm_add(fmm_sub(fmm_neg(b0), b1), b2));  // operand of M7
    st(5, fmm_add(fmm_sub(fmm_neg(b2), b5), b8));  // operand of M8
    st(6, fmm_add(b0, b1));  // operand of M9
    st(7, fmm_add(fmm_neg(b5), b8));  // operand of M11
    st(8, fmm_add(b1, b4));  // operand of M12
    st(9, fmm_add(fmm_neg(b7), b8));  // operand of M13
    st(10, fmm_add(fmm_sub(b0, b4), b5));  // operand of M14
    st(11, fmm_sub(fmm_add(b3, b4), b5));  // operand of M17
    st(12, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(b1, b2), b4), b5), b7), b8));  // operand of M18
    st(13, fmm_add(fmm_add(b0, b1), b5));  // operand of M19
    st(14, fmm_add(fmm_neg(b4), b7));  // operand of M20
    st(15, fmm_add(b0, b3));  // operand of M22
    st(16, fmm_add(fmm_add(fmm_neg(b5), b6), b7));  // operand of M23
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(m0, m1), m15), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(m0, m1), m15));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(m2, m7), m8), m11), m15), m17), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(m2, m7), m8), m11), m15), m17));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_neg(m4), m6), m7), m8), m18), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_neg(m4), m6), m7), m8), m18));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(m5, m13), m14), m16), m19), m21), m22), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(m5, m13), m14), m16), m19), m21), m22));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m2, m7), m9), m17), m19), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_add(m2, m7), m9), m17), m19));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m2, m5), m7), m9), m10), m12), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m2, m5), m7), m9), m10), m12));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(m3, m5), m13), m16), m19), m22), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(m3, m5), m13), m16), m19), m22));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m3), m5), m8), m13), m18), m19), m20), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m3), m5), m8), m13), m18), m19), m20));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m6, m8), m10), m18), m20), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_sub(fmm_add(m6, m8), m10), m18), m20));
  }
};

// grey333_23_221  <3,3,3; 23>  (reference header algorithms/fast333_23_221.hpp, coefficients codegen/algorithms/grey333-23-221)
struct FmmAlg_grey333_23_221 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 3, kR = 23;
  static constexpr int kNumAOut = 18, kNumBOut = 19;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_add(fmm_sub(fmm_sub(a4, a5), a7), a8));  // operand of M2
    st(1, fmm_sub(a3, a4));  // operand of M3
    st(2, fmm_add(a1, a7));  // operand of M4
    st(3, fmm_sub(a1, a2));  // operand of M5
    st(4, fmm_add(fmm_sub(fmm_sub(fmm_add(a2, a3), a5), a6), a8));  // operand of M7
    st(5, fmm_add(fmm_sub(fmm_sub(a3, a5), a6), a8));  // operand of M8
    st(6, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(a0, a1), a3), a4), a6), a7));  // operand of M9
    st(7, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(a0, a1), a3), a5), a6), a8));  // operand of M10
    st(8, fmm_add(fmm_neg(a3), a6));  // operand of M13
    st(9, fmm_sub(fmm_add(fmm_sub(a1, a2), a7), a8));  // operand of M14
    st(10, fmm_sub(fmm_add(fmm_add(fmm_sub(a1, a2), a5), a7), a8));  // operand of M15
    st(11, fmm_sub(fmm_add(fmm_add(fmm_neg(a3), a5), a7), a8));  // operand of M16
    st(12, fmm_add(fmm_sub(fmm_add(fmm_neg(a0), a1), a6), a7));  // operand of M17
    st(13, fmm_add(fmm_sub(a2, a5), a8));  // operand of M18
    st(14, fmm_add(fmm_sub(fmm_add(fmm_neg(a0), a1), a4), a7));  // operand of M19
    st(15, fmm_sub(a3, a7));  // operand of M20
    st(16, fmm_sub(a0, a1));  // operand of M21
    st(17, fmm_add(fmm_sub(a3, a7), a8));  // operand of M23
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    st(0, fmm_add(fmm_add(fmm_add(b0, b1), b3), b4));  // operand of M1
    st(1, fmm_sub(fmm_add(b0, b1), b5));  // operand of M3
    st(2, fmm_add(fmm_add(b0, b3), b6));  // operand of M4
    st(3, fmm_sub(fmm_neg(b1), b4));  // operand of M5
    st(4, fmm_add(b2, b5));  // operand of M6
    st(5, fmm_add(fmm_add(fmm_sub(fmm_neg(b1), b4), b6), b8));  // operand of M7
    st(6, fmm_add(fmm_add(fmm_neg(b4), b6), b8));  // operand of M8
    st(7, fmm_add(b0, b1));  // operand of M9
    st(8, fmm_add(fmm_add(b6, b7), b8));  // operand of M11
    st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), b2), b3), b4), b5));  // operand of M12
    st(10, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(b1), b2), b4), b6), b8));  // operand of M13
    st(11, fmm_sub(fmm_add(b1, b4), b6));  // operand of M15
    st(12, fmm_add(fmm_add(fmm_neg(b1), b6), b7));  // operand of M16
    st(13, fmm_add(fmm_add(b1, b4), b7));  // operand of M18
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), b3), b4), b5));  // operand of M19
    st(15, fmm_add(fmm_add(fmm_neg(b5), b6), b7));  // operand of M20
    st(16, fmm_add(fmm_add(b3, b4), b5));  // operand of M21
    st(17, fmm_add(fmm_add(b6, b7), b8));  // operand of M22
    st(18, fmm_add(b6, b7));  // operand of M23
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m2), m3), m4), m6), m7), m8), m14), m15), m16), m17), m18), m19), m20), m21), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m2), m3), m4), m6), m7), m8), m14), m15), m16), m17), m18), m19), m20), m21));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m4), m6), m7), m9), m21), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m4), m6), m7), m9), m21));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(m0, m2), m3), m8), m9), m11), m14), m15), m16), m17), m18), m19), m21), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(m0, m2), m3), m8), m9), m11), m14), m15), m16), m17), m18), m19), m21));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(m0, m1), m4), m8), m9), m13), m14), m16), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(m0, m1), m4), m8), m9), m13), m14), m16));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m1, m4), m13), m14), m15), m22), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m1, m4), m13), m14), m15), m22));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(m2, m5), m8), m9), m10), m15), m16), m22), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(m2, m5), m8), m9), m10), m15), m16), m22));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(m0, m2), m4), m6), m7), m8), m13), m14), m15), m17), m18), m19), m20), m21), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(m0, m2), m4), m6), m7), m8), m13), m14), m15), m17), m18), m19), m20), m21));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m4, m6), m7), m13), m14), m15), m17), m21), m22), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m4, m6), m7), m13), m14), m15), m17), m21), m22));
    if (kBeta) st(8, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m5, m6), m10), m12), m17), m19), m21), m22), fmm_mul(beta, ldc(8)))); else st(8, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m5, m6), m10), m12), m17), m19), m21), m22));
  }
};

// grey333_23_125  <3,3,3; 23>  (reference header algorithms/fast333_23_125.hpp, coefficients codegen/algorithms/eliminated/grey333-23-125)
struct FmmAlg_grey333_23_125 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 3, kR = 23;
  static constexpr int kNumAOut = 14, kNumBOut = 16;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T ax0 = fmm_add(a2, a3);
    const T ax1 = fmm_sub(a3, a4);
    const T ax2 = fmm_sub(a6, a7);
    const T ax3 = fmm_sub(fmm_neg(a0), a6);
    const T ax4 = fmm_add(fmm_neg(a0), a1);
    const T ax5 = fmm_sub(fmm_neg(a5), a8);
    st(0, ax0);
    st(1, ax1);
    st(2, ax4);
    st(3, ax5);
    st(4, fmm_add(ax1, ax2));  // operand of M4
    st(5, fmm_add(fmm_neg(a2), ax3));  // operand of M5
    st(6, fmm_add(a8, ax1));  // operand of M6
    st(7, fmm_sub(fmm_add(a4, a5), ax0));  // operand of M10
    st(8, fmm_sub(a1, a3));  // operand of M12
    st(9, fmm_add(fmm_neg(a3), ax5));  // operand of M13
    st(10, fmm_add(fmm_neg(a7), ax1));  // operand of M14
    st(11, fmm_sub(fmm_neg(a1), ax3));  // operand of M19
    st(12, fmm_add(fmm_sub(a8, ax2), ax4));  // operand of M21
    st(13, fmm_add(a4, a7));  // operand of M22
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T bx0 = fmm_sub(fmm_neg(b0), b3);
    const T bx1 = fmm_add(b2, b5);
    const T bx2 = fmm_sub(b7, b8);
    const T bx3 = fmm_add(fmm_neg(b5), b7);
    const T bx4 = fmm_sub(fmm_neg(b0), b1);
    const T bx5 = fmm_add(b1, b4);
    const T bx6 = fmm_add(fmm_neg(b4), b5);
    st(0, bx0);
    st(1, bx1);
    st(2, bx2);
    st(3, bx3);
    st(4, bx4);
    st(5, bx5);
    st(6, fmm_add(bx1, bx2));  // operand of M3
    st(7, fmm_add(b2, bx4));  // operand of M7
    st(8, fmm_sub(b8, bx1));  // operand of M8
    st(9, fmm_add(fmm_neg(b5), b8));  // operand of M11
    st(10, fmm_add(b0, bx6));  // operand of M14
    st(11, fmm_sub(b3, bx6));  // operand of M17
    st(12, fmm_add(fmm_sub(fmm_neg(bx1), bx2), bx5));  // operand of M18
    st(13, fmm_sub(b5, bx4));  // operand of M19
    st(14, fmm_add(fmm_neg(b4), b7));  // operand of M20
    st(15, fmm_add(b6, bx3));  // operand of M23
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T mx0 = fmm_add(m2, m7);
    const T mx1 = fmm_sub(fmm_neg(m6), m8);
    const T mx2 = fmm_add(m5, m13);
    const T mx3 = fmm_sub(fmm_neg(m16), m19);
    const T mx4 = fmm_add(m18, m20);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(m0, m1), m15), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(m0, m1), m15));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m8), m11), m15), m17), mx0), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m8), m11), m15), m17), mx0));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m4), m7), m18), mx1), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_sub(fmm_add(fmm_neg(m4), m7), m18), mx1));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m14, m21), m22), mx2), mx3), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_sub(fmm_add(m14, m21), m22), mx2), mx3));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(m9, m17), m19), mx0), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(m9, m17), m19), mx0));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(m5, m9), m10), m12), mx0), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_sub(fmm_add(fmm_add(m5, m9), m10), m12), mx0));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_sub(fmm_add(m3, m22), mx2), mx3), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_sub(fmm_add(m3, m22), mx2), mx3));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m3), m8), m19), mx2), mx4), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m3), m8), m19), mx2), mx4));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_sub(fmm_neg(m10), mx1), mx4), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_sub(fmm_neg(m10), mx1), mx4));
  }
};

// smirnov333_23_139  <3,3,3; 23>  (reference header algorithms/smirnov333_23_139.hpp, coefficients codegen/algorithms/smirnov333-23-139)
struct FmmAlg_smirnov333_23_139 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 3, kR = 23;
  static constexpr int kNumAOut = 20, kNumBOut = 14;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_add(a4, a8));  // operand of M2
    st(1, fmm_add(fmm_add(fmm_add(a0, a1), a6), a7));  // operand of M3
    st(2, fmm_add(fmm_neg(a0), a3));  // operand of M4
    st(3, fmm_sub(fmm_neg(a6), a7));  // operand of M5
    st(4, fmm_add(a4, a5));  // operand of M6
    st(5, fmm_sub(fmm_neg(a3), a8));  // operand of M7
    st(6, fmm_add(a6, a8));  // operand of M8
    st(7, fmm_sub(a4, a7));  // operand of M10
    st(8, fmm_sub(fmm_neg(a7), a8));  // operand of M11
    st(9, fmm_add(fmm_add(fmm_neg(a2), a4), a5));  // operand of M12
    st(10, fmm_add(a2, a8));  // operand of M13
    st(11, fmm_add(a0, a6));  // operand of M14
    st(12, fmm_add(fmm_neg(a0), a8));  // operand of M15
    st(13, fmm_add(fmm_neg(a2), a5));  // operand of M16
    st(14, fmm_add(fmm_add(fmm_sub(fmm_neg(a1), a2), a4), a5));  // operand of M17
    st(15, fmm_add(fmm_neg(a5), a8));  // operand of M18
    st(16, fmm_sub(fmm_sub(fmm_neg(a0), a6), a7));  // operand of M19
    st(17, fmm_sub(fmm_neg(a0), a2));  // operand of M20
    st(18, fmm_sub(fmm_neg(a3), a4));  // operand of M22
    st(19, fmm_add(fmm_neg(a1), a8));  // operand of M23
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    st(0, fmm_add(fmm_sub(fmm_neg(b0), b3), b6));  // operand of M1
    st(1, fmm_add(fmm_neg(b3), b7));  // operand of M2
    st(2, fmm_add(b1, b2));  // operand of M4
    st(3, fmm_sub(fmm_add(fmm_neg(b1), b4), b7));  // operand of M9
    st(4, fmm_sub(fmm_add(b1, b3), b4));  // operand of M10
    st(5, fmm_sub(fmm_add(b4, b5), b7));  // operand of M12
    st(6, fmm_add(b6, b8));  // operand of M13
    st(7, fmm_sub(fmm_add(b0, b2), b5));  // operand of M14
    st(8, fmm_add(b0, b8));  // operand of M15
    st(9, fmm_add(fmm_add(fmm_sub(fmm_neg(b4), b5), b7), b8));  // operand of M16
    st(10, fmm_sub(fmm_neg(b4), b5));  // operand of M17
    st(11, fmm_add(fmm_neg(b6), b7));  // operand of M18
    st(12, fmm_sub(fmm_neg(b1), b5));  // operand of M19
    st(13, fmm_add(fmm_sub(fmm_neg(b1), b2), b8));  // operand of M21
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(m0), m12), m14), m19), m22), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(m0), m12), m14), m19), m22));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m2), m4), m5), m11), m16), m18), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m2), m4), m5), m11), m16), m18));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m2, m4), m18), m19), m20), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_sub(fmm_sub(fmm_add(m2, m4), m18), m19), m20));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(m0, m1), m5), m6), m17), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(m0, m1), m5), m6), m17));
    if (kBeta) st(4, fmm_add(fmm_sub(fmm_add(m5, m8), m21), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(fmm_add(m5, m8), m21));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(m3, m8), m11), m15), m19), m20), m21), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(m3, m8), m11), m15), m19), m20), m21));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_add(m0, m7), m10), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_add(m0, m7), m10));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m1, m4), m8), m9), m10), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_add(fmm_add(fmm_add(m1, m4), m8), m9), m10));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m4), m7), m13), m14), m18), m20), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m4), m7), m13), m14), m18), m20));
  }
};

// smirnov333_23_128  <3,3,3; 23>  (reference header algorithms/smirnov333_23_128.hpp, coefficients codegen/algorithms/eliminated/smirnov333-23-128)
struct FmmAlg_smirnov333_23_128 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 3, kR = 23;
  static constexpr int kNumAOut = 20, kNumBOut = 14;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T ax0 = fmm_add(a0, a6);
    const T ax1 = fmm_add(a4, a5);
    st(0, ax0);
    st(1, ax1);
    st(2, fmm_add(a4, a8));  // operand of M2
    st(3, fmm_add(fmm_add(a1, a7), ax0));  // operand of M3
    st(4, fmm_add(fmm_neg(a0), a3));  // operand of M4
    st(5, fmm_sub(fmm_neg(a6), a7));  // operand of M5
    st(6, fmm_sub(fmm_neg(a3), a8));  // operand of M7
    st(7, fmm_add(a6, a8));  // operand of M8
    st(8, fmm_sub(a4, a7));  // operand of M10
    st(9, fmm_sub(fmm_neg(a7), a8));  // operand of M11
    st(10, fmm_add(fmm_neg(a2), ax1));  // operand of M12
    st(11, fmm_add(a2, a8));  // operand of M13
    st(12, fmm_add(fmm_neg(a0), a8));  // operand of M15
    st(13, fmm_add(fmm_neg(a2), a5));  // operand of M16
    st(14, fmm_add(fmm_sub(fmm_neg(a1), a2), ax1));  // operand of M17
    st(15, fmm_add(fmm_neg(a5), a8));  // operand of M18
    st(16, fmm_sub(fmm_neg(a7), ax0));  // operand of M19
    st(17, fmm_sub(fmm_neg(a0), a2));  // operand of M20
    st(18, fmm_sub(fmm_neg(a3), a4));  // operand of M22
    st(19, fmm_add(fmm_neg(a1), a8));  // operand of M23
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T bx0 = fmm_add(b1, b2);
    const T bx1 = fmm_add(fmm_neg(b1), b4);
    const T bx2 = fmm_add(b4, b5);
    st(0, bx0);
    st(1, bx2);
    st(2, fmm_add(fmm_sub(fmm_neg(b0), b3), b6));  // operand of M1
    st(3, fmm_add(fmm_neg(b3), b7));  // operand of M2
    st(4, fmm_add(fmm_neg(b7), bx1));  // operand of M9
    st(5, fmm_sub(b3, bx1));  // operand of M10
    st(6, fmm_add(fmm_neg(b7), bx2));  // operand of M12
    st(7, fmm_add(b6, b8));  // operand of M13
    st(8, fmm_sub(fmm_add(b0, b2), b5));  // operand of M14
    st(9, fmm_add(b0, b8));  // operand of M15
    st(10, fmm_sub(fmm_add(b7, b8), bx2));  // operand of M16
    st(11, fmm_add(fmm_neg(b6), b7));  // operand of M18
    st(12, fmm_sub(fmm_neg(b1), b5));  // operand of M19
    st(13, fmm_sub(b8, bx0));  // operand of M21
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T mx0 = fmm_sub(fmm_neg(m2), m4);
    const T mx1 = fmm_sub(fmm_neg(m18), m20);
    const T mx2 = fmm_sub(m8, m21);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(m0), m12), m14), m19), m22), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(m0), m12), m14), m19), m22));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m5, m11), m16), m18), mx0), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(m5, m11), m16), m18), mx0));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_sub(fmm_neg(m19), mx0), mx1), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_sub(fmm_neg(m19), mx0), mx1));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(m0, m1), m5), m6), m17), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(m0, m1), m5), m6), m17));
    if (kBeta) st(4, fmm_add(fmm_add(m5, mx2), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(m5, mx2));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(m3, m11), m15), m19), m20), mx2), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(m3, m11), m15), m19), m20), mx2));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_add(m0, m7), m10), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_add(m0, m7), m10));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m1, m4), m8), m9), m10), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_add(fmm_add(fmm_add(m1, m4), m8), m9), m10));
    if (kBeta) st(8, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_neg(m4), m7), m13), m14), mx1), fmm_mul(beta, ldc(8)))); else st(8, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_neg(m4), m7), m13), m14), mx1));
  }
};

// classical333_27_81  <3,3,3; 27>  (reference header algorithms/classical333.hpp, coefficients codegen/algorithms/classical333-27-81)
struct FmmAlg_classical333_27_81 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 3, kR = 27;
  static constexpr int kNumAOut = 0, kNumBOut = 0;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T m26 = ld(26);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(m0, m1), m2), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(m0, m1), m2));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(m3, m4), m5), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(m3, m4), m5));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(m6, m7), m8), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(m6, m7), m8));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(m9, m10), m11), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(m9, m10), m11));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(m12, m13), m14), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(m12, m13), m14));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(m15, m16), m17), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(m15, m16), m17));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(m18, m19), m20), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(m18, m19), m20));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(m21, m22), m23), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(m21, m22), m23));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(m24, m25), m26), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(m24, m25), m26));
  }
};

// schonhage333_21_117_approx  <3,3,3; 21>  (reference header algorithms/schonhage333_21_117_approx.hpp, coefficients codegen/algorithms/schonhage333-21-117-approx)
struct FmmAlg_schonhage333_21_117_approx {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 3, kR = 21;
  static constexpr int kNumAOut = 18, kNumBOut = 18;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_add(a0, fmm_mul(cf[1], a1)));  // operand of M1
    st(1, fmm_add(a0, fmm_mul(cf[1], a4)));  // operand of M2
    st(2, fmm_add(a0, fmm_mul(cf[1], a7)));  // operand of M3
    st(3, fmm_add(fmm_mul(cf[1], a1), a3));  // operand of M4
    st(4, fmm_add(a3, fmm_mul(cf[1], a4)));  // operand of M5
    st(5, fmm_add(a3, fmm_mul(cf[1], a7)));  // operand of M6
    st(6, fmm_add(fmm_mul(cf[1], a1), a6));  // operand of M7
    st(7, fmm_add(fmm_mul(cf[1], a4), a6));  // operand of M8
    st(8, fmm_add(a6, fmm_mul(cf[1], a7)));  // operand of M9
    st(9, fmm_add(a0, fmm_mul(cf[1], a2)));  // operand of M10
    st(10, fmm_add(a0, fmm_mul(cf[1], a5)));  // operand of M11
    st(11, fmm_add(a0, fmm_mul(cf[1], a8)));  // operand of M12
    st(12, fmm_add(fmm_mul(cf[1], a2), a3));  // operand of M13
    st(13, fmm_add(a3, fmm_mul(cf[1], a5)));  // operand of M14
    st(14, fmm_add(a3, fmm_mul(cf[1], a8)));  // operand of M15
    st(15, fmm_add(fmm_mul(cf[1], a2), a6));  // operand of M16
    st(16, fmm_add(fmm_mul(cf[1], a5), a6));  // operand of M17
    st(17, fmm_add(a6, fmm_mul(cf[1], a8)));  // operand of M18
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    st(0, fmm_add(fmm_mul(cf[1], b0), b3));  // operand of M1
    st(1, fmm_add(fmm_mul(cf[2], b1), b3));  // operand of M2
    st(2, fmm_add(fmm_mul(cf[2], b2), b3));  // operand of M3
    st(3, fmm_add(fmm_mul(cf[2], b0), b4));  // operand of M4
    st(4, fmm_add(fmm_mul(cf[1], b1), b4));  // operand of M5
    st(5, fmm_add(fmm_mul(cf[2], b2), b4));  // operand of M6
    st(6, fmm_add(fmm_mul(cf[2], b0), b5));  // operand of M7
    st(7, fmm_add(fmm_mul(cf[2], b1), b5));  // operand of M8
    st(8, fmm_add(fmm_mul(cf[1], b2), b5));  // operand of M9
    st(9, fmm_add(fmm_mul(cf[3], b1), b6));  // operand of M11
    st(10, fmm_add(fmm_mul(cf[3], b2), b6));  // operand of M12
    st(11, fmm_add(fmm_mul(cf[3], b0), b7));  // operand of M13
    st(12, fmm_add(fmm_mul(cf[3], b2), b7));  // operand of M15
    st(13, fmm_add(fmm_mul(cf[3], b0), b8));  // operand of M16
    st(14, fmm_add(fmm_mul(cf[3], b1), b8));  // operand of M17
    st(15, fmm_add(b3, b6));  // operand of M19
    st(16, fmm_add(b4, b7));  // operand of M20
    st(17, fmm_add(b5, b8));  // operand of M21
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m0), fmm_mul(cf[4], m9)), fmm_mul(cf[5], m18)), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_mul(cf[4], m0), fmm_mul(cf[4], m9)), fmm_mul(cf[5], m18)));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m3), fmm_mul(cf[6], m9)), fmm_mul(cf[7], m10)), fmm_mul(cf[4], m12)), fmm_mul(cf[5], m19)), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m3), fmm_mul(cf[6], m9)), fmm_mul(cf[7], m10)), fmm_mul(cf[4], m12)), fmm_mul(cf[5], m19)));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m6), fmm_mul(cf[6], m9)), fmm_mul(cf[7], m11)), fmm_mul(cf[4], m15)), fmm_mul(cf[5], m20)), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m6), fmm_mul(cf[6], m9)), fmm_mul(cf[7], m11)), fmm_mul(cf[4], m15)), fmm_mul(cf[5], m20)));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m1), fmm_mul(cf[4], m10)), fmm_mul(cf[7], m12)), fmm_mul(cf[6], m13)), fmm_mul(cf[5], m18)), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m1), fmm_mul(cf[4], m10)), fmm_mul(cf[7], m12)), fmm_mul(cf[6], m13)), fmm_mul(cf[5], m18)));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m4), fmm_mul(cf[4], m13)), fmm_mul(cf[5], m19)), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_mul(cf[4], m4), fmm_mul(cf[4], m13)), fmm_mul(cf[5], m19)));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m7), fmm_mul(cf[6], m13)), fmm_mul(cf[7], m14)), fmm_mul(cf[4], m16)), fmm_mul(cf[5], m20)), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m7), fmm_mul(cf[6], m13)), fmm_mul(cf[7], m14)), fmm_mul(cf[4], m16)), fmm_mul(cf[5], m20)));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m2), fmm_mul(cf[4], m11)), fmm_mul(cf[7], m15)), fmm_mul(cf[6], m17)), fmm_mul(cf[5], m18)), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m2), fmm_mul(cf[4], m11)), fmm_mul(cf[7], m15)), fmm_mul(cf[6], m17)), fmm_mul(cf[5], m18)));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m5), fmm_mul(cf[4], m14)), fmm_mul(cf[7], m16)), fmm_mul(cf[6], m17)), fmm_mul(cf[5], m19)), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m5), fmm_mul(cf[4], m14)), fmm_mul(cf[7], m16)), fmm_mul(cf[6], m17)), fmm_mul(cf[5], m19)));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m8), fmm_mul(cf[4], m17)), fmm_mul(cf[5], m20)), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_mul(cf[4], m8), fmm_mul(cf[4], m17)), fmm_mul(cf[5], m20)));
  }
};

// smirnov333_20_182_approx  <3,3,3; 20>  (reference header algorithms/smirnov333_20_182_approx.hpp, coefficients codegen/algorithms/smirnov333-20-182-approx)
struct FmmAlg_smirnov333_20_182_approx {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 3, kR = 20;
  static constexpr int kNumAOut = 16, kNumBOut = 17;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_add(fmm_add(fmm_add(fmm_mul(cf[0], a0), fmm_mul(cf[5], a2)), fmm_mul(cf[11], a6)), fmm_mul(cf[7], a8)));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_add(fmm_mul(cf[6], a2), fmm_mul(cf[7], a3)), fmm_mul(cf[8], a4)), fmm_mul(cf[12], a8)));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_mul(cf[8], a3), a4), fmm_mul(cf[9], a7)));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_add(fmm_neg(a0), fmm_mul(cf[0], a1)), fmm_mul(cf[9], a6)), fmm_mul(cf[11], a7)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_mul(cf[5], a2), fmm_mul(cf[7], a3)), fmm_mul(cf[7], a8)));  // operand of M5
    st(5, fmm_add(fmm_mul(cf[7], a6), fmm_mul(cf[8], a7)));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(fmm_mul(cf[0], a0), fmm_mul(cf[2], a1)), fmm_mul(cf[7], a6)), fmm_mul(cf[8], a7)));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[0], a0), fmm_mul(cf[5], a2)), fmm_mul(cf[9], a3)), a5), fmm_mul(cf[11], a6)));  // operand of M8
    st(8, fmm_add(fmm_mul(cf[9], a3), fmm_mul(cf[11], a4)));  // operand of M9
    st(9, fmm_sub(fmm_mul(cf[7], a3), a5));  // operand of M11
    st(10, fmm_add(fmm_add(fmm_add(fmm_mul(cf[3], a1), fmm_mul(cf[9], a3)), a5), a7));  // operand of M12
    st(11, fmm_add(fmm_add(fmm_add(fmm_neg(a3), fmm_mul(cf[0], a4)), fmm_mul(cf[7], a6)), fmm_mul(cf[8], a7)));  // operand of M13
    st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(a0), fmm_mul(cf[0], a1)), fmm_mul(cf[3], a2)), fmm_mul(cf[9], a6)), fmm_mul(cf[11], a7)));  // operand of M14
    st(13, fmm_sub(fmm_add(fmm_mul(cf[4], a1), fmm_mul(cf[7], a3)), a7));  // operand of M16
    st(14, fmm_add(fmm_add(fmm_mul(cf[8], a3), a4), fmm_mul(cf[0], a5)));  // operand of M18
    st(15, fmm_add(fmm_add(fmm_neg(a3), fmm_mul(cf[3], a5)), fmm_mul(cf[7], a8)));  // operand of M19
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    st(0, fmm_add(fmm_add(fmm_add(fmm_add(b0, fmm_mul(cf[0], b1)), fmm_mul(cf[11], b3)), fmm_mul(cf[7], b6)), fmm_mul(cf[13], b8)));  // operand of M1
    st(1, fmm_add(fmm_mul(cf[6], b5), fmm_mul(cf[11], b8)));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_mul(cf[11], b3), b4), fmm_mul(cf[4], b5)));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_mul(cf[0], b0), b3), fmm_mul(cf[11], b6)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, fmm_mul(cf[0], b1)), fmm_mul(cf[11], b3)), fmm_mul(cf[7], b6)), fmm_mul(cf[11], b7)), fmm_mul(cf[6], b8)));  // operand of M5
    st(5, fmm_add(fmm_mul(cf[3], b2), fmm_mul(cf[7], b3)));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_mul(cf[0], b0), fmm_mul(cf[6], b2)), fmm_mul(cf[11], b3)));  // operand of M7
    st(7, fmm_add(fmm_mul(cf[0], b2), fmm_mul(cf[7], b6)));  // operand of M8
    st(8, fmm_add(fmm_mul(cf[0], b4), fmm_mul(cf[11], b8)));  // operand of M9
    st(9, fmm_add(fmm_add(fmm_mul(cf[6], b2), fmm_mul(cf[11], b3)), b4));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_mul(cf[0], b2), b5), b7));  // operand of M11
    st(11, fmm_add(fmm_neg(b5), fmm_mul(cf[7], b6)));  // operand of M12
    st(12, fmm_add(fmm_mul(cf[7], b7), fmm_mul(cf[4], b8)));  // operand of M15
    st(13, fmm_add(fmm_sub(fmm_add(b0, fmm_mul(cf[11], b3)), b4), fmm_mul(cf[7], b6)));  // operand of M16
    st(14, fmm_add(fmm_add(fmm_add(fmm_mul(cf[12], b1), fmm_mul(cf[6], b2)), fmm_mul(cf[11], b3)), fmm_mul(cf[14], b8)));  // operand of M17
    st(15, fmm_add(b5, fmm_mul(cf[11], b8)));  // operand of M18
    st(16, fmm_add(fmm_add(fmm_add(fmm_mul(cf[0], b1), b4), fmm_mul(cf[11], b7)), fmm_mul(cf[6], b8)));  // operand of M20
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[12], m1), fmm_mul(cf[0], m2)), fmm_mul(cf[8], m3)), m5), fmm_mul(cf[8], m6)), fmm_mul(cf[12], m8)), fmm_mul(cf[0], m9)), fmm_mul(cf[12], m12)), fmm_mul(cf[11], m13)), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[12], m1), fmm_mul(cf[0], m2)), fmm_mul(cf[8], m3)), m5), fmm_mul(cf[8], m6)), fmm_mul(cf[12], m8)), fmm_mul(cf[0], m9)), fmm_mul(cf[12], m12)), fmm_mul(cf[11], m13)));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_mul(cf[7], m0), fmm_mul(cf[7], m3)), fmm_mul(cf[9], m4)), m5), m9), fmm_mul(cf[11], m14)), fmm_mul(cf[7], m15)), fmm_mul(cf[7], m16)), fmm_mul(cf[7], m19)), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_mul(cf[7], m0), fmm_mul(cf[7], m3)), fmm_mul(cf[9], m4)), m5), m9), fmm_mul(cf[11], m14)), fmm_mul(cf[7], m15)), fmm_mul(cf[7], m16)), fmm_mul(cf[7], m19)));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[7], m1), fmm_mul(cf[9], m2)), fmm_mul(cf[9], m5)), fmm_mul(cf[7], m7)), fmm_mul(cf[7], m8)), fmm_mul(cf[9], m9)), fmm_mul(cf[7], m10)), fmm_mul(cf[9], m11)), fmm_mul(cf[7], m12)), fmm_mul(cf[7], m13)), fmm_mul(cf[9], m14)), fmm_mul(cf[7], m18)), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[7], m1), fmm_mul(cf[9], m2)), fmm_mul(cf[9], m5)), fmm_mul(cf[7], m7)), fmm_mul(cf[7], m8)), fmm_mul(cf[9], m9)), fmm_mul(cf[7], m10)), fmm_mul(cf[9], m11)), fmm_mul(cf[7], m12)), fmm_mul(cf[7], m13)), fmm_mul(cf[9], m14)), fmm_mul(cf[7], m18)));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m0), fmm_mul(cf[12], m1)), fmm_mul(cf[15], m2)), fmm_mul(cf[3], m4)), fmm_mul(cf[16], m7)), fmm_mul(cf[12], m8)), fmm_mul(cf[0], m9)), fmm_mul(cf[12], m10)), fmm_mul(cf[0], m11)), fmm_mul(cf[17], m12)), fmm_mul(cf[12], m13)), fmm_mul(cf[5], m14)), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[4], m0), fmm_mul(cf[12], m1)), fmm_mul(cf[15], m2)), fmm_mul(cf[3], m4)), fmm_mul(cf[16], m7)), fmm_mul(cf[12], m8)), fmm_mul(cf[0], m9)), fmm_mul(cf[12], m10)), fmm_mul(cf[0], m11)), fmm_mul(cf[17], m12)), fmm_mul(cf[12], m13)), fmm_mul(cf[5], m14)));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m1, fmm_mul(cf[18], m8)), m14), fmm_mul(cf[3], m17)), m18), fmm_mul(cf[0], m19)), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m1, fmm_mul(cf[18], m8)), m14), fmm_mul(cf[3], m17)), m18), fmm_mul(cf[0], m19)));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[0], m1), fmm_mul(cf[0], m10)), fmm_mul(cf[12], m14)), m17), fmm_mul(cf[0], m18)), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[0], m1), fmm_mul(cf[0], m10)), fmm_mul(cf[12], m14)), m17), fmm_mul(cf[0], m18)));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[17], m0), fmm_mul(cf[17], m3)), fmm_mul(cf[19], m5)), fmm_mul(cf[0], m6)), fmm_mul(cf[0], m16)), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(cf[17], m0), fmm_mul(cf[17], m3)), fmm_mul(cf[19], m5)), fmm_mul(cf[0], m6)), fmm_mul(cf[0], m16)));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(cf[3], m5), fmm_mul(cf[3], m9)), fmm_mul(cf[17], m14)), m16), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_add(fmm_add(fmm_mul(cf[3], m5), fmm_mul(cf[3], m9)), fmm_mul(cf[17], m14)), m16));
    if (kBeta) st(8, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m2), m5), m8), m9), m12), fmm_mul(beta, ldc(8)))); else st(8, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m2), m5), m8), m9), m12));
  }
};

// grey422_14_84  <4,2,2; 14>  (reference header algorithms/fast422_14_84.hpp, coefficients codegen/algorithms/grey422-14-84)
struct FmmAlg_grey422_14_84 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 2, kR = 14;
  static constexpr int kNumAOut = 10, kNumBOut = 10;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    st(0, fmm_add(fmm_sub(fmm_sub(a2, a3), a4), a5));  // operand of M1
    st(1, fmm_sub(fmm_add(fmm_neg(a1), a3), a5));  // operand of M2
    st(2, fmm_sub(fmm_add(fmm_neg(a0), a2), a4));  // operand of M3
    st(3, fmm_add(a5, a6));  // operand of M5
    st(4, fmm_add(a5, a7));  // operand of M6
    st(5, fmm_add(fmm_add(fmm_neg(a0), a2), a6));  // operand of M8
    st(6, fmm_add(fmm_sub(a0, a3), a5));  // operand of M9
    st(7, fmm_add(fmm_neg(a0), a1));  // operand of M10
    st(8, fmm_sub(a4, a5));  // operand of M11
    st(9, fmm_add(fmm_neg(a6), a7));  // operand of M12
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    st(0, fmm_add(fmm_neg(b2), b3));  // operand of M2
    st(1, fmm_add(fmm_neg(b0), b1));  // operand of M3
    st(2, fmm_add(b0, b2));  // operand of M4
    st(3, fmm_add(b1, b2));  // operand of M5
    st(4, fmm_add(fmm_neg(b2), b3));  // operand of M6
    st(5, fmm_add(b0, b2));  // operand of M7
    st(6, fmm_sub(b0, b1));  // operand of M8
    st(7, fmm_add(b1, b2));  // operand of M9
    st(8, fmm_add(b1, b3));  // operand of M13
    st(9, fmm_add(b1, b3));  // operand of M14
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    if (kBeta) st(0, fmm_add(fmm_sub(m6, m9), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(m6, m9));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m1), m8), m9), m12), m13), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m1), m8), m9), m12), m13));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(m0, m3), m4), m6), m7), m8), m10), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(m0, m3), m4), m6), m7), m8), m10));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(m0, m10), m13), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(m0, m10), m13));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m2, m3), m4), m7), m10), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_sub(m2, m3), m4), m7), m10));
    if (kBeta) st(5, fmm_add(fmm_sub(m10, m12), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(m10, m12));
    if (kBeta) st(6, fmm_add(fmm_add(m3, m11), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(m3, m11));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_add(m4, m5), m11), m12), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_add(m4, m5), m11), m12));
  }
};

// grey432_20_144  <4,3,2; 20>  (reference header algorithms/fast432_20_144.hpp, coefficients codegen/algorithms/grey432-20-144)
struct FmmAlg_grey432_20_144 {
  static constexpr int kM0 = 4, kK0 = 3, kN0 = 2, kR = 20;
  static constexpr int kNumAOut = 16, kNumBOut = 16;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    const T a10 = ld(10);
    const T a11 = ld(11);
    st(0, fmm_add(a3, a4));  // operand of M2
    st(1, fmm_add(fmm_add(a0, a1), a2));  // operand of M3
    st(2, fmm_sub(fmm_sub(fmm_neg(a0), a1), a11));  // operand of M4
    st(3, fmm_sub(fmm_add(a7, a8), a9));  // operand of M6
    st(4, fmm_sub(a0, a3));  // operand of M7
    st(5, fmm_add(fmm_add(fmm_sub(fmm_add(a3, a4), a6), a8), a9));  // operand of M9
    st(6, fmm_add(fmm_sub(fmm_sub(fmm_neg(a0), a1), a9), a10));  // operand of M10
    st(7, fmm_add(fmm_add(fmm_sub(fmm_neg(a7), a8), a10), a11));  // operand of M11
    st(8, fmm_sub(fmm_sub(fmm_neg(a3), a4), a8));  // operand of M12
    st(9, fmm_add(fmm_add(fmm_neg(a6), a7), a8));  // operand of M14
    st(10, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_neg(a0), a2), a4), a5), a11));  // operand of M15
    st(11, fmm_add(a7, a8));  // operand of M16
    st(12, fmm_add(fmm_neg(a5), a8));  // operand of M17
    st(13, fmm_sub(fmm_sub(fmm_neg(a0), a4), a5));  // operand of M18
    st(14, fmm_add(a0, a1));  // operand of M19
    st(15, fmm_add(a4, a5));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_add(fmm_neg(b0), b2));  // operand of M1
    st(1, fmm_add(fmm_neg(b3), b5));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_neg(b2), b3), b4));  // operand of M4
    st(3, fmm_sub(fmm_add(fmm_add(fmm_neg(b2), b3), b4), b5));  // operand of M5
    st(4, fmm_add(b0, b3));  // operand of M6
    st(5, fmm_add(fmm_sub(b1, b3), b5));  // operand of M7
    st(6, fmm_add(fmm_neg(b2), b4));  // operand of M8
    st(7, fmm_add(fmm_neg(b0), b1));  // operand of M9
    st(8, fmm_add(fmm_neg(b2), b3));  // operand of M11
    st(9, fmm_add(fmm_sub(fmm_add(fmm_neg(b0), b1), b3), b5));  // operand of M12
    st(10, fmm_add(b1, b3));  // operand of M13
    st(11, fmm_sub(fmm_neg(b0), b2));  // operand of M16
    st(12, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b1), b2), b3), b4), b5));  // operand of M17
    st(13, fmm_sub(fmm_add(fmm_sub(fmm_sub(b0, b1), b2), b3), b5));  // operand of M18
    st(14, fmm_add(fmm_neg(b2), b4));  // operand of M19
    st(15, fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b1), b2), b3));  // operand of M20
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_sub(fmm_neg(m0), m2), m18), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_sub(fmm_neg(m0), m2), m18));
    if (kBeta) st(1, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m3), m4), m14), m17), m18), m19), fmm_mul(beta, ldc(1)))); else st(1, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m3), m4), m14), m17), m18), m19));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m6), m7), m11), m16), m17), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m6), m7), m11), m16), m17));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_neg(m0), m1), m6), m17), m19), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_neg(m0), m1), m6), m17), m19));
    if (kBeta) st(4, fmm_add(fmm_sub(fmm_add(m7, m13), m15), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(fmm_add(m7, m13), m15));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_neg(m1), m5), m8), m11), m12), m13), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_neg(m1), m5), m8), m11), m12), m13));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m5), m9), m10), m15), m18), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m5), m9), m10), m15), m18));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m3), m4), m9), m12), m18), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m3), m4), m9), m12), m18));
  }
};

// grey423_20_144  <4,2,3; 20>  (reference header algorithms/fast423_20_144.hpp, coefficients codegen/algorithms/grey423-20-144)
struct FmmAlg_grey423_20_144 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 3, kR = 20;
  static constexpr int kNumAOut = 15, kNumBOut = 16;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    st(0, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a0), a1), a2), a3));  // operand of M1
    st(1, fmm_sub(fmm_neg(a3), a5));  // operand of M2
    st(2, fmm_sub(fmm_sub(fmm_neg(a1), a6), a7));  // operand of M4
    st(3, fmm_add(a1, a7));  // operand of M5
    st(4, fmm_sub(a5, a6));  // operand of M6
    st(5, fmm_sub(fmm_neg(a2), a3));  // operand of M7
    st(6, fmm_add(a2, a4));  // operand of M8
    st(7, fmm_add(a6, a7));  // operand of M10
    st(8, fmm_sub(a2, a5));  // operand of M12
    st(9, fmm_add(a5, a7));  // operand of M13
    st(10, fmm_add(a4, a5));  // operand of M14
    st(11, fmm_sub(fmm_neg(a4), a6));  // operand of M16
    st(12, fmm_add(fmm_add(a1, a2), a3));  // operand of M18
    st(13, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a0), a1), a6), a7));  // operand of M19
    st(14, fmm_sub(fmm_neg(a1), a3));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_add(fmm_neg(b0), b1));  // operand of M1
    st(1, fmm_add(fmm_neg(b4), b5));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_neg(b1), b2), b4));  // operand of M4
    st(3, fmm_sub(fmm_add(fmm_add(fmm_neg(b1), b2), b4), b5));  // operand of M5
    st(4, fmm_add(b0, b4));  // operand of M6
    st(5, fmm_add(fmm_sub(b3, b4), b5));  // operand of M7
    st(6, fmm_add(fmm_neg(b1), b2));  // operand of M8
    st(7, fmm_add(fmm_neg(b0), b3));  // operand of M9
    st(8, fmm_add(fmm_neg(b1), b4));  // operand of M11
    st(9, fmm_add(fmm_sub(fmm_add(fmm_neg(b0), b3), b4), b5));  // operand of M12
    st(10, fmm_add(b3, b4));  // operand of M13
    st(11, fmm_sub(fmm_neg(b0), b1));  // operand of M16
    st(12, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(b0), b1), b2), b3), b4), b5));  // operand of M17
    st(13, fmm_sub(fmm_add(fmm_sub(fmm_sub(b0, b1), b3), b4), b5));  // operand of M18
    st(14, fmm_add(fmm_neg(b1), b2));  // operand of M19
    st(15, fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b1), b3), b4));  // operand of M20
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(m0, m2), m3), m6), m9), m14), m17), m18), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(m0, m2), m3), m6), m9), m14), m17), m18));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_sub(fmm_sub(m2, m3), m9), m18), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_sub(fmm_sub(m2, m3), m9), m18));
    if (kBeta) st(2, fmm_add(fmm_add(m2, m14), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(m2, m14));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(m1, m6), m8), m11), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_sub(m1, m6), m8), m11));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m1, m8), m11), m14), m17), m19), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m1, m8), m11), m14), m17), m19));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(m14), m16), m17), m19), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_sub(fmm_sub(fmm_neg(m14), m16), m17), m19));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_neg(m8), m13), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_neg(m8), m13));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_sub(m5, m10), m13), m15), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_sub(m5, m10), m13), m15));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(m5, m7), m8), m10), m11), m13), m15), m16), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(m5, m7), m8), m10), m11), m13), m15), m16));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m5), m8), m9), m12), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_sub(fmm_add(fmm_neg(m5), m8), m9), m12));
    if (kBeta) st(10, fmm_add(fmm_add(m9, m10), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(m9, m10));
    if (kBeta) st(11, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m4), m10), m14), fmm_mul(beta, ldc(11)))); else st(11, fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m4), m10), m14));
  }
};

// grey324_20_144  <3,2,4; 20>  (reference header algorithms/fast324_20_144.hpp, coefficients codegen/algorithms/grey324-20-144)
struct FmmAlg_grey324_20_144 {
  static constexpr int kM0 = 3, kK0 = 2, kN0 = 4, kR = 20;
  static constexpr int kNumAOut = 16, kNumBOut = 15;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    st(0, fmm_add(fmm_neg(a0), a2));  // operand of M1
    st(1, fmm_add(fmm_neg(a3), a5));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_neg(a2), a3), a4));  // operand of M4
    st(3, fmm_sub(fmm_add(fmm_add(fmm_neg(a2), a3), a4), a5));  // operand of M5
    st(4, fmm_add(a0, a3));  // operand of M6
    st(5, fmm_add(fmm_sub(a1, a3), a5));  // operand of M7
    st(6, fmm_add(fmm_neg(a2), a4));  // operand of M8
    st(7, fmm_add(fmm_neg(a0), a1));  // operand of M9
    st(8, fmm_add(fmm_neg(a2), a3));  // operand of M11
    st(9, fmm_add(fmm_sub(fmm_add(fmm_neg(a0), a1), a3), a5));  // operand of M12
    st(10, fmm_add(a1, a3));  // operand of M13
    st(11, fmm_sub(fmm_neg(a0), a2));  // operand of M16
    st(12, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a1), a2), a3), a4), a5));  // operand of M17
    st(13, fmm_sub(fmm_add(fmm_sub(fmm_sub(a0, a1), a2), a3), a5));  // operand of M18
    st(14, fmm_add(fmm_neg(a2), a4));  // operand of M19
    st(15, fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a1), a2), a3));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    st(0, fmm_sub(fmm_sub(fmm_sub(fmm_neg(b0), b1), b4), b5));  // operand of M1
    st(1, fmm_sub(fmm_neg(b5), b6));  // operand of M2
    st(2, fmm_sub(fmm_sub(fmm_neg(b3), b4), b7));  // operand of M4
    st(3, fmm_add(b4, b7));  // operand of M5
    st(4, fmm_add(fmm_neg(b3), b6));  // operand of M6
    st(5, fmm_sub(fmm_neg(b1), b5));  // operand of M7
    st(6, fmm_add(b1, b2));  // operand of M8
    st(7, fmm_add(b3, b7));  // operand of M10
    st(8, fmm_sub(b1, b6));  // operand of M12
    st(9, fmm_add(b6, b7));  // operand of M13
    st(10, fmm_add(b2, b6));  // operand of M14
    st(11, fmm_sub(fmm_neg(b2), b3));  // operand of M16
    st(12, fmm_add(fmm_add(b1, b4), b5));  // operand of M18
    st(13, fmm_sub(fmm_sub(fmm_sub(fmm_neg(b0), b3), b4), b7));  // operand of M19
    st(14, fmm_sub(fmm_neg(b4), b5));  // operand of M20
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(m0, m2), m3), m6), m9), m14), m17), m18), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(m0, m2), m3), m6), m9), m14), m17), m18));
    if (kBeta) st(1, fmm_add(fmm_sub(fmm_add(fmm_sub(m1, m6), m8), m11), fmm_mul(beta, ldc(1)))); else st(1, fmm_sub(fmm_add(fmm_sub(m1, m6), m8), m11));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_neg(m8), m13), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_neg(m8), m13));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m5), m8), m9), m12), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(fmm_add(fmm_neg(m5), m8), m9), m12));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_sub(fmm_sub(m2, m3), m9), m18), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_sub(fmm_sub(m2, m3), m9), m18));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m1, m8), m11), m14), m17), m19), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m1, m8), m11), m14), m17), m19));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_sub(m5, m10), m13), m15), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_sub(m5, m10), m13), m15));
    if (kBeta) st(7, fmm_add(fmm_add(m9, m10), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(m9, m10));
    if (kBeta) st(8, fmm_add(fmm_add(m2, m14), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(m2, m14));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(m14), m16), m17), m19), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_sub(fmm_sub(fmm_neg(m14), m16), m17), m19));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(m5, m7), m8), m10), m11), m13), m15), m16), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(m5, m7), m8), m10), m11), m13), m15), m16));
    if (kBeta) st(11, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m4), m10), m14), fmm_mul(beta, ldc(11)))); else st(11, fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m4), m10), m14));
  }
};

// grey342_20_144  <3,4,2; 20>  (reference header algorithms/fast342_20_144.hpp, coefficients codegen/algorithms/grey342-20-144)
struct FmmAlg_grey342_20_144 {
  static constexpr int kM0 = 3, kK0 = 4, kN0 = 2, kR = 20;
  static constexpr int kNumAOut = 16, kNumBOut = 15;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    const T a10 = ld(10);
    const T a11 = ld(11);
    st(0, fmm_add(a1, a5));  // operand of M2
    st(1, fmm_add(fmm_add(a0, a4), a8));  // operand of M3
    st(2, fmm_sub(fmm_sub(fmm_neg(a0), a4), a11));  // operand of M4
    st(3, fmm_add(fmm_add(fmm_neg(a3), a6), a10));  // operand of M6
    st(4, fmm_sub(a0, a1));  // operand of M7
    st(5, fmm_add(fmm_add(fmm_add(fmm_sub(a1, a2), a3), a5), a10));  // operand of M9
    st(6, fmm_add(fmm_sub(fmm_sub(fmm_neg(a0), a3), a4), a7));  // operand of M10
    st(7, fmm_add(fmm_sub(fmm_add(fmm_neg(a6), a7), a10), a11));  // operand of M11
    st(8, fmm_sub(fmm_sub(fmm_neg(a1), a5), a10));  // operand of M12
    st(9, fmm_add(fmm_add(fmm_neg(a2), a6), a10));  // operand of M14
    st(10, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_neg(a0), a5), a8), a9), a11));  // operand of M15
    st(11, fmm_add(a6, a10));  // operand of M16
    st(12, fmm_add(fmm_neg(a9), a10));  // operand of M17
    st(13, fmm_sub(fmm_sub(fmm_neg(a0), a5), a9));  // operand of M18
    st(14, fmm_add(a0, a4));  // operand of M19
    st(15, fmm_add(a5, a9));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    st(0, fmm_sub(fmm_sub(fmm_sub(fmm_neg(b0), b1), b2), b3));  // operand of M1
    st(1, fmm_sub(fmm_neg(b3), b5));  // operand of M2
    st(2, fmm_sub(fmm_sub(fmm_neg(b1), b6), b7));  // operand of M4
    st(3, fmm_add(b1, b7));  // operand of M5
    st(4, fmm_sub(b5, b6));  // operand of M6
    st(5, fmm_sub(fmm_neg(b2), b3));  // operand of M7
    st(6, fmm_add(b2, b4));  // operand of M8
    st(7, fmm_add(b6, b7));  // operand of M10
    st(8, fmm_sub(b2, b5));  // operand of M12
    st(9, fmm_add(b5, b7));  // operand of M13
    st(10, fmm_add(b4, b5));  // operand of M14
    st(11, fmm_sub(fmm_neg(b4), b6));  // operand of M16
    st(12, fmm_add(fmm_add(b1, b2), b3));  // operand of M18
    st(13, fmm_sub(fmm_sub(fmm_sub(fmm_neg(b0), b1), b6), b7));  // operand of M19
    st(14, fmm_sub(fmm_neg(b1), b3));  // operand of M20
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_neg(m0), m5), m8), m11), m13), m15), m16), m17), m19), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_neg(m0), m5), m8), m11), m13), m15), m16), m17), m19));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m6, m8), m11), m12), m16), m17), m19), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m6, m8), m11), m12), m16), m17), m19));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m0, m3), m4), m7), m10), m15), m16), m17), m18), m19), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m0, m3), m4), m7), m10), m15), m16), m17), m18), m19));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m1), m3), m4), m5), m6), m9), m10), m11), m12), m16), m17), m19), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m1), m3), m4), m5), m6), m9), m10), m11), m12), m16), m17), m19));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m2), m3), m4), m7), m16), m18), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m2), m3), m4), m7), m16), m18));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m1, m4), m6), m11), m14), m16), m17), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m1, m4), m6), m11), m14), m16), m17));
  }
};

// grey234_20_144  <2,3,4; 20>  (reference header algorithms/fast234_20_144.hpp, coefficients codegen/algorithms/grey234-20-144)
struct FmmAlg_grey234_20_144 {
  static constexpr int kM0 = 2, kK0 = 3, kN0 = 4, kR = 20;
  static constexpr int kNumAOut = 16, kNumBOut = 16;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    st(0, fmm_add(fmm_neg(a0), a1));  // operand of M1
    st(1, fmm_add(fmm_neg(a4), a5));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_neg(a1), a2), a4));  // operand of M4
    st(3, fmm_sub(fmm_add(fmm_add(fmm_neg(a1), a2), a4), a5));  // operand of M5
    st(4, fmm_add(a0, a4));  // operand of M6
    st(5, fmm_add(fmm_sub(a3, a4), a5));  // operand of M7
    st(6, fmm_add(fmm_neg(a1), a2));  // operand of M8
    st(7, fmm_add(fmm_neg(a0), a3));  // operand of M9
    st(8, fmm_add(fmm_neg(a1), a4));  // operand of M11
    st(9, fmm_add(fmm_sub(fmm_add(fmm_neg(a0), a3), a4), a5));  // operand of M12
    st(10, fmm_add(a3, a4));  // operand of M13
    st(11, fmm_sub(fmm_neg(a0), a1));  // operand of M16
    st(12, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(a0), a1), a2), a3), a4), a5));  // operand of M17
    st(13, fmm_sub(fmm_add(fmm_sub(fmm_sub(a0, a1), a3), a4), a5));  // operand of M18
    st(14, fmm_add(fmm_neg(a1), a2));  // operand of M19
    st(15, fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a1), a3), a4));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T b9 = ld(9);
    const T b10 = ld(10);
    const T b11 = ld(11);
    st(0, fmm_add(b1, b5));  // operand of M2
    st(1, fmm_add(fmm_add(b0, b4), b8));  // operand of M3
    st(2, fmm_sub(fmm_sub(fmm_neg(b0), b4), b11));  // operand of M4
    st(3, fmm_add(fmm_add(fmm_neg(b3), b6), b10));  // operand of M6
    st(4, fmm_sub(b0, b1));  // operand of M7
    st(5, fmm_add(fmm_add(fmm_add(fmm_sub(b1, b2), b3), b5), b10));  // operand of M9
    st(6, fmm_add(fmm_sub(fmm_sub(fmm_neg(b0), b3), b4), b7));  // operand of M10
    st(7, fmm_add(fmm_sub(fmm_add(fmm_neg(b6), b7), b10), b11));  // operand of M11
    st(8, fmm_sub(fmm_sub(fmm_neg(b1), b5), b10));  // operand of M12
    st(9, fmm_add(fmm_add(fmm_neg(b2), b6), b10));  // operand of M14
    st(10, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_neg(b0), b5), b8), b9), b11));  // operand of M15
    st(11, fmm_add(b6, b10));  // operand of M16
    st(12, fmm_add(fmm_neg(b9), b10));  // operand of M17
    st(13, fmm_sub(fmm_sub(fmm_neg(b0), b5), b9));  // operand of M18
    st(14, fmm_add(b0, b4));  // operand of M19
    st(15, fmm_add(b5, b9));  // operand of M20
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_sub(fmm_neg(m0), m2), m18), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_sub(fmm_neg(m0), m2), m18));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m6), m7), m11), m16), m17), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m6), m7), m11), m16), m17));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_add(m7, m13), m15), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_add(m7, m13), m15));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m5), m9), m10), m15), m18), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m5), m9), m10), m15), m18));
    if (kBeta) st(4, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m3), m4), m14), m17), m18), m19), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m3), m4), m14), m17), m18), m19));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_neg(m0), m1), m6), m17), m19), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_neg(m0), m1), m6), m17), m19));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_neg(m1), m5), m8), m11), m12), m13), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_neg(m1), m5), m8), m11), m12), m13));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m3), m4), m9), m12), m18), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m3), m4), m9), m12), m18));
  }
};

// grey243_20_144  <2,4,3; 20>  (reference header algorithms/fast243_20_144.hpp, coefficients codegen/algorithms/grey243-20-144)
struct FmmAlg_grey243_20_144 {
  static constexpr int kM0 = 2, kK0 = 4, kN0 = 3, kR = 20;
  static constexpr int kNumAOut = 15, kNumBOut = 16;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    st(0, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a0), a1), a4), a5));  // operand of M1
    st(1, fmm_sub(fmm_neg(a5), a6));  // operand of M2
    st(2, fmm_sub(fmm_sub(fmm_neg(a3), a4), a7));  // operand of M4
    st(3, fmm_add(a4, a7));  // operand of M5
    st(4, fmm_add(fmm_neg(a3), a6));  // operand of M6
    st(5, fmm_sub(fmm_neg(a1), a5));  // operand of M7
    st(6, fmm_add(a1, a2));  // operand of M8
    st(7, fmm_add(a3, a7));  // operand of M10
    st(8, fmm_sub(a1, a6));  // operand of M12
    st(9, fmm_add(a6, a7));  // operand of M13
    st(10, fmm_add(a2, a6));  // operand of M14
    st(11, fmm_sub(fmm_neg(a2), a3));  // operand of M16
    st(12, fmm_add(fmm_add(a1, a4), a5));  // operand of M18
    st(13, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a0), a3), a4), a7));  // operand of M19
    st(14, fmm_sub(fmm_neg(a4), a5));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T b9 = ld(9);
    const T b10 = ld(10);
    const T b11 = ld(11);
    st(0, fmm_add(b3, b4));  // operand of M2
    st(1, fmm_add(fmm_add(b0, b1), b2));  // operand of M3
    st(2, fmm_sub(fmm_sub(fmm_neg(b0), b1), b11));  // operand of M4
    st(3, fmm_sub(fmm_add(b7, b8), b9));  // operand of M6
    st(4, fmm_sub(b0, b3));  // operand of M7
    st(5, fmm_add(fmm_add(fmm_sub(fmm_add(b3, b4), b6), b8), b9));  // operand of M9
    st(6, fmm_add(fmm_sub(fmm_sub(fmm_neg(b0), b1), b9), b10));  // operand of M10
    st(7, fmm_add(fmm_add(fmm_sub(fmm_neg(b7), b8), b10), b11));  // operand of M11
    st(8, fmm_sub(fmm_sub(fmm_neg(b3), b4), b8));  // operand of M12
    st(9, fmm_add(fmm_add(fmm_neg(b6), b7), b8));  // operand of M14
    st(10, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_neg(b0), b2), b4), b5), b11));  // operand of M15
    st(11, fmm_add(b7, b8));  // operand of M16
    st(12, fmm_add(fmm_neg(b5), b8));  // operand of M17
    st(13, fmm_sub(fmm_sub(fmm_neg(b0), b4), b5));  // operand of M18
    st(14, fmm_add(b0, b1));  // operand of M19
    st(15, fmm_add(b4, b5));  // operand of M20
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_neg(m0), m5), m8), m11), m13), m15), m16), m17), m19), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_neg(m0), m5), m8), m11), m13), m15), m16), m17), m19));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m0, m3), m4), m7), m10), m15), m16), m17), m18), m19), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m0, m3), m4), m7), m10), m15), m16), m17), m18), m19));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m2), m3), m4), m7), m16), m18), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m2), m3), m4), m7), m16), m18));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m6, m8), m11), m12), m16), m17), m19), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m6, m8), m11), m12), m16), m17), m19));
    if (kBeta) st(4, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m1), m3), m4), m5), m6), m9), m10), m11), m12), m16), m17), m19), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m1), m3), m4), m5), m6), m9), m10), m11), m12), m16), m17), m19));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m1, m4), m6), m11), m14), m16), m17), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m1, m4), m6), m11), m14), m16), m17));
  }
};

// classical423_24_72  <4,2,3; 24>  (reference header algorithms/classical423.hpp, coefficients codegen/algorithms/classical423-24-72)
struct FmmAlg_classical423_24_72 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 3, kR = 24;
  static constexpr int kNumAOut = 0, kNumBOut = 0;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    if (kBeta) st(0, fmm_add(fmm_add(m0, m1), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(m0, m1));
    if (kBeta) st(1, fmm_add(fmm_add(m8, m9), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(m8, m9));
    if (kBeta) st(2, fmm_add(fmm_add(m16, m17), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(m16, m17));
    if (kBeta) st(3, fmm_add(fmm_add(m2, m3), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(m2, m3));
    if (kBeta) st(4, fmm_add(fmm_add(m10, m11), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(m10, m11));
    if (kBeta) st(5, fmm_add(fmm_add(m18, m19), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(m18, m19));
    if (kBeta) st(6, fmm_add(fmm_add(m4, m5), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(m4, m5));
    if (kBeta) st(7, fmm_add(fmm_add(m12, m13), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(m12, m13));
    if (kBeta) st(8, fmm_add(fmm_add(m20, m21), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(m20, m21));
    if (kBeta) st(9, fmm_add(fmm_add(m6, m7), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(m6, m7));
    if (kBeta) st(10, fmm_add(fmm_add(m14, m15), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(m14, m15));
    if (kBeta) st(11, fmm_add(fmm_add(m22, m23), fmm_mul(beta, ldc(11)))); else st(11, fmm_add(m22, m23));
  }
};

// fast423_130  <4,2,3; 20>  (reference header algorithms/fast423_20_130.hpp, coefficients codegen/algorithms/fast423-130)
struct FmmAlg_fast423_130 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 3, kR = 20;
  static constexpr int kNumAOut = 16, kNumBOut = 14;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    st(0, fmm_sub(fmm_neg(a4), a5));  // operand of M1
    st(1, fmm_sub(fmm_neg(a4), a6));  // operand of M2
    st(2, fmm_sub(a3, a6));  // operand of M3
    st(3, fmm_add(fmm_neg(a0), a5));  // operand of M5
    st(4, fmm_add(a2, a6));  // operand of M6
    st(5, fmm_add(a0, a1));  // operand of M7
    st(6, fmm_add(a1, a5));  // operand of M9
    st(7, fmm_add(a2, a3));  // operand of M10
    st(8, fmm_add(a5, a7));  // operand of M11
    st(9, fmm_add(fmm_neg(a0), a3));  // operand of M12
    st(10, fmm_add(fmm_neg(a5), a6));  // operand of M13
    st(11, fmm_add(a6, a7));  // operand of M14
    st(12, fmm_add(a1, a3));  // operand of M16
    st(13, fmm_sub(fmm_neg(a3), a7));  // operand of M17
    st(14, fmm_add(a0, a4));  // operand of M18
    st(15, fmm_add(a0, a2));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_sub(fmm_sub(fmm_add(fmm_neg(b1), b2), b3), b5));  // operand of M3
    st(1, fmm_add(fmm_neg(b1), b4));  // operand of M4
    st(2, fmm_add(b0, b4));  // operand of M5
    st(3, fmm_add(b0, b1));  // operand of M6
    st(4, fmm_sub(fmm_sub(fmm_add(b0, b2), b3), b5));  // operand of M8
    st(5, fmm_add(b3, b4));  // operand of M9
    st(6, fmm_add(fmm_neg(b1), b2));  // operand of M10
    st(7, fmm_add(fmm_add(fmm_neg(b1), b2), b4));  // operand of M12
    st(8, fmm_sub(fmm_sub(b0, b3), b5));  // operand of M13
    st(9, fmm_add(b3, b5));  // operand of M14
    st(10, fmm_sub(b0, b3));  // operand of M15
    st(11, fmm_sub(fmm_neg(b3), b4));  // operand of M17
    st(12, fmm_add(b0, b1));  // operand of M18
    st(13, fmm_sub(fmm_add(fmm_add(fmm_neg(b1), b2), b4), b5));  // operand of M19
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m4), m6), m8), m14), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_sub(fmm_neg(m4), m6), m8), m14));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_neg(m3), m6), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_neg(m3), m6));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m11), m15), m18), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_add(fmm_sub(fmm_neg(m3), m11), m15), m18));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m2), m3), m5), m7), m9), m11), m18), m19), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m2), m3), m5), m7), m9), m11), m18), m19));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_sub(m3, m9), m11), m19), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_sub(m3, m9), m11), m19));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(m3, m11), m18), m19), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(m3, m11), m18), m19));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_neg(m0), m14), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_neg(m0), m14));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_add(m0, m3), m4), m17), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_add(m0, m3), m4), m17));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_sub(m1, m7), m12), m14), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_sub(m1, m7), m12), m14));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m10), m12), m13), m14), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_add(fmm_add(fmm_neg(m10), m12), m13), m14));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(m2, m7), m10), m12), m13), m14), m16), m18), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(m2, m7), m10), m12), m13), m14), m16), m18));
    if (kBeta) st(11, fmm_add(fmm_sub(fmm_sub(fmm_add(m7, m10), m12), m14), fmm_mul(beta, ldc(11)))); else st(11, fmm_sub(fmm_sub(fmm_add(m7, m10), m12), m14));
  }
};

// fast423_134  <4,2,3; 20>  (reference header algorithms/fast423_20_134.hpp, coefficients codegen/algorithms/fast423-134)
struct FmmAlg_fast423_134 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 3, kR = 20;
  static constexpr int kNumAOut = 16, kNumBOut = 14;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    st(0, fmm_sub(a3, a5));  // operand of M1
    st(1, fmm_sub(a4, a5));  // operand of M2
    st(2, fmm_sub(a0, a1));  // operand of M3
    st(3, fmm_add(fmm_neg(a2), a7));  // operand of M4
    st(4, fmm_sub(a2, a4));  // operand of M5
    st(5, fmm_add(fmm_neg(a3), a7));  // operand of M6
    st(6, fmm_add(a0, a5));  // operand of M7
    st(7, fmm_add(a1, a5));  // operand of M8
    st(8, fmm_add(a0, a6));  // operand of M9
    st(9, fmm_add(fmm_neg(a2), a3));  // operand of M10
    st(10, fmm_sub(a2, a6));  // operand of M13
    st(11, fmm_add(a0, a4));  // operand of M14
    st(12, fmm_sub(a2, a5));  // operand of M16
    st(13, fmm_sub(fmm_neg(a1), a7));  // operand of M18
    st(14, fmm_add(a0, a7));  // operand of M19
    st(15, fmm_sub(a6, a7));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_add(fmm_sub(fmm_neg(b3), b4), b5));  // operand of M1
    st(1, fmm_add(b3, b5));  // operand of M3
    st(2, fmm_sub(fmm_sub(fmm_neg(b1), b3), b4));  // operand of M4
    st(3, fmm_add(fmm_sub(fmm_neg(b0), b1), b2));  // operand of M5
    st(4, fmm_add(fmm_add(b2, b3), b5));  // operand of M7
    st(5, fmm_add(fmm_sub(b0, b1), b2));  // operand of M9
    st(6, fmm_add(b3, b4));  // operand of M10
    st(7, fmm_add(fmm_add(fmm_add(b0, b2), b3), b5));  // operand of M11
    st(8, fmm_add(b1, b4));  // operand of M12
    st(9, fmm_add(b2, b5));  // operand of M15
    st(10, fmm_add(fmm_add(b2, b3), b4));  // operand of M16
    st(11, fmm_add(fmm_add(fmm_add(b0, b1), b3), b4));  // operand of M17
    st(12, fmm_sub(fmm_add(fmm_neg(b3), b4), b5));  // operand of M18
    st(13, fmm_add(fmm_add(b1, b3), b5));  // operand of M19
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(m6), m7), m10), m14), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_sub(fmm_sub(fmm_neg(m6), m7), m10), m14));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(m2), m11), m17), m18), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_sub(fmm_sub(fmm_neg(m2), m11), m17), m18));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m2), m6), m7), m14), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_add(fmm_add(fmm_neg(m2), m6), m7), m14));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(m3), m5), m11), m16), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(fmm_sub(fmm_neg(m3), m5), m11), m16));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(m3, m5), m9), m11), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(m3, m5), m9), m11));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(m0, m9), m14), m15), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(m0, m9), m14), m15));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_add(fmm_add(m6, m10), m13), m14), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_add(fmm_add(m6, m10), m13), m14));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m1, m4), m6), m10), m13), m14), m15), m16), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m1, m4), m6), m10), m13), m14), m15), m16));
    if (kBeta) st(8, fmm_add(fmm_add(m1, m14), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(m1, m14));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(m3), m11), m12), m16), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_sub(fmm_sub(fmm_neg(m3), m11), m12), m16));
    if (kBeta) st(10, fmm_add(fmm_add(m11, m19), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(m11, m19));
    if (kBeta) st(11, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m3, m8), m10), m11), m12), m16), m18), m19), fmm_mul(beta, ldc(11)))); else st(11, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(m3, m8), m10), m11), m12), m16), m18), m19));
  }
};

// fast423_138  <4,2,3; 20>  (reference header algorithms/fast423_20_138.hpp, coefficients codegen/algorithms/fast423-138)
struct FmmAlg_fast423_138 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 3, kR = 20;
  static constexpr int kNumAOut = 14, kNumBOut = 14;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    st(0, fmm_sub(fmm_neg(a0), a4));  // operand of M1
    st(1, fmm_add(fmm_sub(fmm_sub(a0, a1), a2), a3));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_neg(a5), a6), a7));  // operand of M3
    st(3, fmm_sub(fmm_sub(fmm_add(a4, a5), a6), a7));  // operand of M4
    st(4, fmm_add(a6, a7));  // operand of M5
    st(5, fmm_sub(a0, a2));  // operand of M9
    st(6, fmm_add(fmm_neg(a5), a7));  // operand of M10
    st(7, fmm_sub(fmm_sub(a0, a1), a2));  // operand of M11
    st(8, fmm_sub(a3, a7));  // operand of M12
    st(9, fmm_add(fmm_sub(a0, a1), a4));  // operand of M13
    st(10, fmm_add(fmm_add(fmm_neg(a3), a6), a7));  // operand of M14
    st(11, fmm_sub(fmm_sub(fmm_add(a2, a3), a6), a7));  // operand of M16
    st(12, fmm_add(fmm_neg(a0), a1));  // operand of M17
    st(13, fmm_sub(fmm_add(fmm_sub(a0, a1), a4), a5));  // operand of M19
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_sub(fmm_neg(b1), b4));  // operand of M1
    st(1, fmm_add(fmm_sub(b2, b3), b4));  // operand of M3
    st(2, fmm_add(fmm_neg(b3), b4));  // operand of M5
    st(3, fmm_sub(fmm_add(fmm_sub(b0, b2), b3), b5));  // operand of M6
    st(4, fmm_add(fmm_sub(fmm_sub(b0, b1), b3), b4));  // operand of M8
    st(5, fmm_add(b2, b5));  // operand of M9
    st(6, fmm_add(fmm_neg(b2), b5));  // operand of M10
    st(7, fmm_sub(fmm_sub(b0, b2), b5));  // operand of M11
    st(8, fmm_add(fmm_neg(b1), b4));  // operand of M12
    st(9, fmm_add(fmm_sub(b0, b2), b4));  // operand of M13
    st(10, fmm_sub(fmm_add(b1, b3), b4));  // operand of M14
    st(11, fmm_add(fmm_add(fmm_neg(b0), b1), b2));  // operand of M15
    st(12, fmm_sub(b0, b2));  // operand of M17
    st(13, fmm_add(fmm_add(fmm_neg(b3), b4), b5));  // operand of M18
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_add(m5, m6), m8), m10), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_add(m5, m6), m8), m10));
    if (kBeta) st(1, fmm_add(fmm_sub(fmm_sub(fmm_sub(m0, m12), m14), m16), fmm_mul(beta, ldc(1)))); else st(1, fmm_sub(fmm_sub(fmm_sub(m0, m12), m14), m16));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(m6, m8), m10), m16), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(m6, m8), m10), m16));
    if (kBeta) st(3, fmm_add(fmm_add(m6, m19), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(m6, m19));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(m4, m13), m15), m19), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(m4, m13), m15), m19));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(m1, m6), m10), m16), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(m1, m6), m10), m16));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m2, m3), m4), m12), m16), m18), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m2, m3), m4), m12), m16), m18));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_add(m12, m14), m16), m18), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_add(m12, m14), m16), m18));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_sub(fmm_add(m2, m3), m4), m17), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_sub(fmm_add(m2, m3), m4), m17));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m7), m11), m13), m19), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_add(fmm_sub(fmm_neg(m7), m11), m13), m19));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_sub(m4, m11), m13), m19), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_sub(m4, m11), m13), m19));
    if (kBeta) st(11, fmm_add(fmm_add(fmm_add(fmm_sub(m2, m4), m9), m17), fmm_mul(beta, ldc(11)))); else st(11, fmm_add(fmm_add(fmm_sub(m2, m4), m9), m17));
  }
};

// fast423_156  <4,2,3; 20>  (reference header algorithms/fast423_20_156.hpp, coefficients codegen/algorithms/fast423-156)
struct FmmAlg_fast423_156 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 3, kR = 20;
  static constexpr int kNumAOut = 13, kNumBOut = 11;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    st(0, fmm_sub(fmm_sub(a1, a3), a5));  // operand of M4
    st(1, fmm_sub(fmm_add(fmm_add(fmm_neg(a2), a3), a6), a7));  // operand of M5
    st(2, fmm_add(fmm_neg(a2), a3));  // operand of M6
    st(3, fmm_sub(a3, a7));  // operand of M7
    st(4, fmm_add(a2, a5));  // operand of M8
    st(5, fmm_sub(a4, a5));  // operand of M9
    st(6, fmm_add(fmm_sub(a2, a3), a7));  // operand of M10
    st(7, fmm_sub(fmm_add(fmm_sub(a0, a4), a5), a6));  // operand of M13
    st(8, fmm_add(fmm_add(fmm_neg(a0), a4), a6));  // operand of M15
    st(9, fmm_sub(fmm_neg(a2), a4));  // operand of M17
    st(10, fmm_sub(a1, a7));  // operand of M18
    st(11, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(a0, a1), a4), a5), a6), a7));  // operand of M19
    st(12, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(a0), a3), a4), a6), a7));  // operand of M20
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    st(0, fmm_add(b0, b2));  // operand of M5
    st(1, fmm_add(fmm_add(fmm_add(b0, b2), b3), b5));  // operand of M7
    st(2, fmm_add(fmm_add(b0, b1), b3));  // operand of M8
    st(3, fmm_add(b0, b1));  // operand of M9
    st(4, fmm_add(fmm_add(b0, b2), b3));  // operand of M10
    st(5, fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), b3), b4), b5));  // operand of M13
    st(6, fmm_add(b0, b3));  // operand of M14
    st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), b2), b3), b4), b5));  // operand of M15
    st(8, fmm_add(fmm_add(fmm_add(b0, b1), b3), b4));  // operand of M16
    st(9, fmm_sub(fmm_sub(fmm_neg(b3), b4), b5));  // operand of M19
    st(10, fmm_add(fmm_add(fmm_add(fmm_add(b0, b2), b3), b4), b5));  // operand of M20
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m0, m3), m4), m5), m6), m7), m8), m9), m12), m13), m14), m15), m16), m17), m18), m19), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m0, m3), m4), m5), m6), m7), m8), m9), m12), m13), m14), m15), m16), m17), m18), m19));
    if (kBeta) st(1, fmm_add(fmm_add(m1, m10), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(m1, m10));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(m2, m11), m17), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(m2, m11), m17));
    if (kBeta) st(3, fmm_add(fmm_sub(m5, m13), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(m5, m13));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m3, m7), m10), m13), m15), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_add(m3, m7), m10), m13), m15));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(m6, m9), m11), m13), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(m6, m9), m11), m13));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(m7, m8), m13), m16), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(m7, m8), m13), m16));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m7), m13), m15), m16), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_sub(fmm_sub(fmm_neg(m7), m13), m15), m16));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m0, m2), m12), m14), m15), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_add(fmm_add(m0, m2), m12), m14), m15));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_add(fmm_add(m0, m4), m5), m9), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_add(fmm_add(m0, m4), m5), m9));
    if (kBeta) st(10, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m1, m3), m6), m7), m10), m13), m14), m15), m16), m19), fmm_mul(beta, ldc(10)))); else st(10, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m1, m3), m6), m7), m10), m13), m14), m15), m16), m19));
    if (kBeta) st(11, fmm_add(fmm_add(fmm_neg(m0), m11), fmm_mul(beta, ldc(11)))); else st(11, fmm_add(fmm_neg(m0), m11));
  }
};

// grey433_29_234  <4,3,3; 29>  (reference header algorithms/fast433_29_234.hpp, coefficients codegen/algorithms/grey433-29-234)
struct FmmAlg_grey433_29_234 {
  static constexpr int kM0 = 4, kK0 = 3, kN0 = 3, kR = 29;
  static constexpr int kNumAOut = 21, kNumBOut = 24;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    const T a10 = ld(10);
    const T a11 = ld(11);
    st(0, fmm_add(a5, a8));  // operand of M3
    st(1, fmm_sub(fmm_sub(fmm_neg(a5), a8), a9));  // operand of M6
    st(2, fmm_add(fmm_add(fmm_neg(a2), a8), a11));  // operand of M7
    st(3, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(a0), a1), a2), a6), a7), a8), a9), a10), a11));  // operand of M8
    st(4, fmm_add(a4, a7));  // operand of M9
    st(5, fmm_add(fmm_add(fmm_neg(a3), a4), a10));  // operand of M10
    st(6, fmm_sub(fmm_sub(fmm_sub(a2, a8), a10), a11));  // operand of M11
    st(7, fmm_add(fmm_add(fmm_neg(a0), a5), a8));  // operand of M12
    st(8, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(a0), a4), a6), a7), a9));  // operand of M13
    st(9, fmm_add(fmm_neg(a2), a8));  // operand of M14
    st(10, fmm_sub(fmm_sub(a3, a4), a7));  // operand of M16
    st(11, fmm_sub(fmm_add(fmm_neg(a5), a9), a11));  // operand of M18
    st(12, fmm_sub(fmm_neg(a1), a4));  // operand of M19
    st(13, fmm_sub(fmm_sub(a0, a6), a9));  // operand of M20
    st(14, fmm_sub(a1, a5));  // operand of M21
    st(15, fmm_add(fmm_add(fmm_add(a5, a8), a10), a11));  // operand of M22
    st(16, fmm_add(fmm_sub(a5, a6), a8));  // operand of M24
    st(17, fmm_sub(fmm_sub(a0, a1), a2));  // operand of M26
    st(18, fmm_add(fmm_sub(fmm_add(fmm_sub(a3, a4), a6), a7), a9));  // operand of M27
    st(19, fmm_add(fmm_neg(a5), a7));  // operand of M28
    st(20, fmm_sub(a5, a10));  // operand of M29
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    st(0, fmm_add(b0, b6));  // operand of M1
    st(1, fmm_add(fmm_sub(fmm_add(fmm_neg(b1), b2), b4), b5));  // operand of M2
    st(2, fmm_sub(fmm_neg(b2), b8));  // operand of M3
    st(3, fmm_add(fmm_neg(b0), b2));  // operand of M4
    st(4, fmm_sub(b3, b6));  // operand of M5
    st(5, fmm_add(fmm_sub(b2, b7), b8));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(b3, b4), b5), b6), b7), b8));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_neg(b3), b4), b5));  // operand of M8
    st(8, fmm_add(b1, b4));  // operand of M9
    st(9, fmm_add(fmm_neg(b4), b5));  // operand of M10
    st(10, fmm_add(fmm_sub(fmm_sub(b3, b4), b5), b7));  // operand of M11
    st(11, fmm_add(b2, b6));  // operand of M12
    st(12, fmm_add(fmm_add(fmm_sub(b1, b3), b4), b5));  // operand of M13
    st(13, fmm_sub(b6, b8));  // operand of M14
    st(14, fmm_sub(b0, b2));  // operand of M15
    st(15, fmm_add(fmm_sub(fmm_neg(b1), b4), b5));  // operand of M16
    st(16, fmm_sub(b5, b8));  // operand of M17
    st(17, fmm_sub(b7, b8));  // operand of M18
    st(18, fmm_add(fmm_neg(b3), b5));  // operand of M19
    st(19, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b1), b2), b3), b4), b5));  // operand of M20
    st(20, fmm_sub(b5, b6));  // operand of M21
    st(21, fmm_sub(b4, b7));  // operand of M23
    st(22, fmm_add(fmm_sub(fmm_add(fmm_neg(b1), b2), b7), b8));  // operand of M25
    st(23, fmm_sub(b5, b7));  // operand of M29
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T m26 = ld(26);
    const T m27 = ld(27);
    const T m28 = ld(28);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_sub(m0, m4), m25), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_sub(m0, m4), m25));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m7, m8), m9), m10), m12), m15), m18), m21), m22), m26), m27), m28), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m7, m8), m9), m10), m12), m15), m18), m21), m22), m26), m27), m28));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m2), m11), m13), m16), m20), m25), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(m2), m11), m13), m16), m20), m25));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m1, m4), m8), m14), m15), m18), m20), m27), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m1, m4), m8), m14), m15), m18), m20), m27));
    if (kBeta) st(4, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m8, m9), m15), m22), m27), m28), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m8, m9), m15), m22), m27), m28));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(m1, m8), m15), m16), m27), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_sub(fmm_sub(fmm_add(m1, m8), m15), m16), m27));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m0, m3), m4), m8), m11), m12), m18), m19), m20), m23), m27), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m0, m3), m4), m8), m11), m12), m18), m19), m20), m23), m27));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m2), m5), m9), m15), m22), m24), m26), m27), m28), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m2), m5), m9), m15), m22), m24), m26), m27), m28));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m2), m16), m23), m27), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_sub(fmm_add(fmm_neg(m2), m16), m23), m27));
    if (kBeta) st(9, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m2, m3), m5), m6), m10), m13), m16), m17), m21), m22), m28), fmm_mul(beta, ldc(9)))); else st(9, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m2, m3), m5), m6), m10), m13), m16), m17), m21), m22), m28));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m2, m5), m21), m22), m24), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_add(fmm_sub(m2, m5), m21), m22), m24));
    if (kBeta) st(11, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(m2, m5), m16), m17), m21), m28), fmm_mul(beta, ldc(11)))); else st(11, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(m2, m5), m16), m17), m21), m28));
  }
};

// grey343_29_234  <3,4,3; 29>  (reference header algorithms/fast343_29_234.hpp, coefficients codegen/algorithms/grey343-29-234)
struct FmmAlg_grey343_29_234 {
  static constexpr int kM0 = 3, kK0 = 4, kN0 = 3, kR = 29;
  static constexpr int kNumAOut = 21, kNumBOut = 25;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    const T a10 = ld(10);
    const T a11 = ld(11);
    st(0, fmm_add(a9, a10));  // operand of M3
    st(1, fmm_sub(fmm_sub(fmm_neg(a3), a9), a10));  // operand of M6
    st(2, fmm_add(fmm_add(fmm_neg(a8), a10), a11));  // operand of M7
    st(3, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(a0), a2), a3), a4), a6), a7), a8), a10), a11));  // operand of M8
    st(4, fmm_add(a5, a6));  // operand of M9
    st(5, fmm_add(fmm_add(fmm_neg(a1), a5), a7));  // operand of M10
    st(6, fmm_sub(fmm_sub(fmm_add(fmm_neg(a7), a8), a10), a11));  // operand of M11
    st(7, fmm_add(fmm_add(fmm_neg(a0), a9), a10));  // operand of M12
    st(8, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a2), a3), a5), a6));  // operand of M13
    st(9, fmm_add(fmm_neg(a8), a10));  // operand of M14
    st(10, fmm_sub(fmm_sub(a1, a5), a6));  // operand of M16
    st(11, fmm_sub(fmm_sub(a3, a9), a11));  // operand of M18
    st(12, fmm_sub(fmm_neg(a4), a5));  // operand of M19
    st(13, fmm_sub(fmm_sub(a0, a2), a3));  // operand of M20
    st(14, fmm_sub(a4, a9));  // operand of M21
    st(15, fmm_add(fmm_add(fmm_add(a7, a9), a10), a11));  // operand of M22
    st(16, fmm_add(fmm_add(fmm_neg(a2), a9), a10));  // operand of M24
    st(17, fmm_sub(fmm_sub(a0, a4), a8));  // operand of M26
    st(18, fmm_sub(fmm_sub(fmm_add(fmm_add(a1, a2), a3), a5), a6));  // operand of M27
    st(19, fmm_sub(a6, a9));  // operand of M28
    st(20, fmm_add(fmm_neg(a7), a9));  // operand of M29
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T b9 = ld(9);
    const T b10 = ld(10);
    const T b11 = ld(11);
    st(0, fmm_add(b0, b6));  // operand of M1
    st(1, fmm_add(b3, b5));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(b2), b7), b8), b9), b10), b11));  // operand of M3
    st(3, fmm_sub(b6, b9));  // operand of M4
    st(4, fmm_sub(fmm_add(fmm_neg(b0), b3), b6));  // operand of M5
    st(5, fmm_sub(fmm_sub(fmm_sub(b7, b9), b10), b11));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b1), b3), b4), b5), b6));  // operand of M9
    st(7, fmm_add(fmm_sub(b1, b4), b7));  // operand of M10
    st(8, fmm_sub(b1, b9));  // operand of M11
    st(9, fmm_add(fmm_neg(b2), b6));  // operand of M12
    st(10, fmm_add(fmm_neg(b1), b6));  // operand of M13
    st(11, fmm_sub(b2, b9));  // operand of M14
    st(12, fmm_add(fmm_sub(fmm_sub(fmm_sub(b1, b3), b4), b5), b7));  // operand of M16
    st(13, fmm_add(fmm_add(fmm_add(fmm_sub(b2, b5), b8), b9), b11));  // operand of M17
    st(14, fmm_add(b9, b11));  // operand of M18
    st(15, fmm_sub(fmm_add(b1, b3), b6));  // operand of M19
    st(16, fmm_sub(fmm_add(b2, b3), b6));  // operand of M21
    st(17, fmm_add(fmm_add(fmm_add(b1, b9), b10), b11));  // operand of M22
    st(18, fmm_add(fmm_add(fmm_add(fmm_sub(b1, b4), b7), b9), b10));  // operand of M23
    st(19, fmm_sub(fmm_neg(b6), b8));  // operand of M24
    st(20, fmm_add(fmm_neg(b7), b10));  // operand of M25
    st(21, fmm_add(b0, b2));  // operand of M26
    st(22, fmm_sub(fmm_neg(b1), b7));  // operand of M27
    st(23, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(b1, b3), b4), b5), b6), b7), b8));  // operand of M28
    st(24, fmm_sub(fmm_sub(fmm_add(fmm_sub(b1, b4), b7), b9), b11));  // operand of M29
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T m26 = ld(26);
    const T m27 = ld(27);
    const T m28 = ld(28);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_sub(m0, m3), m14), m19), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_sub(m0, m3), m14), m19));
    if (kBeta) st(1, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m8), m12), m15), m19), m24), m26), fmm_mul(beta, ldc(1)))); else st(1, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m8), m12), m15), m19), m24), m26));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(m1, m2), m3), m5), m11), m14), m19), m23), m24), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(m1, m2), m3), m5), m11), m14), m19), m23), m24));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(m4, m6), m7), m10), m12), m18), m19), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(m4, m6), m7), m10), m12), m18), m19));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_neg(m1), m6), m7), m8), m9), m10), m12), m15), m19), m22), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_neg(m1), m6), m7), m8), m9), m10), m12), m15), m19), m22));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m1, m6), m7), m9), m10), m12), m15), m16), m18), m19), m20), m27), m28), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m1, m6), m7), m9), m10), m12), m15), m16), m18), m19), m20), m27), m28));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(m0, m4), m6), m11), m13), m20), m25), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(m0, m4), m6), m11), m13), m20), m25));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m5), m6), m10), m17), m21), m22), m24), m28), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m5), m6), m10), m17), m21), m22), m24), m28));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(m2), m5), m6), m13), m16), m17), m24), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(m2), m5), m6), m13), m16), m17), m24));
  }
};

// grey442_26_257  <4,4,2; 26>  (reference header algorithms/fast442_26_257.hpp, coefficients codegen/algorithms/grey442-26-257)
struct FmmAlg_grey442_26_257 {
  static constexpr int kM0 = 4, kK0 = 4, kN0 = 2, kR = 26;
  static constexpr int kNumAOut = 24, kNumBOut = 20;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    const T a10 = ld(10);
    const T a11 = ld(11);
    const T a12 = ld(12);
    const T a13 = ld(13);
    const T a14 = ld(14);
    const T a15 = ld(15);
    st(0, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(a4, a5), a6), a9), a10), a12));  // operand of M2
    st(1, fmm_add(fmm_add(fmm_neg(a0), fmm_mul(0.5, a7)), fmm_mul(0.5, a11)));  // operand of M4
    st(2, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(a7, a9), a10), a13), a14), a15));  // operand of M5
    st(3, fmm_sub(fmm_neg(a1), a2));  // operand of M6
    st(4, fmm_add(fmm_mul(-0.5, a7), fmm_mul(-0.5, a11)));  // operand of M7
    st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a4), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)), fmm_mul(0.5, a8)), fmm_mul(0.5, a10)), fmm_mul(-0.5, a11)));  // operand of M8
    st(6, fmm_add(fmm_neg(a0), a12));  // operand of M9
    st(7, fmm_add(fmm_mul(-0.5, a7), fmm_mul(0.5, a11)));  // operand of M10
    st(8, fmm_add(fmm_sub(fmm_add(a1, a2), a7), a15));  // operand of M11
    st(9, fmm_add(fmm_sub(fmm_add(a1, a2), a3), a7));  // operand of M12
    st(10, fmm_add(fmm_sub(fmm_add(a1, a2), a5), a13));  // operand of M13
    st(11, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(a0), a2), a3), a7), a15));  // operand of M14
    st(12, fmm_add(fmm_neg(a7), a15));  // operand of M15
    st(13, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a5), fmm_mul(-0.5, a8)), fmm_mul(0.5, a9)), fmm_mul(0.5, a12)));  // operand of M16
    st(14, fmm_add(fmm_mul(0.5, a8), fmm_mul(-0.5, a12)));  // operand of M17
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a7), fmm_mul(0.5, a8)), fmm_mul(0.5, a10)), fmm_mul(-0.5, a11)), fmm_mul(-0.5, a12)), fmm_mul(-0.5, a14)));  // operand of M18
    st(16, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a4), fmm_mul(-0.5, a6)), fmm_mul(0.5, a12)), fmm_mul(0.5, a14)));  // operand of M19
    st(17, fmm_add(fmm_mul(0.5, a5), fmm_mul(0.5, a9)));  // operand of M20
    st(18, fmm_add(fmm_add(fmm_neg(a2), fmm_mul(0.5, a7)), fmm_mul(-0.5, a11)));  // operand of M21
    st(19, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a5), a6), a9), a10));  // operand of M22
    st(20, fmm_add(a9, a10));  // operand of M23
    st(21, fmm_add(a2, a5));  // operand of M24
    st(22, fmm_sub(fmm_add(fmm_add(fmm_neg(a5), a9), a10), a14));  // operand of M25
    st(23, fmm_sub(a4, a12));  // operand of M26
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    st(0, fmm_add(b0, b6));  // operand of M1
    st(1, fmm_add(fmm_sub(fmm_neg(b0), b1), b4));  // operand of M2
    st(2, fmm_sub(fmm_sub(b2, b4), b6));  // operand of M3
    st(3, fmm_add(fmm_add(b0, b1), b6));  // operand of M4
    st(4, fmm_sub(b2, b3));  // operand of M5
    st(5, fmm_add(b3, b7));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(b0, b1), b6), b7));  // operand of M7
    st(7, fmm_add(b0, b1));  // operand of M8
    st(8, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(b2, b3), b4), b5), b6), b7));  // operand of M10
    st(9, fmm_add(fmm_add(fmm_neg(b2), b3), b7));  // operand of M11
    st(10, fmm_sub(fmm_add(fmm_sub(b2, b3), b6), b7));  // operand of M15
    st(11, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(b0, b1), b2), b3), b4), b5));  // operand of M16
    st(12, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(b0, b1), b2), b3), b4), b5));  // operand of M17
    st(13, fmm_add(fmm_sub(fmm_sub(b2, b3), b4), b5));  // operand of M18
    st(14, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(b0, b1), b2), b3), b4), b5));  // operand of M20
    st(15, fmm_sub(fmm_add(fmm_sub(fmm_sub(b2, b3), b4), b5), b6));  // operand of M21
    st(16, fmm_sub(fmm_sub(fmm_add(b0, b1), b4), b5));  // operand of M22
    st(17, fmm_sub(b3, b5));  // operand of M24
    st(18, fmm_add(fmm_sub(b2, b3), b5));  // operand of M25
    st(19, fmm_sub(b0, b4));  // operand of M26
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m0, m2), m5), m10), m13), m14), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m0, m2), m5), m10), m13), m14));
    if (kBeta) st(1, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m0), m2), m3), m5), m6), m9), m11), m20), fmm_mul(beta, ldc(1)))); else st(1, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m0), m2), m3), m5), m6), m9), m11), m20));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m0, fmm_mul(0.5, m1)), m2), m3), m7), m8), m15), m17), m18), m20), m23), fmm_mul(-0.5, m24)), m25), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m0, fmm_mul(0.5, m1)), m2), m3), m7), m8), m15), m17), m18), m20), m23), fmm_mul(-0.5, m24)), m25));
    if (kBeta) st(3, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m0), m1), m2), m3), m6), m8), m9), m20), m21), m22), m23), m25), fmm_mul(beta, ldc(3)))); else st(3, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m0), m1), m2), m3), m6), m8), m9), m20), m21), m22), m23), m25));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m0, fmm_mul(0.5, m1)), m2), m3), m7), m8), m16), m17), m18), m19), m20), m23), fmm_mul(0.5, m24)), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m0, fmm_mul(0.5, m1)), m2), m3), m7), m8), m16), m17), m18), m19), m20), m23), fmm_mul(0.5, m24)));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_neg(m0), m2), m3), m6), m8), m9), m15), m16), m19), m20), m22), m23), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_neg(m0), m2), m3), m6), m8), m9), m15), m16), m19), m20), m22), m23));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m0, fmm_mul(0.5, m1)), m2), m3), m5), m7), m8), m10), m12), m14), m15), m17), m18), m20), m23), fmm_mul(-0.5, m24)), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m0, fmm_mul(0.5, m1)), m2), m3), m5), m7), m8), m10), m12), m14), m15), m17), m18), m20), m23), fmm_mul(-0.5, m24)));
    if (kBeta) st(7, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m0), m2), m3), m4), m5), m6), m8), m9), m10), m12), m20), m22), m23), m24), fmm_mul(beta, ldc(7)))); else st(7, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m0), m2), m3), m4), m5), m6), m8), m9), m10), m12), m20), m22), m23), m24));
  }
};

// grey424_26_257  <4,2,4; 26>  (reference header algorithms/fast424_26_257.hpp, coefficients codegen/algorithms/grey424-26-257)
struct FmmAlg_grey424_26_257 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 4, kR = 26;
  static constexpr int kNumAOut = 22, kNumBOut = 20;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    st(0, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(a0, a1), a2), a3), a4), a5), a6), a7));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_sub(fmm_mul(0.5, a2), a3), fmm_mul(0.5, a4)), fmm_mul(0.5, a6)));  // operand of M2
    st(2, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_neg(a0), a1), a2), a3), a4), a5), a6), a7));  // operand of M3
    st(3, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(a1), a2), a3), a4), a5), a6), a7));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_sub(fmm_neg(a0), a1), a6), a7));  // operand of M6
    st(5, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a1), a3), a5), a7));  // operand of M7
    st(6, fmm_add(fmm_add(a2, a4), a6));  // operand of M8
    st(7, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(a2, a3), a4), a5), a6), a7));  // operand of M9
    st(8, fmm_sub(fmm_add(fmm_sub(fmm_neg(a1), a3), a5), a7));  // operand of M10
    st(9, fmm_add(fmm_add(fmm_neg(a0), a6), a7));  // operand of M11
    st(10, fmm_sub(fmm_neg(a6), a7));  // operand of M13
    st(11, fmm_add(fmm_neg(a0), a6));  // operand of M15
    st(12, fmm_add(fmm_sub(a2, a5), a6));  // operand of M16
    st(13, fmm_sub(a4, a5));  // operand of M17
    st(14, fmm_add(fmm_sub(a2, a4), a6));  // operand of M18
    st(15, fmm_sub(fmm_sub(a2, a4), a6));  // operand of M19
    st(16, fmm_add(a4, a5));  // operand of M20
    st(17, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(a1), a2), a3), a4), a5), a6), a7));  // operand of M21
    st(18, fmm_sub(fmm_sub(a3, a5), a7));  // operand of M23
    st(19, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(a2, a3), a4), a5), a6), a7));  // operand of M24
    st(20, fmm_sub(fmm_add(fmm_add(fmm_mul(-0.5, a2), fmm_mul(0.5, a4)), fmm_mul(-0.5, a6)), a7));  // operand of M25
    st(21, fmm_sub(a2, a3));  // operand of M26
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    st(0, fmm_add(b0, b3));  // operand of M1
    st(1, fmm_sub(fmm_add(fmm_neg(b0), b2), b4));  // operand of M2
    st(2, fmm_sub(fmm_sub(b1, b2), b3));  // operand of M3
    st(3, fmm_add(fmm_add(b0, b3), b4));  // operand of M4
    st(4, fmm_sub(b1, b5));  // operand of M5
    st(5, fmm_add(b5, b7));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(b0, b3), b4), b7));  // operand of M7
    st(7, fmm_add(b0, b4));  // operand of M8
    st(8, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(b1, b2), b3), b5), b6), b7));  // operand of M10
    st(9, fmm_add(fmm_add(fmm_neg(b1), b5), b7));  // operand of M11
    st(10, fmm_sub(fmm_sub(fmm_add(b1, b3), b5), b7));  // operand of M15
    st(11, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(b0, b1), b2), b4), b5), b6));  // operand of M16
    st(12, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(b0, b1), b2), b4), b5), b6));  // operand of M17
    st(13, fmm_add(fmm_sub(fmm_sub(b1, b2), b5), b6));  // operand of M18
    st(14, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(b0, b1), b2), b4), b5), b6));  // operand of M20
    st(15, fmm_add(fmm_sub(fmm_sub(fmm_sub(b1, b2), b3), b5), b6));  // operand of M21
    st(16, fmm_sub(fmm_add(fmm_sub(b0, b2), b4), b6));  // operand of M22
    st(17, fmm_sub(b5, b6));  // operand of M24
    st(18, fmm_add(fmm_sub(b1, b5), b6));  // operand of M25
    st(19, fmm_sub(b0, b2));  // operand of M26
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_sub(fmm_sub(m0, m3), m8), m13), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_sub(fmm_sub(m0, m3), m8), m13));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m5), m10), m11), m12), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_neg(m5), m10), m11), m12));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(m2, m5), m10), m11), m12), m13), m20), m23), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(m2, m5), m10), m11), m12), m13), m20), m23));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_neg(m11), m13), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_neg(m11), m13));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(m1, fmm_mul(0.5, m7)), fmm_mul(-0.5, m18)), m25), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(m1, fmm_mul(0.5, m7)), fmm_mul(-0.5, m18)), m25));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m1, m12), fmm_mul(0.5, m15)), fmm_mul(0.5, m19)), m21), m23), m24), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m1, m12), fmm_mul(0.5, m15)), fmm_mul(0.5, m19)), m21), m23), m24));
    if (kBeta) st(6, fmm_add(fmm_sub(fmm_add(fmm_add(m1, fmm_mul(0.5, m7)), fmm_mul(-0.5, m18)), m21), fmm_mul(beta, ldc(6)))); else st(6, fmm_sub(fmm_add(fmm_add(m1, fmm_mul(0.5, m7)), fmm_mul(-0.5, m18)), m21));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m3), m4), fmm_mul(-0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(-0.5, m9)), m10), m11), m13), m14), fmm_mul(0.5, m17)), fmm_mul(0.5, m20)), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m3), m4), fmm_mul(-0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(-0.5, m9)), m10), m11), m13), m14), fmm_mul(0.5, m17)), fmm_mul(0.5, m20)));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m7), fmm_mul(-0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(0.5, m17)), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m7), fmm_mul(-0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(0.5, m17)));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m1, m4), fmm_mul(0.5, m15)), fmm_mul(0.5, m19)), m21), m22), m24), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m1, m4), fmm_mul(0.5, m15)), fmm_mul(0.5, m19)), m21), m22), m24));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m1, m4), fmm_mul(0.5, m7)), fmm_mul(0.5, m17)), m21), m22), m24), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(m1, m4), fmm_mul(0.5, m7)), fmm_mul(0.5, m17)), m21), m22), m24));
    if (kBeta) st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m3), fmm_mul(-0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(0.5, m9)), fmm_mul(-0.5, m17)), fmm_mul(-0.5, m20)), fmm_mul(beta, ldc(11)))); else st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m3), fmm_mul(-0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(0.5, m9)), fmm_mul(-0.5, m17)), fmm_mul(-0.5, m20)));
    if (kBeta) st(12, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m1), m8), fmm_mul(0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), m25), fmm_mul(beta, ldc(12)))); else st(12, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m1), m8), fmm_mul(0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), m25));
    if (kBeta) st(13, fmm_add(fmm_add(m4, m12), fmm_mul(beta, ldc(13)))); else st(13, fmm_add(m4, m12));
    if (kBeta) st(14, fmm_add(fmm_sub(fmm_add(fmm_add(m4, fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), m24), fmm_mul(beta, ldc(14)))); else st(14, fmm_sub(fmm_add(fmm_add(m4, fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), m24));
    if (kBeta) st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m4), m10), m13), m14), fmm_mul(beta, ldc(15)))); else st(15, fmm_add(fmm_add(fmm_add(fmm_neg(m4), m10), m13), m14));
  }
};

// grey424_26_206  <4,2,4; 26>  (reference header algorithms/fast424_26_206.hpp, coefficients codegen/algorithms/eliminated/grey424-26-206)
struct FmmAlg_grey424_26_206 {
  static constexpr int kM0 = 4, kK0 = 2, kN0 = 4, kR = 26;
  static constexpr int kNumAOut = 22, kNumBOut = 20;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T ax0 = fmm_add(a0, a2);
    const T ax1 = fmm_sub(fmm_neg(a1), a3);
    const T ax2 = fmm_sub(a4, a5);
    const T ax3 = fmm_sub(a6, a7);
    const T ax4 = fmm_add(a4, a5);
    const T ax5 = fmm_sub(fmm_neg(a6), a7);
    st(0, ax2);
    st(1, ax4);
    st(2, ax5);
    st(3, fmm_add(fmm_add(fmm_add(ax0, ax1), ax2), ax3));  // operand of M1
    st(4, fmm_add(fmm_add(fmm_sub(fmm_mul(0.5, a2), a3), fmm_mul(0.5, a4)), fmm_mul(0.5, a6)));  // operand of M2
    st(5, fmm_add(fmm_add(fmm_add(fmm_neg(ax0), ax1), ax4), ax5));  // operand of M3
    st(6, fmm_add(fmm_add(fmm_add(a2, ax1), ax2), ax3));  // operand of M4
    st(7, fmm_sub(fmm_sub(fmm_neg(a0), a1), ax5));  // operand of M6
    st(8, fmm_add(fmm_sub(fmm_neg(a5), a7), ax1));  // operand of M7
    st(9, fmm_add(fmm_add(a2, a4), a6));  // operand of M8
    st(10, fmm_add(fmm_add(fmm_sub(a2, a3), ax2), ax3));  // operand of M9
    st(11, fmm_add(fmm_sub(a5, a7), ax1));  // operand of M10
    st(12, fmm_sub(fmm_neg(a0), ax5));  // operand of M11
    st(13, fmm_add(fmm_neg(a0), a6));  // operand of M15
    st(14, fmm_add(fmm_sub(a2, a5), a6));  // operand of M16
    st(15, fmm_add(fmm_sub(a2, a4), a6));  // operand of M18
    st(16, fmm_sub(fmm_sub(a2, a4), a6));  // operand of M19
    st(17, fmm_add(fmm_add(fmm_add(fmm_neg(a2), ax1), ax4), ax5));  // operand of M21
    st(18, fmm_sub(fmm_sub(a3, a5), a7));  // operand of M23
    st(19, fmm_sub(fmm_sub(fmm_add(a2, a3), ax4), ax5));  // operand of M24
    st(20, fmm_sub(fmm_add(fmm_add(fmm_mul(-0.5, a2), fmm_mul(0.5, a4)), fmm_mul(-0.5, a6)), a7));  // operand of M25
    st(21, fmm_sub(a2, a3));  // operand of M26
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T bx0 = fmm_add(b0, b3);
    const T bx1 = fmm_add(fmm_neg(b0), b2);
    const T bx2 = fmm_sub(b1, b2);
    const T bx3 = fmm_sub(b1, b5);
    const T bx4 = fmm_sub(fmm_neg(b3), b5);
    const T bx5 = fmm_add(fmm_neg(b4), b6);
    st(0, bx0);
    st(1, bx1);
    st(2, bx3);
    st(3, fmm_add(fmm_neg(b4), bx1));  // operand of M2
    st(4, fmm_add(fmm_neg(b3), bx2));  // operand of M3
    st(5, fmm_add(b4, bx0));  // operand of M4
    st(6, fmm_add(b5, b7));  // operand of M6
    st(7, fmm_add(fmm_add(b4, b7), bx0));  // operand of M7
    st(8, fmm_add(b0, b4));  // operand of M8
    st(9, fmm_add(fmm_add(fmm_add(b6, b7), bx2), bx4));  // operand of M10
    st(10, fmm_sub(b7, bx3));  // operand of M11
    st(11, fmm_add(fmm_sub(b3, b7), bx3));  // operand of M15
    st(12, fmm_add(fmm_sub(fmm_add(b4, b6), bx1), bx3));  // operand of M16
    st(13, fmm_add(fmm_add(fmm_neg(bx1), bx3), bx5));  // operand of M17
    st(14, fmm_add(fmm_add(fmm_neg(b5), b6), bx2));  // operand of M18
    st(15, fmm_sub(fmm_sub(fmm_add(b1, b5), bx1), bx5));  // operand of M20
    st(16, fmm_add(fmm_add(b6, bx2), bx4));  // operand of M21
    st(17, fmm_sub(fmm_neg(bx1), bx5));  // operand of M22
    st(18, fmm_sub(b5, b6));  // operand of M24
    st(19, fmm_add(b6, bx3));  // operand of M25
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T mx0 = fmm_add(fmm_neg(m5), m10);
    const T mx1 = fmm_add(m11, m12);
    const T mx2 = fmm_add(m1, fmm_mul(0.5, m7));
    const T mx3 = fmm_add(fmm_mul(-0.5, m18), m25);
    const T mx4 = fmm_add(m1, fmm_mul(0.5, m15));
    const T mx5 = fmm_sub(fmm_mul(0.5, m19), m21);
    const T mx6 = fmm_add(fmm_mul(0.5, m3), fmm_mul(-0.5, m6));
    const T mx7 = fmm_sub(m4, m10);
    const T mx8 = fmm_add(fmm_mul(-0.5, m9), fmm_mul(0.5, m17));
    const T mx9 = fmm_sub(fmm_neg(m13), m14);
    const T mx10 = fmm_add(fmm_mul(-0.5, m15), fmm_mul(0.5, m16));
    const T mx11 = fmm_add(fmm_neg(m4), m22);
    const T mx12 = fmm_add(fmm_mul(0.5, m17), m24);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_sub(fmm_sub(m0, m3), m8), m13), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_sub(fmm_sub(m0, m3), m8), m13));
    if (kBeta) st(1, fmm_add(fmm_add(mx0, mx1), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(mx0, mx1));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(m2, m13), m20), m23), mx0), mx1), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(m2, m13), m20), m23), mx0), mx1));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_neg(m11), m13), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_neg(m11), m13));
    if (kBeta) st(4, fmm_add(fmm_add(mx2, mx3), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(mx2, mx3));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m12), m23), m24), mx4), mx5), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m12), m23), m24), mx4), mx5));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_sub(fmm_mul(-0.5, m18), m21), mx2), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_sub(fmm_mul(-0.5, m18), m21), mx2));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m7), m11), fmm_mul(0.5, m20)), mx6), mx7), mx8), mx9), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m7), m11), fmm_mul(0.5, m20)), mx6), mx7), mx8), mx9));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m7), fmm_mul(0.5, m17)), mx10), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_mul(0.5, m7), fmm_mul(0.5, m17)), mx10));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_add(fmm_add(m24, mx4), mx5), mx11), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_add(fmm_add(m24, mx4), mx5), mx11));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m21), mx2), mx11), mx12), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_add(fmm_neg(m21), mx2), mx11), mx12));
    if (kBeta) st(11, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(-0.5, m7), fmm_mul(-0.5, m20)), mx6), mx8), fmm_mul(beta, ldc(11)))); else st(11, fmm_sub(fmm_add(fmm_add(fmm_mul(-0.5, m7), fmm_mul(-0.5, m20)), mx6), mx8));
    if (kBeta) st(12, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m8), fmm_mul(-0.5, m17)), mx3), mx10), fmm_mul(beta, ldc(12)))); else st(12, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(m1), m8), fmm_mul(-0.5, m17)), mx3), mx10));
    if (kBeta) st(13, fmm_add(fmm_add(m4, m12), fmm_mul(beta, ldc(13)))); else st(13, fmm_add(m4, m12));
    if (kBeta) st(14, fmm_add(fmm_sub(fmm_add(m4, fmm_mul(0.5, m18)), mx12), fmm_mul(beta, ldc(14)))); else st(14, fmm_sub(fmm_add(m4, fmm_mul(0.5, m18)), mx12));
    if (kBeta) st(15, fmm_add(fmm_sub(fmm_neg(mx7), mx9), fmm_mul(beta, ldc(15)))); else st(15, fmm_sub(fmm_neg(mx7), mx9));
  }
};

// grey522_18_99  <5,2,2; 18>  (reference header algorithms/fast522_18_99.hpp, coefficients codegen/algorithms/grey522-18-99)
struct FmmAlg_grey522_18_99 {
  static constexpr int kM0 = 5, kK0 = 2, kN0 = 2, kR = 18;
  static constexpr int kNumAOut = 12, kNumBOut = 9;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    st(0, fmm_add(a6, a9));  // operand of M2
    st(1, fmm_add(fmm_sub(fmm_sub(a0, a1), a2), a3));  // operand of M5
    st(2, fmm_sub(fmm_neg(a6), a8));  // operand of M7
    st(3, fmm_sub(a1, a3));  // operand of M9
    st(4, fmm_add(a7, a9));  // operand of M10
    st(5, fmm_add(a1, a5));  // operand of M11
    st(6, fmm_sub(fmm_add(fmm_neg(a2), a3), a4));  // operand of M12
    st(7, fmm_add(fmm_neg(a6), a7));  // operand of M13
    st(8, fmm_sub(fmm_add(fmm_sub(fmm_neg(a1), a2), a3), a4));  // operand of M14
    st(9, fmm_add(a0, a4));  // operand of M15
    st(10, fmm_add(a2, a4));  // operand of M16
    st(11, fmm_sub(a8, a9));  // operand of M18
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    st(0, fmm_add(b0, b3));  // operand of M2
    st(1, fmm_add(b0, b2));  // operand of M4
    st(2, fmm_add(fmm_neg(b0), b1));  // operand of M5
    st(3, fmm_add(b1, b3));  // operand of M6
    st(4, fmm_sub(b0, b1));  // operand of M7
    st(5, fmm_add(fmm_sub(fmm_add(fmm_neg(b0), b1), b2), b3));  // operand of M9
    st(6, fmm_add(fmm_neg(b2), b3));  // operand of M10
    st(7, fmm_add(fmm_add(fmm_neg(b0), b1), b3));  // operand of M14
    st(8, fmm_add(b1, b3));  // operand of M16
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_add(m0, m2), m10), m14), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_add(m0, m2), m10), m14));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(m4, m7), m11), m13), m14), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_sub(fmm_add(fmm_sub(m4, m7), m11), m13), m14));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m0, m2), m8), m10), m13), m15), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m0, m2), m8), m10), m13), m15));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_neg(m7), m11), m15), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_neg(m7), m11), m15));
    if (kBeta) st(4, fmm_add(fmm_sub(fmm_neg(m0), m2), fmm_mul(beta, ldc(4)))); else st(4, fmm_sub(fmm_neg(m0), m2));
    if (kBeta) st(5, fmm_add(fmm_sub(m7, m16), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(m7, m16));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_sub(fmm_sub(m1, m3), m9), m12), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_sub(fmm_sub(m1, m3), m9), m12));
    if (kBeta) st(7, fmm_add(fmm_add(m5, m12), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(m5, m12));
    if (kBeta) st(8, fmm_add(fmm_add(m3, m17), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(m3, m17));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_add(fmm_sub(m1, m5), m6), m17), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_add(fmm_sub(m1, m5), m6), m17));
  }
};

// grey252_18_99  <2,5,2; 18>  (reference header algorithms/fast252_18_99.hpp, coefficients codegen/algorithms/grey252-18-99)
struct FmmAlg_grey252_18_99 {
  static constexpr int kM0 = 2, kK0 = 5, kN0 = 2, kR = 18;
  static constexpr int kNumAOut = 12, kNumBOut = 13;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    st(0, fmm_add(a3, a9));  // operand of M2
    st(1, fmm_add(fmm_sub(fmm_sub(a0, a1), a5), a6));  // operand of M5
    st(2, fmm_sub(fmm_neg(a3), a4));  // operand of M7
    st(3, fmm_sub(a5, a6));  // operand of M9
    st(4, fmm_add(a8, a9));  // operand of M10
    st(5, fmm_add(a5, a7));  // operand of M11
    st(6, fmm_add(fmm_sub(fmm_neg(a1), a2), a6));  // operand of M12
    st(7, fmm_add(fmm_neg(a3), a8));  // operand of M13
    st(8, fmm_add(fmm_sub(fmm_sub(fmm_neg(a1), a2), a5), a6));  // operand of M14
    st(9, fmm_add(a0, a2));  // operand of M15
    st(10, fmm_add(a1, a2));  // operand of M16
    st(11, fmm_sub(a4, a9));  // operand of M18
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T b9 = ld(9);
    st(0, fmm_sub(fmm_add(b0, b2), b4));  // operand of M1
    st(1, fmm_add(b6, b9));  // operand of M2
    st(2, fmm_sub(fmm_add(b0, b2), b4));  // operand of M3
    st(3, fmm_add(fmm_neg(b6), b8));  // operand of M4
    st(4, fmm_sub(b7, b9));  // operand of M6
    st(5, fmm_add(fmm_sub(fmm_neg(b1), b3), b5));  // operand of M8
    st(6, fmm_add(b0, b2));  // operand of M11
    st(7, fmm_add(b1, b3));  // operand of M12
    st(8, fmm_add(b6, b7));  // operand of M13
    st(9, fmm_add(fmm_neg(b1), b2));  // operand of M14
    st(10, fmm_add(b0, b1));  // operand of M15
    st(11, fmm_add(b2, b3));  // operand of M16
    st(12, fmm_add(b8, b9));  // operand of M18
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(m1, m2), m3), m4), m6), m8), m13), m14), m17), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(m1, m2), m3), m4), m6), m8), m13), m14), m17));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m4, m5), m6), m7), m8), m13), m15), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(m4, m5), m6), m7), m8), m13), m15));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(m0, m3), m8), m9), m10), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_sub(fmm_sub(fmm_add(m0, m3), m8), m9), m10));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m1, m5), m8), m9), m11), m12), m13), m15), m16), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(m1, m5), m8), m9), m11), m12), m13), m15), m16));
  }
};

// smirnov336_40_960  <3,3,6; 40>  (reference header algorithms/smirnov336_40_960.hpp, coefficients codegen/algorithms/smirnov336-40-960)
struct FmmAlg_smirnov336_40_960 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 6, kR = 40;
  static constexpr int kNumAOut = 40, kNumBOut = 40;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(a0, a2), a4), a5), a6), a7));  // operand of M1
    st(1, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(a0, a2), a4), a5), a6), a7));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M4
    st(4, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(a0, a2), a4), a5), a6), a7));  // operand of M5
    st(5, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M6
    st(6, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(a0, a2), a4), a5), a6), a7));  // operand of M8
    st(8, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M9
    st(9, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(a0, a2), a4), a5), a6), a7));  // operand of M11
    st(11, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(a0, a2), a4), a5), a6), a7));  // operand of M12
    st(12, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M13
    st(13, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M14
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(a0), a2), a4), a5), a6), a7));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(a0, a2), a4), a5), a6), a7));  // operand of M16
    st(16, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a3), a4), a6), a7));  // operand of M17
    st(17, fmm_sub(fmm_sub(fmm_add(a0, a1), a6), a7));  // operand of M18
    st(18, fmm_add(fmm_sub(fmm_add(fmm_neg(a3), a4), a6), a7));  // operand of M19
    st(19, fmm_add(fmm_add(fmm_add(a1, a2), a4), a5));  // operand of M20
    st(20, fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a2), a3), a5));  // operand of M21
    st(21, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a0), a2), a3), a5));  // operand of M22
    st(22, fmm_add(fmm_sub(fmm_add(fmm_neg(a4), a5), a7), a8));  // operand of M23
    st(23, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a4), a5), a7), a8));  // operand of M24
    st(24, fmm_sub(fmm_add(fmm_add(fmm_neg(a0), a1), a6), a7));  // operand of M25
    st(25, fmm_sub(fmm_add(fmm_add(fmm_neg(a1), a2), a4), a5));  // operand of M26
    st(26, fmm_sub(fmm_sub(fmm_add(a0, a2), a6), a8));  // operand of M27
    st(27, fmm_sub(fmm_sub(fmm_sub(fmm_neg(a0), a2), a6), a8));  // operand of M28
    st(28, fmm_sub(fmm_add(fmm_sub(a0, a2), a6), a8));  // operand of M29
    st(29, fmm_add(fmm_sub(fmm_sub(a4, a5), a7), a8));  // operand of M30
    st(30, fmm_add(fmm_add(fmm_sub(fmm_neg(a4), a5), a7), a8));  // operand of M31
    st(31, fmm_add(fmm_sub(fmm_sub(a0, a2), a6), a8));  // operand of M32
    st(32, fmm_sub(fmm_add(fmm_sub(a0, a1), a6), a7));  // operand of M33
    st(33, fmm_sub(fmm_add(fmm_sub(a0, a2), a3), a5));  // operand of M34
    st(34, fmm_sub(fmm_add(fmm_sub(a1, a2), a4), a5));  // operand of M35
    st(35, fmm_add(fmm_add(fmm_add(a0, a1), a6), a7));  // operand of M36
    st(36, fmm_sub(fmm_add(fmm_add(fmm_neg(a3), a4), a6), a7));  // operand of M37
    st(37, fmm_add(fmm_add(fmm_sub(fmm_neg(a3), a4), a6), a7));  // operand of M38
    st(38, fmm_add(fmm_add(fmm_sub(fmm_neg(a1), a2), a4), a5));  // operand of M39
    st(39, fmm_add(fmm_add(fmm_sub(fmm_neg(a0), a2), a3), a5));  // operand of M40
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T b9 = ld(9);
    const T b10 = ld(10);
    const T b11 = ld(11);
    const T b12 = ld(12);
    const T b13 = ld(13);
    const T b14 = ld(14);
    const T b15 = ld(15);
    const T b16 = ld(16);
    const T b17 = ld(17);
    st(0, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, b1), b4), fmm_mul(0.125, b5)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), b10), b12), fmm_mul(0.125, b14)), fmm_mul(0.125, b17)));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_mul(-0.125, b2), fmm_mul(-0.125, b3)), b4), fmm_mul(0.125, b7)), b10), fmm_mul(-0.125, b11)), b12), fmm_mul(-0.125, b13)), fmm_mul(0.125, b15)));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(0.125, b2)), fmm_mul(-0.125, b5)), b6), fmm_mul(0.125, b7)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b13)), b16), fmm_mul(-0.125, b17)));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_mul(-0.125, b1), b4), fmm_mul(-0.125, b5)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b9)), b10), b12), fmm_mul(-0.125, b14)), fmm_mul(0.125, b17)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, b2), fmm_mul(0.125, b3)), b4), fmm_mul(-0.125, b7)), b10), fmm_mul(-0.125, b11)), b12), fmm_mul(0.125, b13)), fmm_mul(0.125, b15)));  // operand of M5
    st(5, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(-0.125, b1)), fmm_mul(0.125, b3)), b6), fmm_mul(0.125, b8)), fmm_mul(0.125, b11)), fmm_mul(-0.125, b14)), fmm_mul(-0.125, b15)), b16));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(0.125, b2)), fmm_mul(0.125, b5)), b6), fmm_mul(-0.125, b7)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b13)), b16), fmm_mul(0.125, b17)));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_mul(0.125, b1), b4), fmm_mul(0.125, b5)), fmm_mul(0.125, b8)), fmm_mul(-0.125, b9)), b10), b12), fmm_mul(-0.125, b14)), fmm_mul(0.125, b17)));  // operand of M8
    st(8, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(-0.125, b2)), fmm_mul(-0.125, b5)), b6), fmm_mul(0.125, b7)), fmm_mul(-0.125, b9)), fmm_mul(-0.125, b13)), b16), fmm_mul(0.125, b17)));  // operand of M9
    st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(0.125, b1)), fmm_mul(-0.125, b3)), b6), fmm_mul(-0.125, b8)), fmm_mul(-0.125, b11)), fmm_mul(-0.125, b14)), fmm_mul(-0.125, b15)), b16));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(0.125, b1)), fmm_mul(0.125, b3)), b6), fmm_mul(0.125, b8)), fmm_mul(-0.125, b11)), fmm_mul(-0.125, b14)), fmm_mul(0.125, b15)), b16));  // operand of M11
    st(11, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, b2), fmm_mul(-0.125, b3)), b4), fmm_mul(0.125, b7)), b10), fmm_mul(-0.125, b11)), b12), fmm_mul(0.125, b13)), fmm_mul(-0.125, b15)));  // operand of M12
    st(12, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_mul(-0.125, b1), b4), fmm_mul(0.125, b5)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), b10), b12), fmm_mul(-0.125, b14)), fmm_mul(-0.125, b17)));  // operand of M13
    st(13, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, fmm_mul(0.125, b2)), fmm_mul(-0.125, b5)), b6), fmm_mul(0.125, b7)), fmm_mul(0.125, b9)), fmm_mul(0.125, b13)), b16), fmm_mul(0.125, b17)));  // operand of M14
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, fmm_mul(0.125, b1)), fmm_mul(0.125, b3)), b6), fmm_mul(0.125, b8)), fmm_mul(-0.125, b11)), fmm_mul(0.125, b14)), fmm_mul(-0.125, b15)), b16));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b2), fmm_mul(-0.125, b3)), b4), fmm_mul(0.125, b7)), b10), fmm_mul(0.125, b11)), b12), fmm_mul(0.125, b13)), fmm_mul(0.125, b15)));  // operand of M16
    st(16, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(-0.125, b1)), fmm_mul(0.125, b2)), fmm_mul(-0.125, b3)), b4), fmm_mul(-0.125, b5)), b6), b10), fmm_mul(0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M17
    st(17, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(b0), b4), b6), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b9)), b10), fmm_mul(0.125, b11)), fmm_mul(-0.125, b13)), fmm_mul(-0.125, b14)));  // operand of M18
    st(18, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(-0.125, b1)), fmm_mul(0.125, b2)), fmm_mul(0.125, b3)), b4), fmm_mul(0.125, b5)), b6), b10), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M19
    st(19, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b4), b6), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), b10), fmm_mul(-0.125, b11)), fmm_mul(0.125, b13)), fmm_mul(0.125, b14)));  // operand of M20
    st(20, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, fmm_mul(0.125, b1)), fmm_mul(0.125, b2)), fmm_mul(-0.125, b3)), b4), fmm_mul(0.125, b5)), b6), b10), fmm_mul(0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M21
    st(21, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, fmm_mul(-0.125, b1)), fmm_mul(-0.125, b2)), fmm_mul(-0.125, b3)), b4), fmm_mul(0.125, b5)), b6), b10), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M22
    st(22, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b3), fmm_mul(0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), b12), fmm_mul(0.125, b13)), fmm_mul(-0.125, b14)), fmm_mul(-0.125, b15)), b16), fmm_mul(0.125, b17)));  // operand of M23
    st(23, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b3), fmm_mul(0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), b12), fmm_mul(-0.125, b13)), fmm_mul(0.125, b14)), fmm_mul(-0.125, b15)), b16), fmm_mul(0.125, b17)));  // operand of M24
    st(24, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(b0, b4), b6), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), b10), fmm_mul(0.125, b11)), fmm_mul(0.125, b13)), fmm_mul(0.125, b14)));  // operand of M25
    st(25, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b4), b6), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(-0.125, b9)), b10), fmm_mul(0.125, b11)), fmm_mul(-0.125, b13)), fmm_mul(-0.125, b14)));  // operand of M26
    st(26, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b3), fmm_mul(0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), b12), fmm_mul(0.125, b13)), fmm_mul(0.125, b14)), fmm_mul(0.125, b15)), b16), fmm_mul(0.125, b17)));  // operand of M27
    st(27, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b3), fmm_mul(0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), b12), fmm_mul(-0.125, b13)), fmm_mul(-0.125, b14)), fmm_mul(0.125, b15)), b16), fmm_mul(0.125, b17)));  // operand of M28
    st(28, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b3), fmm_mul(0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), b12), fmm_mul(-0.125, b13)), fmm_mul(-0.125, b14)), fmm_mul(-0.125, b15)), b16), fmm_mul(-0.125, b17)));  // operand of M29
    st(29, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b3), fmm_mul(0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), b12), fmm_mul(0.125, b13)), fmm_mul(-0.125, b14)), fmm_mul(0.125, b15)), b16), fmm_mul(-0.125, b17)));  // operand of M30
    st(30, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b3), fmm_mul(0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), b12), fmm_mul(-0.125, b13)), fmm_mul(0.125, b14)), fmm_mul(0.125, b15)), b16), fmm_mul(-0.125, b17)));  // operand of M31
    st(31, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, b3), fmm_mul(0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), b12), fmm_mul(0.125, b13)), fmm_mul(0.125, b14)), fmm_mul(-0.125, b15)), b16), fmm_mul(-0.125, b17)));  // operand of M32
    st(32, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b4), b6), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), b10), fmm_mul(0.125, b11)), fmm_mul(-0.125, b13)), fmm_mul(-0.125, b14)));  // operand of M33
    st(33, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, fmm_mul(0.125, b1)), fmm_mul(0.125, b2)), fmm_mul(0.125, b3)), b4), fmm_mul(-0.125, b5)), b6), b10), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M34
    st(34, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(b0), b4), b6), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), b10), fmm_mul(-0.125, b11)), fmm_mul(-0.125, b13)), fmm_mul(-0.125, b14)));  // operand of M35
    st(35, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_neg(b0), b4), b6), fmm_mul(-0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(-0.125, b9)), b10), fmm_mul(-0.125, b11)), fmm_mul(-0.125, b13)), fmm_mul(-0.125, b14)));  // operand of M36
    st(36, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(0.125, b1)), fmm_mul(-0.125, b2)), fmm_mul(-0.125, b3)), b4), fmm_mul(-0.125, b5)), b6), b10), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M37
    st(37, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(b0, fmm_mul(-0.125, b1)), fmm_mul(0.125, b2)), fmm_mul(-0.125, b3)), b4), fmm_mul(-0.125, b5)), b6), b10), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M38
    st(38, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(b0, b4), b6), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(-0.125, b9)), b10), fmm_mul(0.125, b11)), fmm_mul(0.125, b13)), fmm_mul(0.125, b14)));  // operand of M39
    st(39, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(b0), fmm_mul(0.125, b1)), fmm_mul(0.125, b2)), fmm_mul(-0.125, b3)), b4), fmm_mul(0.125, b5)), b6), b10), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M40
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T m26 = ld(26);
    const T m27 = ld(27);
    const T m28 = ld(28);
    const T m29 = ld(29);
    const T m30 = ld(30);
    const T m31 = ld(31);
    const T m32 = ld(32);
    const T m33 = ld(33);
    const T m34 = ld(34);
    const T m35 = ld(35);
    const T m36 = ld(36);
    const T m37 = ld(37);
    const T m38 = ld(38);
    const T m39 = ld(39);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m0), fmm_mul(0.125, m1)), fmm_mul(-0.125, m3)), fmm_mul(-0.125, m4)), fmm_mul(0.125, m7)), fmm_mul(-0.125, m11)), fmm_mul(-0.125, m12)), fmm_mul(-0.125, m15)), fmm_mul(-0.125, m16)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m18)), fmm_mul(0.125, m19)), fmm_mul(-0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(-0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(-0.125, m32)), fmm_mul(0.125, m33)), fmm_mul(-0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(0.125, m38)), fmm_mul(0.125, m39)), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m0), fmm_mul(0.125, m1)), fmm_mul(-0.125, m3)), fmm_mul(-0.125, m4)), fmm_mul(0.125, m7)), fmm_mul(-0.125, m11)), fmm_mul(-0.125, m12)), fmm_mul(-0.125, m15)), fmm_mul(-0.125, m16)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m18)), fmm_mul(0.125, m19)), fmm_mul(-0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(-0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(-0.125, m32)), fmm_mul(0.125, m33)), fmm_mul(-0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(0.125, m38)), fmm_mul(0.125, m39)));
    if (kBeta) st(1, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m0), m3), m5), m7), m9), m10), m12), m14), m17), m19), m22), m23), m24), m25), m26), m27), m28), m29), m30), m31), m32), m34), m35), m38), fmm_mul(beta, ldc(1)))); else st(1, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m0), m3), m5), m7), m9), m10), m12), m14), m17), m19), m22), m23), m24), m25), m26), m27), m28), m29), m30), m31), m32), m34), m35), m38));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m1), m2), m4), m6), m8), m11), m13), m15), m17), m19), m22), m23), m24), m25), m26), m27), m28), m29), m30), m31), m32), m34), m35), m38), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m1), m2), m4), m6), m8), m11), m13), m15), m17), m19), m22), m23), m24), m25), m26), m27), m28), m29), m30), m31), m32), m34), m35), m38));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m1), m4), m5), m9), m10), m11), m14), m15), m17), m19), m24), m25), m32), m34), m35), m38), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_neg(m1), m4), m5), m9), m10), m11), m14), m15), m17), m19), m24), m25), m32), m34), m35), m38));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m2), fmm_mul(-0.125, m5)), fmm_mul(-0.125, m6)), fmm_mul(-0.125, m8)), fmm_mul(-0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(0.125, m13)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m16)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m18)), fmm_mul(-0.125, m19)), fmm_mul(-0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(-0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(-0.125, m32)), fmm_mul(0.125, m33)), fmm_mul(0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(-0.125, m38)), fmm_mul(0.125, m39)), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m2), fmm_mul(-0.125, m5)), fmm_mul(-0.125, m6)), fmm_mul(-0.125, m8)), fmm_mul(-0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(0.125, m13)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m16)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m18)), fmm_mul(-0.125, m19)), fmm_mul(-0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(-0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(-0.125, m32)), fmm_mul(0.125, m33)), fmm_mul(0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(-0.125, m38)), fmm_mul(0.125, m39)));
    if (kBeta) st(5, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(m0, m2), m3), m6), m7), m8), m12), m13), m17), m19), m24), m25), m32), m34), m35), m38), fmm_mul(beta, ldc(5)))); else st(5, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(m0, m2), m3), m6), m7), m8), m12), m13), m17), m19), m24), m25), m32), m34), m35), m38));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m0), fmm_mul(0.125, m1)), fmm_mul(0.125, m3)), fmm_mul(0.125, m4)), fmm_mul(-0.125, m7)), fmm_mul(-0.125, m11)), fmm_mul(-0.125, m12)), fmm_mul(0.125, m15)), fmm_mul(0.125, m16)), fmm_mul(0.125, m17)), fmm_mul(0.125, m18)), fmm_mul(0.125, m19)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(-0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(-0.125, m32)), fmm_mul(0.125, m33)), fmm_mul(-0.125, m34)), fmm_mul(0.125, m35)), fmm_mul(0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(-0.125, m38)), fmm_mul(-0.125, m39)), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m0), fmm_mul(0.125, m1)), fmm_mul(0.125, m3)), fmm_mul(0.125, m4)), fmm_mul(-0.125, m7)), fmm_mul(-0.125, m11)), fmm_mul(-0.125, m12)), fmm_mul(0.125, m15)), fmm_mul(0.125, m16)), fmm_mul(0.125, m17)), fmm_mul(0.125, m18)), fmm_mul(0.125, m19)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(-0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(-0.125, m32)), fmm_mul(0.125, m33)), fmm_mul(-0.125, m34)), fmm_mul(0.125, m35)), fmm_mul(0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(-0.125, m38)), fmm_mul(-0.125, m39)));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(m1, m2), m4), m6), m8), m11), m13), m15), m16), m18), m20), m21), m33), m36), m37), m39), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(m1, m2), m4), m6), m8), m11), m13), m15), m16), m18), m20), m21), m33), m36), m37), m39));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(m0, m3), m5), m7), m9), m10), m12), m14), m16), m18), m20), m21), m33), m36), m37), m39), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(m0, m3), m5), m7), m9), m10), m12), m14), m16), m18), m20), m21), m33), m36), m37), m39));
    if (kBeta) st(9, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(m0, m2), m3), m6), m7), m8), m12), m13), m16), m18), m20), m21), m22), m23), m26), m27), m28), m29), m30), m31), m33), m36), m37), m39), fmm_mul(beta, ldc(9)))); else st(9, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(m0, m2), m3), m6), m7), m8), m12), m13), m16), m18), m20), m21), m22), m23), m26), m27), m28), m29), m30), m31), m33), m36), m37), m39));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m2), fmm_mul(0.125, m5)), fmm_mul(0.125, m6)), fmm_mul(0.125, m8)), fmm_mul(0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(0.125, m13)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m16)), fmm_mul(-0.125, m17)), fmm_mul(-0.125, m18)), fmm_mul(-0.125, m19)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(0.125, m32)), fmm_mul(0.125, m33)), fmm_mul(0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(-0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(0.125, m38)), fmm_mul(-0.125, m39)), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m2), fmm_mul(0.125, m5)), fmm_mul(0.125, m6)), fmm_mul(0.125, m8)), fmm_mul(0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(0.125, m13)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m16)), fmm_mul(-0.125, m17)), fmm_mul(-0.125, m18)), fmm_mul(-0.125, m19)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(0.125, m32)), fmm_mul(0.125, m33)), fmm_mul(0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(-0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(0.125, m38)), fmm_mul(-0.125, m39)));
    if (kBeta) st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m1), m4), m5), m9), m10), m11), m14), m15), m16), m18), m20), m21), m22), m23), m26), m27), m28), m29), m30), m31), m33), m36), m37), m39), fmm_mul(beta, ldc(11)))); else st(11, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m1), m4), m5), m9), m10), m11), m14), m15), m16), m18), m20), m21), m22), m23), m26), m27), m28), m29), m30), m31), m33), m36), m37), m39));
    if (kBeta) st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m2), fmm_mul(0.125, m5)), fmm_mul(0.125, m6)), fmm_mul(-0.125, m8)), fmm_mul(-0.125, m9)), fmm_mul(-0.125, m10)), fmm_mul(-0.125, m13)), fmm_mul(0.125, m14)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(-0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(beta, ldc(12)))); else st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m2), fmm_mul(0.125, m5)), fmm_mul(0.125, m6)), fmm_mul(-0.125, m8)), fmm_mul(-0.125, m9)), fmm_mul(-0.125, m10)), fmm_mul(-0.125, m13)), fmm_mul(0.125, m14)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(-0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)));
    if (kBeta) st(13, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m0, m3), m5), m7), m9), m10), m12), m14), m17), m19), m22), m23), m24), m25), m26), m27), m28), m29), m30), m31), m32), m34), m35), m38), fmm_mul(beta, ldc(13)))); else st(13, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(m0, m3), m5), m7), m9), m10), m12), m14), m17), m19), m22), m23), m24), m25), m26), m27), m28), m29), m30), m31), m32), m34), m35), m38));
    if (kBeta) st(14, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(m1, m2), m4), m6), m8), m11), m13), m15), m17), m19), m22), m23), m24), m25), m26), m27), m28), m29), m30), m31), m32), m34), m35), m38), fmm_mul(beta, ldc(14)))); else st(14, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(m1, m2), m4), m6), m8), m11), m13), m15), m17), m19), m22), m23), m24), m25), m26), m27), m28), m29), m30), m31), m32), m34), m35), m38));
    if (kBeta) st(15, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m0, m2), m3), m6), m7), m8), m12), m13), m16), m18), m20), m21), m22), m23), m26), m27), m28), m29), m30), m31), m33), m36), m37), m39), fmm_mul(beta, ldc(15)))); else st(15, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m0, m2), m3), m6), m7), m8), m12), m13), m16), m18), m20), m21), m22), m23), m26), m27), m28), m29), m30), m31), m33), m36), m37), m39));
    if (kBeta) st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m0), fmm_mul(0.125, m1)), fmm_mul(-0.125, m3)), fmm_mul(-0.125, m4)), fmm_mul(-0.125, m7)), fmm_mul(0.125, m11)), fmm_mul(0.125, m12)), fmm_mul(0.125, m15)), fmm_mul(-0.125, m22)), fmm_mul(-0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(-0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(beta, ldc(16)))); else st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m0), fmm_mul(0.125, m1)), fmm_mul(-0.125, m3)), fmm_mul(-0.125, m4)), fmm_mul(-0.125, m7)), fmm_mul(0.125, m11)), fmm_mul(0.125, m12)), fmm_mul(0.125, m15)), fmm_mul(-0.125, m22)), fmm_mul(-0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(-0.125, m30)), fmm_mul(0.125, m31)));
    if (kBeta) st(17, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m1), m4), m5), m9), m10), m11), m14), m15), m16), m18), m20), m21), m22), m23), m26), m27), m28), m29), m30), m31), m33), m36), m37), m39), fmm_mul(beta, ldc(17)))); else st(17, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(m1), m4), m5), m9), m10), m11), m14), m15), m16), m18), m20), m21), m22), m23), m26), m27), m28), m29), m30), m31), m33), m36), m37), m39));
  }
};

// smirnov363_40_960  <3,6,3; 40>  (reference header algorithms/smirnov363_40_960.hpp, coefficients codegen/algorithms/smirnov363-40-960)
struct FmmAlg_smirnov363_40_960 {
  static constexpr int kM0 = 3, kK0 = 6, kN0 = 3, kR = 40;
  static constexpr int kNumAOut = 40, kNumBOut = 40;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    const T a10 = ld(10);
    const T a11 = ld(11);
    const T a12 = ld(12);
    const T a13 = ld(13);
    const T a14 = ld(14);
    const T a15 = ld(15);
    const T a16 = ld(16);
    const T a17 = ld(17);
    st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_mul(-0.125, a0), a1), a5), fmm_mul(-0.125, a6)), a8), a9), a13), a15), fmm_mul(-0.125, a16)));  // operand of M1
    st(1, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_mul(0.125, a0), a2), a3), fmm_mul(0.125, a6)), a7), a11), a14), fmm_mul(0.125, a16)), a17));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(a2), fmm_mul(-0.125, a4)), a5), a7), a9), fmm_mul(-0.125, a10)), fmm_mul(-0.125, a12)), a14), a15));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), a1), a5), fmm_mul(0.125, a6)), a8), a9), a13), a15), fmm_mul(-0.125, a16)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_mul(-0.125, a0), a2), a3), fmm_mul(0.125, a6)), a7), a11), a14), fmm_mul(-0.125, a16)), a17));  // operand of M5
    st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(a1, a3), fmm_mul(-0.125, a4)), a8), fmm_mul(0.125, a10)), a11), fmm_mul(0.125, a12)), a13), a17));  // operand of M6
    st(6, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_neg(a2), fmm_mul(-0.125, a4)), a5), a7), a9), fmm_mul(0.125, a10)), fmm_mul(0.125, a12)), a14), a15));  // operand of M7
    st(7, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), a1), a5), fmm_mul(-0.125, a6)), a8), a9), a13), a15), fmm_mul(-0.125, a16)));  // operand of M8
    st(8, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(a2, fmm_mul(-0.125, a4)), a5), a7), a9), fmm_mul(0.125, a10)), fmm_mul(-0.125, a12)), a14), a15));  // operand of M9
    st(9, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(a1), a3), fmm_mul(-0.125, a4)), a8), fmm_mul(0.125, a10)), a11), fmm_mul(-0.125, a12)), a13), a17));  // operand of M10
    st(10, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(a1, a3), fmm_mul(0.125, a4)), a8), fmm_mul(0.125, a10)), a11), fmm_mul(-0.125, a12)), a13), a17));  // operand of M11
    st(11, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_mul(-0.125, a0), a2), a3), fmm_mul(-0.125, a6)), a7), a11), a14), fmm_mul(0.125, a16)), a17));  // operand of M12
    st(12, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_mul(-0.125, a0), a1), a5), fmm_mul(-0.125, a6)), a8), a9), a13), a15), fmm_mul(0.125, a16)));  // operand of M13
    st(13, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(a2), fmm_mul(0.125, a4)), a5), a7), a9), fmm_mul(0.125, a10)), fmm_mul(-0.125, a12)), a14), a15));  // operand of M14
    st(14, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(a1), a3), fmm_mul(0.125, a4)), a8), fmm_mul(0.125, a10)), a11), fmm_mul(0.125, a12)), a13), a17));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_mul(-0.125, a0), a2), a3), fmm_mul(0.125, a6)), a7), a11), a14), fmm_mul(0.125, a16)), a17));  // operand of M16
    st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a4)), fmm_mul(0.125, a6)), a7), a8), a9), fmm_mul(-0.125, a10)), a11), a15), a17));  // operand of M17
    st(17, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_mul(-0.125, a0), a1), a2), a3), fmm_mul(-0.125, a4)), a5), fmm_mul(0.125, a6)), fmm_mul(-0.125, a10)), a13), a14));  // operand of M18
    st(18, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a4)), fmm_mul(0.125, a6)), a7), a8), a9), fmm_mul(-0.125, a10)), a11), a15), a17));  // operand of M19
    st(19, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), a1), a2), a3), fmm_mul(-0.125, a4)), a5), fmm_mul(0.125, a6)), fmm_mul(-0.125, a10)), a13), a14));  // operand of M20
    st(20, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a4)), fmm_mul(0.125, a6)), a7), a8), a9), fmm_mul(0.125, a10)), a11), a15), a17));  // operand of M21
    st(21, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a4)), fmm_mul(-0.125, a6)), a7), a8), a9), fmm_mul(-0.125, a10)), a11), a15), a17));  // operand of M22
    st(22, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(a1, a2), a9), a11), fmm_mul(0.125, a12)), a13), a14), a15), fmm_mul(-0.125, a16)), a17));  // operand of M23
    st(23, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(a1), a2), a9), a11), fmm_mul(0.125, a12)), a13), a14), a15), fmm_mul(-0.125, a16)), a17));  // operand of M24
    st(24, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_mul(-0.125, a0), a1), a2), a3), fmm_mul(-0.125, a4)), a5), fmm_mul(-0.125, a6)), fmm_mul(0.125, a10)), a13), a14));  // operand of M25
    st(25, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_mul(-0.125, a0), a1), a2), a3), fmm_mul(0.125, a4)), a5), fmm_mul(0.125, a6)), fmm_mul(-0.125, a10)), a13), a14));  // operand of M26
    st(26, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(a1, a2), a9), a11), fmm_mul(0.125, a12)), a13), a14), a15), fmm_mul(0.125, a16)), a17));  // operand of M27
    st(27, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(a1, a2), a9), a11), fmm_mul(-0.125, a12)), a13), a14), a15), fmm_mul(-0.125, a16)), a17));  // operand of M28
    st(28, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(a1, a2), a9), a11), fmm_mul(0.125, a12)), a13), a14), a15), fmm_mul(0.125, a16)), a17));  // operand of M29
    st(29, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(a1, a2), a9), a11), fmm_mul(-0.125, a12)), a13), a14), a15), fmm_mul(0.125, a16)), a17));  // operand of M30
    st(30, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(a1, a2), a9), a11), fmm_mul(0.125, a12)), a13), a14), a15), fmm_mul(-0.125, a16)), a17));  // operand of M31
    st(31, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(a1), a2), a9), a11), fmm_mul(0.125, a12)), a13), a14), a15), fmm_mul(0.125, a16)), a17));  // operand of M32
    st(32, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_mul(-0.125, a0), a1), a2), a3), fmm_mul(-0.125, a4)), a5), fmm_mul(-0.125, a6)), fmm_mul(0.125, a10)), a13), a14));  // operand of M33
    st(33, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a4)), fmm_mul(0.125, a6)), a7), a8), a9), fmm_mul(0.125, a10)), a11), a15), a17));  // operand of M34
    st(34, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), a1), a2), a3), fmm_mul(0.125, a4)), a5), fmm_mul(-0.125, a6)), fmm_mul(0.125, a10)), a13), a14));  // operand of M35
    st(35, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_mul(-0.125, a0), a1), a2), a3), fmm_mul(-0.125, a4)), a5), fmm_mul(0.125, a6)), fmm_mul(-0.125, a10)), a13), a14));  // operand of M36
    st(36, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a4)), fmm_mul(0.125, a6)), a7), a8), a9), fmm_mul(-0.125, a10)), a11), a15), a17));  // operand of M37
    st(37, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a4)), fmm_mul(-0.125, a6)), a7), a8), a9), fmm_mul(0.125, a10)), a11), a15), a17));  // operand of M38
    st(38, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_mul(0.125, a0), a1), a2), a3), fmm_mul(-0.125, a4)), a5), fmm_mul(-0.125, a6)), fmm_mul(0.125, a10)), a13), a14));  // operand of M39
    st(39, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a4)), fmm_mul(-0.125, a6)), a7), a8), a9), fmm_mul(-0.125, a10)), a11), a15), a17));  // operand of M40
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T b9 = ld(9);
    const T b10 = ld(10);
    const T b11 = ld(11);
    const T b12 = ld(12);
    const T b13 = ld(13);
    const T b14 = ld(14);
    const T b15 = ld(15);
    const T b16 = ld(16);
    const T b17 = ld(17);
    st(0, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(-0.125, b3)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b10)), b12), b13), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(-0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(0.125, b11)), b12), b13), fmm_mul(-0.125, b16)));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b1), fmm_mul(0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b6)), fmm_mul(0.125, b10)), b14), fmm_mul(-0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(-0.125, b3)), fmm_mul(-0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b10)), b12), b13), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(-0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(-0.125, b6)), fmm_mul(0.125, b9)), fmm_mul(0.125, b11)), b12), b13), fmm_mul(-0.125, b16)));  // operand of M5
    st(5, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(-0.125, b3)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b11)), b14), fmm_mul(0.125, b16)));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(-0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b6)), fmm_mul(0.125, b10)), b14), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(b2, fmm_mul(0.125, b3)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(-0.125, b10)), b12), b13), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M8
    st(8, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(-0.125, b6)), fmm_mul(-0.125, b10)), b14), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M9
    st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(0.125, b3)), fmm_mul(-0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(-0.125, b9)), fmm_mul(-0.125, b11)), b14), fmm_mul(-0.125, b16)));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b1), fmm_mul(0.125, b3)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(0.125, b11)), b14), fmm_mul(-0.125, b16)));  // operand of M11
    st(11, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(-0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(-0.125, b11)), b12), b13), fmm_mul(-0.125, b16)));  // operand of M12
    st(12, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(-0.125, b3)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b10)), b12), b13), fmm_mul(0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M13
    st(13, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), fmm_mul(0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b6)), fmm_mul(0.125, b10)), b14), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M14
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), fmm_mul(0.125, b3)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b11)), b14), fmm_mul(-0.125, b16)));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b2, fmm_mul(0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(0.125, b11)), b12), b13), fmm_mul(0.125, b16)));  // operand of M16
    st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b1), fmm_mul(-0.125, b3)), fmm_mul(0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(0.125, b11)), b12), b13), fmm_mul(-0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M17
    st(17, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b1), fmm_mul(0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(-0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b10)), b12), b13), fmm_mul(0.125, b16)));  // operand of M18
    st(18, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(-0.125, b3)), fmm_mul(0.125, b6)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b11)), b12), b13), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M19
    st(19, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), fmm_mul(0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b10)), b12), b13), fmm_mul(-0.125, b16)));  // operand of M20
    st(20, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(b0, b1), fmm_mul(0.125, b3)), fmm_mul(0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(0.125, b11)), b12), b13), fmm_mul(0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M21
    st(21, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), fmm_mul(-0.125, b3)), fmm_mul(-0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(-0.125, b11)), b12), b13), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M22
    st(22, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b2, fmm_mul(-0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b11)), b14), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M23
    st(23, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(-0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b11)), b14), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M24
    st(24, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(b0, b1), fmm_mul(-0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b10)), b12), b13), fmm_mul(0.125, b16)));  // operand of M25
    st(25, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(-0.125, b10)), b12), b13), fmm_mul(0.125, b16)));  // operand of M26
    st(26, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(-0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(0.125, b11)), b14), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M27
    st(27, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b2, fmm_mul(-0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(0.125, b11)), b14), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M28
    st(28, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(-0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b11)), b14), fmm_mul(0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M29
    st(29, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b2), fmm_mul(-0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(0.125, b11)), b14), fmm_mul(0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M30
    st(30, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b2, fmm_mul(-0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(0.125, b11)), b14), fmm_mul(0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M31
    st(31, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b2, fmm_mul(-0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b11)), b14), fmm_mul(0.125, b15)), fmm_mul(-0.125, b17)));  // operand of M32
    st(32, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(-0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b10)), b12), b13), fmm_mul(0.125, b16)));  // operand of M33
    st(33, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), fmm_mul(0.125, b3)), fmm_mul(0.125, b6)), fmm_mul(0.125, b9)), fmm_mul(-0.125, b11)), b12), b13), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M34
    st(34, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b1), fmm_mul(0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(0.125, b10)), b12), b13), fmm_mul(-0.125, b16)));  // operand of M35
    st(35, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b1), fmm_mul(-0.125, b4)), fmm_mul(-0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(-0.125, b8)), fmm_mul(-0.125, b10)), b12), b13), fmm_mul(-0.125, b16)));  // operand of M36
    st(36, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(0.125, b3)), fmm_mul(-0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(-0.125, b11)), b12), b13), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M37
    st(37, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(b0, b1), fmm_mul(-0.125, b3)), fmm_mul(0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(-0.125, b11)), b12), b13), fmm_mul(-0.125, b15)), fmm_mul(0.125, b17)));  // operand of M38
    st(38, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(b0, b1), fmm_mul(0.125, b4)), fmm_mul(0.125, b5)), fmm_mul(0.125, b7)), fmm_mul(0.125, b8)), fmm_mul(-0.125, b10)), b12), b13), fmm_mul(0.125, b16)));  // operand of M39
    st(39, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b1), fmm_mul(0.125, b3)), fmm_mul(0.125, b6)), fmm_mul(-0.125, b9)), fmm_mul(-0.125, b11)), b12), b13), fmm_mul(0.125, b15)), fmm_mul(0.125, b17)));  // operand of M40
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T m26 = ld(26);
    const T m27 = ld(27);
    const T m28 = ld(28);
    const T m29 = ld(29);
    const T m30 = ld(30);
    const T m31 = ld(31);
    const T m32 = ld(32);
    const T m33 = ld(33);
    const T m34 = ld(34);
    const T m35 = ld(35);
    const T m36 = ld(36);
    const T m37 = ld(37);
    const T m38 = ld(38);
    const T m39 = ld(39);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m17), m20), m21), m24), m26), m27), m28), m31), m32), m33), m35), m39), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m17), m20), m21), m24), m26), m27), m28), m31), m32), m33), m35), m39));
    if (kBeta) st(1, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(m17, m19), m24), m25), m32), m34), m35), m38), fmm_mul(beta, ldc(1)))); else st(1, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(m17, m19), m24), m25), m32), m34), m35), m38));
    if (kBeta) st(2, fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m19), m20), m21), m25), m26), m27), m28), m31), m33), m34), m38), m39), fmm_mul(beta, ldc(2)))); else st(2, fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m19), m20), m21), m25), m26), m27), m28), m31), m33), m34), m38), m39));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m16), m18), m20), m21), m33), m36), m37), m39), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(m16), m18), m20), m21), m33), m36), m37), m39));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m16), m18), m19), m22), m23), m25), m29), m30), m34), m36), m37), m38), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m16), m18), m19), m22), m23), m25), m29), m30), m34), m36), m37), m38));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m19), m20), m21), m22), m23), m25), m29), m30), m33), m34), m38), m39), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m19), m20), m21), m22), m23), m25), m29), m30), m33), m34), m38), m39));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m16), m17), m18), m24), m26), m27), m28), m31), m32), m35), m36), m37), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_neg(m0), m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m16), m17), m18), m24), m26), m27), m28), m31), m32), m35), m36), m37));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m16), m17), m18), m22), m23), m24), m29), m30), m32), m35), m36), m37), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(m0, m1), m2), m3), m4), m5), m6), m7), m8), m9), m10), m11), m12), m13), m14), m15), m16), m17), m18), m22), m23), m24), m29), m30), m32), m35), m36), m37));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m22, m23), m26), m27), m28), m29), m30), m31), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(m22, m23), m26), m27), m28), m29), m30), m31));
  }
};

// smirnov633_40_960  <6,3,3; 40>  (reference header algorithms/smirnov633_40_960.hpp, coefficients codegen/algorithms/smirnov633-40-960)
struct FmmAlg_smirnov633_40_960 {
  static constexpr int kM0 = 6, kK0 = 3, kN0 = 3, kR = 40;
  static constexpr int kNumAOut = 40, kNumBOut = 40;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    const T a10 = ld(10);
    const T a11 = ld(11);
    const T a12 = ld(12);
    const T a13 = ld(13);
    const T a14 = ld(14);
    const T a15 = ld(15);
    const T a16 = ld(16);
    const T a17 = ld(17);
    st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a1)), a3), a5), a7), a10), a11), fmm_mul(-0.125, a14)), a15));  // operand of M1
    st(1, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a1)), a4), a6), a8), a9), fmm_mul(0.125, a14)), a16), a17));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_mul(-0.125, a2), a4), a6), a8), a10), a11), fmm_mul(-0.125, a12)), fmm_mul(-0.125, a13)), a15));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(0.125, a1)), a3), a5), a7), a10), a11), fmm_mul(-0.125, a14)), a15));  // operand of M4
    st(4, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_mul(-0.125, a0), fmm_mul(0.125, a1)), a4), a6), a8), a9), fmm_mul(-0.125, a14)), a16), a17));  // operand of M5
    st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a2), a3), a5), a7), a9), fmm_mul(-0.125, a12)), fmm_mul(0.125, a13)), a16), a17));  // operand of M6
    st(6, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_mul(0.125, a2), a4), a6), a8), a10), a11), fmm_mul(-0.125, a12)), fmm_mul(0.125, a13)), a15));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(-0.125, a1)), a3), a5), a7), a10), a11), fmm_mul(-0.125, a14)), a15));  // operand of M8
    st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_mul(-0.125, a2), a4), a6), a8), a10), a11), fmm_mul(-0.125, a12)), fmm_mul(0.125, a13)), a15));  // operand of M9
    st(9, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_mul(-0.125, a2), a3), a5), a7), a9), fmm_mul(-0.125, a12)), fmm_mul(0.125, a13)), a16), a17));  // operand of M10
    st(10, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(-0.125, a2), a3), a5), a7), a9), fmm_mul(0.125, a12)), fmm_mul(0.125, a13)), a16), a17));  // operand of M11
    st(11, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a1)), a4), a6), a8), a9), fmm_mul(0.125, a14)), a16), a17));  // operand of M12
    st(12, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a1)), a3), a5), a7), a10), a11), fmm_mul(0.125, a14)), a15));  // operand of M13
    st(13, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_mul(-0.125, a2), a4), a6), a8), a10), a11), fmm_mul(0.125, a12)), fmm_mul(0.125, a13)), a15));  // operand of M14
    st(14, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_mul(0.125, a2), a3), a5), a7), a9), fmm_mul(0.125, a12)), fmm_mul(0.125, a13)), a16), a17));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(0.125, a1)), a4), a6), a8), a9), fmm_mul(0.125, a14)), a16), a17));  // operand of M16
    st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(0.125, a1)), a4), a7), a10), a11), fmm_mul(-0.125, a12)), fmm_mul(-0.125, a13)), a16), a17));  // operand of M17
    st(17, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(0.125, a1)), a3), a5), a6), a8), a9), fmm_mul(-0.125, a12)), fmm_mul(-0.125, a13)), a15));  // operand of M18
    st(18, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a1)), a4), a7), a10), a11), fmm_mul(0.125, a12)), fmm_mul(-0.125, a13)), a16), a17));  // operand of M19
    st(19, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a1)), a3), a5), a6), a8), a9), fmm_mul(-0.125, a12)), fmm_mul(-0.125, a13)), a15));  // operand of M20
    st(20, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(0.125, a1)), a4), a7), a10), a11), fmm_mul(-0.125, a12)), fmm_mul(0.125, a13)), a16), a17));  // operand of M21
    st(21, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a1)), a4), a7), a10), a11), fmm_mul(-0.125, a12)), fmm_mul(-0.125, a13)), a16), a17));  // operand of M22
    st(22, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a2), a3), a5), a6), a8), a10), a11), fmm_mul(-0.125, a14)), a16), a17));  // operand of M23
    st(23, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_mul(0.125, a2), a3), a5), a6), a8), a10), a11), fmm_mul(-0.125, a14)), a16), a17));  // operand of M24
    st(24, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a1)), a3), a5), a6), a8), a9), fmm_mul(-0.125, a12)), fmm_mul(0.125, a13)), a15));  // operand of M25
    st(25, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_mul(-0.125, a0), fmm_mul(0.125, a1)), a3), a5), a6), a8), a9), fmm_mul(0.125, a12)), fmm_mul(-0.125, a13)), a15));  // operand of M26
    st(26, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_mul(0.125, a2), a3), a5), a6), a8), a10), a11), fmm_mul(0.125, a14)), a16), a17));  // operand of M27
    st(27, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a2), a3), a5), a6), a8), a10), a11), fmm_mul(-0.125, a14)), a16), a17));  // operand of M28
    st(28, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a2), a3), a5), a6), a8), a10), a11), fmm_mul(0.125, a14)), a16), a17));  // operand of M29
    st(29, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a2), a3), a5), a6), a8), a10), a11), fmm_mul(0.125, a14)), a16), a17));  // operand of M30
    st(30, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_mul(0.125, a2), a3), a5), a6), a8), a10), a11), fmm_mul(-0.125, a14)), a16), a17));  // operand of M31
    st(31, fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_mul(0.125, a2), a3), a5), a6), a8), a10), a11), fmm_mul(0.125, a14)), a16), a17));  // operand of M32
    st(32, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a1)), a3), a5), a6), a8), a9), fmm_mul(-0.125, a12)), fmm_mul(0.125, a13)), a15));  // operand of M33
    st(33, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a1)), a4), a7), a10), a11), fmm_mul(0.125, a12)), fmm_mul(0.125, a13)), a16), a17));  // operand of M34
    st(34, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, a0), fmm_mul(-0.125, a1)), a3), a5), a6), a8), a9), fmm_mul(0.125, a12)), fmm_mul(0.125, a13)), a15));  // operand of M35
    st(35, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_mul(-0.125, a0), fmm_mul(0.125, a1)), a3), a5), a6), a8), a9), fmm_mul(-0.125, a12)), fmm_mul(-0.125, a13)), a15));  // operand of M36
    st(36, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_mul(0.125, a0), fmm_mul(0.125, a1)), a4), a7), a10), a11), fmm_mul(0.125, a12)), fmm_mul(-0.125, a13)), a16), a17));  // operand of M37
    st(37, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(-0.125, a1)), a4), a7), a10), a11), fmm_mul(0.125, a12)), fmm_mul(0.125, a13)), a16), a17));  // operand of M38
    st(38, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_mul(0.125, a0), fmm_mul(-0.125, a1)), a3), a5), a6), a8), a9), fmm_mul(-0.125, a12)), fmm_mul(0.125, a13)), a15));  // operand of M39
    st(39, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, a0), fmm_mul(-0.125, a1)), a4), a7), a10), a11), fmm_mul(0.125, a12)), fmm_mul(-0.125, a13)), a16), a17));  // operand of M40
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    st(0, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(b0, b2), b4), b5), b6), b7));  // operand of M1
    st(1, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(b0, b2), b4), b5), b6), b7));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M4
    st(4, fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(b0, b2), b4), b5), b6), b7));  // operand of M5
    st(5, fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M6
    st(6, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(b0, b2), b4), b5), b6), b7));  // operand of M8
    st(8, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M9
    st(9, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(b0, b2), b4), b5), b6), b7));  // operand of M11
    st(11, fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(b0, b2), b4), b5), b6), b7));  // operand of M12
    st(12, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M13
    st(13, fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M14
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(b0), b2), b4), b5), b6), b7));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(b0, b2), b4), b5), b6), b7));  // operand of M16
    st(16, fmm_sub(fmm_sub(fmm_sub(fmm_neg(b3), b4), b6), b7));  // operand of M17
    st(17, fmm_sub(fmm_sub(fmm_add(b0, b1), b6), b7));  // operand of M18
    st(18, fmm_add(fmm_sub(fmm_add(fmm_neg(b3), b4), b6), b7));  // operand of M19
    st(19, fmm_add(fmm_add(fmm_add(b1, b2), b4), b5));  // operand of M20
    st(20, fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b2), b3), b5));  // operand of M21
    st(21, fmm_sub(fmm_sub(fmm_sub(fmm_neg(b0), b2), b3), b5));  // operand of M22
    st(22, fmm_add(fmm_sub(fmm_add(fmm_neg(b4), b5), b7), b8));  // operand of M23
    st(23, fmm_sub(fmm_sub(fmm_sub(fmm_neg(b4), b5), b7), b8));  // operand of M24
    st(24, fmm_sub(fmm_add(fmm_add(fmm_neg(b0), b1), b6), b7));  // operand of M25
    st(25, fmm_sub(fmm_add(fmm_add(fmm_neg(b1), b2), b4), b5));  // operand of M26
    st(26, fmm_sub(fmm_sub(fmm_add(b0, b2), b6), b8));  // operand of M27
    st(27, fmm_sub(fmm_sub(fmm_sub(fmm_neg(b0), b2), b6), b8));  // operand of M28
    st(28, fmm_sub(fmm_add(fmm_sub(b0, b2), b6), b8));  // operand of M29
    st(29, fmm_add(fmm_sub(fmm_sub(b4, b5), b7), b8));  // operand of M30
    st(30, fmm_add(fmm_add(fmm_sub(fmm_neg(b4), b5), b7), b8));  // operand of M31
    st(31, fmm_add(fmm_sub(fmm_sub(b0, b2), b6), b8));  // operand of M32
    st(32, fmm_sub(fmm_add(fmm_sub(b0, b1), b6), b7));  // operand of M33
    st(33, fmm_sub(fmm_add(fmm_sub(b0, b2), b3), b5));  // operand of M34
    st(34, fmm_sub(fmm_add(fmm_sub(b1, b2), b4), b5));  // operand of M35
    st(35, fmm_add(fmm_add(fmm_add(b0, b1), b6), b7));  // operand of M36
    st(36, fmm_sub(fmm_add(fmm_add(fmm_neg(b3), b4), b6), b7));  // operand of M37
    st(37, fmm_add(fmm_add(fmm_sub(fmm_neg(b3), b4), b6), b7));  // operand of M38
    st(38, fmm_add(fmm_add(fmm_sub(fmm_neg(b1), b2), b4), b5));  // operand of M39
    st(39, fmm_add(fmm_add(fmm_sub(fmm_neg(b0), b2), b3), b5));  // operand of M40
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T m26 = ld(26);
    const T m27 = ld(27);
    const T m28 = ld(28);
    const T m29 = ld(29);
    const T m30 = ld(30);
    const T m31 = ld(31);
    const T m32 = ld(32);
    const T m33 = ld(33);
    const T m34 = ld(34);
    const T m35 = ld(35);
    const T m36 = ld(36);
    const T m37 = ld(37);
    const T m38 = ld(38);
    const T m39 = ld(39);
    if (kBeta) st(0, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m2), m5), m6), m8), m9), m10), m13), m14), m16), m17), m18), m19), m20), m21), m24), m25), m32), m33), m34), m35), m36), m37), m38), m39), fmm_mul(beta, ldc(0)))); else st(0, fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m2), m5), m6), m8), m9), m10), m13), m14), m16), m17), m18), m19), m20), m21), m24), m25), m32), m33), m34), m35), m36), m37), m38), m39));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m2), m5), m6), m8), m9), m10), m13), m14), m16), m17), m18), m19), m20), m21), m24), m25), m32), m33), m34), m35), m36), m37), m38), m39), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_neg(m2), m5), m6), m8), m9), m10), m13), m14), m16), m17), m18), m19), m20), m21), m24), m25), m32), m33), m34), m35), m36), m37), m38), m39));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m0), m1), m3), m4), m7), m11), m12), m15), m22), m23), m26), m27), m28), m29), m30), m31), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_neg(m0), m1), m3), m4), m7), m11), m12), m15), m22), m23), m26), m27), m28), m29), m30), m31));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m0), fmm_mul(-0.125, m3)), fmm_mul(-0.125, m5)), fmm_mul(0.125, m7)), fmm_mul(0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(-0.125, m12)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m16)), fmm_mul(-0.125, m18)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(0.125, m33)), fmm_mul(0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(0.125, m39)), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m0), fmm_mul(-0.125, m3)), fmm_mul(-0.125, m5)), fmm_mul(0.125, m7)), fmm_mul(0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(-0.125, m12)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m16)), fmm_mul(-0.125, m18)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(0.125, m33)), fmm_mul(0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(0.125, m39)));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m1), fmm_mul(0.125, m2)), fmm_mul(-0.125, m4)), fmm_mul(-0.125, m6)), fmm_mul(0.125, m8)), fmm_mul(0.125, m11)), fmm_mul(0.125, m13)), fmm_mul(0.125, m15)), fmm_mul(0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(-0.125, m22)), fmm_mul(-0.125, m23)), fmm_mul(-0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(-0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(-0.125, m29)), fmm_mul(-0.125, m30)), fmm_mul(-0.125, m31)), fmm_mul(-0.125, m32)), fmm_mul(0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m38)), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m1), fmm_mul(0.125, m2)), fmm_mul(-0.125, m4)), fmm_mul(-0.125, m6)), fmm_mul(0.125, m8)), fmm_mul(0.125, m11)), fmm_mul(0.125, m13)), fmm_mul(0.125, m15)), fmm_mul(0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(-0.125, m22)), fmm_mul(-0.125, m23)), fmm_mul(-0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(-0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(-0.125, m29)), fmm_mul(-0.125, m30)), fmm_mul(-0.125, m31)), fmm_mul(-0.125, m32)), fmm_mul(0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m38)));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m1), fmm_mul(-0.125, m2)), fmm_mul(0.125, m4)), fmm_mul(-0.125, m6)), fmm_mul(-0.125, m8)), fmm_mul(0.125, m11)), fmm_mul(0.125, m13)), fmm_mul(0.125, m15)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(0.125, m22)), fmm_mul(-0.125, m23)), fmm_mul(0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(-0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(-0.125, m32)), fmm_mul(-0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m38)), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m1), fmm_mul(-0.125, m2)), fmm_mul(0.125, m4)), fmm_mul(-0.125, m6)), fmm_mul(-0.125, m8)), fmm_mul(0.125, m11)), fmm_mul(0.125, m13)), fmm_mul(0.125, m15)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(0.125, m22)), fmm_mul(-0.125, m23)), fmm_mul(0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(-0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(-0.125, m32)), fmm_mul(-0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m38)));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m1), fmm_mul(0.125, m2)), fmm_mul(-0.125, m4)), fmm_mul(0.125, m6)), fmm_mul(-0.125, m8)), fmm_mul(-0.125, m11)), fmm_mul(0.125, m13)), fmm_mul(0.125, m15)), fmm_mul(0.125, m16)), fmm_mul(0.125, m18)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(0.125, m33)), fmm_mul(-0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(0.125, m39)), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m1), fmm_mul(0.125, m2)), fmm_mul(-0.125, m4)), fmm_mul(0.125, m6)), fmm_mul(-0.125, m8)), fmm_mul(-0.125, m11)), fmm_mul(0.125, m13)), fmm_mul(0.125, m15)), fmm_mul(0.125, m16)), fmm_mul(0.125, m18)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(0.125, m33)), fmm_mul(-0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(0.125, m39)));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(-0.125, m3)), fmm_mul(0.125, m5)), fmm_mul(0.125, m7)), fmm_mul(-0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(0.125, m12)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(0.125, m32)), fmm_mul(0.125, m34)), fmm_mul(0.125, m35)), fmm_mul(0.125, m38)), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(-0.125, m3)), fmm_mul(0.125, m5)), fmm_mul(0.125, m7)), fmm_mul(-0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(0.125, m12)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(0.125, m32)), fmm_mul(0.125, m34)), fmm_mul(0.125, m35)), fmm_mul(0.125, m38)));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(-0.125, m3)), fmm_mul(-0.125, m5)), fmm_mul(-0.125, m7)), fmm_mul(-0.125, m9)), fmm_mul(-0.125, m10)), fmm_mul(-0.125, m12)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(-0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(-0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(-0.125, m32)), fmm_mul(-0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m38)), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(-0.125, m3)), fmm_mul(-0.125, m5)), fmm_mul(-0.125, m7)), fmm_mul(-0.125, m9)), fmm_mul(-0.125, m10)), fmm_mul(-0.125, m12)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(-0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(0.125, m26)), fmm_mul(-0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(-0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(-0.125, m32)), fmm_mul(-0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m38)));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m1), fmm_mul(0.125, m4)), fmm_mul(0.125, m5)), fmm_mul(-0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(-0.125, m11)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m15)), fmm_mul(-0.125, m16)), fmm_mul(0.125, m18)), fmm_mul(-0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(0.125, m33)), fmm_mul(-0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(-0.125, m39)), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m1), fmm_mul(0.125, m4)), fmm_mul(0.125, m5)), fmm_mul(-0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(-0.125, m11)), fmm_mul(0.125, m14)), fmm_mul(-0.125, m15)), fmm_mul(-0.125, m16)), fmm_mul(0.125, m18)), fmm_mul(-0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(0.125, m33)), fmm_mul(-0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(-0.125, m39)));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(0.125, m2)), fmm_mul(0.125, m3)), fmm_mul(0.125, m6)), fmm_mul(-0.125, m7)), fmm_mul(-0.125, m8)), fmm_mul(0.125, m12)), fmm_mul(0.125, m13)), fmm_mul(0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(0.125, m32)), fmm_mul(0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(-0.125, m38)), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(0.125, m2)), fmm_mul(0.125, m3)), fmm_mul(0.125, m6)), fmm_mul(-0.125, m7)), fmm_mul(-0.125, m8)), fmm_mul(0.125, m12)), fmm_mul(0.125, m13)), fmm_mul(0.125, m17)), fmm_mul(0.125, m19)), fmm_mul(0.125, m24)), fmm_mul(-0.125, m25)), fmm_mul(0.125, m32)), fmm_mul(0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(-0.125, m38)));
    if (kBeta) st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m1), fmm_mul(0.125, m4)), fmm_mul(-0.125, m5)), fmm_mul(-0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(-0.125, m11)), fmm_mul(-0.125, m14)), fmm_mul(0.125, m15)), fmm_mul(0.125, m16)), fmm_mul(-0.125, m18)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(-0.125, m22)), fmm_mul(-0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(-0.125, m31)), fmm_mul(-0.125, m33)), fmm_mul(-0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(-0.125, m39)), fmm_mul(beta, ldc(11)))); else st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m1), fmm_mul(0.125, m4)), fmm_mul(-0.125, m5)), fmm_mul(-0.125, m9)), fmm_mul(0.125, m10)), fmm_mul(-0.125, m11)), fmm_mul(-0.125, m14)), fmm_mul(0.125, m15)), fmm_mul(0.125, m16)), fmm_mul(-0.125, m18)), fmm_mul(0.125, m20)), fmm_mul(-0.125, m21)), fmm_mul(-0.125, m22)), fmm_mul(-0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(-0.125, m31)), fmm_mul(-0.125, m33)), fmm_mul(-0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(-0.125, m39)));
    if (kBeta) st(12, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(m0, m1), m3), m4), m7), m11), m12), m15), m16), m17), m18), m19), m20), m21), m24), m25), m32), m33), m34), m35), m36), m37), m38), m39), fmm_mul(beta, ldc(12)))); else st(12, fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(m0, m1), m3), m4), m7), m11), m12), m15), m16), m17), m18), m19), m20), m21), m24), m25), m32), m33), m34), m35), m36), m37), m38), m39));
    if (kBeta) st(13, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(m0), m1), m3), m4), m7), m11), m12), m15), m16), m17), m18), m19), m20), m21), m24), m25), m32), m33), m34), m35), m36), m37), m38), m39), fmm_mul(beta, ldc(13)))); else st(13, fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_sub(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_neg(m0), m1), m3), m4), m7), m11), m12), m15), m16), m17), m18), m19), m20), m21), m24), m25), m32), m33), m34), m35), m36), m37), m38), m39));
    if (kBeta) st(14, fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(m2, m5), m6), m8), m9), m10), m13), m14), m22), m23), m26), m27), m28), m29), m30), m31), fmm_mul(beta, ldc(14)))); else st(14, fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_sub(fmm_add(fmm_add(fmm_add(fmm_add(fmm_sub(fmm_add(fmm_sub(m2, m5), m6), m8), m9), m10), m13), m14), m22), m23), m26), m27), m28), m29), m30), m31));
    if (kBeta) st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(-0.125, m2)), fmm_mul(-0.125, m3)), fmm_mul(0.125, m6)), fmm_mul(0.125, m7)), fmm_mul(-0.125, m8)), fmm_mul(0.125, m12)), fmm_mul(-0.125, m13)), fmm_mul(-0.125, m16)), fmm_mul(0.125, m18)), fmm_mul(0.125, m20)), fmm_mul(0.125, m21)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(-0.125, m33)), fmm_mul(-0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(0.125, m39)), fmm_mul(beta, ldc(15)))); else st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(-0.125, m2)), fmm_mul(-0.125, m3)), fmm_mul(0.125, m6)), fmm_mul(0.125, m7)), fmm_mul(-0.125, m8)), fmm_mul(0.125, m12)), fmm_mul(-0.125, m13)), fmm_mul(-0.125, m16)), fmm_mul(0.125, m18)), fmm_mul(0.125, m20)), fmm_mul(0.125, m21)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(0.125, m28)), fmm_mul(0.125, m29)), fmm_mul(0.125, m30)), fmm_mul(0.125, m31)), fmm_mul(-0.125, m33)), fmm_mul(-0.125, m36)), fmm_mul(-0.125, m37)), fmm_mul(0.125, m39)));
    if (kBeta) st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m1), fmm_mul(-0.125, m4)), fmm_mul(0.125, m5)), fmm_mul(-0.125, m9)), fmm_mul(-0.125, m10)), fmm_mul(-0.125, m11)), fmm_mul(-0.125, m14)), fmm_mul(0.125, m15)), fmm_mul(0.125, m17)), fmm_mul(-0.125, m19)), fmm_mul(0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(0.125, m32)), fmm_mul(-0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m38)), fmm_mul(beta, ldc(16)))); else st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.125, m1), fmm_mul(-0.125, m4)), fmm_mul(0.125, m5)), fmm_mul(-0.125, m9)), fmm_mul(-0.125, m10)), fmm_mul(-0.125, m11)), fmm_mul(-0.125, m14)), fmm_mul(0.125, m15)), fmm_mul(0.125, m17)), fmm_mul(-0.125, m19)), fmm_mul(0.125, m24)), fmm_mul(0.125, m25)), fmm_mul(0.125, m32)), fmm_mul(-0.125, m34)), fmm_mul(-0.125, m35)), fmm_mul(0.125, m38)));
    if (kBeta) st(17, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(-0.125, m2)), fmm_mul(0.125, m3)), fmm_mul(0.125, m6)), fmm_mul(0.125, m7)), fmm_mul(0.125, m8)), fmm_mul(-0.125, m12)), fmm_mul(0.125, m13)), fmm_mul(-0.125, m16)), fmm_mul(0.125, m18)), fmm_mul(-0.125, m20)), fmm_mul(0.125, m21)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(-0.125, m29)), fmm_mul(-0.125, m30)), fmm_mul(-0.125, m31)), fmm_mul(0.125, m33)), fmm_mul(0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(0.125, m39)), fmm_mul(beta, ldc(17)))); else st(17, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.125, m0), fmm_mul(-0.125, m2)), fmm_mul(0.125, m3)), fmm_mul(0.125, m6)), fmm_mul(0.125, m7)), fmm_mul(0.125, m8)), fmm_mul(-0.125, m12)), fmm_mul(0.125, m13)), fmm_mul(-0.125, m16)), fmm_mul(0.125, m18)), fmm_mul(-0.125, m20)), fmm_mul(0.125, m21)), fmm_mul(0.125, m22)), fmm_mul(0.125, m23)), fmm_mul(0.125, m26)), fmm_mul(0.125, m27)), fmm_mul(-0.125, m28)), fmm_mul(-0.125, m29)), fmm_mul(-0.125, m30)), fmm_mul(-0.125, m31)), fmm_mul(0.125, m33)), fmm_mul(0.125, m36)), fmm_mul(0.125, m37)), fmm_mul(0.125, m39)));
  }
};

// tichavsky_kovac336_40_960  <3,3,6; 40>  (reference header algorithms/tichavsky_kovac336_40_960.hpp, coefficients codegen/algorithms/tichavsky_kovac336-40-960)
struct FmmAlg_tichavsky_kovac336_40_960 {
  static constexpr int kM0 = 3, kK0 = 3, kN0 = 6, kR = 40;
  static constexpr int kNumAOut = 40, kNumBOut = 40;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a2)), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M5
    st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)));  // operand of M8
    st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M9
    st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a2)), fmm_mul(-0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)));  // operand of M11
    st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M12
    st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a2)), fmm_mul(-0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)));  // operand of M13
    st(13, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M14
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)));  // operand of M16
    st(16, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a3), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M17
    st(17, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a1)), fmm_mul(-0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M18
    st(18, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a3), fmm_mul(0.5, a4)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)));  // operand of M19
    st(19, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)));  // operand of M20
    st(20, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(-0.5, a5)));  // operand of M21
    st(21, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(-0.5, a3)), fmm_mul(-0.5, a5)));  // operand of M22
    st(22, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a4), fmm_mul(0.5, a5)), fmm_mul(-0.5, a7)), fmm_mul(0.5, a8)));  // operand of M23
    st(23, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a4), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a7)), fmm_mul(-0.5, a8)));  // operand of M24
    st(24, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a1)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M25
    st(25, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a1), fmm_mul(0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)));  // operand of M26
    st(26, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a2)), fmm_mul(-0.5, a6)), fmm_mul(-0.5, a8)));  // operand of M27
    st(27, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(-0.5, a6)), fmm_mul(-0.5, a8)));  // operand of M28
    st(28, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a8)));  // operand of M29
    st(29, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a4), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a7)), fmm_mul(0.5, a8)));  // operand of M30
    st(30, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a4), fmm_mul(-0.5, a5)), fmm_mul(0.5, a7)), fmm_mul(0.5, a8)));  // operand of M31
    st(31, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a8)));  // operand of M32
    st(32, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(-0.5, a1)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M33
    st(33, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(-0.5, a5)));  // operand of M34
    st(34, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(-0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)));  // operand of M35
    st(35, fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a1)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)));  // operand of M36
    st(36, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a3), fmm_mul(0.5, a4)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)));  // operand of M37
    st(37, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a3), fmm_mul(-0.5, a4)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)));  // operand of M38
    st(38, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a1), fmm_mul(-0.5, a2)), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)));  // operand of M39
    st(39, fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(0.5, a5)));  // operand of M40
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T b9 = ld(9);
    const T b10 = ld(10);
    const T b11 = ld(11);
    const T b12 = ld(12);
    const T b13 = ld(13);
    const T b14 = ld(14);
    const T b15 = ld(15);
    const T b16 = ld(16);
    const T b17 = ld(17);
    st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b1), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b14)), fmm_mul(0.5, b17)));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b3)), fmm_mul(-0.5, b4)), fmm_mul(0.5, b7)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b15)));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b2)), fmm_mul(-0.5, b5)), fmm_mul(-0.5, b6)), fmm_mul(0.5, b7)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b16)), fmm_mul(-0.5, b17)));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b1), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b17)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b15)));  // operand of M5
    st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(0.5, b8)), fmm_mul(0.5, b11)), fmm_mul(-0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(-0.5, b16)));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b2)), fmm_mul(0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b16)), fmm_mul(0.5, b17)));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b1), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b10)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b17)));  // operand of M8
    st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b2)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b16)), fmm_mul(0.5, b17)));  // operand of M9
    st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b8)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b16)));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(-0.5, b6)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(0.5, b16)));  // operand of M11
    st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(-0.5, b15)));  // operand of M12
    st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b1), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b14)), fmm_mul(-0.5, b17)));  // operand of M13
    st(13, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b2)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(0.5, b7)), fmm_mul(0.5, b9)), fmm_mul(0.5, b13)), fmm_mul(0.5, b16)), fmm_mul(0.5, b17)));  // operand of M14
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b16)));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b2), fmm_mul(-0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(0.5, b7)), fmm_mul(0.5, b10)), fmm_mul(0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b15)));  // operand of M16
    st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b2)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(-0.5, b6)), fmm_mul(0.5, b10)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M17
    st(17, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b6)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b10)), fmm_mul(0.5, b11)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b14)));  // operand of M18
    st(18, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b2)), fmm_mul(0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M19
    st(19, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b4)), fmm_mul(0.5, b6)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b13)), fmm_mul(0.5, b14)));  // operand of M20
    st(20, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b2)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(-0.5, b6)), fmm_mul(0.5, b10)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M21
    st(21, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(-0.5, b2)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M22
    st(22, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b3), fmm_mul(0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(-0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(-0.5, b16)), fmm_mul(0.5, b17)));  // operand of M23
    st(23, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b3), fmm_mul(0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b16)), fmm_mul(0.5, b17)));  // operand of M24
    st(24, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b4)), fmm_mul(-0.5, b6)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b10)), fmm_mul(0.5, b11)), fmm_mul(0.5, b13)), fmm_mul(0.5, b14)));  // operand of M25
    st(25, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b4)), fmm_mul(0.5, b6)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b10)), fmm_mul(0.5, b11)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b14)));  // operand of M26
    st(26, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b3), fmm_mul(0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b16)), fmm_mul(0.5, b17)));  // operand of M27
    st(27, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b3), fmm_mul(0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(0.5, b16)), fmm_mul(0.5, b17)));  // operand of M28
    st(28, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b3), fmm_mul(0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(-0.5, b16)), fmm_mul(-0.5, b17)));  // operand of M29
    st(29, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b3), fmm_mul(0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(0.5, b16)), fmm_mul(-0.5, b17)));  // operand of M30
    st(30, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b3), fmm_mul(0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b16)), fmm_mul(-0.5, b17)));  // operand of M31
    st(31, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b3), fmm_mul(0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b16)), fmm_mul(-0.5, b17)));  // operand of M32
    st(32, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b4)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(0.5, b10)), fmm_mul(0.5, b11)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b14)));  // operand of M33
    st(33, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b2)), fmm_mul(0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M34
    st(34, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b6)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b14)));  // operand of M35
    st(35, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b6)), fmm_mul(-0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b14)));  // operand of M36
    st(36, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(-0.5, b2)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M37
    st(37, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b2)), fmm_mul(-0.5, b3)), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M38
    st(38, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b4)), fmm_mul(-0.5, b6)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b9)), fmm_mul(0.5, b10)), fmm_mul(0.5, b11)), fmm_mul(0.5, b13)), fmm_mul(0.5, b14)));  // operand of M39
    st(39, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b2)), fmm_mul(-0.5, b3)), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M40
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T m26 = ld(26);
    const T m27 = ld(27);
    const T m28 = ld(28);
    const T m29 = ld(29);
    const T m30 = ld(30);
    const T m31 = ld(31);
    const T m32 = ld(32);
    const T m33 = ld(33);
    const T m34 = ld(34);
    const T m35 = ld(35);
    const T m36 = ld(36);
    const T m37 = ld(37);
    const T m38 = ld(38);
    const T m39 = ld(39);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(0.5, m1)), fmm_mul(-0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(-0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), fmm_mul(0.5, m19)), fmm_mul(-0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(-0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(-0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(0.5, m38)), fmm_mul(0.5, m39)), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(0.5, m1)), fmm_mul(-0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(-0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), fmm_mul(0.5, m19)), fmm_mul(-0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(-0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(-0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(0.5, m38)), fmm_mul(0.5, m39)));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(0.5, m3)), fmm_mul(0.5, m5)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m12)), fmm_mul(-0.5, m14)), fmm_mul(0.5, m17)), fmm_mul(0.5, m19)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(-0.5, m38)), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(0.5, m3)), fmm_mul(0.5, m5)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m12)), fmm_mul(-0.5, m14)), fmm_mul(0.5, m17)), fmm_mul(0.5, m19)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(-0.5, m38)));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m1), fmm_mul(-0.5, m2)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m8)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m19)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m38)), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m1), fmm_mul(-0.5, m2)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m8)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m19)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m38)));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m1), fmm_mul(0.5, m4)), fmm_mul(-0.5, m5)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m14)), fmm_mul(-0.5, m15)), fmm_mul(0.5, m17)), fmm_mul(0.5, m19)), fmm_mul(0.5, m24)), fmm_mul(0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(0.5, m38)), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m1), fmm_mul(0.5, m4)), fmm_mul(-0.5, m5)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m14)), fmm_mul(-0.5, m15)), fmm_mul(0.5, m17)), fmm_mul(0.5, m19)), fmm_mul(0.5, m24)), fmm_mul(0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(0.5, m38)));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m2), fmm_mul(-0.5, m5)), fmm_mul(-0.5, m6)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), fmm_mul(-0.5, m19)), fmm_mul(-0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(-0.5, m24)), fmm_mul(0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(-0.5, m38)), fmm_mul(0.5, m39)), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m2), fmm_mul(-0.5, m5)), fmm_mul(-0.5, m6)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), fmm_mul(-0.5, m19)), fmm_mul(-0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(-0.5, m24)), fmm_mul(0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(-0.5, m38)), fmm_mul(0.5, m39)));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m17)), fmm_mul(-0.5, m19)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(-0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(-0.5, m38)), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m17)), fmm_mul(-0.5, m19)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(-0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(-0.5, m38)));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(0.5, m1)), fmm_mul(0.5, m3)), fmm_mul(0.5, m4)), fmm_mul(-0.5, m7)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(0.5, m17)), fmm_mul(0.5, m18)), fmm_mul(0.5, m19)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(-0.5, m24)), fmm_mul(0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(-0.5, m34)), fmm_mul(0.5, m35)), fmm_mul(0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(-0.5, m38)), fmm_mul(-0.5, m39)), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(0.5, m1)), fmm_mul(0.5, m3)), fmm_mul(0.5, m4)), fmm_mul(-0.5, m7)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(0.5, m17)), fmm_mul(0.5, m18)), fmm_mul(0.5, m19)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(-0.5, m24)), fmm_mul(0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(-0.5, m34)), fmm_mul(0.5, m35)), fmm_mul(0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(-0.5, m38)), fmm_mul(-0.5, m39)));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m1), fmm_mul(0.5, m2)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m8)), fmm_mul(0.5, m11)), fmm_mul(0.5, m13)), fmm_mul(0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(0.5, m33)), fmm_mul(-0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(0.5, m39)), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m1), fmm_mul(0.5, m2)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m8)), fmm_mul(0.5, m11)), fmm_mul(0.5, m13)), fmm_mul(0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(0.5, m33)), fmm_mul(-0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(0.5, m39)));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m3)), fmm_mul(0.5, m5)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m9)), fmm_mul(-0.5, m10)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(0.5, m33)), fmm_mul(0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(0.5, m39)), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m3)), fmm_mul(0.5, m5)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m9)), fmm_mul(-0.5, m10)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(0.5, m33)), fmm_mul(0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(0.5, m39)));
    if (kBeta) st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m2)), fmm_mul(-0.5, m3)), fmm_mul(0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(-0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(-0.5, m22)), fmm_mul(0.5, m23)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(-0.5, m28)), fmm_mul(-0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(0.5, m33)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(-0.5, m39)), fmm_mul(beta, ldc(9)))); else st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m2)), fmm_mul(-0.5, m3)), fmm_mul(0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(-0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(-0.5, m22)), fmm_mul(0.5, m23)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(-0.5, m28)), fmm_mul(-0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(0.5, m33)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(-0.5, m39)));
    if (kBeta) st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m2), fmm_mul(0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(0.5, m8)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(-0.5, m18)), fmm_mul(-0.5, m19)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(-0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(0.5, m38)), fmm_mul(-0.5, m39)), fmm_mul(beta, ldc(10)))); else st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m2), fmm_mul(0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(0.5, m8)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(-0.5, m18)), fmm_mul(-0.5, m19)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(-0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(0.5, m38)), fmm_mul(-0.5, m39)));
    if (kBeta) st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m1), fmm_mul(-0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m33)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(0.5, m39)), fmm_mul(beta, ldc(11)))); else st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m1), fmm_mul(-0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m33)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(0.5, m39)));
    if (kBeta) st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m2), fmm_mul(0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(-0.5, m10)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m22)), fmm_mul(0.5, m23)), fmm_mul(0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(-0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(beta, ldc(12)))); else st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m2), fmm_mul(0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(-0.5, m10)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m22)), fmm_mul(0.5, m23)), fmm_mul(0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(-0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(0.5, m31)));
    if (kBeta) st(13, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(-0.5, m3)), fmm_mul(0.5, m5)), fmm_mul(0.5, m7)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m12)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m17)), fmm_mul(-0.5, m19)), fmm_mul(0.5, m22)), fmm_mul(0.5, m23)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(0.5, m38)), fmm_mul(beta, ldc(13)))); else st(13, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(-0.5, m3)), fmm_mul(0.5, m5)), fmm_mul(0.5, m7)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m12)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m17)), fmm_mul(-0.5, m19)), fmm_mul(0.5, m22)), fmm_mul(0.5, m23)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(-0.5, m35)), fmm_mul(0.5, m38)));
    if (kBeta) st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m1), fmm_mul(0.5, m2)), fmm_mul(0.5, m4)), fmm_mul(-0.5, m6)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m15)), fmm_mul(0.5, m17)), fmm_mul(0.5, m19)), fmm_mul(-0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m24)), fmm_mul(0.5, m25)), fmm_mul(-0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(-0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(-0.5, m32)), fmm_mul(-0.5, m34)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m38)), fmm_mul(beta, ldc(14)))); else st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m1), fmm_mul(0.5, m2)), fmm_mul(0.5, m4)), fmm_mul(-0.5, m6)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m11)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m15)), fmm_mul(0.5, m17)), fmm_mul(0.5, m19)), fmm_mul(-0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m24)), fmm_mul(0.5, m25)), fmm_mul(-0.5, m26)), fmm_mul(0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(-0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(-0.5, m32)), fmm_mul(-0.5, m34)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m38)));
    if (kBeta) st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(0.5, m12)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(-0.5, m22)), fmm_mul(0.5, m23)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m33)), fmm_mul(-0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(-0.5, m39)), fmm_mul(beta, ldc(15)))); else st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(0.5, m12)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(-0.5, m22)), fmm_mul(0.5, m23)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m33)), fmm_mul(-0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(-0.5, m39)));
    if (kBeta) st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(0.5, m1)), fmm_mul(-0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m7)), fmm_mul(0.5, m11)), fmm_mul(0.5, m12)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(beta, ldc(16)))); else st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(0.5, m1)), fmm_mul(-0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m7)), fmm_mul(0.5, m11)), fmm_mul(0.5, m12)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(0.5, m31)));
    if (kBeta) st(17, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m1), fmm_mul(0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(0.5, m9)), fmm_mul(-0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(-0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(-0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m33)), fmm_mul(-0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(-0.5, m39)), fmm_mul(beta, ldc(17)))); else st(17, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m1), fmm_mul(0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(0.5, m9)), fmm_mul(-0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(-0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(0.5, m16)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(0.5, m21)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(-0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m33)), fmm_mul(-0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(-0.5, m39)));
  }
};

// tichavsky_kovac363_40_960  <3,6,3; 40>  (reference header algorithms/tichavsky_kovac363_40_960.hpp, coefficients codegen/algorithms/tichavsky_kovac363-40-960)
struct FmmAlg_tichavsky_kovac363_40_960 {
  static constexpr int kM0 = 3, kK0 = 6, kN0 = 3, kR = 40;
  static constexpr int kNumAOut = 40, kNumBOut = 40;
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_s(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T a0 = ld(0);
    const T a1 = ld(1);
    const T a2 = ld(2);
    const T a3 = ld(3);
    const T a4 = ld(4);
    const T a5 = ld(5);
    const T a6 = ld(6);
    const T a7 = ld(7);
    const T a8 = ld(8);
    const T a9 = ld(9);
    const T a10 = ld(10);
    const T a11 = ld(11);
    const T a12 = ld(12);
    const T a13 = ld(13);
    const T a14 = ld(14);
    const T a15 = ld(15);
    const T a16 = ld(16);
    const T a17 = ld(17);
    st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a1)), fmm_mul(0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a8)), fmm_mul(0.5, a9)), fmm_mul(0.5, a13)), fmm_mul(0.5, a15)), fmm_mul(-0.5, a16)));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(-0.5, a3)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(-0.5, a11)), fmm_mul(0.5, a14)), fmm_mul(0.5, a16)), fmm_mul(-0.5, a17)));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a2), fmm_mul(-0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a7)), fmm_mul(0.5, a9)), fmm_mul(-0.5, a10)), fmm_mul(-0.5, a12)), fmm_mul(0.5, a14)), fmm_mul(0.5, a15)));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a1)), fmm_mul(0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(0.5, a8)), fmm_mul(-0.5, a9)), fmm_mul(-0.5, a13)), fmm_mul(0.5, a15)), fmm_mul(-0.5, a16)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)), fmm_mul(-0.5, a11)), fmm_mul(0.5, a14)), fmm_mul(-0.5, a16)), fmm_mul(0.5, a17)));  // operand of M5
    st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(-0.5, a3)), fmm_mul(-0.5, a4)), fmm_mul(0.5, a8)), fmm_mul(0.5, a10)), fmm_mul(0.5, a11)), fmm_mul(0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(0.5, a17)));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a2), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a7)), fmm_mul(0.5, a9)), fmm_mul(0.5, a10)), fmm_mul(0.5, a12)), fmm_mul(-0.5, a14)), fmm_mul(0.5, a15)));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a1)), fmm_mul(0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a8)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a15)), fmm_mul(-0.5, a16)));  // operand of M8
    st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a2), fmm_mul(-0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a7)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a10)), fmm_mul(-0.5, a12)), fmm_mul(-0.5, a14)), fmm_mul(0.5, a15)));  // operand of M9
    st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a1), fmm_mul(0.5, a3)), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a8)), fmm_mul(0.5, a10)), fmm_mul(-0.5, a11)), fmm_mul(-0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(0.5, a17)));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(0.5, a3)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a8)), fmm_mul(0.5, a10)), fmm_mul(0.5, a11)), fmm_mul(-0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a17)));  // operand of M11
    st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a2)), fmm_mul(-0.5, a3)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(-0.5, a11)), fmm_mul(-0.5, a14)), fmm_mul(0.5, a16)), fmm_mul(0.5, a17)));  // operand of M12
    st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a1)), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(-0.5, a8)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a13)), fmm_mul(0.5, a15)), fmm_mul(0.5, a16)));  // operand of M13
    st(13, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a2), fmm_mul(0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a7)), fmm_mul(0.5, a9)), fmm_mul(0.5, a10)), fmm_mul(-0.5, a12)), fmm_mul(-0.5, a14)), fmm_mul(-0.5, a15)));  // operand of M14
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a1), fmm_mul(-0.5, a3)), fmm_mul(0.5, a4)), fmm_mul(0.5, a8)), fmm_mul(0.5, a10)), fmm_mul(-0.5, a11)), fmm_mul(0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a17)));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a2)), fmm_mul(-0.5, a3)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(0.5, a11)), fmm_mul(0.5, a14)), fmm_mul(0.5, a16)), fmm_mul(0.5, a17)));  // operand of M16
    st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a4)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(-0.5, a8)), fmm_mul(0.5, a9)), fmm_mul(-0.5, a10)), fmm_mul(0.5, a11)), fmm_mul(0.5, a15)), fmm_mul(0.5, a17)));  // operand of M17
    st(17, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a1)), fmm_mul(-0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(-0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a10)), fmm_mul(-0.5, a13)), fmm_mul(0.5, a14)));  // operand of M18
    st(18, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a4)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(-0.5, a8)), fmm_mul(-0.5, a9)), fmm_mul(-0.5, a10)), fmm_mul(-0.5, a11)), fmm_mul(-0.5, a15)), fmm_mul(-0.5, a17)));  // operand of M19
    st(19, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a1)), fmm_mul(0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a10)), fmm_mul(-0.5, a13)), fmm_mul(0.5, a14)));  // operand of M20
    st(20, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a4)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(0.5, a8)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a10)), fmm_mul(0.5, a11)), fmm_mul(0.5, a15)), fmm_mul(0.5, a17)));  // operand of M21
    st(21, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(0.5, a8)), fmm_mul(0.5, a9)), fmm_mul(-0.5, a10)), fmm_mul(-0.5, a11)), fmm_mul(0.5, a15)), fmm_mul(0.5, a17)));  // operand of M22
    st(22, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(0.5, a2)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a11)), fmm_mul(0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a14)), fmm_mul(-0.5, a15)), fmm_mul(-0.5, a16)), fmm_mul(0.5, a17)));  // operand of M23
    st(23, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a1), fmm_mul(-0.5, a2)), fmm_mul(0.5, a9)), fmm_mul(-0.5, a11)), fmm_mul(0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a14)), fmm_mul(0.5, a15)), fmm_mul(-0.5, a16)), fmm_mul(-0.5, a17)));  // operand of M24
    st(24, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a1)), fmm_mul(0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(-0.5, a4)), fmm_mul(0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a10)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a14)));  // operand of M25
    st(25, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a1)), fmm_mul(-0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a10)), fmm_mul(-0.5, a13)), fmm_mul(0.5, a14)));  // operand of M26
    st(26, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(0.5, a2)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a11)), fmm_mul(0.5, a12)), fmm_mul(-0.5, a13)), fmm_mul(-0.5, a14)), fmm_mul(-0.5, a15)), fmm_mul(0.5, a16)), fmm_mul(-0.5, a17)));  // operand of M27
    st(27, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(0.5, a2)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a11)), fmm_mul(-0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(0.5, a14)), fmm_mul(-0.5, a15)), fmm_mul(-0.5, a16)), fmm_mul(-0.5, a17)));  // operand of M28
    st(28, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(0.5, a2)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a11)), fmm_mul(0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(0.5, a14)), fmm_mul(0.5, a15)), fmm_mul(0.5, a16)), fmm_mul(0.5, a17)));  // operand of M29
    st(29, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(0.5, a2)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a11)), fmm_mul(-0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a14)), fmm_mul(0.5, a15)), fmm_mul(0.5, a16)), fmm_mul(-0.5, a17)));  // operand of M30
    st(30, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a1), fmm_mul(0.5, a2)), fmm_mul(-0.5, a9)), fmm_mul(0.5, a11)), fmm_mul(0.5, a12)), fmm_mul(-0.5, a13)), fmm_mul(0.5, a14)), fmm_mul(0.5, a15)), fmm_mul(-0.5, a16)), fmm_mul(-0.5, a17)));  // operand of M31
    st(31, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a1), fmm_mul(-0.5, a2)), fmm_mul(0.5, a9)), fmm_mul(-0.5, a11)), fmm_mul(0.5, a12)), fmm_mul(0.5, a13)), fmm_mul(0.5, a14)), fmm_mul(-0.5, a15)), fmm_mul(0.5, a16)), fmm_mul(-0.5, a17)));  // operand of M32
    st(32, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a1)), fmm_mul(-0.5, a2)), fmm_mul(-0.5, a3)), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a10)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a14)));  // operand of M33
    st(33, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a4)), fmm_mul(0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(0.5, a8)), fmm_mul(0.5, a9)), fmm_mul(0.5, a10)), fmm_mul(-0.5, a11)), fmm_mul(-0.5, a15)), fmm_mul(-0.5, a17)));  // operand of M34
    st(34, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(0.5, a1)), fmm_mul(0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a10)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a14)));  // operand of M35
    st(35, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, a0), fmm_mul(-0.5, a1)), fmm_mul(0.5, a2)), fmm_mul(-0.5, a3)), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a10)), fmm_mul(-0.5, a13)), fmm_mul(0.5, a14)));  // operand of M36
    st(36, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a4)), fmm_mul(0.5, a6)), fmm_mul(-0.5, a7)), fmm_mul(0.5, a8)), fmm_mul(0.5, a9)), fmm_mul(-0.5, a10)), fmm_mul(0.5, a11)), fmm_mul(-0.5, a15)), fmm_mul(-0.5, a17)));  // operand of M37
    st(37, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a4)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(-0.5, a8)), fmm_mul(0.5, a9)), fmm_mul(0.5, a10)), fmm_mul(0.5, a11)), fmm_mul(-0.5, a15)), fmm_mul(-0.5, a17)));  // operand of M38
    st(38, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(-0.5, a1)), fmm_mul(-0.5, a2)), fmm_mul(0.5, a3)), fmm_mul(-0.5, a4)), fmm_mul(-0.5, a5)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a10)), fmm_mul(0.5, a13)), fmm_mul(-0.5, a14)));  // operand of M39
    st(39, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, a0), fmm_mul(0.5, a4)), fmm_mul(-0.5, a6)), fmm_mul(0.5, a7)), fmm_mul(0.5, a8)), fmm_mul(-0.5, a9)), fmm_mul(-0.5, a10)), fmm_mul(0.5, a11)), fmm_mul(-0.5, a15)), fmm_mul(-0.5, a17)));  // operand of M40
  }
  template <class T, class Ld, class St>
  __device__ __forceinline__ static void form_t(const double* __restrict__ cf, Ld&& ld, St&& st) {
    (void)cf;
    const T b0 = ld(0);
    const T b1 = ld(1);
    const T b2 = ld(2);
    const T b3 = ld(3);
    const T b4 = ld(4);
    const T b5 = ld(5);
    const T b6 = ld(6);
    const T b7 = ld(7);
    const T b8 = ld(8);
    const T b9 = ld(9);
    const T b10 = ld(10);
    const T b11 = ld(11);
    const T b12 = ld(12);
    const T b13 = ld(13);
    const T b14 = ld(14);
    const T b15 = ld(15);
    const T b16 = ld(16);
    const T b17 = ld(17);
    st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b3)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b10)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M1
    st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(-0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(-0.5, b16)));  // operand of M2
    st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(0.5, b10)), fmm_mul(0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M3
    st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b3)), fmm_mul(-0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M4
    st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(-0.5, b6)), fmm_mul(0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(-0.5, b16)));  // operand of M5
    st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b16)));  // operand of M6
    st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(0.5, b10)), fmm_mul(0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M7
    st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b2), fmm_mul(0.5, b3)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M8
    st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(-0.5, b6)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M9
    st(9, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(-0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b14)), fmm_mul(-0.5, b16)));  // operand of M10
    st(10, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(0.5, b14)), fmm_mul(-0.5, b16)));  // operand of M11
    st(11, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(-0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b16)));  // operand of M12
    st(12, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b3)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M13
    st(13, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(0.5, b10)), fmm_mul(0.5, b14)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M14
    st(14, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b14)), fmm_mul(-0.5, b16)));  // operand of M15
    st(15, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b2), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b16)));  // operand of M16
    st(16, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(-0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M17
    st(17, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(-0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b16)));  // operand of M18
    st(18, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M19
    st(19, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b10)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b16)));  // operand of M20
    st(20, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M21
    st(21, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(-0.5, b3)), fmm_mul(-0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M22
    st(22, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M23
    st(23, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M24
    st(24, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b10)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b16)));  // operand of M25
    st(25, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b16)));  // operand of M26
    st(26, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M27
    st(27, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M28
    st(28, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M29
    st(29, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M30
    st(30, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(0.5, b11)), fmm_mul(-0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M31
    st(31, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b2), fmm_mul(-0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b14)), fmm_mul(0.5, b15)), fmm_mul(-0.5, b17)));  // operand of M32
    st(32, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b16)));  // operand of M33
    st(33, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M34
    st(34, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(-0.5, b16)));  // operand of M35
    st(35, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(-0.5, b4)), fmm_mul(-0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(-0.5, b8)), fmm_mul(-0.5, b10)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b16)));  // operand of M36
    st(36, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(-0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M37
    st(37, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(0.5, b1)), fmm_mul(-0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(-0.5, b15)), fmm_mul(0.5, b17)));  // operand of M38
    st(38, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, b0), fmm_mul(-0.5, b1)), fmm_mul(0.5, b4)), fmm_mul(0.5, b5)), fmm_mul(0.5, b7)), fmm_mul(0.5, b8)), fmm_mul(-0.5, b10)), fmm_mul(0.5, b12)), fmm_mul(0.5, b13)), fmm_mul(0.5, b16)));  // operand of M39
    st(39, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, b0), fmm_mul(0.5, b1)), fmm_mul(0.5, b3)), fmm_mul(0.5, b6)), fmm_mul(-0.5, b9)), fmm_mul(-0.5, b11)), fmm_mul(-0.5, b12)), fmm_mul(-0.5, b13)), fmm_mul(0.5, b15)), fmm_mul(0.5, b17)));  // operand of M40
  }
  template <class T, bool kBeta, class Ld, class LdC, class St>
  __device__ __forceinline__ static void combine(const double* __restrict__ cf, double beta, Ld&& ld, LdC&& ldc, St&& st) {
    (void)cf; (void)beta;
    const T m0 = ld(0);
    const T m1 = ld(1);
    const T m2 = ld(2);
    const T m3 = ld(3);
    const T m4 = ld(4);
    const T m5 = ld(5);
    const T m6 = ld(6);
    const T m7 = ld(7);
    const T m8 = ld(8);
    const T m9 = ld(9);
    const T m10 = ld(10);
    const T m11 = ld(11);
    const T m12 = ld(12);
    const T m13 = ld(13);
    const T m14 = ld(14);
    const T m15 = ld(15);
    const T m16 = ld(16);
    const T m17 = ld(17);
    const T m18 = ld(18);
    const T m19 = ld(19);
    const T m20 = ld(20);
    const T m21 = ld(21);
    const T m22 = ld(22);
    const T m23 = ld(23);
    const T m24 = ld(24);
    const T m25 = ld(25);
    const T m26 = ld(26);
    const T m27 = ld(27);
    const T m28 = ld(28);
    const T m29 = ld(29);
    const T m30 = ld(30);
    const T m31 = ld(31);
    const T m32 = ld(32);
    const T m33 = ld(33);
    const T m34 = ld(34);
    const T m35 = ld(35);
    const T m36 = ld(36);
    const T m37 = ld(37);
    const T m38 = ld(38);
    const T m39 = ld(39);
    if (kBeta) st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m1)), fmm_mul(-0.5, m2)), fmm_mul(-0.5, m3)), fmm_mul(0.5, m4)), fmm_mul(-0.5, m5)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(-0.5, m13)), fmm_mul(-0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(0.5, m17)), fmm_mul(-0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(-0.5, m24)), fmm_mul(0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m31)), fmm_mul(0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m39)), fmm_mul(beta, ldc(0)))); else st(0, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m1)), fmm_mul(-0.5, m2)), fmm_mul(-0.5, m3)), fmm_mul(0.5, m4)), fmm_mul(-0.5, m5)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(-0.5, m13)), fmm_mul(-0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(0.5, m17)), fmm_mul(-0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(-0.5, m24)), fmm_mul(0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(0.5, m31)), fmm_mul(0.5, m32)), fmm_mul(0.5, m33)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m39)));
    if (kBeta) st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m17), fmm_mul(0.5, m19)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m38)), fmm_mul(beta, ldc(1)))); else st(1, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m17), fmm_mul(0.5, m19)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m34)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m38)));
    if (kBeta) st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(-0.5, m1)), fmm_mul(-0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m15)), fmm_mul(0.5, m19)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m25)), fmm_mul(0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(-0.5, m28)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m33)), fmm_mul(-0.5, m34)), fmm_mul(-0.5, m38)), fmm_mul(-0.5, m39)), fmm_mul(beta, ldc(2)))); else st(2, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(-0.5, m1)), fmm_mul(-0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(-0.5, m15)), fmm_mul(0.5, m19)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m25)), fmm_mul(0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(-0.5, m28)), fmm_mul(-0.5, m31)), fmm_mul(-0.5, m33)), fmm_mul(-0.5, m34)), fmm_mul(-0.5, m38)), fmm_mul(-0.5, m39)));
    if (kBeta) st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m16), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m33)), fmm_mul(-0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(0.5, m39)), fmm_mul(beta, ldc(3)))); else st(3, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m16), fmm_mul(-0.5, m18)), fmm_mul(0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m33)), fmm_mul(-0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(0.5, m39)));
    if (kBeta) st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m1)), fmm_mul(0.5, m2)), fmm_mul(-0.5, m3)), fmm_mul(0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(0.5, m9)), fmm_mul(-0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(0.5, m18)), fmm_mul(0.5, m19)), fmm_mul(-0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(0.5, m25)), fmm_mul(0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(0.5, m34)), fmm_mul(0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(0.5, m38)), fmm_mul(beta, ldc(4)))); else st(4, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m1)), fmm_mul(0.5, m2)), fmm_mul(-0.5, m3)), fmm_mul(0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(0.5, m9)), fmm_mul(-0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(0.5, m18)), fmm_mul(0.5, m19)), fmm_mul(-0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(0.5, m25)), fmm_mul(0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(0.5, m34)), fmm_mul(0.5, m36)), fmm_mul(-0.5, m37)), fmm_mul(0.5, m38)));
    if (kBeta) st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(-0.5, m1)), fmm_mul(-0.5, m2)), fmm_mul(-0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(-0.5, m8)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(0.5, m19)), fmm_mul(-0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(-0.5, m33)), fmm_mul(-0.5, m34)), fmm_mul(0.5, m38)), fmm_mul(0.5, m39)), fmm_mul(beta, ldc(5)))); else st(5, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(-0.5, m1)), fmm_mul(-0.5, m2)), fmm_mul(-0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(-0.5, m7)), fmm_mul(-0.5, m8)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(0.5, m12)), fmm_mul(0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(0.5, m19)), fmm_mul(-0.5, m20)), fmm_mul(-0.5, m21)), fmm_mul(0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m25)), fmm_mul(-0.5, m29)), fmm_mul(-0.5, m30)), fmm_mul(-0.5, m33)), fmm_mul(-0.5, m34)), fmm_mul(0.5, m38)), fmm_mul(0.5, m39)));
    if (kBeta) st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(-0.5, m1)), fmm_mul(0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m5)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(-0.5, m31)), fmm_mul(0.5, m32)), fmm_mul(0.5, m35)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(beta, ldc(6)))); else st(6, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(-0.5, m0), fmm_mul(-0.5, m1)), fmm_mul(0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(-0.5, m5)), fmm_mul(-0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(0.5, m8)), fmm_mul(0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(0.5, m11)), fmm_mul(-0.5, m12)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(-0.5, m18)), fmm_mul(0.5, m24)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(0.5, m28)), fmm_mul(-0.5, m31)), fmm_mul(0.5, m32)), fmm_mul(0.5, m35)), fmm_mul(0.5, m36)), fmm_mul(0.5, m37)));
    if (kBeta) st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m1)), fmm_mul(0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(-0.5, m11)), fmm_mul(0.5, m12)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), fmm_mul(-0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m24)), fmm_mul(-0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m36)), fmm_mul(0.5, m37)), fmm_mul(beta, ldc(7)))); else st(7, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m0), fmm_mul(0.5, m1)), fmm_mul(0.5, m2)), fmm_mul(0.5, m3)), fmm_mul(-0.5, m4)), fmm_mul(0.5, m5)), fmm_mul(0.5, m6)), fmm_mul(0.5, m7)), fmm_mul(-0.5, m8)), fmm_mul(-0.5, m9)), fmm_mul(0.5, m10)), fmm_mul(-0.5, m11)), fmm_mul(0.5, m12)), fmm_mul(-0.5, m13)), fmm_mul(0.5, m14)), fmm_mul(0.5, m15)), fmm_mul(-0.5, m16)), fmm_mul(-0.5, m17)), fmm_mul(0.5, m18)), fmm_mul(-0.5, m22)), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m24)), fmm_mul(-0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(-0.5, m32)), fmm_mul(0.5, m35)), fmm_mul(-0.5, m36)), fmm_mul(0.5, m37)));
    if (kBeta) st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m22), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(-0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(0.5, m31)), fmm_mul(beta, ldc(8)))); else st(8, fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_add(fmm_mul(0.5, m22), fmm_mul(-0.5, m23)), fmm_mul(-0.5, m26)), fmm_mul(-0.5, m27)), fmm_mul(-0.5, m28)), fmm_mul(0.5, m29)), fmm_mul(0.5, m30)), fmm_mul(0.5, m31)));
  }
};

#define FMM_FOR_EACH_ALGORITHM(X) \
  X(0, FmmAlg_strassen) \
  X(1, FmmAlg_classical222_8_24) \
  X(2, FmmAlg_grey322_11_50) \
  X(3, FmmAlg_bini322_10_52_approx) \
  X(4, FmmAlg_grey332_15_103) \
  X(5, FmmAlg_grey323_15_103) \
  X(6, FmmAlg_hk332_15_94) \
  X(7, FmmAlg_hk323_15_94) \
  X(8, FmmAlg_hk323_15_84) \
  X(9, FmmAlg_grey323_15_89) \
  X(10, FmmAlg_grey333_23_152) \
  X(11, FmmAlg_grey333_23_221) \
  X(12, FmmAlg_grey333_23_125) \
  X(13, FmmAlg_smirnov333_23_139) \
  X(14, FmmAlg_smirnov333_23_128) \
  X(15, FmmAlg_classical333_27_81) \
  X(16, FmmAlg_schonhage333_21_117_approx) \
  X(17, FmmAlg_smirnov333_20_182_approx) \
  X(18, FmmAlg_grey422_14_84) \
  X(19, FmmAlg_grey432_20_144) \
  X(20, FmmAlg_grey423_20_144) \
  X(21, FmmAlg_grey324_20_144) \
  X(22, FmmAlg_grey342_20_144) \
  X(23, FmmAlg_grey234_20_144) \
  X(24, FmmAlg_grey243_20_144) \
  X(25, FmmAlg_classical423_24_72) \
  X(26, FmmAlg_fast423_130) \
  X(27, FmmAlg_fast423_134) \
  X(28, FmmAlg_fast423_138) \
  X(29, FmmAlg_fast423_156) \
  X(30, FmmAlg_grey433_29_234) \
  X(31, FmmAlg_grey343_29_234) \
  X(32, FmmAlg_grey442_26_257) \
  X(33, FmmAlg_grey424_26_257) \
  X(34, FmmAlg_grey424_26_206) \
  X(35, FmmAlg_grey522_18_99) \
  X(36, FmmAlg_grey252_18_99) \
  X(37, FmmAlg_smirnov336_40_960) \
  X(38, FmmAlg_smirnov363_40_960) \
  X(39, FmmAlg_smirnov633_40_960) \
  X(40, FmmAlg_tichavsky_kovac336_40_960) \
  X(41, FmmAlg_tichavsky_kovac363_40_960)
