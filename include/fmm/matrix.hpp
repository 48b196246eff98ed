// C++ drop-in surface of the engine: the reference's Matrix<Scalar> view,
// MatMul, MaxRelativeDiff and RandomMatrix (linalg/linalg.hpp), with the
// products running on the B200 through the C ABI (include/fmm.h).
//
// Matrices live in host memory, column-major, exactly as in the reference
// (linalg/linalg.hpp:41-192): a Matrix owns its data unless constructed from
// a pointer, Subblock/Submatrix return views, the copy constructor deep
// copies, and every matrix carries a scalar multiplier.  Each FastMatmul /
// MatMul call copies its operands to the device, computes there and copies
// C back.  Scalar is double or float; float matrices run through the FP32
// entry points (widened to FP64 on the device, rounded back once).
//
// Engine failures throw std::runtime_error with the engine's message (the
// reference has no error reporting; its FastMatmul returns elapsed ms).
#pragma once

#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include "fmm.h"

template <typename Scalar>
class Matrix {
 public:
  Matrix(Scalar* data, int stride, int m, int n, Scalar multiplier, bool is_view)
      : data_(data), stride_(stride), m_(m), n_(n), is_view_(is_view), multiplier_(multiplier) {
    if (!is_view) allocate();
  }
  Matrix(Scalar* data, int stride, int m, int n, Scalar multiplier) : Matrix(data, stride, m, n, multiplier, true) {}
  Matrix(Scalar* data, int stride, int m, int n) : Matrix(data, stride, m, n, Scalar(1)) {}
  Matrix(int m, int n, Scalar multiplier) : Matrix(nullptr, m, m, n, multiplier, false) {}
  Matrix(int m, int n) : Matrix(m, n, Scalar(1)) {}
  Matrix(int n = 0) : Matrix(n, n) {}

  // deep copy, as the reference's copy constructor (linalg/linalg.hpp:61-70)
  Matrix(const Matrix& that) : Matrix(nullptr, that.m_, that.m_, that.n_, that.multiplier_, false) {
    for (int j = 0; j < n_; ++j)
      for (int i = 0; i < m_; ++i) data_[i + (long)j * stride_] = that.data_[i + (long)j * that.stride_];
  }
  Matrix(Matrix&& that) noexcept : Matrix() { swap(*this, that); }
  Matrix& operator=(Matrix that) {
    swap(*this, that);
    return *this;
  }
  friend void swap(Matrix& a, Matrix& b) noexcept {
    using std::swap;
    swap(a.m_, b.m_);
    swap(a.n_, b.n_);
    swap(a.stride_, b.stride_);
    swap(a.is_view_, b.is_view_);
    swap(a.data_, b.data_);
    swap(a.multiplier_, b.multiplier_);
  }
  ~Matrix() {
    if (!is_view_) deallocate();
  }

  // block (row_ind, col_ind), 1-based, of a num_block_rows x num_block_cols
  // floor split (linalg/linalg.hpp:97-102, 179-184)
  Matrix Subblock(int num_block_rows, int num_block_cols, int row_ind, int col_ind) {
    const int rs = m_ / num_block_rows, cs = n_ / num_block_cols;
    return Submatrix(rs * (row_ind - 1), cs * (col_ind - 1), rs, cs);
  }
  Matrix Submatrix(int start_row, int start_col, int num_rows, int num_cols) {
    return Matrix(data(start_row, start_col), stride_, num_rows, num_cols, multiplier_);
  }

  Scalar* data() { return data_; }
  Scalar* data(int i, int j) { return data_ + i + (long)j * stride_; }
  int stride() const { return stride_; }
  int m() const { return m_; }
  int n() const { return n_; }
  int height() const { return m_; }
  int width() const { return n_; }
  const Scalar& operator()(int i, int j) const { return data_[i + (long)j * stride_]; }
  Scalar& operator()(int i, int j) { return data_[i + (long)j * stride_]; }

  void allocate() {
    if (m_ > 0 && n_ > 0) data_ = new Scalar[(size_t)m_ * (size_t)n_];
  }
  void deallocate() {
    delete[] data_;
    data_ = nullptr;
  }
  void UpdateMultiplier(Scalar multiplier) { multiplier_ *= multiplier; }
  void set_multiplier(Scalar multiplier) { multiplier_ = multiplier; }
  Scalar multiplier() const { return multiplier_; }

 private:
  Scalar* data_;
  int stride_;
  int m_;
  int n_;
  bool is_view_;
  Scalar multiplier_;
};

namespace fmm {

// Device used by this thread's engine handle (default 0); set before the
// first product.
inline int& Device() {
  static int device = 0;
  return device;
}

namespace detail {

inline void Check(fmm_status s) {
  if (s != FMM_OK) throw std::runtime_error(std::string("fmm: ") + fmm_last_error());
}

class HandleHolder {
 public:
  HandleHolder() { Check(fmm_handle_create(&h_, Device())); }
  ~HandleHolder() { fmm_handle_destroy(h_); }
  fmm_handle get() const { return h_; }

 private:
  fmm_handle h_ = nullptr;
};

inline fmm_handle ThreadHandle() {
  thread_local HandleHolder holder;
  return holder.get();
}

// <ns>::FastMatmul(A, B, C, num_steps, x, alpha, beta) (algorithms/strassen.hpp:661-722).
// Multiplier side effects as in the reference: A's multiplier is set to
// alpha, then A's and B's multipliers are folded into C's and reset to 1
// (:669, :380-383), so C keeps multiplier = C.mult * alpha * B.mult.
inline fmm_status FastHost(int alg, double* A, int lda, double* B, int ldb, double* C, int ldc, int m, int k, int n,
                           int steps, double x, double alpha, double beta, double* ms) {
  return fmm_fast_matmul_host(ThreadHandle(), alg, A, lda, B, ldb, C, ldc, m, k, n, steps, x, alpha, beta, nullptr,
                              ms);
}

inline fmm_status FastHost(int alg, float* A, int lda, float* B, int ldb, float* C, int ldc, int m, int k, int n,
                           int steps, double x, float alpha, float beta, double* ms) {
  return fmm_fast_matmul_f32_host(ThreadHandle(), alg, A, lda, B, ldb, C, ldc, m, k, n, steps, x, alpha, beta,
                                  nullptr, ms);
}

inline fmm_status GemmHost(double* A, int lda, double* B, int ldb, double* C, int ldc, int m, int k, int n,
                           double alpha, double beta) {
  return fmm_dgemm_host(ThreadHandle(), A, lda, B, ldb, C, ldc, m, k, n, alpha, beta);
}

inline fmm_status GemmHost(float* A, int lda, float* B, int ldb, float* C, int ldc, int m, int k, int n, float alpha,
                           float beta) {
  return fmm_sgemm_host(ThreadHandle(), A, lda, B, ldb, C, ldc, m, k, n, alpha, beta, nullptr);
}

template <typename Scalar>
double RunFastMatmul(int alg, Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps, double x,
                     Scalar alpha, Scalar beta) {
  static_assert(std::is_same<Scalar, double>::value || std::is_same<Scalar, float>::value,
                "the B200 engine computes with Scalar = double or float");
  A.set_multiplier(alpha);
  C.UpdateMultiplier(A.multiplier());
  C.UpdateMultiplier(B.multiplier());
  A.set_multiplier(Scalar(1));
  B.set_multiplier(Scalar(1));
  double ms = 0.0;
  Check(FastHost(alg, A.data(), A.stride(), B.data(), B.stride(), C.data(), C.stride(), C.m(), A.n(), C.n(),
                 num_steps, x, C.multiplier(), beta, &ms));
  return ms;
}

}  // namespace detail
}  // namespace fmm

// C <- C.multiplier * A * B + beta * C (linalg/linalg.hpp:261-269), on the
// engine's FP64 GEMM.
// Scalar = float: sgemm's role, through fmm_sgemm_host.
template <typename Scalar>
void MatMul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, Scalar beta = Scalar(0.0)) {
  static_assert(std::is_same<Scalar, double>::value || std::is_same<Scalar, float>::value,
                "the B200 engine computes with Scalar = double or float");
  fmm::detail::Check(fmm::detail::GemmHost(A.data(), A.stride(), B.data(), B.stride(), C.data(), C.stride(), C.m(),
                                           A.n(), C.n(), C.multiplier(), beta));
}

// max_ij |a_ij - b_ij| / |a_ij| (linalg/linalg.hpp:280-295)
template <typename Scalar>
double MaxRelativeDiff(Matrix<Scalar>& A, Matrix<Scalar>& B) {
  double mx = 0.0;
  for (int j = 0; j < A.n(); ++j)
    for (int i = 0; i < A.m(); ++i) {
      const Scalar a = A(i, j), b = B(i, j);
      const Scalar d = std::abs(a - b) / std::abs(a);
      if (d > mx) mx = d;
    }
  return mx;
}

// max_ij |a_ij - b_ij|
template <typename Scalar>
double MaxAbsDiff(Matrix<Scalar>& A, Matrix<Scalar>& B) {
  double mx = 0.0;
  for (int j = 0; j < A.n(); ++j)
    for (int i = 0; i < A.m(); ++i) {
      const Scalar d = std::abs(A(i, j) - B(i, j));
      if (d > mx) mx = d;
    }
  return mx;
}

// Uniform [0, 1] entries from rand(), like linalg/linalg.hpp:422-433.
template <typename Scalar>
Matrix<Scalar> RandomMatrix(int m, int n) {
  Matrix<Scalar> A(m, n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) A(i, j) = static_cast<Scalar>(static_cast<double>(rand()) / RAND_MAX);
  return A;
}
