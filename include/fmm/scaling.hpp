// C++ drop-in for the reference's scaling/scaling.hpp: the scaling types,
// Scaling and PostProcessScaling over the adapter's host Matrix<double> or
// Matrix<float> (include/fmm/matrix.hpp), computed on the B200 through
// fmm_diagonal_scaling[_f32]_host / fmm_scaling_postprocess[_f32]_host
// (include/fmm.h).
// Results are the reference's bit for bit: every factor is the same
// correctly rounded division, square root or product.
#pragma once

#include <stdexcept>
#include <type_traits>
#include <vector>

#include "fmm/matrix.hpp"

// The reference's scaling types (scaling/scaling.hpp:19-24).
enum {
  OUTSIDE_INSIDE = FMM_SCALING_OUTSIDE_INSIDE,
  INSIDE_OUTSIDE = FMM_SCALING_INSIDE_OUTSIDE,
  INSIDE = FMM_SCALING_INSIDE,
  OUTSIDE = FMM_SCALING_OUTSIDE,
};

namespace fmm {
namespace detail {

inline fmm_status ScalingHost(double* A, int lda, double* B, int ldb, int m, int k, int n, int steps, int type,
                              double* r, double* s) {
  return fmm_diagonal_scaling_host(ThreadHandle(), A, lda, B, ldb, m, k, n, steps, type, r, s);
}

inline fmm_status ScalingHost(float* A, int lda, float* B, int ldb, int m, int k, int n, int steps, int type, float* r,
                              float* s) {
  return fmm_diagonal_scaling_f32_host(ThreadHandle(), A, lda, B, ldb, m, k, n, steps, type, r, s);
}

inline fmm_status PostHost(double* C, int ldc, int m, int n, const double* r, const double* s) {
  return fmm_scaling_postprocess_host(ThreadHandle(), C, ldc, m, n, r, s);
}

inline fmm_status PostHost(float* C, int ldc, int m, int n, const float* r, const float* s) {
  return fmm_scaling_postprocess_f32_host(ThreadHandle(), C, ldc, m, n, r, s);
}

}  // namespace detail
}  // namespace fmm

// C := diag(r_vals) * C * diag(s_vals), rows first (scaling/scaling.hpp:143-148).
template <typename Scalar>
void PostProcessScaling(Matrix<Scalar>& C, std::vector<Scalar>& r_vals, std::vector<Scalar>& s_vals) {
  static_assert(std::is_same<Scalar, double>::value || std::is_same<Scalar, float>::value,
                "the B200 engine computes with Scalar = double or float");
  if ((int)r_vals.size() < C.m() || (int)s_vals.size() < C.n())
    throw std::runtime_error("fmm: PostProcessScaling: factor vectors shorter than C");
  fmm::detail::Check(fmm::detail::PostHost(C.data(), C.stride(), C.m(), C.n(), r_vals.data(), s_vals.data()));
}

// num_steps steps of outer and / or inner scaling of A and B in place, the
// outer maxima multiplied into r_vals and s_vals (scaling/scaling.hpp:153-196).
template <typename Scalar>
void Scaling(Matrix<Scalar>& A, Matrix<Scalar>& B, int num_steps, std::vector<Scalar>& r_vals,
             std::vector<Scalar>& s_vals, int scaling_type) {
  static_assert(std::is_same<Scalar, double>::value || std::is_same<Scalar, float>::value,
                "the B200 engine computes with Scalar = double or float");
  r_vals.resize(A.height(), 1.0);
  s_vals.resize(B.width(), 1.0);
  if (scaling_type < OUTSIDE_INSIDE || scaling_type > OUTSIDE) throw std::runtime_error("Unknown iteration type.");
  fmm::detail::Check(fmm::detail::ScalingHost(A.data(), A.stride(), B.data(), B.stride(), A.m(), A.n(), B.n(),
                                              num_steps, scaling_type, r_vals.data(), s_vals.data()));
}
