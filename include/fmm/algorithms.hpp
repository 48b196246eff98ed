// Generated by fast_matmul_b200/codegen/gen_cuda.py from the fast-matmul coefficient files. Do not edit.
// The reference's per-algorithm entry points (one namespace per generated
// header, e.g. algorithms/strassen.hpp:661-722), routed to the B200 engine.
#pragma once
#include "fmm/matrix.hpp"

namespace fmm {
enum AlgorithmId {
  kAlg_strassen = 0,
  kAlg_classical222_8_24 = 1,
  kAlg_grey322_11_50 = 2,
  kAlg_bini322_10_52_approx = 3,
  kAlg_grey332_15_103 = 4,
  kAlg_grey323_15_103 = 5,
  kAlg_hk332_15_94 = 6,
  kAlg_hk323_15_94 = 7,
  kAlg_hk323_15_84 = 8,
  kAlg_grey323_15_89 = 9,
  kAlg_grey333_23_152 = 10,
  kAlg_grey333_23_221 = 11,
  kAlg_grey333_23_125 = 12,
  kAlg_smirnov333_23_139 = 13,
  kAlg_smirnov333_23_128 = 14,
  kAlg_classical333_27_81 = 15,
  kAlg_schonhage333_21_117_approx = 16,
  kAlg_smirnov333_20_182_approx = 17,
  kAlg_grey422_14_84 = 18,
  kAlg_grey432_20_144 = 19,
  kAlg_grey423_20_144 = 20,
  kAlg_grey324_20_144 = 21,
  kAlg_grey342_20_144 = 22,
  kAlg_grey234_20_144 = 23,
  kAlg_grey243_20_144 = 24,
  kAlg_classical423_24_72 = 25,
  kAlg_fast423_130 = 26,
  kAlg_fast423_134 = 27,
  kAlg_fast423_138 = 28,
  kAlg_fast423_156 = 29,
  kAlg_grey433_29_234 = 30,
  kAlg_grey343_29_234 = 31,
  kAlg_grey442_26_257 = 32,
  kAlg_grey424_26_257 = 33,
  kAlg_grey424_26_206 = 34,
  kAlg_grey522_18_99 = 35,
  kAlg_grey252_18_99 = 36,
  kAlg_smirnov336_40_960 = 37,
  kAlg_smirnov363_40_960 = 38,
  kAlg_smirnov633_40_960 = 39,
  kAlg_tichavsky_kovac336_40_960 = 40,
  kAlg_tichavsky_kovac363_40_960 = 41,
};
}  // namespace fmm

namespace strassen {
// C := alpha * A * B + beta * C with <2,2,2;7>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_strassen, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace strassen

namespace classical222_8_24 {
// C := alpha * A * B + beta * C with <2,2,2;8>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_classical222_8_24, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace classical222_8_24

namespace grey322_11_50 {
// C := alpha * A * B + beta * C with <3,2,2;11>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey322_11_50, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey322_11_50

namespace bini322_10_52_approx {
// C := alpha * A * B + beta * C with <3,2,2;10>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_bini322_10_52_approx, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace bini322_10_52_approx

namespace grey332_15_103 {
// C := alpha * A * B + beta * C with <3,3,2;15>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey332_15_103, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey332_15_103

namespace grey323_15_103 {
// C := alpha * A * B + beta * C with <3,2,3;15>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey323_15_103, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey323_15_103

namespace hk332_15_94 {
// C := alpha * A * B + beta * C with <3,3,2;15>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_hk332_15_94, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace hk332_15_94

namespace hk323_15_94 {
// C := alpha * A * B + beta * C with <3,2,3;15>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_hk323_15_94, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace hk323_15_94

namespace hk323_15_84 {
// C := alpha * A * B + beta * C with <3,2,3;15>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_hk323_15_84, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace hk323_15_84

namespace grey323_15_89 {
// C := alpha * A * B + beta * C with <3,2,3;15>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey323_15_89, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey323_15_89

namespace grey333_23_152 {
// C := alpha * A * B + beta * C with <3,3,3;23>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey333_23_152, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey333_23_152

namespace grey333_23_221 {
// C := alpha * A * B + beta * C with <3,3,3;23>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey333_23_221, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey333_23_221

namespace grey333_23_125 {
// C := alpha * A * B + beta * C with <3,3,3;23>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey333_23_125, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey333_23_125

namespace smirnov333_23_139 {
// C := alpha * A * B + beta * C with <3,3,3;23>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_smirnov333_23_139, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace smirnov333_23_139

namespace smirnov333_23_128 {
// C := alpha * A * B + beta * C with <3,3,3;23>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_smirnov333_23_128, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace smirnov333_23_128

namespace classical333_27_81 {
// C := alpha * A * B + beta * C with <3,3,3;27>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_classical333_27_81, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace classical333_27_81

namespace schonhage333_21_117_approx {
// C := alpha * A * B + beta * C with <3,3,3;21>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_schonhage333_21_117_approx, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace schonhage333_21_117_approx

namespace smirnov333_20_182_approx {
// C := alpha * A * B + beta * C with <3,3,3;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_smirnov333_20_182_approx, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace smirnov333_20_182_approx

namespace grey422_14_84 {
// C := alpha * A * B + beta * C with <4,2,2;14>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey422_14_84, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey422_14_84

namespace grey432_20_144 {
// C := alpha * A * B + beta * C with <4,3,2;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey432_20_144, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey432_20_144

namespace grey423_20_144 {
// C := alpha * A * B + beta * C with <4,2,3;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey423_20_144, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey423_20_144

namespace grey324_20_144 {
// C := alpha * A * B + beta * C with <3,2,4;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey324_20_144, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey324_20_144

namespace grey342_20_144 {
// C := alpha * A * B + beta * C with <3,4,2;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey342_20_144, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey342_20_144

namespace grey234_20_144 {
// C := alpha * A * B + beta * C with <2,3,4;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey234_20_144, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey234_20_144

namespace grey243_20_144 {
// C := alpha * A * B + beta * C with <2,4,3;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey243_20_144, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey243_20_144

namespace classical423_24_72 {
// C := alpha * A * B + beta * C with <4,2,3;24>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_classical423_24_72, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace classical423_24_72

namespace fast423_130 {
// C := alpha * A * B + beta * C with <4,2,3;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_fast423_130, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace fast423_130

namespace fast423_134 {
// C := alpha * A * B + beta * C with <4,2,3;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_fast423_134, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace fast423_134

namespace fast423_138 {
// C := alpha * A * B + beta * C with <4,2,3;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_fast423_138, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace fast423_138

namespace fast423_156 {
// C := alpha * A * B + beta * C with <4,2,3;20>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_fast423_156, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace fast423_156

namespace grey433_29_234 {
// C := alpha * A * B + beta * C with <4,3,3;29>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey433_29_234, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey433_29_234

namespace grey343_29_234 {
// C := alpha * A * B + beta * C with <3,4,3;29>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey343_29_234, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey343_29_234

namespace grey442_26_257 {
// C := alpha * A * B + beta * C with <4,4,2;26>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey442_26_257, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey442_26_257

namespace grey424_26_257 {
// C := alpha * A * B + beta * C with <4,2,4;26>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey424_26_257, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey424_26_257

namespace grey424_26_206 {
// C := alpha * A * B + beta * C with <4,2,4;26>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey424_26_206, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey424_26_206

namespace grey522_18_99 {
// C := alpha * A * B + beta * C with <5,2,2;18>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey522_18_99, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey522_18_99

namespace grey252_18_99 {
// C := alpha * A * B + beta * C with <2,5,2;18>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_grey252_18_99, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace grey252_18_99

namespace smirnov336_40_960 {
// C := alpha * A * B + beta * C with <3,3,6;40>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_smirnov336_40_960, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace smirnov336_40_960

namespace smirnov363_40_960 {
// C := alpha * A * B + beta * C with <3,6,3;40>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_smirnov363_40_960, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace smirnov363_40_960

namespace smirnov633_40_960 {
// C := alpha * A * B + beta * C with <6,3,3;40>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_smirnov633_40_960, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace smirnov633_40_960

namespace tichavsky_kovac336_40_960 {
// C := alpha * A * B + beta * C with <3,3,6;40>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_tichavsky_kovac336_40_960, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace tichavsky_kovac336_40_960

namespace tichavsky_kovac363_40_960 {
// C := alpha * A * B + beta * C with <3,6,3;40>, num_steps recursive levels.
template <typename Scalar>
double FastMatmul(Matrix<Scalar>& A, Matrix<Scalar>& B, Matrix<Scalar>& C, int num_steps,
                  double x = 1e-8, Scalar alpha = Scalar(1.0), Scalar beta = Scalar(0.0)) {
  return ::fmm::detail::RunFastMatmul(::fmm::kAlg_tichavsky_kovac363_40_960, A, B, C, num_steps, x, alpha, beta);
}
}  // namespace tichavsky_kovac363_40_960
