// Operand formation (S/T) and product combination (M -> C) kernels.
//
// The reference evaluates every S_r, T_r and C_ij as its own loop nest over
// the block (S_Add*/T_Add*/M_Add*, e.g. algorithms/strassen.hpp:9-375), which
// re-reads each input block once per output that uses it.  Here one thread
// handles one element position (two with 16-byte vectors) of a block and
// produces ALL outputs of the level there: it loads the M0*K0 input blocks
// (or the R products) once, keeps common-subexpression temporaries in
// registers, and writes each output once -- the minimum HBM traffic for the
// level.  The per-algorithm arithmetic is emitted by codegen/gen_cuda.py in
// the reference's term order; the helpers below round every multiply and
// add separately (no contraction), so results are bit-identical to the
// reference's write-once additions.
//
// One launch covers every sub-problem of a breadth-first level: grid.y walks
// the sub-problems (S side, then T side), grid.x strides over block rows x
// columns.

#include <cuda_runtime.h>

#include <cstdint>

#include "device_checks.cuh"
#include "fmm_internal.h"

namespace fmm {
namespace {

__device__ __forceinline__ double fmm_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fmm_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fmm_mul(double c, double a) { return __dmul_rn(c, a); }
__device__ __forceinline__ double fmm_neg(double a) { return -a; }

__device__ __forceinline__ double2 fmm_add(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 fmm_sub(double2 a, double2 b) {
  return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
__device__ __forceinline__ double2 fmm_mul(double c, double2 a) {
  return make_double2(__dmul_rn(c, a.x), __dmul_rn(c, a.y));
}
__device__ __forceinline__ double2 fmm_neg(double2 a) { return make_double2(-a.x, -a.y); }

#include "generated/fmm_alg_kernels.cuh"

template <int VEC>
struct VecT;
template <>
struct VecT<1> {
  using T = double;
};
template <>
struct VecT<2> {
  using T = double2;
};

template <class T>
__device__ __forceinline__ T ld_block(const double* p) {
  return *reinterpret_cast<const T*>(p);
}
template <class T>
__device__ __forceinline__ void st_block(double* p, T v) {
  *reinterpret_cast<T*>(p) = v;
}

constexpr int kAddThreads = 128;

template <class ALG, int VEC>
__global__ void __launch_bounds__(kAddThreads) form_kernel(FormLaunch L, CoefSlots cf) {
  using T = typename VecT<VEC>::T;
  const int nall = L.n_s + L.n_t;
  for (int pp = blockIdx.y; pp < nall; pp += gridDim.y) {
    const bool s_side = pp < L.n_s;
    const FormDesc d = s_side ? L.s_desc[pp] : L.t_desc[pp - L.n_s];
    const int64_t rows = d.rows;
    const int64_t cols = d.cols;
    const int nbc = s_side ? ALG::kK0 : ALG::kN0;
    const int64_t rows_v = rows / VEC;
    const int64_t chunks = (rows_v + kAddThreads - 1) / kAddThreads;
    const int64_t items = chunks * cols;
    for (int64_t w = blockIdx.x; w < items; w += gridDim.x) {
      const int64_t j = w / chunks;
      const int64_t i = ((w - j * chunks) * kAddThreads + threadIdx.x) * VEC;
      if (i >= rows) continue;
      const double* in = d.in + i + j * d.ld_in;
      double* out = d.out + i + j * d.ld_out;
      auto ld = [&](int b) -> T {
        const int bi = b / nbc, bj = b % nbc;
        return ld_block<T>(in + bi * rows + bj * cols * d.ld_in);
      };
      auto st = [&](int o, T v) {
        double* p = out + o * d.out_stride;
        if (FMM_CHECK(FMM_IN_WORKSPACE(p, sizeof(T)), kCheckFormOut)) st_block<T>(p, v);
      };
      if (s_side)
        ALG::template form_s<T>(cf.v, ld, st);
      else
        ALG::template form_t<T>(cf.v, ld, st);
    }
  }
}

template <class ALG, int VEC>
__global__ void __launch_bounds__(kAddThreads) combine_kernel(CombineLaunch L, CoefSlots cf) {
  using T = typename VecT<VEC>::T;
  for (int p = blockIdx.y; p < L.n; p += gridDim.y) {
    const CombineDesc d = L.desc[p];
    const int64_t rows = d.rows, cols = d.cols;
    const int64_t rows_v = rows / VEC;
    const int64_t chunks = (rows_v + kAddThreads - 1) / kAddThreads;
    const int64_t items = chunks * cols;
    const bool with_beta = d.beta != 0.0;
    for (int64_t w = blockIdx.x; w < items; w += gridDim.x) {
      const int64_t j = w / chunks;
      const int64_t i = ((w - j * chunks) * kAddThreads + threadIdx.x) * VEC;
      if (i >= rows) continue;
      const double* mp = d.m + i + j * d.ld_m;
      double* cp = d.c + i + j * d.ld_c;
      auto ld = [&](int r) -> T {
        const double* p = mp + r * d.m_stride;
        return FMM_CHECK(FMM_IN_WORKSPACE(p, sizeof(T)), kCheckCombineIn) ? ld_block<T>(p) : T{};
      };
      auto cptr = [&](int c) -> double* {
        const int ci = c / ALG::kN0, cj = c % ALG::kN0;
        return cp + ci * rows + cj * cols * d.ld_c;
      };
      auto ldc = [&](int c) -> T { return ld_block<T>(cptr(c)); };
      auto st = [&](int c, T v) { st_block<T>(cptr(c), v); };
      if (with_beta)
        ALG::template combine<T, true>(cf.v, d.beta, ld, ldc, st);
      else
        ALG::template combine<T, false>(cf.v, 0.0, ld, ldc, st);
    }
  }
}

inline void add_grid(int64_t items_per_problem, int nprob, int num_sms, dim3* grid) {
  const int gy = nprob < 65535 ? nprob : 65535;
  int64_t target = (int64_t)num_sms * 16;  // resident 128-thread CTAs
  int64_t gx = target / gy;
  if (gx < 1) gx = 1;
  if (gx > items_per_problem) gx = items_per_problem;
  if (gx < 1) gx = 1;
  if (gx > 2147483647) gx = 2147483647;
  *grid = dim3((unsigned)gx, (unsigned)gy, 1);
}

template <class ALG>
cudaError_t launch_form(const FormLaunch& L, const CoefSlots& cf, bool vec2, int num_sms, cudaStream_t stream) {
  const int nall = L.n_s + L.n_t;
  if (nall == 0) return cudaSuccess;
  const int64_t it = L.max_items;
  if (it == 0) return cudaSuccess;
  dim3 grid;
  add_grid(it, nall, num_sms, &grid);
  if (vec2)
    form_kernel<ALG, 2><<<grid, kAddThreads, 0, stream>>>(L, cf);
  else
    form_kernel<ALG, 1><<<grid, kAddThreads, 0, stream>>>(L, cf);
  return cudaGetLastError();
}

template <class ALG>
cudaError_t launch_combine(const CombineLaunch& L, const CoefSlots& cf, bool vec2, int num_sms, cudaStream_t stream) {
  if (L.n == 0 || L.max_items == 0) return cudaSuccess;
  dim3 grid;
  add_grid(L.max_items, L.n, num_sms, &grid);
  if (vec2)
    combine_kernel<ALG, 2><<<grid, kAddThreads, 0, stream>>>(L, cf);
  else
    combine_kernel<ALG, 1><<<grid, kAddThreads, 0, stream>>>(L, cf);
  return cudaGetLastError();
}

}  // namespace

bool device_checks_built() { return kDeviceChecks; }

cudaError_t device_checks_arm(const void* ws, size_t bytes, cudaStream_t stream) {
  if (!kDeviceChecks) return cudaSuccess;
  const uintptr_t lo = reinterpret_cast<uintptr_t>(ws);
  cudaError_t e = fmm_checks_arm_tu(CheckRange{lo, ws ? lo + bytes : 0}, stream);
  if (e == cudaSuccess) e = gemm_checks_arm(ws, bytes, stream);
  if (e == cudaSuccess) e = thin_checks_arm(ws, bytes, stream);
  return e;
}

cudaError_t device_checks_take(unsigned* word) {
  *word = 0;
  cudaError_t e = fmm_checks_take_tu(word);
  if (e == cudaSuccess) e = gemm_checks_take(word);
  if (e == cudaSuccess) e = thin_checks_take(word);
  return e;
}

cudaError_t form_launch(int alg, const FormLaunch& L, const CoefSlots& cf, bool vec2, int num_sms,
                        cudaStream_t stream) {
  switch (alg) {
#define FMM_FORM_CASE(idx, ALG) \
  case idx:                     \
    return launch_form<ALG>(L, cf, vec2, num_sms, stream);
    FMM_FOR_EACH_ALGORITHM(FMM_FORM_CASE)
#undef FMM_FORM_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t combine_launch(int alg, const CombineLaunch& L, const CoefSlots& cf, bool vec2, int num_sms,
                           cudaStream_t stream) {
  switch (alg) {
#define FMM_COMBINE_CASE(idx, ALG) \
  case idx:                        \
    return launch_combine<ALG>(L, cf, vec2, num_sms, stream);
    FMM_FOR_EACH_ALGORITHM(FMM_COMBINE_CASE)
#undef FMM_COMBINE_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace fmm
