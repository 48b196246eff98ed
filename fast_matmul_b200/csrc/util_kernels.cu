// Seeded input generation and the max-relative-difference error metric.

#include <cuda_runtime.h>

#include <cstdint>

#include "fmm_internal.h"

namespace fmm {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// out(i, j) = lo + (hi - lo) * u(e), e = i + j * rows: a counter-based
// splitmix64 stream, bit-identical to the host generator of the tests.
__global__ void fill_uniform_kernel(double* out, int64_t rows, int64_t cols, int64_t ld, uint64_t seed,
                                    uint64_t stream_id, double lo, double hi) {
  const uint64_t key = seed * 0xD1B54A32D192ED03ULL + stream_id * 0x8CB92BA72F3D8DD7ULL;
  const int64_t total = rows * cols;
  const double span = __dsub_rn(hi, lo);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t z = mix64(key + (uint64_t)(e + 1) * 0x9E3779B97F4A7C15ULL);
    const double u = __dmul_rn((double)(z >> 11), 1.0 / 9007199254740992.0);
    const int64_t j = e / rows, i = e - j * rows;
    out[i + j * ld] = __dadd_rn(lo, __dmul_rn(span, u));
  }
}

// Non-negative doubles order like their bit patterns, so an unsigned max
// over the bits is a max over the values (NaN terms are skipped, as in the
// reference's `curr > max` comparison).
__global__ void max_rel_diff_kernel(const double* a, int64_t lda, const double* b, int64_t ldb, int64_t m, int64_t n,
                                    unsigned long long* out) {
  double best_rel = 0.0, best_abs = 0.0;
  const int64_t total = m * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / m, i = e - j * m;
    const double x = a[i + j * lda], y = b[i + j * ldb];
    const double d = fabs(x - y);
    const double r = d / fabs(x);
    if (r > best_rel) best_rel = r;
    if (d > best_abs) best_abs = d;
  }
  for (int off = 16; off > 0; off >>= 1) {
    const double o1 = __shfl_xor_sync(0xffffffffu, best_rel, off);
    const double o2 = __shfl_xor_sync(0xffffffffu, best_abs, off);
    if (o1 > best_rel) best_rel = o1;
    if (o2 > best_abs) best_abs = o2;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, (unsigned long long)__double_as_longlong(best_rel));
    atomicMax(out + 1, (unsigned long long)__double_as_longlong(best_abs));
  }
}

}  // namespace

cudaError_t fill_uniform_launch(double* out, int64_t rows, int64_t cols, int64_t ld, uint64_t seed, uint64_t stream_id,
                                double lo, double hi, cudaStream_t stream) {
  const int64_t total = rows * cols;
  if (total <= 0) return cudaSuccess;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  fill_uniform_kernel<<<(unsigned)blocks, 256, 0, stream>>>(out, rows, cols, ld, seed, stream_id, lo, hi);
  return cudaGetLastError();
}

cudaError_t max_rel_diff_launch(const double* a, int64_t lda, const double* b, int64_t ldb, int64_t m, int64_t n,
                                double* d_out, cudaStream_t stream) {
  cudaError_t err = cudaMemsetAsync(d_out, 0, 2 * sizeof(double), stream);
  if (err != cudaSuccess) return err;
  const int64_t total = m * n;
  if (total <= 0) return cudaSuccess;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  max_rel_diff_kernel<<<(unsigned)blocks, 256, 0, stream>>>(a, lda, b, ldb, m, n,
                                                           reinterpret_cast<unsigned long long*>(d_out));
  return cudaGetLastError();
}

}  // namespace fmm
