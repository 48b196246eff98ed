// Element conversions between FP32 and FP64 column-major matrices, for the
// FP32 entry points: their operands are widened once into FP64 staging, the
// engine runs there, and the result is rounded back to FP32 once.

#include <cuda_runtime.h>

#include <cstdint>

#include "fmm_internal.h"

namespace fmm {
namespace {

// One thread per element, rows fastest (consecutive threads read and write
// consecutive addresses of a column).
__global__ void widen_kernel(const float* __restrict__ src, int64_t lds, double* __restrict__ dst, int64_t ldd,
                             int64_t rows, int64_t cols) {
  const int64_t total = rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / rows, i = e - j * rows;
    dst[i + j * ldd] = (double)src[i + j * lds];  // exact
  }
}

// Round to nearest (ties to even), the IEEE conversion.
__global__ void narrow_kernel(const double* __restrict__ src, int64_t lds, float* __restrict__ dst, int64_t ldd,
                              int64_t rows, int64_t cols) {
  const int64_t total = rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / rows, i = e - j * rows;
    dst[i + j * ldd] = __double2float_rn(src[i + j * lds]);
  }
}

unsigned grid_of(int64_t total, int num_sms) {
  const int64_t want = (total + 255) / 256;
  const int64_t cap = (int64_t)num_sms * 32;
  return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

cudaError_t widen_launch(const float* src, int64_t lds, double* dst, int64_t ldd, int64_t rows, int64_t cols,
                         int num_sms, cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return cudaSuccess;
  widen_kernel<<<grid_of(rows * cols, num_sms), 256, 0, stream>>>(src, lds, dst, ldd, rows, cols);
  return cudaGetLastError();
}

cudaError_t narrow_launch(const double* src, int64_t lds, float* dst, int64_t ldd, int64_t rows, int64_t cols,
                          int num_sms, cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return cudaSuccess;
  narrow_kernel<<<grid_of(rows * cols, num_sms), 256, 0, stream>>>(src, lds, dst, ldd, rows, cols);
  return cudaGetLastError();
}

}  // namespace fmm
