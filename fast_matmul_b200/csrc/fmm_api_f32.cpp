// FP32 entry points: <ns>::FastMatmul and MatMul with Scalar = float.
//
// The operands are widened to FP64 once (exact), the FP64 engine runs on
// them -- by default with split-INT8 leaf products of 5 slices, 34 bits per
// operand entry against FP32's 24 -- and the result is rounded to FP32 once.
// The reference computes every addition and leaf product in FP32
// (Scalar = float, algorithms/*.hpp; sgemm, linalg/blas_wrap.hpp:116-120),
// so these results are at least as accurate as the reference's.

#include <cuda_runtime.h>

#include <chrono>

#include "api_internal.h"
#include "fmm.h"
#include "fmm_internal.h"

using fmm::api::check_alg;
using fmm::api::check_dims;
using fmm::api::DeviceGuard;
using fmm::api::ensure_device_buffer;
using fmm::api::fail;

namespace {

size_t pad32(size_t v) { return (v + 31) & ~(size_t)31; }

void f32_options(const fmm_options* opts, fmm_options* o) {
  fmm_options_init(o);
  if (opts) {
    *o = *opts;
  } else {
    o->precision = FMM_PRECISION_SPLIT_INT8;
    o->split_slices = FMM_F32_DEFAULT_SLICES;
  }
}

// FP64 staging for m x k, k x n and m x n operands in the handle.
fmm_status stage(fmm_handle h, int64_t m, int64_t k, int64_t n, double** a, double** b, double** c) {
  const size_t na = pad32((size_t)m * (size_t)k), nb = pad32((size_t)k * (size_t)n), nc = pad32((size_t)m * (size_t)n);
  fmm_status s = ensure_device_buffer(h, &h->wide, &h->wide_cap, (na + nb + nc) * sizeof(double), "FP64 staging");
  if (s != FMM_OK) return s;
  *a = static_cast<double*>(h->wide);
  *b = *a + na;
  *c = *b + nb;
  return FMM_OK;
}

// Widens A, B (and C when it is read) into the staging; ld of the staged
// matrices is their row count.
fmm_status widen_operands(fmm_handle h, const float* A, int64_t lda, const float* B, int64_t ldb, const float* C,
                          int64_t ldc, int64_t m, int64_t k, int64_t n, bool read_c, double* a, double* b,
                          double* c) {
  FMM_CUDA_TRY(fmm::widen_launch(A, lda, a, m > 1 ? m : 1, m, k, h->num_sms, h->stream), "widen A");
  FMM_CUDA_TRY(fmm::widen_launch(B, ldb, b, k > 1 ? k : 1, k, n, h->num_sms, h->stream), "widen B");
  h->launches += (m * k > 0) + (k * n > 0);
  if (read_c) {
    FMM_CUDA_TRY(fmm::widen_launch(C, ldc, c, m > 1 ? m : 1, m, n, h->num_sms, h->stream), "widen C");
    ++h->launches;
  }
  return FMM_OK;
}

fmm_status narrow_result(fmm_handle h, const double* c, float* C, int64_t ldc, int64_t m, int64_t n) {
  FMM_CUDA_TRY(fmm::narrow_launch(c, m > 1 ? m : 1, C, ldc, m, n, h->num_sms, h->stream), "round C to FP32");
  ++h->launches;
  return FMM_OK;
}

// Device FP32 copies of host operands (for the _host entry points).
fmm_status stage_host(fmm_handle h, const float* A, int64_t lda, const float* B, int64_t ldb, const float* C,
                      int64_t ldc, int64_t m, int64_t k, int64_t n, bool read_c, float** a, float** b, float** c) {
  const size_t na = pad32((size_t)m * (size_t)k), nb = pad32((size_t)k * (size_t)n), nc = pad32((size_t)m * (size_t)n);
  fmm_status s =
      ensure_device_buffer(h, &h->narrow_io, &h->narrow_io_cap, (na + nb + nc) * sizeof(float), "host-call operands");
  if (s != FMM_OK) return s;
  *a = static_cast<float*>(h->narrow_io);
  *b = *a + na;
  *c = *b + nb;
  const int64_t lda_d = m > 1 ? m : 1, ldb_d = k > 1 ? k : 1;
  if (m * k > 0)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(*a, lda_d * sizeof(float), A, lda * sizeof(float), m * sizeof(float), k,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy A to device");
  if (k * n > 0)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(*b, ldb_d * sizeof(float), B, ldb * sizeof(float), k * sizeof(float), n,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy B to device");
  if (read_c)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(*c, lda_d * sizeof(float), C, ldc * sizeof(float), m * sizeof(float), n,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy C to device");
  return FMM_OK;
}

fmm_status copy_back(fmm_handle h, const float* c, float* C, int64_t ldc, int64_t m, int64_t n) {
  FMM_CUDA_TRY(cudaMemcpy2DAsync(C, ldc * sizeof(float), c, (m > 1 ? m : 1) * sizeof(float), m * sizeof(float), n,
                                 cudaMemcpyDeviceToHost, h->stream),
               "copy C to host");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  return FMM_OK;
}

}  // namespace

extern "C" {

fmm_status fmm_fast_matmul_f32(fmm_handle h, int alg, const float* A, int64_t lda, const float* B, int64_t ldb,
                               float* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                               float alpha, float beta, const fmm_options* opts) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_alg(alg);
  if (s != FMM_OK) return s;
  if ((s = check_dims(m, k, n, lda, ldb, ldc)) != FMM_OK) return s;
  if (num_steps < 0 || num_steps > 16) return fail(FMM_ERR_INVALID_ARGUMENT, "num_steps must be in [0, 16]");
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  fmm_options o;
  f32_options(opts, &o);
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  double *a, *b, *c;
  if ((s = stage(h, m, k, n, &a, &b, &c)) != FMM_OK) return s;
  // FastMatmul with num_steps == 0 ignores beta (one classical product)
  const bool read_c = beta != 0.0f && num_steps > 0;
  if ((s = widen_operands(h, A, lda, B, ldb, C, ldc, m, k, n, read_c, a, b, c)) != FMM_OK) return s;
  s = fmm_fast_matmul(h, alg, a, m > 1 ? m : 1, b, k > 1 ? k : 1, c, m > 1 ? m : 1, m, k, n, num_steps, x,
                      (double)alpha, (double)beta, &o);
  if (s != FMM_OK) return s;
  return narrow_result(h, c, C, ldc, m, n);
}

fmm_status fmm_sgemm(fmm_handle h, const float* A, int64_t lda, const float* B, int64_t ldb, float* C, int64_t ldc,
                     int64_t m, int64_t k, int64_t n, float alpha, float beta, const fmm_options* opts) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_dims(m, k, n, lda, ldb, ldc);
  if (s != FMM_OK) return s;
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  fmm_options o;
  f32_options(opts, &o);
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  double *a, *b, *c;
  if ((s = stage(h, m, k, n, &a, &b, &c)) != FMM_OK) return s;
  const bool read_c = beta != 0.0f;
  if ((s = widen_operands(h, A, lda, B, ldb, C, ldc, m, k, n, read_c, a, b, c)) != FMM_OK) return s;
  const int64_t lm = m > 1 ? m : 1, lk = k > 1 ? k : 1;
  if (o.precision == FMM_PRECISION_SPLIT_BF16)
    s = fmm_dgemm_split_bf16(h, a, lm, b, lk, c, lm, m, k, n, (double)alpha, (double)beta, o.split_slices);
  else if (o.precision == FMM_PRECISION_SPLIT_INT8)
    s = fmm_dgemm_split_int8(h, a, lm, b, lk, c, lm, m, k, n, (double)alpha, (double)beta, o.split_slices);
  else
    s = fmm_dgemm(h, a, lm, b, lk, c, lm, m, k, n, (double)alpha, (double)beta);
  if (s != FMM_OK) return s;
  return narrow_result(h, c, C, ldc, m, n);
}

fmm_status fmm_fast_matmul_f32_host(fmm_handle h, int alg, const float* A, int64_t lda, const float* B, int64_t ldb,
                                    float* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                                    float alpha, float beta, const fmm_options* opts, double* elapsed_ms) {
  auto t0 = std::chrono::steady_clock::now();
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_alg(alg);
  if (s != FMM_OK) return s;
  if ((s = check_dims(m, k, n, lda, ldb, ldc)) != FMM_OK) return s;
  if (num_steps < 0 || num_steps > 16) return fail(FMM_ERR_INVALID_ARGUMENT, "num_steps must be in [0, 16]");
  if (m == 0 || n == 0) {
    if (elapsed_ms) *elapsed_ms = 0.0;
    return FMM_OK;
  }
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  float *a, *b, *c;
  const bool read_c = beta != 0.0f && num_steps > 0;
  if ((s = stage_host(h, A, lda, B, ldb, C, ldc, m, k, n, read_c, &a, &b, &c)) != FMM_OK) return s;
  const int64_t lm = m > 1 ? m : 1, lk = k > 1 ? k : 1;
  s = fmm_fast_matmul_f32(h, alg, a, lm, b, lk, c, lm, m, k, n, num_steps, x, alpha, beta, opts);
  if (s != FMM_OK) return s;
  if ((s = copy_back(h, c, C, ldc, m, n)) != FMM_OK) return s;
  if (elapsed_ms)
    *elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return FMM_OK;
}

fmm_status fmm_sgemm_host(fmm_handle h, const float* A, int64_t lda, const float* B, int64_t ldb, float* C,
                          int64_t ldc, int64_t m, int64_t k, int64_t n, float alpha, float beta,
                          const fmm_options* opts) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_dims(m, k, n, lda, ldb, ldc);
  if (s != FMM_OK) return s;
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  float *a, *b, *c;
  const bool read_c = beta != 0.0f;
  if ((s = stage_host(h, A, lda, B, ldb, C, ldc, m, k, n, read_c, &a, &b, &c)) != FMM_OK) return s;
  const int64_t lm = m > 1 ? m : 1, lk = k > 1 ? k : 1;
  s = fmm_sgemm(h, a, lm, b, lk, c, lm, m, k, n, alpha, beta, opts);
  if (s != FMM_OK) return s;
  return copy_back(h, c, C, ldc, m, n);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Diagonal scaling with Scalar = float: Scaling<float> / PostProcessScaling
// (scaling/scaling.hpp:143-196), as the reference's scaling/fast_scaling.cpp
// runs it on Matrix<float>.

extern "C" {

fmm_status fmm_diagonal_scaling_f32(fmm_handle h, float* A, int64_t lda, float* B, int64_t ldb, int64_t m, int64_t k,
                                    int64_t n, int num_steps, int type, float* r, float* s) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status st = check_dims(m, k, n, lda, ldb, m > 1 ? m : 1);
  if (st != FMM_OK) return st;
  if (num_steps < 0) return fail(FMM_ERR_INVALID_ARGUMENT, "num_steps must be >= 0");
  if (type < FMM_SCALING_OUTSIDE_INSIDE || type > FMM_SCALING_OUTSIDE)
    return fail(FMM_ERR_INVALID_ARGUMENT, "Unknown iteration type.");
  if ((m > 0 && !r) || (n > 0 && !s)) return fail(FMM_ERR_INVALID_ARGUMENT, "null factor pointer");
  if ((m * k > 0 && !A) || (k * n > 0 && !B)) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  st = ensure_device_buffer(h, &h->scal, &h->scal_cap, fmm::scaling_scratch_bytes(m, k, n), "scaling scratch");
  if (st != FMM_OK) return st;
  FMM_CUDA_TRY(fmm::scaling_launch(A, lda, B, ldb, (int)m, (int)k, (int)n, num_steps, type, r, s, h->scal, h->stream,
                                   &h->launches),
               "diagonal scaling");
  return FMM_OK;
}

fmm_status fmm_scaling_postprocess_f32(fmm_handle h, float* C, int64_t ldc, int64_t m, int64_t n, const float* r,
                                       const float* s) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status st = check_dims(m, 0, n, m > 1 ? m : 1, 1, ldc);
  if (st != FMM_OK) return st;
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || !r || !s) return fail(FMM_ERR_INVALID_ARGUMENT, "null pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  FMM_CUDA_TRY(fmm::scaling_postprocess_launch(C, ldc, (int)m, (int)n, r, s, h->stream, &h->launches),
               "scaling postprocess");
  return FMM_OK;
}

fmm_status fmm_diagonal_scaling_f32_host(fmm_handle h, float* A, int64_t lda, float* B, int64_t ldb, int64_t m,
                                         int64_t k, int64_t n, int num_steps, int type, float* r, float* s) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status st = check_dims(m, k, n, lda, ldb, m > 1 ? m : 1);
  if (st != FMM_OK) return st;
  if ((m > 0 && !r) || (n > 0 && !s)) return fail(FMM_ERR_INVALID_ARGUMENT, "null factor pointer");
  if ((m * k > 0 && !A) || (k * n > 0 && !B)) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  const size_t na = pad32((size_t)m * (size_t)k), nb = pad32((size_t)k * (size_t)n);
  if ((st = ensure_device_buffer(h, &h->narrow_io, &h->narrow_io_cap,
                                 (na + nb + pad32((size_t)m) + pad32((size_t)n)) * sizeof(float),
                                 "host-call operands")) != FMM_OK)
    return st;
  float* dA = static_cast<float*>(h->narrow_io);
  float* dB = dA + na;
  float* dr = dB + nb;
  float* ds = dr + pad32((size_t)m);
  const int64_t ldA = m > 1 ? m : 1, ldB = k > 1 ? k : 1;
  if (m * k > 0)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dA, ldA * sizeof(float), A, lda * sizeof(float), m * sizeof(float), k,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy A to device");
  if (k * n > 0)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dB, ldB * sizeof(float), B, ldb * sizeof(float), k * sizeof(float), n,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy B to device");
  if (m) FMM_CUDA_TRY(cudaMemcpyAsync(dr, r, m * sizeof(float), cudaMemcpyHostToDevice, h->stream), "copy r");
  if (n) FMM_CUDA_TRY(cudaMemcpyAsync(ds, s, n * sizeof(float), cudaMemcpyHostToDevice, h->stream), "copy s");
  st = fmm_diagonal_scaling_f32(h, dA, ldA, dB, ldB, m, k, n, num_steps, type, dr, ds);
  if (st != FMM_OK) return st;
  if (m * k > 0)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(A, lda * sizeof(float), dA, ldA * sizeof(float), m * sizeof(float), k,
                                   cudaMemcpyDeviceToHost, h->stream),
                 "copy A to host");
  if (k * n > 0)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(B, ldb * sizeof(float), dB, ldB * sizeof(float), k * sizeof(float), n,
                                   cudaMemcpyDeviceToHost, h->stream),
                 "copy B to host");
  if (m) FMM_CUDA_TRY(cudaMemcpyAsync(r, dr, m * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "copy r back");
  if (n) FMM_CUDA_TRY(cudaMemcpyAsync(s, ds, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "copy s back");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  return FMM_OK;
}

fmm_status fmm_scaling_postprocess_f32_host(fmm_handle h, float* C, int64_t ldc, int64_t m, int64_t n,
                                            const float* r, const float* s) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status st = check_dims(m, 0, n, m > 1 ? m : 1, 1, ldc);
  if (st != FMM_OK) return st;
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || !r || !s) return fail(FMM_ERR_INVALID_ARGUMENT, "null pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  const size_t nc = pad32((size_t)m * (size_t)n);
  if ((st = ensure_device_buffer(h, &h->narrow_io, &h->narrow_io_cap,
                                 (nc + pad32((size_t)m) + pad32((size_t)n)) * sizeof(float),
                                 "host-call operands")) != FMM_OK)
    return st;
  float* dC = static_cast<float*>(h->narrow_io);
  float* dr = dC + nc;
  float* ds = dr + pad32((size_t)m);
  FMM_CUDA_TRY(cudaMemcpy2DAsync(dC, m * sizeof(float), C, ldc * sizeof(float), m * sizeof(float), n,
                                 cudaMemcpyHostToDevice, h->stream),
               "copy C to device");
  FMM_CUDA_TRY(cudaMemcpyAsync(dr, r, m * sizeof(float), cudaMemcpyHostToDevice, h->stream), "copy r");
  FMM_CUDA_TRY(cudaMemcpyAsync(ds, s, n * sizeof(float), cudaMemcpyHostToDevice, h->stream), "copy s");
  st = fmm_scaling_postprocess_f32(h, dC, m, m, n, dr, ds);
  if (st != FMM_OK) return st;
  FMM_CUDA_TRY(cudaMemcpy2DAsync(C, ldc * sizeof(float), dC, m * sizeof(float), m * sizeof(float), n,
                                 cudaMemcpyDeviceToHost, h->stream),
               "copy C to host");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  return FMM_OK;
}

}  // extern "C"
