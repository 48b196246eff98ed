// C ABI of the engine (include/fmm.h).  No exception crosses this boundary;
// every entry point returns an fmm_status and leaves a message for
// fmm_last_error() on failure.

#include "fmm.h"

#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "api_internal.h"
#include "fmm_internal.h"
#include "plan.h"

namespace fmm {
namespace api {

thread_local std::string g_last_error;

fmm_status fail(fmm_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

fmm_status cuda_fail(cudaError_t e, const char* where) {
  return fail(FMM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

}  // namespace api

void set_last_error(const std::string& msg) { api::g_last_error = msg; }

}  // namespace fmm

using namespace fmm::api;

namespace fmm {
namespace api {

fmm_status ensure_device_buffer(fmm_handle h, void** buf, size_t* cap, size_t need, const char* what) {
  if (need <= *cap) return FMM_OK;
  if (*buf) {
    // in-flight work on the handle's stream may still use the old buffer
    FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    cudaFree(*buf);
    *buf = nullptr;
    *cap = 0;
  }
  size_t alloc = need + need / 8;
  cudaError_t e = cudaMalloc(buf, alloc);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(buf, need);
    alloc = need;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *buf = nullptr;
    return fail(FMM_ERR_OUT_OF_MEMORY, std::string("cannot allocate ") + std::to_string(need) + " bytes of " + what);
  }
  *cap = alloc;
  return FMM_OK;
}

fmm_status stage_descriptors(fmm_handle h, const fmm::Program& prog) {
  const size_t need = prog.desc.size();
  if (need == 0) return FMM_OK;
  if (h->desc_pending) {
    FMM_CUDA_TRY(cudaEventSynchronize(h->desc_done), "cudaEventSynchronize");
    h->desc_pending = false;
  }
  if (need > h->h_desc_cap) {
    if (h->h_desc) cudaFreeHost(h->h_desc);
    h->h_desc = nullptr;
    h->h_desc_cap = 0;
    const size_t alloc = need + need / 4;
    FMM_CUDA_TRY(cudaMallocHost(&h->h_desc, alloc), "cudaMallocHost(descriptors)");
    h->h_desc_cap = alloc;
  }
  fmm_status s = ensure_device_buffer(h, &h->d_desc, &h->d_desc_cap, need, "launch descriptors");
  if (s != FMM_OK) return s;
  std::memcpy(h->h_desc, prog.desc.data(), need);
  return FMM_OK;
}

fmm_status run_staged(fmm_handle h, const fmm::Program& prog) {
  // desc_done marks the end of the descriptor copy: the pinned staging
  // buffer can take the next call's descriptors while this call still runs
  cudaError_t e = fmm::run_program(prog, h->h_desc, h->d_desc, h->num_sms, h->stream, &h->launches,
                                   h->profiling ? &h->prof : nullptr, h->d_err, h->desc_done);
  if (!prog.desc.empty()) h->desc_pending = true;
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  return FMM_OK;
}

fmm_status check_alg(int alg) {
  if (alg < 0 || alg >= FMM_NUM_ALGORITHMS)
    return fail(FMM_ERR_UNKNOWN_ALGORITHM, "unknown algorithm index " + std::to_string(alg));
  return FMM_OK;
}

fmm_status check_dims(int64_t m, int64_t k, int64_t n, int64_t lda, int64_t ldb, int64_t ldc) {
  if (m < 0 || k < 0 || n < 0) return fail(FMM_ERR_INVALID_ARGUMENT, "negative matrix dimension");
  if (m > 2147483647 || k > 2147483647 || n > 2147483647)
    return fail(FMM_ERR_INVALID_ARGUMENT, "matrix dimension above 2^31-1");
  if (lda < (m > 1 ? m : 1) || ldb < (k > 1 ? k : 1) || ldc < (m > 1 ? m : 1))
    return fail(FMM_ERR_INVALID_ARGUMENT, "leading dimension smaller than the number of rows");
  return FMM_OK;
}

void resolve_options(const fmm_options* opts, fmm_options* out) {
  fmm_options_init(out);
  if (opts) *out = *opts;
}

fmm_status split_slices_for(int precision, int requested, int* slices) {
  *slices = 0;
  if (precision == FMM_PRECISION_FP64) return FMM_OK;
  if (precision == FMM_PRECISION_SPLIT_INT8) {
    const int s = requested == 0 ? FMM_SPLIT_INT8_DEFAULT_SLICES : requested;
    if (s < FMM_SPLIT_MIN_SLICES || s > FMM_SPLIT_INT8_MAX_SLICES)
      return fail(FMM_ERR_INVALID_ARGUMENT, "split_slices must be in [2, 8] for SPLIT_INT8");
    *slices = fmm::kSplitInt8Code + s;
    return FMM_OK;
  }
  if (precision != FMM_PRECISION_SPLIT_BF16) return fail(FMM_ERR_INVALID_ARGUMENT, "unknown precision");
  const int s = requested == 0 ? FMM_SPLIT_DEFAULT_SLICES : requested;
  if (s < FMM_SPLIT_MIN_SLICES || s > FMM_SPLIT_MAX_SLICES)
    return fail(FMM_ERR_INVALID_ARGUMENT, "split_slices must be in [2, 6]");
  *slices = s;
  return FMM_OK;
}

fmm_status check_device_errors(fmm_handle h) {
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  int code = 0;
  FMM_CUDA_TRY(cudaMemcpy(&code, h->d_err, sizeof(int), cudaMemcpyDeviceToHost), "read device error word");
  if (code != 0) {
    FMM_CUDA_TRY(cudaMemset(h->d_err, 0, sizeof(int)), "clear device error word");
    return fail(FMM_ERR_TIMEOUT, "a split-BF16 tensor-core kernel gave up a bounded wait (code " +
                                     std::to_string(code) + "); its results are not valid");
  }
  return FMM_OK;
}

// Depth-first levels for a schedule: the fewest that fit the limit.
fmm_status choose_dfs_levels(fmm_handle h, int alg, int64_t m, int64_t k, int64_t n, int steps,
                             const fmm_options& o, int* dfs_levels, size_t* bytes) {
  const fmm_alg_table& t = fmm_algorithms[alg];
  const size_t limit = o.workspace_limit ? o.workspace_limit : h->ws_limit;
  int slices = 0;
  fmm_status ss = split_slices_for(o.precision, o.split_slices, &slices);
  if (ss != FMM_OK) return ss;
  auto fits = [&](int d, size_t* b) {
    *b = fmm::workspace_bytes(t, m, k, n, steps, d, slices);
    return *b <= limit;
  };
  switch (o.schedule) {
    case FMM_SCHEDULE_BFS:
      *dfs_levels = 0;
      *bytes = fmm::workspace_bytes(t, m, k, n, steps, 0, slices);
      break;
    case FMM_SCHEDULE_DFS:
      *dfs_levels = steps;
      *bytes = fmm::workspace_bytes(t, m, k, n, steps, steps, slices);
      break;
    case FMM_SCHEDULE_HYBRID:
    case FMM_SCHEDULE_AUTO: {
      if (o.schedule == FMM_SCHEDULE_HYBRID && o.dfs_levels >= 0) {
        if (o.dfs_levels > steps) return fail(FMM_ERR_INVALID_ARGUMENT, "dfs_levels exceeds num_steps");
        *dfs_levels = o.dfs_levels;
        *bytes = fmm::workspace_bytes(t, m, k, n, steps, o.dfs_levels, slices);
        break;
      }
      // dfs_levels 0 and 1 plan identically (the root level has a single
      // sub-problem); 2 is the first split that differs from BFS.  From 3
      // steps on, two depth-first levels above breadth-first ones measured
      // as fast as BFS or faster (16384^3 Strassen 46.1 either way; 16384 x
      // 1600 x 16384 grey333 16.4 against 14.9, 65536 x 2400 x 2400 14.1
      // against 12.9), so AUTO takes that split too.
      const int lo = steps >= 3 ? 2 : 0;
      int d = lo;
      size_t b = 0;
      while (d < steps && !fits(d, &b)) ++d;
      if (d == steps) fits(d, &b);
      *dfs_levels = d;
      *bytes = b;
      break;
    }
    default:
      return fail(FMM_ERR_INVALID_ARGUMENT, "unknown schedule");
  }
  if (*bytes > limit)
    return fail(FMM_ERR_OUT_OF_MEMORY, "workspace of " + std::to_string(*bytes) + " bytes exceeds the limit of " +
                                           std::to_string(limit) + " bytes");
  return FMM_OK;
}

}  // namespace api
}  // namespace fmm

extern "C" {

void fmm_options_init(fmm_options* opts) {
  if (!opts) return;
  opts->schedule = FMM_SCHEDULE_AUTO;
  opts->precision = FMM_PRECISION_FP64;
  opts->split_slices = 0;
  opts->dfs_levels = -1;
  opts->workspace_limit = 0;
  opts->gemm_tile = FMM_GEMM_TILE_AUTO;
}

const char* fmm_last_error(void) { return fmm::api::g_last_error.c_str(); }

fmm_status fmm_handle_create(fmm_handle* out, int device) {
  if (!out) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle pointer");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(FMM_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  if (device < 0 || device >= count) return fail(FMM_ERR_INVALID_ARGUMENT, "device index out of range");
  DeviceGuard g(device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  cudaDeviceProp prop;
  FMM_CUDA_TRY(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  if (prop.major != 10)
    return fail(FMM_ERR_NOT_SUPPORTED, std::string("device ") + prop.name + " is not sm_100 (B200)");
  fmm_handle h = new (std::nothrow) fmm_handle_s();
  if (!h) return fail(FMM_ERR_OUT_OF_MEMORY, "host allocation failed");
  h->device = device;
  h->num_sms = prop.multiProcessorCount;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = (size_t)8 << 30;
  h->ws_limit = (size_t)(0.6 * (double)free_b);
  if (cudaEventCreateWithFlags(&h->desc_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc(&h->d_small, 2 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->d_err, 256) != cudaSuccess || cudaMemset(h->d_err, 0, 256) != cudaSuccess) {
    cudaGetLastError();
    if (h->desc_done) cudaEventDestroy(h->desc_done);
    if (h->d_small) cudaFree(h->d_small);
  if (h->scal) cudaFree(h->scal);
  if (h->wide) cudaFree(h->wide);
  if (h->narrow_io) cudaFree(h->narrow_io);
    if (h->d_err) cudaFree(h->d_err);
    delete h;
    return fail(FMM_ERR_CUDA, "handle setup failed");
  }
  *out = h;
  return FMM_OK;
}

fmm_status fmm_handle_destroy(fmm_handle h) {
  if (!h) return FMM_OK;
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  if (h->ws) cudaFree(h->ws);
  if (h->d_desc) cudaFree(h->d_desc);
  if (h->h_desc) cudaFreeHost(h->h_desc);
  if (h->io) cudaFree(h->io);
  if (h->wide) cudaFree(h->wide);
  if (h->narrow_io) cudaFree(h->narrow_io);
  if (h->d2h) cudaStreamSynchronize(h->d2h);
  for (auto& sl : h->slots) {
    if (sl.io) cudaFree(sl.io);
    for (cudaEvent_t e : {sl.in_ready, sl.out_ready, sl.free})
      if (e) cudaEventDestroy(e);
  }
  if (h->h2d) cudaStreamDestroy(h->h2d);
  if (h->d2h) cudaStreamDestroy(h->d2h);
  if (h->d_small) cudaFree(h->d_small);
  if (h->scal) cudaFree(h->scal);
  if (h->d_err) cudaFree(h->d_err);
  if (h->desc_done) cudaEventDestroy(h->desc_done);
  delete h;
  return FMM_OK;
}

fmm_status fmm_debug_fill_workspace(fmm_handle h, size_t bytes, int pattern) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  if (pattern < 0 || pattern > 255) return fail(FMM_ERR_INVALID_ARGUMENT, "pattern must be a byte value");
  DeviceGuard g(h->device);
  fmm_status s = ensure_device_buffer(h, &h->ws, &h->ws_cap, bytes ? bytes : 256, "workspace");
  if (s != FMM_OK) return s;
  FMM_CUDA_TRY(cudaMemsetAsync(h->ws, pattern, h->ws_cap, h->stream), "cudaMemsetAsync(workspace)");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  return FMM_OK;
}

fmm_status fmm_debug_check_flags(unsigned* flags) {
  if (!flags) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  *flags = 0;
  if (!fmm::device_checks_built())
    return fail(FMM_ERR_NOT_SUPPORTED, "this library was built without device checks (FMM_DEVICE_CHECKS)");
  FMM_CUDA_TRY(fmm::device_checks_take(flags), "reading the device check word");
  return FMM_OK;
}

fmm_status fmm_release_workspace(fmm_handle h) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  DeviceGuard g(h->device);
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  if (h->d2h) FMM_CUDA_TRY(cudaStreamSynchronize(h->d2h), "cudaStreamSynchronize(copy-out)");
  void** bufs[] = {&h->ws, reinterpret_cast<void**>(&h->io), &h->wide, &h->narrow_io,
                   reinterpret_cast<void**>(&h->slots[0].io), reinterpret_cast<void**>(&h->slots[1].io)};
  size_t* caps[] = {&h->ws_cap, &h->io_cap, &h->wide_cap, &h->narrow_io_cap, &h->slots[0].cap, &h->slots[1].cap};
  for (int i = 0; i < 6; ++i) {
    if (*bufs[i]) cudaFree(*bufs[i]);
    *bufs[i] = nullptr;
    *caps[i] = 0;
  }
  h->slots[0].used = h->slots[1].used = false;
  return FMM_OK;
}

fmm_status fmm_set_stream(fmm_handle h, void* stream) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  h->stream = static_cast<cudaStream_t>(stream);
  return FMM_OK;
}

fmm_status fmm_set_workspace_limit(fmm_handle h, size_t bytes) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  if (bytes == 0) {
    DeviceGuard g(h->device);
    size_t free_b = 0, total_b = 0;
    FMM_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    bytes = (size_t)(0.6 * (double)(free_b + h->ws_cap));
  }
  h->ws_limit = bytes;
  return FMM_OK;
}

int fmm_num_algorithms(void) { return FMM_NUM_ALGORITHMS; }

const char* fmm_algorithm_name(int alg) {
  if (alg < 0 || alg >= FMM_NUM_ALGORITHMS) return nullptr;
  return fmm_algorithms[alg].name;
}

const char* fmm_algorithm_header(int alg) {
  if (alg < 0 || alg >= FMM_NUM_ALGORITHMS) return nullptr;
  return fmm_algorithms[alg].header;
}

int fmm_algorithm_lookup(const char* name) {
  if (!name) return -1;
  for (int i = 0; i < FMM_NUM_ALGORITHMS; ++i) {
    if (std::strcmp(fmm_algorithms[i].name, name) == 0) return i;
    if (std::strcmp(fmm_algorithms[i].header, name) == 0) return i;
    // header name without the .hpp suffix, e.g. "fast424_26_206"
    const char* hd = fmm_algorithms[i].header;
    const size_t len = std::strlen(hd);
    if (len > 4 && std::strlen(name) == len - 4 && std::strncmp(hd, name, len - 4) == 0) return i;
  }
  return -1;
}

fmm_status fmm_algorithm_info(int alg, int* m0, int* k0, int* n0, int* rank, int* approximate) {
  fmm_status s = check_alg(alg);
  if (s != FMM_OK) return s;
  const fmm_alg_table& t = fmm_algorithms[alg];
  if (m0) *m0 = t.m0;
  if (k0) *k0 = t.k0;
  if (n0) *n0 = t.n0;
  if (rank) *rank = t.rank;
  if (approximate) *approximate = t.approximate;
  return FMM_OK;
}

fmm_status fmm_workspace_query(fmm_handle h, int alg, int64_t m, int64_t k, int64_t n, int num_steps,
                               const fmm_options* opts, size_t* bytes) {
  if (!h || !bytes) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  fmm_status s = check_alg(alg);
  if (s != FMM_OK) return s;
  if (num_steps < 0) return fail(FMM_ERR_INVALID_ARGUMENT, "num_steps < 0");
  fmm_options o;
  resolve_options(opts, &o);
  int d = 0;
  return choose_dfs_levels(h, alg, m, k, n, num_steps, o, &d, bytes);
}

fmm_status fmm_fast_matmul(fmm_handle h, int alg, const double* A, int64_t lda, const double* B, int64_t ldb,
                           double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                           double alpha, double beta, const fmm_options* opts) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_alg(alg);
  if (s != FMM_OK) return s;
  if ((s = check_dims(m, k, n, lda, ldb, ldc)) != FMM_OK) return s;
  if (num_steps < 0 || num_steps > 16) return fail(FMM_ERR_INVALID_ARGUMENT, "num_steps must be in [0, 16]");
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  fmm_options o;
  resolve_options(opts, &o);
  int slices = 0;
  if ((s = split_slices_for(o.precision, o.split_slices, &slices)) != FMM_OK) return s;
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  int d = 0;
  size_t bytes = 0;
  if ((s = choose_dfs_levels(h, alg, m, k, n, num_steps, o, &d, &bytes)) != FMM_OK) return s;
  if ((s = ensure_device_buffer(h, &h->ws, &h->ws_cap, bytes ? bytes : 256, "workspace")) != FMM_OK) return s;
  try {
    fmm::build_program(alg, m, k, n, num_steps, x, alpha, beta, d, fmm::Operand{const_cast<double*>(A), lda},
                       fmm::Operand{const_cast<double*>(B), ldb}, fmm::Operand{C, ldc}, h->ws, &h->prog, slices,
                       o.gemm_tile);
  } catch (const std::exception& ex) {
    return fail(FMM_ERR_OUT_OF_MEMORY, std::string("planning failed: ") + ex.what());
  }
  if ((s = stage_descriptors(h, h->prog)) != FMM_OK) return s;
  return run_staged(h, h->prog);
}

fmm_status fmm_fast_matmul_host(fmm_handle h, int alg, const double* A, int64_t lda, const double* B, int64_t ldb,
                                double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                                double alpha, double beta, const fmm_options* opts, double* elapsed_ms) {
  auto t0 = std::chrono::steady_clock::now();
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_alg(alg);
  if (s != FMM_OK) return s;
  if ((h->slots[0].used || h->slots[1].used) && (s = fmm_host_sync(h)) != FMM_OK) return s;
  if ((s = check_dims(m, k, n, lda, ldb, ldc)) != FMM_OK) return s;
  if (m == 0 || n == 0) {
    if (elapsed_ms) *elapsed_ms = 0.0;
    return FMM_OK;
  }
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  const size_t na = (size_t)m * (size_t)k, nb = (size_t)k * (size_t)n, nc = (size_t)m * (size_t)n;
  void* io = h->io;
  size_t cap = h->io_cap;
  if ((s = ensure_device_buffer(h, &io, &cap, (na + nb + nc) * sizeof(double) + 512, "host-call operands")) != FMM_OK)
    return s;
  h->io = static_cast<double*>(io);
  h->io_cap = cap;
  double* dA = h->io;
  double* dB = dA + ((na + 31) & ~(size_t)31);
  double* dC = dB + ((nb + 31) & ~(size_t)31);
  const int64_t ldA = m, ldB = k > 0 ? k : 1, ldC = m;
  if (na)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dA, ldA * sizeof(double), A, lda * sizeof(double), m * sizeof(double), k,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy A to device");
  if (nb)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dB, ldB * sizeof(double), B, ldb * sizeof(double), k * sizeof(double), n,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy B to device");
  if (beta != 0.0 && num_steps > 0)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dC, ldC * sizeof(double), C, ldc * sizeof(double), m * sizeof(double), n,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy C to device");
  s = fmm_fast_matmul(h, alg, dA, ldA, dB, ldB, dC, ldC, m, k, n, num_steps, x, alpha, beta, opts);
  if (s != FMM_OK) return s;
  FMM_CUDA_TRY(cudaMemcpy2DAsync(C, ldc * sizeof(double), dC, ldC * sizeof(double), m * sizeof(double), n,
                                 cudaMemcpyDeviceToHost, h->stream),
               "copy C to host");
  if ((s = check_device_errors(h)) != FMM_OK) return s;
  if (elapsed_ms)
    *elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return FMM_OK;
}

fmm_status fmm_fast_matmul_host_async(fmm_handle h, int alg, const double* A, int64_t lda, const double* B,
                                      int64_t ldb, double* C, int64_t ldc, int64_t m, int64_t k, int64_t n,
                                      int num_steps, double x, double alpha, double beta, const fmm_options* opts) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_alg(alg);
  if (s != FMM_OK) return s;
  if ((s = check_dims(m, k, n, lda, ldb, ldc)) != FMM_OK) return s;
  if (num_steps < 0 || num_steps > 16) return fail(FMM_ERR_INVALID_ARGUMENT, "num_steps must be in [0, 16]");
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  if (!h->h2d) {
    FMM_CUDA_TRY(cudaStreamCreateWithFlags(&h->h2d, cudaStreamNonBlocking), "cudaStreamCreate(copy-in)");
    FMM_CUDA_TRY(cudaStreamCreateWithFlags(&h->d2h, cudaStreamNonBlocking), "cudaStreamCreate(copy-out)");
    for (auto& sl : h->slots)
      for (cudaEvent_t* e : {&sl.in_ready, &sl.out_ready, &sl.free})
        FMM_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
  }
  fmm_handle_s::HostSlot& sl = h->slots[h->next_slot];
  fmm_handle_s::HostSlot& other = h->slots[h->next_slot ^ 1];
  const size_t na = (size_t)m * (size_t)k, nb = (size_t)k * (size_t)n, nc = (size_t)m * (size_t)n;
  const size_t need = (((na + 31) & ~(size_t)31) + ((nb + 31) & ~(size_t)31) + nc) * sizeof(double) + 512;
  if (need > sl.cap) {
    // the slot's previous call must be finished before its buffer goes
    if (sl.used) FMM_CUDA_TRY(cudaEventSynchronize(sl.free), "cudaEventSynchronize(slot)");
    if (sl.io) cudaFree(sl.io);
    sl.io = nullptr;
    sl.cap = 0;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(FMM_ERR_OUT_OF_MEMORY, "cannot allocate " + std::to_string(need) + " bytes of host-call operands");
    }
    sl.io = static_cast<double*>(p);
    sl.cap = need;
  }
  double* dA = sl.io;
  double* dB = dA + ((na + 31) & ~(size_t)31);
  double* dC = dB + ((nb + 31) & ~(size_t)31);
  const int64_t ldA = m, ldB = k > 0 ? k : 1, ldC = m;
  const bool read_c = beta != 0.0 && num_steps > 0;
  // copy-in: after this slot's previous call has returned its C (the slot's
  // buffers are free again); a call that reads C also waits for the other
  // slot's copy-out, which may write the same host C
  if (sl.used) FMM_CUDA_TRY(cudaStreamWaitEvent(h->h2d, sl.free, 0), "cudaStreamWaitEvent");
  if (read_c && other.used) FMM_CUDA_TRY(cudaStreamWaitEvent(h->h2d, other.free, 0), "cudaStreamWaitEvent");
  if (na)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dA, ldA * sizeof(double), A, lda * sizeof(double), m * sizeof(double), k,
                                   cudaMemcpyHostToDevice, h->h2d),
                 "copy A to device");
  if (nb)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dB, ldB * sizeof(double), B, ldb * sizeof(double), k * sizeof(double), n,
                                   cudaMemcpyHostToDevice, h->h2d),
                 "copy B to device");
  if (read_c)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dC, ldC * sizeof(double), C, ldc * sizeof(double), m * sizeof(double), n,
                                   cudaMemcpyHostToDevice, h->h2d),
                 "copy C to device");
  FMM_CUDA_TRY(cudaEventRecord(sl.in_ready, h->h2d), "cudaEventRecord");
  FMM_CUDA_TRY(cudaStreamWaitEvent(h->stream, sl.in_ready, 0), "cudaStreamWaitEvent");
  s = fmm_fast_matmul(h, alg, dA, ldA, dB, ldB, dC, ldC, m, k, n, num_steps, x, alpha, beta, opts);
  if (s != FMM_OK) return s;
  FMM_CUDA_TRY(cudaEventRecord(sl.out_ready, h->stream), "cudaEventRecord");
  FMM_CUDA_TRY(cudaStreamWaitEvent(h->d2h, sl.out_ready, 0), "cudaStreamWaitEvent");
  FMM_CUDA_TRY(cudaMemcpy2DAsync(C, ldc * sizeof(double), dC, ldC * sizeof(double), m * sizeof(double), n,
                                 cudaMemcpyDeviceToHost, h->d2h),
               "copy C to host");
  FMM_CUDA_TRY(cudaEventRecord(sl.free, h->d2h), "cudaEventRecord");
  sl.used = true;
  h->next_slot ^= 1;
  return FMM_OK;
}

fmm_status fmm_host_sync(fmm_handle h) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  DeviceGuard g(h->device);
  if (h->d2h) FMM_CUDA_TRY(cudaStreamSynchronize(h->d2h), "cudaStreamSynchronize(copy-out)");
  h->slots[0].used = h->slots[1].used = false;
  return check_device_errors(h);
}

fmm_status fmm_dgemm(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                     int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta) {
  return fmm::api::dgemm_tiled(h, A, lda, B, ldb, C, ldc, m, k, n, alpha, beta, FMM_GEMM_TILE_AUTO);
}

}  // extern "C"

namespace fmm {
namespace api {

fmm_status dgemm_tiled(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                       int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta, int tile_choice) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_dims(m, k, n, lda, ldb, ldc);
  if (s != FMM_OK) return s;
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  fmm::Program& prog = h->prog;
  prog.clear();
  fmm::GemmDesc d{};
  d.A = A;
  d.B = B;
  d.C = C;
  d.lda = lda;
  d.ldb = ldb;
  d.ldc = ldc;
  d.m = (int)m;
  d.n = (int)n;
  d.k = (int)k;
  d.alpha = alpha;
  d.beta = beta;
  const int tile = (tile_choice == fmm::kGemmTileLarge || tile_choice == fmm::kGemmTileSmall)
                       ? tile_choice
                       : fmm::gemm_tile_rule(d.m);
  const int64_t tiles = fmm::gemm_prepare(&d, 1, fmm::kGemmBN, fmm::gemm_tile_rows(tile));
  prog.desc.resize(sizeof(d));
  std::memcpy(prog.desc.data(), &d, sizeof(d));
  fmm::Op op;
  op.kind = fmm::OpKind::kGemm;
  op.n = 1;
  op.total_tiles = tiles;
  op.gemm_tile = tile;
  op.desc_off = 0;
  op.flops = 2.0 * (double)m * (double)n * (double)k;
  prog.ops.push_back(op);
  if ((s = stage_descriptors(h, prog)) != FMM_OK) return s;
  return run_staged(h, prog);
}

}  // namespace api
}  // namespace fmm

extern "C" {

fmm_status fmm_dgemm_host(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                          int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_dims(m, k, n, lda, ldb, ldc);
  if (s != FMM_OK) return s;
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  const size_t na = (size_t)m * (size_t)k, nb = (size_t)k * (size_t)n, nc = (size_t)m * (size_t)n;
  void* io = h->io;
  size_t cap = h->io_cap;
  if ((s = ensure_device_buffer(h, &io, &cap, (na + nb + nc) * sizeof(double) + 512, "host-call operands")) != FMM_OK)
    return s;
  h->io = static_cast<double*>(io);
  h->io_cap = cap;
  double* dA = h->io;
  double* dB = dA + ((na + 31) & ~(size_t)31);
  double* dC = dB + ((nb + 31) & ~(size_t)31);
  const int64_t ldA = m, ldB = k > 0 ? k : 1, ldC = m;
  if (na)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dA, ldA * sizeof(double), A, lda * sizeof(double), m * sizeof(double), k,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy A to device");
  if (nb)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dB, ldB * sizeof(double), B, ldb * sizeof(double), k * sizeof(double), n,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy B to device");
  if (beta != 0.0)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dC, ldC * sizeof(double), C, ldc * sizeof(double), m * sizeof(double), n,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy C to device");
  s = fmm_dgemm(h, dA, ldA, dB, ldB, dC, ldC, m, k, n, alpha, beta);
  if (s != FMM_OK) return s;
  FMM_CUDA_TRY(cudaMemcpy2DAsync(C, ldc * sizeof(double), dC, ldC * sizeof(double), m * sizeof(double), n,
                                 cudaMemcpyDeviceToHost, h->stream),
               "copy C to host");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  return FMM_OK;
}

// One classical split product (BF16 or INT8 digits, by `precision`).
static fmm_status dgemm_split(fmm_handle h, int precision, const double* A, int64_t lda, const double* B, int64_t ldb,
                       double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta,
                       int slices) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status s = check_dims(m, k, n, lda, ldb, ldc);
  if (s != FMM_OK) return s;
  int sl = 0;
  if ((s = split_slices_for(precision, slices, &sl)) != FMM_OK) return s;
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  fmm::Program& prog = h->prog;
  prog.clear();
  fmm::SplitDesc d{};
  d.A = A;
  d.B = B;
  d.C = C;
  d.lda = lda;
  d.ldb = ldb;
  d.ldc = ldc;
  d.m = (int)m;
  d.n = (int)n;
  d.k = (int)k;
  d.alpha = alpha;
  d.beta = beta;
  const fmm::SplitPlan plan = fmm::split_prepare(&d, 1, sl);
  if ((s = ensure_device_buffer(h, &h->ws, &h->ws_cap, plan.bytes, "split scratch")) != FMM_OK) return s;
  prog.desc.resize(sizeof(d));
  std::memcpy(prog.desc.data(), &d, sizeof(d));
  prog.split_slices = sl;
  prog.split_scratch = static_cast<char*>(h->ws);
  prog.split_bytes = plan.bytes;
  prog.workspace_bytes = plan.bytes;
  fmm::Op op;
  op.kind = fmm::OpKind::kSplitGemm;
  op.n = 1;
  op.total_tiles = plan.tiles;
  op.desc_off = 0;
  op.flops = 2.0 * (double)m * (double)n * (double)k;
  op.split = plan;
  prog.ops.push_back(op);
  if ((s = stage_descriptors(h, prog)) != FMM_OK) return s;
  return run_staged(h, prog);
}

fmm_status fmm_dgemm_split_bf16(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb,
                                double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta,
                                int slices) {
  return dgemm_split(h, FMM_PRECISION_SPLIT_BF16, A, lda, B, ldb, C, ldc, m, k, n, alpha, beta, slices);
}

fmm_status fmm_dgemm_split_int8(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb,
                                double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta,
                                int slices) {
  return dgemm_split(h, FMM_PRECISION_SPLIT_INT8, A, lda, B, ldb, C, ldc, m, k, n, alpha, beta, slices);
}

fmm_status fmm_fill_uniform(fmm_handle h, double* out, int64_t rows, int64_t cols, int64_t ld, uint64_t seed,
                            uint64_t stream, double lo, double hi) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  if (rows < 0 || cols < 0 || ld < (rows > 1 ? rows : 1))
    return fail(FMM_ERR_INVALID_ARGUMENT, "bad matrix shape");
  if (rows * cols > 0 && !out) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  FMM_CUDA_TRY(fmm::fill_uniform_launch(out, rows, cols, ld, seed, stream, lo, hi, h->stream), "fill_uniform");
  ++h->launches;
  return FMM_OK;
}

fmm_status fmm_max_relative_diff(fmm_handle h, const double* a, int64_t lda, const double* b, int64_t ldb,
                                 int64_t m, int64_t n, double* max_rel, double* max_abs) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  if (m < 0 || n < 0 || lda < (m > 1 ? m : 1) || ldb < (m > 1 ? m : 1))
    return fail(FMM_ERR_INVALID_ARGUMENT, "bad matrix shape");
  DeviceGuard g(h->device);
  FMM_CUDA_TRY(fmm::max_rel_diff_launch(a, lda, b, ldb, m, n, h->d_small, h->stream), "max_rel_diff");
  ++h->launches;
  double res[2] = {0.0, 0.0};
  FMM_CUDA_TRY(cudaMemcpyAsync(res, h->d_small, sizeof(res), cudaMemcpyDeviceToHost, h->stream), "copy result");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  if (max_rel) *max_rel = res[0];
  if (max_abs) *max_abs = res[1];
  return FMM_OK;
}

fmm_status fmm_diagonal_scaling(fmm_handle h, double* A, int64_t lda, double* B, int64_t ldb, int64_t m, int64_t k,
                                int64_t n, int num_steps, int type, double* r, double* s) {
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

fmm_status fmm_scaling_postprocess(fmm_handle h, double* C, int64_t ldc, int64_t m, int64_t n, const double* r,
                                   const double* s) {
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

fmm_status fmm_diagonal_scaling_host(fmm_handle h, double* A, int64_t lda, double* B, int64_t ldb, int64_t m,
                                     int64_t k, int64_t n, int num_steps, int type, double* r, double* s) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status st = check_dims(m, k, n, lda, ldb, m > 1 ? m : 1);
  if (st != FMM_OK) return st;
  if ((m > 0 && !r) || (n > 0 && !s)) return fail(FMM_ERR_INVALID_ARGUMENT, "null factor pointer");
  if ((m * k > 0 && !A) || (k * n > 0 && !B)) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  auto pad = [](size_t v) { return (v + 31) & ~(size_t)31; };
  const size_t na = (size_t)m * (size_t)k, nb = (size_t)k * (size_t)n;
  void* io = h->io;
  size_t cap = h->io_cap;
  if ((st = ensure_device_buffer(h, &io, &cap, (pad(na) + pad(nb) + pad(m) + pad(n)) * sizeof(double),
                                 "host-call operands")) != FMM_OK)
    return st;
  h->io = static_cast<double*>(io);
  h->io_cap = cap;
  double* dA = h->io;
  double* dB = dA + pad(na);
  double* dr = dB + pad(nb);
  double* ds = dr + pad(m);
  const int64_t ldA = m > 1 ? m : 1, ldB = k > 1 ? k : 1;
  if (na)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dA, ldA * sizeof(double), A, lda * sizeof(double), m * sizeof(double), k,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy A to device");
  if (nb)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(dB, ldB * sizeof(double), B, ldb * sizeof(double), k * sizeof(double), n,
                                   cudaMemcpyHostToDevice, h->stream),
                 "copy B to device");
  if (m) FMM_CUDA_TRY(cudaMemcpyAsync(dr, r, m * sizeof(double), cudaMemcpyHostToDevice, h->stream), "copy r");
  if (n) FMM_CUDA_TRY(cudaMemcpyAsync(ds, s, n * sizeof(double), cudaMemcpyHostToDevice, h->stream), "copy s");
  st = fmm_diagonal_scaling(h, dA, ldA, dB, ldB, m, k, n, num_steps, type, dr, ds);
  if (st != FMM_OK) return st;
  if (na)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(A, lda * sizeof(double), dA, ldA * sizeof(double), m * sizeof(double), k,
                                   cudaMemcpyDeviceToHost, h->stream),
                 "copy A to host");
  if (nb)
    FMM_CUDA_TRY(cudaMemcpy2DAsync(B, ldb * sizeof(double), dB, ldB * sizeof(double), k * sizeof(double), n,
                                   cudaMemcpyDeviceToHost, h->stream),
                 "copy B to host");
  if (m) FMM_CUDA_TRY(cudaMemcpyAsync(r, dr, m * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "copy r back");
  if (n) FMM_CUDA_TRY(cudaMemcpyAsync(s, ds, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "copy s back");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  return FMM_OK;
}

fmm_status fmm_scaling_postprocess_host(fmm_handle h, double* C, int64_t ldc, int64_t m, int64_t n, const double* r,
                                        const double* s) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  fmm_status st = check_dims(m, 0, n, m > 1 ? m : 1, 1, ldc);
  if (st != FMM_OK) return st;
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || !r || !s) return fail(FMM_ERR_INVALID_ARGUMENT, "null pointer");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  auto pad = [](size_t v) { return (v + 31) & ~(size_t)31; };
  const size_t nc = (size_t)m * (size_t)n;
  void* io = h->io;
  size_t cap = h->io_cap;
  if ((st = ensure_device_buffer(h, &io, &cap, (pad(nc) + pad(m) + pad(n)) * sizeof(double),
                                 "host-call operands")) != FMM_OK)
    return st;
  h->io = static_cast<double*>(io);
  h->io_cap = cap;
  double* dC = h->io;
  double* dr = dC + pad(nc);
  double* ds = dr + pad(m);
  FMM_CUDA_TRY(cudaMemcpy2DAsync(dC, m * sizeof(double), C, ldc * sizeof(double), m * sizeof(double), n,
                                 cudaMemcpyHostToDevice, h->stream),
               "copy C to device");
  FMM_CUDA_TRY(cudaMemcpyAsync(dr, r, m * sizeof(double), cudaMemcpyHostToDevice, h->stream), "copy r");
  FMM_CUDA_TRY(cudaMemcpyAsync(ds, s, n * sizeof(double), cudaMemcpyHostToDevice, h->stream), "copy s");
  st = fmm_scaling_postprocess(h, dC, m, m, n, dr, ds);
  if (st != FMM_OK) return st;
  FMM_CUDA_TRY(cudaMemcpy2DAsync(C, ldc * sizeof(double), dC, m * sizeof(double), m * sizeof(double), n,
                                 cudaMemcpyDeviceToHost, h->stream),
               "copy C to host");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  return FMM_OK;
}

fmm_status fmm_synchronize(fmm_handle h) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  DeviceGuard g(h->device);
  return check_device_errors(h);
}

fmm_status fmm_selftest_wait_timeout(fmm_handle h, double limit_ms, int* code) {
  if (!h || !code) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  if (!(limit_ms > 0.0) || limit_ms > 1000.0) return fail(FMM_ERR_INVALID_ARGUMENT, "limit_ms must be in (0, 1000]");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  FMM_CUDA_TRY(cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream), "clear device error word");
  FMM_CUDA_TRY(fmm::wait_probe_launch(h->d_err, (uint64_t)(limit_ms * 1e6), 99, h->stream), "wait probe launch");
  h->launches++;
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  FMM_CUDA_TRY(cudaMemcpy(code, h->d_err, sizeof(int), cudaMemcpyDeviceToHost), "read device error word");
  FMM_CUDA_TRY(cudaMemset(h->d_err, 0, sizeof(int)), "clear device error word");
  return FMM_OK;
}

int64_t fmm_kernel_launch_count(fmm_handle h) { return h ? h->launches : 0; }

fmm_status fmm_profile_enable(fmm_handle h, int enable) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  h->profiling = enable != 0;
  return FMM_OK;
}

fmm_status fmm_profile_reset(fmm_handle h) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  DeviceGuard g(h->device);
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  h->prof.reset();
  return FMM_OK;
}

fmm_status fmm_profile_read(fmm_handle h, fmm_profile* out) {
  if (!h || !out) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  DeviceGuard g(h->device);
  FMM_CUDA_TRY(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  std::memset(out, 0, sizeof(*out));
  for (const fmm::Profiler::Rec& r : h->prof.recs) {
    float ms = 0.f;
    FMM_CUDA_TRY(cudaEventElapsedTime(&ms, r.start, r.stop), "cudaEventElapsedTime");
    switch (r.kind) {
      case fmm::OpKind::kForm:
        out->form_launches++;
        out->form_ms += ms;
        out->form_bytes += r.bytes;
        break;
      case fmm::OpKind::kCombine:
        out->combine_launches++;
        out->combine_ms += ms;
        out->combine_bytes += r.bytes;
        break;
      case fmm::OpKind::kSplitGemm:
        if (r.mid) {
          float sms = 0.f;
          FMM_CUDA_TRY(cudaEventElapsedTime(&sms, r.start, r.mid), "cudaEventElapsedTime");
          out->split_ms += sms;
        }
        out->split_bf16_flops += r.bf16_flops;
        out->gemm_launches++;
        out->gemm_ms += ms;
        out->gemm_flops += r.flops;
        break;
      case fmm::OpKind::kGemm:
        if (r.peel) {
          out->peel_launches++;
          out->peel_ms += ms;
          out->peel_flops += r.flops;
        } else {
          out->gemm_launches++;
          out->gemm_ms += ms;
          out->gemm_flops += r.flops;
        }
        break;
    }
  }
  return FMM_OK;
}

}  // extern "C"
