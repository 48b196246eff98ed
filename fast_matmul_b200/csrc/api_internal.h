// Handle state and helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "fmm.h"
#include "fmm_internal.h"
#include "plan.h"

#define FMM_CUDA_TRY(expr, where)                  \
  do {                                             \
    cudaError_t e__ = (expr);                      \
    if (e__ != cudaSuccess) {                      \
      return ::fmm::api::cuda_fail(e__, where);    \
    }                                              \
  } while (0)

struct fmm_handle_s {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  size_t ws_limit = 0;
  // device workspace pool (S/T/M temporaries), grown on demand
  void* ws = nullptr;
  size_t ws_cap = 0;
  // launch descriptors: pinned host staging + device copy
  void* h_desc = nullptr;
  size_t h_desc_cap = 0;
  void* d_desc = nullptr;
  size_t d_desc_cap = 0;
  cudaEvent_t desc_done = nullptr;  // staging buffer may be rewritten after this
  bool desc_pending = false;
  // device copies of host operands for the host-memory entry points
  double* io = nullptr;
  size_t io_cap = 0;
  double* d_small = nullptr;  // two doubles for reductions
  void* scal = nullptr;       // maxima and factors of the diagonal scaling
  size_t scal_cap = 0;
  void* wide = nullptr;       // FP64 staging of the FP32 entry points
  size_t wide_cap = 0;
  void* narrow_io = nullptr;  // device copies of host FP32 operands
  size_t narrow_io_cap = 0;
  int* d_err = nullptr;       // error codes of split-BF16 kernels (bounded waits that gave up)
  // pipelined host-pointer calls (fmm_fast_matmul_host_async): two device
  // staging slots used in turn, a copy-in and a copy-out stream
  struct HostSlot {
    double* io = nullptr;
    size_t cap = 0;
    cudaEvent_t in_ready = nullptr;   // copies of this call's operands landed
    cudaEvent_t out_ready = nullptr;  // this call's C is computed
    cudaEvent_t free = nullptr;       // this call's C is back on the host
    bool used = false;
  };
  HostSlot slots[2];
  int next_slot = 0;
  cudaStream_t h2d = nullptr, d2h = nullptr;
  int64_t launches = 0;
  fmm::Program prog;
  bool profiling = false;
  fmm::Profiler prof;
  // autotuner: shape bucket (ceil log2 of m, k, n) -> algorithm (or FMM_ALG_CLASSICAL), steps and
  // the FP64 GEMM tile configuration measured fastest
  struct Tuned {
    int alg, steps, tile;
  };
  std::map<std::tuple<int, int, int>, Tuned> tuned;
};

namespace fmm {
namespace api {

fmm_status fail(fmm_status s, const std::string& msg);
fmm_status cuda_fail(cudaError_t e, const char* where);

// Restores the caller's current device on scope exit.
class DeviceGuard {
 public:
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
    ok_ = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (prev_ >= 0) cudaSetDevice(prev_);
  }
  bool ok() const { return ok_; }

 private:
  int prev_ = -1;
  bool ok_ = false;
};

fmm_status ensure_device_buffer(fmm_handle h, void** buf, size_t* cap, size_t need, const char* what);
fmm_status stage_descriptors(fmm_handle h, const fmm::Program& prog);
fmm_status run_staged(fmm_handle h, const fmm::Program& prog);
fmm_status check_alg(int alg);
// fmm_dgemm with a given tile configuration (fmm_gemm_tile; AUTO: per problem).
fmm_status dgemm_tiled(fmm_handle h, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                       int64_t ldc, int64_t m, int64_t k, int64_t n, double alpha, double beta, int tile);
fmm_status check_dims(int64_t m, int64_t k, int64_t n, int64_t lda, int64_t ldb, int64_t ldc);
void resolve_options(const fmm_options* opts, fmm_options* out);
// Slices of the leaf products for a precision (0 for FP64).
fmm_status split_slices_for(int precision, int requested, int* slices);
// Reads and clears the handle's device error word (synchronises the stream).
fmm_status check_device_errors(fmm_handle h);
fmm_status choose_dfs_levels(fmm_handle h, int alg, int64_t m, int64_t k, int64_t n, int steps,
                             const fmm_options& o, int* dfs_levels, size_t* bytes);
// Batch items with FMM_ALG_AUTO / FMM_ALG_CLASSICAL resolved (batch.cpp);
// items with an empty result are dropped.
fmm_status resolve_items(fmm_handle h, const fmm_batch_item* items, int count, std::vector<fmm::BatchItem>* out);

}  // namespace api
}  // namespace fmm
