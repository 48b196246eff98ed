// Allocation-free FastMatmul (fmm_fast_matmul_noalloc in include/fmm.h).
//
// Same planner and kernels as fmm_fast_matmul; the workspace and the launch
// descriptors come from the static device array below instead of a handle's
// allocations.  In host code `g_noalloc_scratch` is only a stand-in symbol:
// its device address is looked up once per device with cudaGetSymbolAddress
// and that address is what the kernels receive.

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "fmm.h"
#include "fmm_internal.h"
#include "plan.h"

namespace {

constexpr size_t kScratchBytes = FMM_NOALLOC_SCRATCH_BYTES;
constexpr size_t kDescBytes = (size_t)1 << 20;  // launch descriptors at the front
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};
int g_scratch_sms[kMaxDevices] = {};

fmm_status fail(fmm_status s, const std::string& msg) {
  fmm::set_last_error(msg);
  return s;
}

// Device address of the scratch array on `dev` (the current device); looked
// up on the first call for that device.
fmm_status scratch_for_device(int dev, char** addr, int* sms) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return fail(FMM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    }
    int count = 0;
    e = cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(FMM_ERR_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
    }
    g_scratch_sms[dev] = count;
    g_scratch_addr[dev] = p;
  }
  *addr = static_cast<char*>(g_scratch_addr[dev]);
  *sms = g_scratch_sms[dev];
  return FMM_OK;
}

}  // namespace

extern "C" fmm_status fmm_fast_matmul_noalloc(int alg, const double* A, int64_t lda, const double* B, int64_t ldb,
                                              double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps,
                                              double x, double alpha, double beta, void* stream) {
  if (alg < 0 || alg >= FMM_NUM_ALGORITHMS)
    return fail(FMM_ERR_UNKNOWN_ALGORITHM, "unknown algorithm index " + std::to_string(alg));
  if (m < 0 || k < 0 || n < 0 || m > 2147483647 || k > 2147483647 || n > 2147483647)
    return fail(FMM_ERR_INVALID_ARGUMENT, "matrix dimension out of range");
  if (lda < (m > 1 ? m : 1) || ldb < (k > 1 ? k : 1) || ldc < (m > 1 ? m : 1))
    return fail(FMM_ERR_INVALID_ARGUMENT, "leading dimension smaller than the number of rows");
  if (num_steps < 0 || num_steps > 16) return fail(FMM_ERR_INVALID_ARGUMENT, "num_steps must be in [0, 16]");
  if (m == 0 || n == 0) return FMM_OK;
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");

  const fmm_alg_table& t = fmm_algorithms[alg];
  const size_t cap = kScratchBytes - kDescBytes;
  int dfs = 0;
  size_t need = 0;
  for (dfs = 0; dfs <= num_steps; ++dfs) {
    need = fmm::workspace_bytes(t, m, k, n, num_steps, dfs);
    if (need <= cap) break;
  }
  if (dfs > num_steps)
    return fail(FMM_ERR_WORKSPACE_TOO_SMALL,
                "allocation-free call needs " + std::to_string(need) + " bytes of workspace even depth-first; " +
                    "its static scratch holds " + std::to_string(cap) + " (FMM_NOALLOC_SCRATCH_BYTES less " +
                    std::to_string(kDescBytes) + " for launch descriptors)");

  // The launch descriptors are copied from a host buffer that the next call
  // on this thread rewrites.  An ordinary cudaMemcpyAsync from pageable
  // memory has consumed the source when it returns; a copy recorded into a
  // graph would read the buffer again at every replay.  So a stream in
  // capture mode is refused before anything is queued on it.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &capture);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(FMM_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
  }
  if (capture != cudaStreamCaptureStatusNone)
    return fail(FMM_ERR_NOT_SUPPORTED,
                "fmm_fast_matmul_noalloc stages its launch descriptors from reused host memory and does not run "
                "on a stream in capture mode");

  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(FMM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  }
  if (dev < 0 || dev >= kMaxDevices) return fail(FMM_ERR_NOT_SUPPORTED, "device index above 63");
  char* scratch = nullptr;
  int sms = 0;
  fmm_status s = scratch_for_device(dev, &scratch, &sms);
  if (s != FMM_OK) return s;

  thread_local fmm::Program prog;
  try {
    fmm::build_program(alg, m, k, n, num_steps, x, alpha, beta, dfs, fmm::Operand{const_cast<double*>(A), lda},
                       fmm::Operand{const_cast<double*>(B), ldb}, fmm::Operand{C, ldc}, scratch + kDescBytes, &prog);
  } catch (const std::exception& ex) {
    return fail(FMM_ERR_OUT_OF_MEMORY, std::string("planning failed: ") + ex.what());
  }
  if (prog.desc.size() > kDescBytes)
    return fail(FMM_ERR_WORKSPACE_TOO_SMALL, "allocation-free call needs " + std::to_string(prog.desc.size()) +
                                                 " bytes of launch descriptors; the scratch reserves " +
                                                 std::to_string(kDescBytes));
  // descriptors go from ordinary host memory into the front of the scratch
  e = fmm::run_program(prog, prog.desc.data(), scratch, sms, static_cast<cudaStream_t>(stream), nullptr);
  if (e != cudaSuccess) return fail(FMM_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return FMM_OK;
}
