// Device-side bounds checks of the descriptor walks (debug builds only).
//
// Built with -DFMM_DEVICE_CHECKS (python -m fast_matmul_b200.build --checked
// -> libfmm_checked.so), the grouped GEMM and the operand formation and
// combination kernels check what they derive from their launch descriptors:
// the problem and tile a CTA decodes, and that every temporary they write
// (S/T blocks) or read (product blocks M) lies inside the workspace of the
// program being run, which the executor registers before its launches.  A
// failed check sets its bit in a device word and the access is skipped; no
// kernel traps.  fmm_debug_check_flags reads and clears the word.  Without
// the macro every check compiles to `true` and nothing is stored.
//
// Each translation unit that includes this header has its own copy of the
// device state (the library is built without relocatable device code), and
// exports a pair of host functions to arm it and read it back.

#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fmm {

enum CheckBit : unsigned {
  kCheckGemmProblem = 1u << 0,  // GEMM tile whose owning problem or tile index is out of range
  kCheckGemmTile = 1u << 1,     // GEMM tile origin outside its problem
  kCheckFormOut = 1u << 2,      // formation writes outside the workspace
  kCheckCombineIn = 1u << 3,    // combination reads a product block outside the workspace
};

struct CheckRange {
  uintptr_t lo, hi;  // [lo, hi) of the running program's workspace; hi == 0: not armed
};

#ifdef FMM_DEVICE_CHECKS
constexpr bool kDeviceChecks = true;
#else
constexpr bool kDeviceChecks = false;
#endif

}  // namespace fmm

#ifdef FMM_DEVICE_CHECKS
namespace {
__device__ unsigned g_fmm_check_word;
__device__ fmm::CheckRange g_fmm_check_ws;

// cond holds, or bit is recorded (and the caller skips the access).
__device__ __forceinline__ bool fmm_check(bool cond, unsigned bit) {
  if (!cond) atomicOr(&g_fmm_check_word, bit);
  return cond;
}

// [p, p + bytes) inside the registered workspace (true when none is armed).
__device__ __forceinline__ bool fmm_in_workspace(const void* p, size_t bytes) {
  const fmm::CheckRange r = g_fmm_check_ws;
  if (r.hi == 0) return true;
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  return a >= r.lo && a + bytes <= r.hi;
}

// Host side of this translation unit's state.
cudaError_t fmm_checks_arm_tu(fmm::CheckRange ws, cudaStream_t stream) {
  static thread_local fmm::CheckRange staged;  // the copy below reads it once it is issued
  staged = ws;
  return cudaMemcpyToSymbolAsync(g_fmm_check_ws, &staged, sizeof(staged), 0, cudaMemcpyHostToDevice, stream);
}

cudaError_t fmm_checks_take_tu(unsigned* word) {
  unsigned v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_fmm_check_word, sizeof(v));
  if (e != cudaSuccess) return e;
  const unsigned zero = 0;
  e = cudaMemcpyToSymbol(g_fmm_check_word, &zero, sizeof(zero));
  *word |= v;
  return e;
}
}  // namespace
#define FMM_CHECK(cond, bit) fmm_check((cond), (bit))
#define FMM_IN_WORKSPACE(p, bytes) fmm_in_workspace((p), (bytes))
#else
namespace {
inline cudaError_t fmm_checks_arm_tu(fmm::CheckRange, cudaStream_t) { return cudaSuccess; }
inline cudaError_t fmm_checks_take_tu(unsigned*) { return cudaSuccess; }
}  // namespace
#define FMM_CHECK(cond, bit) true
#define FMM_IN_WORKSPACE(p, bytes) true
#endif
