// Recursion planner: turns one FastMatmul call (or a batch of independent
// calls) into a list of grouped launches (operand formation, leaf products,
// combination, peeling) over a device workspace laid out level by level.
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <vector>

#include "fmm_internal.h"

namespace fmm {

struct Operand {
  double* ptr;
  int64_t ld;
};

enum class OpKind { kForm, kGemm, kCombine, kSplitGemm };

struct Op {
  OpKind kind;
  int alg = 0;          // form / combine: algorithm of the kernel
  int cf = 0;           // form / combine: index into Program::coefs
  size_t desc_off = 0;  // byte offset of this launch's descriptors in Program::desc
  int n = 0;            // descriptors
  int n_s = 0, n_t = 0; // form: sub-problems on the A and B side
  int64_t max_items = 0;     // form / combine: largest per-problem work-item count
  int64_t total_tiles = 0;   // gemm
  int gemm_tile = kGemmTileLarge;  // gemm: tile configuration the descriptors were prepared for
  bool vec2 = false;
  bool peel = false;     // gemm: dynamic-peeling fringe products
  int level = 0;         // recursion level the launch belongs to (steps = leaves)
  double flops = 0.0;    // gemm: 2 * m * n * k summed over the problems
  double bytes = 0.0;    // form / combine: algorithmic HBM bytes (each input read once, each output written once)
  SplitPlan split;       // split gemm: scratch layout (offsets from Program::split_scratch)
};

// Per-launch timing with CUDA events (fmm_profile_* in include/fmm.h).
struct Profiler {
  struct Rec {
    OpKind kind;
    bool peel;
    double flops, bytes;
    cudaEvent_t start, stop;
    cudaEvent_t mid = nullptr;  // split gemm: after the splitting kernels
    double bf16_flops = 0.0;    // split gemm: tensor-core FLOPs of the slice products
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  cudaEvent_t get();
  void reset();
  ~Profiler();
};

struct Program {
  std::vector<Op> ops;
  std::vector<unsigned char> desc;
  std::vector<CoefSlots> coefs;
  size_t workspace_bytes = 0;
  int dfs_levels = 0;
  double leaf_flops = 0.0;  // 2 * m * n * k summed over leaf products
  double peel_flops = 0.0;
  int64_t leaf_count = 0;
  int split_slices = 0;         // > 0: split code of the leaf products (slices, BF16 or INT8 digits)
  char* split_scratch = nullptr;  // scratch shared by the split launches (inside the workspace)
  size_t split_bytes = 0;       // its size
  const void* ws_base = nullptr;  // the workspace the program was planned into (workspace_bytes of it)
  void clear();
};

struct LevelDims {
  int64_t m, k, n;
};

// Dimensions of the sub-problems at each level 0..steps: floor splitting
// (linalg/linalg.hpp:179-184), except that block rows and inner dimensions
// of at least kEvenBlockMin are made even (one more row or inner index goes
// to the fringe products), which keeps every block view 16-byte aligned.
constexpr int64_t kEvenBlockMin = 256;
std::vector<LevelDims> level_dims(const fmm_alg_table& t, int64_t m, int64_t k, int64_t n, int steps);

// Workspace bytes for `dfs_levels` depth-first levels (0 = all breadth-first);
// split_slices > 0 (a split code) adds the scratch of split leaf products.
size_t workspace_bytes(const fmm_alg_table& t, int64_t m, int64_t k, int64_t n, int steps, int dfs_levels,
                       int split_slices = 0);

// Builds the launch program of one call.  ws must hold workspace_bytes(...) bytes.
// split_slices > 0 (a split code: slice count, BF16 or INT8 digits) runs
// the leaf products (not the fringe products of dynamic peeling) split.
// gemm_tile (kGemmTileAuto / Large / Small) is the tile configuration of
// the FP64 leaf and fringe products; Auto picks one per problem.
void build_program(int alg, int64_t m, int64_t k, int64_t n, int steps, double x, double alpha, double beta,
                   int dfs_levels, Operand A, Operand B, Operand C, void* ws, Program* out, int split_slices = 0,
                   int gemm_tile = kGemmTileAuto);

// One independent product of a batch.  A classical item is one GEMM
// C = alpha * A * B + beta * C (beta honoured; alg and steps unused); the
// others follow FastMatmul exactly (num_steps == 0 ignores beta).
struct BatchItem {
  int alg;
  int steps;
  int64_t m, k, n;
  Operand A, B, C;
  double x, alpha, beta;
  bool classical;
  int split_slices = 0;  // > 0: split code of this item's leaf products
  int gemm_tile = kGemmTileAuto;  // tile configuration of this item's FP64 products
};

// Workspace of a batch (every item planned breadth-first, regions back to back).
size_t batch_workspace_bytes(const BatchItem* items, int count);

// The same footprint built one item at a time (batch_workspace_bytes uses
// it): a request loop can price each candidate in O(1) instead of laying
// the whole batch out again.
class BatchFootprint {
 public:
  void add(const BatchItem& it);
  size_t bytes() const;

 private:
  size_t fp64_ = 0;                 // FP64 temporaries of the items, 256-byte aligned each
  std::map<int, SplitPlan> split_;  // split leaves per split code (one launch each)
};

// Builds one program for the whole batch: operand formations level by level
// (one launch per algorithm and level over all items), ONE grouped GEMM over
// every item's leaf products, then combinations and fringe products level by
// level upwards.
void build_batch_program(const BatchItem* items, int count, void* ws, Program* out);

// Runs a built program: one host-to-device copy of all descriptors to
// d_desc (which must hold prog.desc.size() bytes), then the launches in order.
// Adds the number of kernels launched to *launches (may be null).
// When prof is non-null every launch is bracketed by CUDA events.  d_err
// (device int) collects the error codes of split launches.  desc_copied
// (may be null) is recorded right after the descriptor copy: from then on
// h_desc may be rewritten.
cudaError_t run_program(const Program& prog, const void* h_desc, void* d_desc, int num_sms, cudaStream_t stream,
                        int64_t* launches, Profiler* prof = nullptr, int* d_err = nullptr,
                        cudaEvent_t desc_copied = nullptr);

}  // namespace fmm
