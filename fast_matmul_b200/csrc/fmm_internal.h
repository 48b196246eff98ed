// Internal interfaces shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "generated/fmm_algorithms.h"

namespace fmm {

// ---------------------------------------------------------------------------
// Grouped FP64 GEMM: C_p = alpha_p * A_p * B_p + beta_p * C_p for a list of
// problems of any shapes, all in one persistent launch (dgemm_dmma.cu).
struct GemmDesc {
  const double* A;
  const double* B;
  double* C;
  int64_t lda, ldb, ldc;
  int m, n, k;
  int tiles_m;      // ceil(m / tile rows)
  int tile_begin;   // first global tile index of this problem
  int flags;        // bit 0: A allows 16-byte copies, bit 1: B allows 16-byte copies
  double alpha, beta;
};

// Tile configurations of the grouped FP64 GEMM (values of fmm_options::gemm_tile):
//   kGemmTileLarge  128 x 64 tiles, 4 warps of 64 x 32, 2 CTAs per SM
//   kGemmTileSmall   64 x 64 tiles, 4 warps of 32 x 32, 3 CTAs per SM
// Both accumulate every output element over the same k16 blocks in the same
// order, so they give bit-identical results.  kGemmTileAuto picks one per
// problem (gemm_tile_rule).
constexpr int kGemmTileAuto = 0;
constexpr int kGemmTileLarge = 1;
constexpr int kGemmTileSmall = 2;
constexpr int kGemmBM = 128;  // tile rows of the large configuration
constexpr int kGemmBN = 64;   // tile columns (both configurations)
constexpr int kGemmBMSmall = 64;
inline int gemm_tile_rows(int tile) { return tile == kGemmTileSmall ? kGemmBMSmall : kGemmBM; }
// Choice for one problem (a launch of several Auto problems applies the same
// test to their padded areas in total): the small tiles where 128-row tiles
// would pad the rows by more than 7% beyond what 64-row tiles pad (the small
// configuration runs about 6% slower on large problems).
inline int gemm_tile_rule(int m) {
  const int64_t large = (int64_t)((m + kGemmBM - 1) / kGemmBM) * kGemmBM;
  const int64_t small = (int64_t)((m + kGemmBMSmall - 1) / kGemmBMSmall) * kGemmBMSmall;
  return (double)large > 1.07 * (double)small ? kGemmTileSmall : kGemmTileLarge;
}

// Device-side checks of the descriptor walks (device_checks.cuh; built in
// with -DFMM_DEVICE_CHECKS): whether the library was compiled with them, registering the
// workspace of the program about to run, and reading (and clearing) the
// word of failed checks.  Without them, arming and reading do nothing.
bool device_checks_built();
cudaError_t device_checks_arm(const void* ws, size_t bytes, cudaStream_t stream);
cudaError_t device_checks_take(unsigned* word);
cudaError_t gemm_checks_arm(const void* ws, size_t bytes, cudaStream_t stream);
cudaError_t gemm_checks_take(unsigned* word);
cudaError_t thin_checks_arm(const void* ws, size_t bytes, cudaStream_t stream);
cudaError_t thin_checks_take(unsigned* word);

// Fringe products with at most kThinMax rows, columns or inner indices
// (thin_gemm.cu): the peeled rows or columns of a sub-problem against its
// whole inner dimension, and the update of its core by its peeled inner
// indices, on the FP64 pipe with each element of the long operand (or of C)
// read once.  A kGemm launch of configuration kGemmTileThin runs those with
// few rows or columns, one of kGemmTileThinInner those with few inner
// indices only; thin_prepare sets tile_begin / tiles_m of their descriptors
// to work items.
constexpr int kGemmTileThin = 3;
constexpr int kGemmTileThinInner = 4;
constexpr int kThinMax = 16;
constexpr int kThinColumnsPerItem = 8;  // few rows: a work item is 8 columns (a warp each)
constexpr int kThinRowsPerItem = 64;    // few columns: a work item is 64 rows
constexpr int kThinBlock = 64;          // few inner indices: a work item is a 64 x 64 block of C
__host__ __device__ inline int64_t thin_items(int64_t m, int64_t n, int64_t k) {
  if (m <= 0 || n <= 0) return 0;
  if (m <= kThinMax) return (n + kThinColumnsPerItem - 1) / kThinColumnsPerItem;
  if (n <= kThinMax) return (m + kThinRowsPerItem - 1) / kThinRowsPerItem;
  (void)k;  // k <= kThinMax
  return ((m + kThinBlock - 1) / kThinBlock) * ((n + kThinBlock - 1) / kThinBlock);
}
int64_t thin_prepare(GemmDesc* descs, int n);
cudaError_t thin_launch(const GemmDesc* d_descs, int n, int64_t total_items, int num_sms, cudaStream_t stream,
                        bool inner);

// Fills tiles_m / tile_begin / flags for descs[0..n) and returns the total
// number of tile_m x tile_n tiles.
int64_t gemm_prepare(GemmDesc* descs, int n, int tile_n = kGemmBN, int tile_m = kGemmBM);
// Launches the grouped GEMM over descs (device copy) with `total_tiles`
// tiles of configuration `tile` (kGemmTileLarge or kGemmTileSmall; the
// descriptors must have been prepared with that configuration's tile), or
// with kGemmTileThin / kGemmTileThinInner the thin kernels over
// `total_tiles` work items.
cudaError_t gemm_launch(const GemmDesc* d_descs, int n, int64_t total_tiles, int num_sms, cudaStream_t stream,
                        int tile = kGemmTileLarge);

// ---------------------------------------------------------------------------
// Split-BF16 leaf products on the tensor cores (split_bf16.cu):
// C_p = alpha_p * A_p * B_p + beta_p * C_p with A_p, B_p split into BF16
// slices after per-row / per-column power-of-two scaling.
constexpr int kSplitMinSlices = 2;
constexpr int kSplitMaxSlices = 6;
constexpr int kSplitDefaultSlices = 5;
constexpr int kSplitTile = 128;   // output tile rows of one CTA, and columns
constexpr int kSplitPairRows = 2 * kSplitTile;  // rows of the tile of a CTA pair (two-SM MMA)
constexpr int kSplitKBlock = 64;  // k-depth of one TMA box (128 bytes of BF16)
constexpr int kSplitChunk = 128;  // k-depth accumulated exactly in FP32 (two k-blocks)

// Split-INT8 leaf products: the same scaling, signed 8-bit digits of 7 bits
// (|d| <= 64), products on the INT8 tensor cores with exact int32 sums.  A
// 128-byte row then holds 128 k values and a chunk (two rows, one pipeline
// stage) 256; a diagonal is accumulated over up to kSplitI8GroupChunks
// chunks: at most 8 slices give at most 8 * 64 * 64 = 2^15 per k, so a sum
// over 32768 k stays below 2^30.
constexpr int kSplitI8MaxSlices = 8;
constexpr int kSplitI8DefaultSlices = 6;
constexpr int kSplitI8KBlock = 128;
constexpr int kSplitI8Chunk = 256;
constexpr int kSplitI8GroupChunks = 128;

// A split form travels through the planner as one int, the split code:
// 0 = FP64 leaves, s = s BF16 slices, kSplitInt8Code + s = s INT8 slices.
constexpr int kSplitInt8Code = 16;
__host__ __device__ inline int split_code_slices(int code) { return code >= kSplitInt8Code ? code - kSplitInt8Code : code; }
__host__ __device__ inline bool split_code_int8(int code) { return code >= kSplitInt8Code; }

// Accumulation groups of one output tile, in order: for each pair of
// 128-deep k-chunks, diagonal 0 over both chunks, diagonal 1 over both, then
// diagonals 2..S-1 of the first chunk and of the second (a last single chunk
// forms its own pair).  Pairs are used at 3 slices or fewer, where they save
// a third of the drains; with more slices every chunk forms its own group
// set (diagonals 0..S-1), which measured faster on Strassen's leaf launches
// and on single products (pairs at 5 slices: 1000 against 1045 TFLOP/s at
// 4096^3, Strassen 2 steps -1.3%; at 4 slices +2%).  With digits
// |d_1| <= 256 and |d_t| <= 128 every FP32 partial sum of a group stays an
// integer of magnitude <= 2^24 -- diagonals
// 0 and 1 add at most 2^16 per k over 256 k, diagonal D >= 2 at most
// (D + 3) 2^14 per k over 128 k -- so the tensor cores accumulate each group
// exactly, and the FP64 recombination adds the groups in this order.
struct SplitGroup {
  int D;       // diagonal: slice pairs (t, D - t), t = 0..D (0-based slices)
  int c0, c1;  // chunks [c0, c1)
};

// Chunks per pair (1 or 2) and groups of a pair of nch chunks.
__host__ __device__ inline int split_chunk_span(int slices) { return slices <= 3 ? 2 : 1; }
__host__ __device__ inline int split_groups_in_pair(int nch, int slices) { return 2 + nch * (slices - 2); }

// Group gi of the chunk pair starting at chunk cp (nch = 1 or 2 chunks).
__host__ __device__ inline SplitGroup split_group(int cp, int nch, int slices, int gi) {
  SplitGroup g;
  if (gi < 2) {
    g.D = gi;
    g.c0 = cp;
    g.c1 = cp + nch;
  } else {
    const int r = gi - 2;
    g.D = 2 + r % (slices - 2);
    g.c0 = cp + r / (slices - 2);
    g.c1 = g.c0 + 1;
  }
  return g;
}

// The exponent recorded for a row of A or column of B holding an Inf or a
// NaN: its digits are zero and every entry of C it reaches is NaN.
constexpr int kSplitNonFinite = 1 << 28;

struct SplitDesc {
  const double* A;
  const double* B;
  double* C;
  int64_t lda, ldb, ldc;
  double alpha, beta;
  int m, n, k;
  int kblocks;          // 128-byte rows of k per padded row / column (padded k / 64 BF16 or / 128 INT8)
  int tiles_m, tiles_n; // padded m / kSplitTile (even: m is padded to kSplitPairRows), padded n / kSplitTile
  int64_t tile_begin;   // first output tile (kSplitPairRows x kSplitTile, one CTA pair) of this problem
  int64_t sa_begin;     // first A-splitting work tile (32 rows x 64 k)
  int64_t a_row;        // first 128-byte row of this problem's A slices
  int64_t b_row;        // first 128-byte row of this problem's B slices
  int64_t e_off;        // first row exponent (tiles_m * 128 entries)
  int64_t f_off;        // first column exponent (tiles_n * 128 entries)
};

// Scratch layout of one split launch (offsets from the scratch base).
struct SplitPlan {
  int slices = 0;        // slice count
  bool int8 = false;     // INT8 digits (else BF16)
  int64_t tiles = 0;     // output tiles (one per CTA pair) over all problems
  int64_t sa_work = 0;   // A-splitting work tiles
  int64_t rows_a = 0, rows_b = 0;  // 128-byte slice rows
  int64_t n_e = 0, n_f = 0;        // row / column exponents
  size_t off_b = 0, off_e = 0, off_f = 0, bytes = 0;
};

// Fills the derived fields of descs[0..n) for split code `code` and returns
// the scratch layout.  Problems with m == 0 or n == 0 get no tiles.
SplitPlan split_prepare(SplitDesc* descs, int n, int code);
// Adds `count` problems of m x k x n to the sizes of *plan (before
// split_finish), the same arithmetic split_prepare applies per descriptor.
void split_accumulate(SplitPlan* plan, int64_t m, int64_t k, int64_t n, int64_t count);
// Computes the region offsets and total bytes of *plan from its sizes.
void split_finish(SplitPlan* plan);
// Scratch bytes split_prepare would report for `count` problems of m x k x n.
size_t split_scratch_bytes(int64_t m, int64_t k, int64_t n, int64_t count, int code);
// The plan of split code `code` with no problems yet.
SplitPlan split_plan_for(int code);
// Launches splitting and the tensor-core product.  `scratch` holds plan.bytes
// bytes (256-byte aligned); *d_err (device) receives a nonzero code if a
// bounded wait inside the product kernel gave up.  Returns the kernel count
// launched through *launches.
cudaError_t split_gemm_launch(const SplitDesc* d_descs, int n, const SplitPlan& plan, void* scratch, int* d_err,
                              int num_sms, cudaStream_t stream, int64_t* launches, cudaEvent_t split_done = nullptr);
// A kernel whose single bounded mbarrier wait is never satisfied: it records
// `code` in *d_err after limit_ns and returns.
cudaError_t wait_probe_launch(int* d_err, uint64_t limit_ns, int code, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Operand formation and product combination (block_adds.cu).
//
// Form: for each sub-problem, read the M0*K0 (K0*N0) blocks of its input
// operand once and write every materialised S (T) operand of the level.
struct FormDesc {
  const double* in;   // sub-problem's A (or B) operand, column-major
  int64_t ld_in;
  double* out;        // first materialised output block
  int64_t ld_out;
  int64_t out_stride; // distance between consecutive output blocks (doubles)
  int64_t rows, cols; // dims of one block of this operand (= of one output)
};

// Combine: for each sub-problem, read its R product blocks once and write the
// M0*N0 blocks of its C operand (+ beta * C).
struct CombineDesc {
  const double* m;    // first product block M_1
  int64_t ld_m;
  int64_t m_stride;   // distance between consecutive product blocks (doubles)
  double* c;          // sub-problem's C operand
  int64_t ld_c;
  int64_t rows, cols; // dims of one C block (= of one product block)
  double beta;        // C blocks = sum (+ beta * C); 0 never reads C
};

struct CoefSlots {
  double v[FMM_MAX_SLOTS > 0 ? FMM_MAX_SLOTS : 1];
};

struct FormLaunch {
  const FormDesc* s_desc;  // A side
  const FormDesc* t_desc;  // B side
  int n_s, n_t;            // number of sub-problems on each side
  int64_t max_items;       // largest per-problem work-item count (grid sizing)
};

struct CombineLaunch {
  const CombineDesc* desc;
  int n;
  int64_t max_items;       // largest per-problem work-item count (grid sizing)
};

// Work items of one block of rows x cols for a kernel of 128-thread chunks
// of `vec` rows.
inline int64_t add_work_items(int64_t rows, int64_t cols, int vec) {
  const int64_t rv = rows / vec;
  return ((rv + 127) / 128) * cols;
}

cudaError_t form_launch(int alg, const FormLaunch& L, const CoefSlots& cf, bool vec2, int num_sms,
                        cudaStream_t stream);
cudaError_t combine_launch(int alg, const CombineLaunch& L, const CoefSlots& cf, bool vec2, int num_sms,
                           cudaStream_t stream);

// ---------------------------------------------------------------------------
// Diagonal scaling (scaling.cu).
//
// Device scratch of scaling_launch for m x k x n operands.
size_t scaling_scratch_bytes(int64_t m, int64_t k, int64_t n);
// Scales A (m x k) and B (k x n) in place, `num_steps` steps of scaling
// `type` (0 outside-inside, 1 inside-outside, 2 inside, 3 outside), and
// multiplies the row factors into r (m) and the column factors into s (n).
cudaError_t scaling_launch(double* A, int64_t lda, double* B, int64_t ldb, int m, int k, int n, int num_steps,
                           int type, double* r, double* s, void* scratch, cudaStream_t stream, int64_t* launches);
// C(i,j) = (C(i,j) * r[i]) * s[j].
cudaError_t scaling_postprocess_launch(double* C, int64_t ldc, int m, int n, const double* r, const double* s,
                                       cudaStream_t stream, int64_t* launches);
// The same with Scalar = float (the reference's Scaling<float> arithmetic).
cudaError_t scaling_launch(float* A, int64_t lda, float* B, int64_t ldb, int m, int k, int n, int num_steps,
                           int type, float* r, float* s, void* scratch, cudaStream_t stream, int64_t* launches);
cudaError_t scaling_postprocess_launch(float* C, int64_t ldc, int m, int n, const float* r, const float* s,
                                       cudaStream_t stream, int64_t* launches);

// ---------------------------------------------------------------------------
// FP32 <-> FP64 conversions of column-major matrices (convert.cu).
cudaError_t widen_launch(const float* src, int64_t lds, double* dst, int64_t ldd, int64_t rows, int64_t cols,
                         int num_sms, cudaStream_t stream);
cudaError_t narrow_launch(const double* src, int64_t lds, float* dst, int64_t ldd, int64_t rows, int64_t cols,
                          int num_sms, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Utilities (util_kernels.cu).
cudaError_t fill_uniform_launch(double* out, int64_t rows, int64_t cols, int64_t ld, uint64_t seed, uint64_t stream_id,
                                double lo, double hi, cudaStream_t stream);
// Writes {max_rel, max_abs} as two doubles into d_out (device).
cudaError_t max_rel_diff_launch(const double* a, int64_t lda, const double* b, int64_t ldb, int64_t m, int64_t n,
                                double* d_out, cudaStream_t stream);

// Sets the message fmm_last_error() returns on this host thread.
void set_last_error(const std::string& msg);

}  // namespace fmm
