// Split-BF16 leaf products on the sm_100a tensor cores (tcgen05, TMA, TMEM).
//
// An FP64 product C = alpha * A * B + beta * C is computed from BF16 slices:
//   * every row i of A is scaled by 2^-e_i (e_i: the least exponent with
//     max_p |a_ip| < 2^e_i), every column j of B by 2^-f_j; scaling by a
//     power of two is exact;
//   * each scaled value x in (-1, 1) is split into S integer digits
//     d_1 = rint(256 x), d_t = rint(256 r_{t-1}) with r the running
//     remainder, so x = sum_t d_t 2^-8t + r_S 2^-8S with |r_S| <= 1/2;
//     |d_1| <= 256 and |d_t| <= 128 are exact BF16 values;
//   * C_ij = alpha 2^(e_i + f_j) sum_{t+u <= S+1} 2^-8(t+u) (dA_t dB_u)_ij,
//     S (S + 1) / 2 slice products.  The products of one diagonal t + u are
//     accumulated by the tensor cores in FP32 over a group of k: 256 deep for
//     the diagonals t + u = 2, 3 at 3 slices or fewer, 128 deep otherwise
//     (SplitGroup in fmm_internal.h); every partial sum is an integer of
//     magnitude <= 2^24,
//     so the accumulation is exact.  Each group's sum is scaled by
//     2^-8(t+u) and added into an FP64 accumulator: all rounding happens in
//     FP64, in a fixed order;
//   * a row of A or column of B holding an Inf or a NaN gets the exponent
//     kSplitNonFinite and zero digits, and the entries of C it reaches are
//     NaN.
// Error: |x - sum_t d_t 2^-8t| <= 2^-(8S+1) 2^e per operand entry plus the
// dropped diagonals, so |C - AB| <~ 3 * 2^-8S * k * max|a_i.| * max|b_.j|.
//
// Split-INT8 (the same kernels, instantiated for 8-bit digits): the scaled x
// is split into signed bytes d_0 = rint(64 x), d_t = rint(128 r_{t-1}), so
// x = sum_t d_t 2^-(6+7t) + r 2^-(7S-1) with |d_t| <= 64 and |r| <= 1/2; the
// slice products run as tcgen05.mma kind::i8 (M256 N128 K32, twice the BF16
// rate) and accumulate in int32, exactly, over up to kSplitI8GroupChunks
// 256-deep chunks per diagonal, so a tile drains each diagonal once instead
// of once per chunk.  Each diagonal sum is scaled by 2^-(12+7D) and added
// into the FP64 accumulator in diagonal order.  A 128-byte slice row holds
// 128 k values, so the tensor maps, TMA boxes and shared-memory descriptors
// are those of the BF16 form byte for byte.  The diagonals run in pairs
// (D, D + 1) in two accumulators: a stage holds A_t with B_{D-t} and
// B_{D+1-t}, so one A tile feeds two products (a third fewer bytes per MMA).
// Error: |C - AB| <~ (S + 2) * 2^-7S * k * max|a_i.| * max|b_.j|.
//
// Product kernel: persistent CTA pairs (clusters of 2) over the 256 x 128
// output tiles of every problem, with the two-SM MMA: one thread of the
// pair leader issues tcgen05.mma.cta_group::2 (M256 N128 K16), which reads
// A rows 0-127 and B columns 0-63 from the leader's shared memory, A rows
// 128-255 and B columns 64-127 from the peer's, and accumulates each CTA's
// 128 rows in its own tensor memory.  One issuing thread thus drives two
// SMs, and each SM reads half of B.  In each CTA warp 0 issues TMA loads of
// its halves of (A_t, B_u) over one 128-deep chunk (48 KB) into a 4-stage
// ring, counted on the leader's full barrier; the leader's warp 1 issues 8
// MMAs per stage into one of four TMEM accumulators of 128 FP32 columns and
// multicasts its commits to both CTAs; the epilogue warps of each CTA (two
// or four warpgroups, splitting the 128 columns) drain each finished
// accumulator into FP64 registers and release it on the leader's barrier.
// Every mbarrier wait is bounded; on a timeout the kernel records a code in
// *err, lets its copies and MMAs in flight finish, frees its TMEM and
// returns.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "fmm_internal.h"
#include "sm100_primitives.cuh"

namespace fmm {
namespace {

using namespace sm100;

constexpr int kBM = kSplitTile, kBN = kSplitTile, kBK = kSplitKBlock;  // per CTA: 128 rows, all 128 columns
constexpr int kBHalf = kBN / 2;                    // columns of B held by each CTA of the pair
constexpr int kChunkBlocks = kSplitChunk / kBK;    // 64-deep k-blocks per chunk (2)
constexpr int kATileBytes = kBM * kBK * 2;         // one 128 x 64 BF16 box: 16 KB
constexpr int kBTileBytes = kBHalf * kBK * 2;      // one 64 x 64 BF16 box: 8 KB
// Two k-blocks of A and of the B half per stage (48 KB per CTA), 4 stages.
constexpr int kStageKBlocks = 2;
constexpr int kStageBytes = kStageKBlocks * (kATileBytes + kBTileBytes);
constexpr int kStages = 4;
constexpr int kAccBufs = 4;  // TMEM accumulators of 128 FP32 columns
constexpr uint16_t kPairMask = 0x3;  // both CTAs of the cluster
// TMA warp, MMA warp, kEpiGroups x 4 epilogue warps, each warpgroup owning
// kBN / kEpiGroups columns of the tile.  Few slices mean few products per
// drained diagonal, so the drains weigh more: 3 slices or fewer use four
// warpgroups of 32 columns (measured +6-8% at 3 slices), more slices two of
// 64 (four were 2% slower at 5).
constexpr int gemm_threads(int epi_groups) { return 32 * (2 + 4 * epi_groups); }
// INT8 digits pair the diagonals (D, D + 1): a stage holds A_t with B_{D-t}
// and B_{D+1-t} (64 KB, two products from one A tile), 3 stages.
constexpr int kI8StageBytes = kStageKBlocks * (kATileBytes + 2 * kBTileBytes);
constexpr int kI8Stages = 3;
constexpr size_t kGemmSmem = (size_t)kStages * kStageBytes + 1024;
static_assert((size_t)kI8Stages * kI8StageBytes + 1024 <= kGemmSmem && kI8Stages <= kStages, "INT8 ring fits");
static_assert(kChunkBlocks == 2 && kChunkBlocks % kStageKBlocks == 0, "stages tile the chunk");
static_assert(kBK * 2 == 128, "one k-block row is one 128-byte swizzle row");
static_assert(kATileBytes % 1024 == 0 && kBTileBytes % 1024 == 0, "128-byte-swizzled tiles start 1024-aligned");

// Largest i in [0, n) with key(d[i]) <= x (keys non-decreasing).
template <typename Key>
__device__ __forceinline__ int find_desc(const SplitDesc* __restrict__ d, int n, int64_t x, Key key) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (key(d[mid]) <= x)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// |x| as ordered bits: the patterns of non-negative doubles order like their
// values, and every NaN orders above Inf, so an integer maximum of these
// finds the largest magnitude and sees a NaN.
__device__ __forceinline__ unsigned long long abs_bits(double x) {
  return (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
}

// The least e with max |x| < 2^e from the maximum of abs_bits, 0 for an
// all-zero row, kSplitNonFinite when it holds an Inf or a NaN.
__device__ __forceinline__ int exponent_above(unsigned long long maxbits) {
  if (maxbits >= 0x7ff0000000000000ull) return kSplitNonFinite;
  if (maxbits == 0) return 0;
  int e;
  frexp(__longlong_as_double((long long)maxbits), &e);  // maxabs = f 2^e, f in [0.5, 1)
  return e;
}

// ---------------------------------------------------------------------------
// splitting

// x * 2^-e, rounded like ldexp(x, -e): a multiplication by the exact power of
// two when 2^-e is a normal double, ldexp otherwise.
__device__ __forceinline__ double scale_pow2(double x, int e) {
  if (e >= -1000 && e <= 1000) return x * __hiloint2double((1023 - e) << 20, 0);
  return ldexp(x, -e);
}

// Row exponents of A.  A block owns 32 padded rows (lane = row, so each
// column load of a warp is 256 contiguous bytes) and its kExpWarps warps
// split the columns, 8 loads in flight per thread; the warps' maxima meet
// in shared memory.  (One thread per row walking all k columns left a
// single large product with a few dozen blocks, latency-bound.)
constexpr int kExpWarps = 16;

__global__ void __launch_bounds__(kExpWarps * 32) split_row_exponents(const SplitDesc* __restrict__ d, int nd,
                                                                      int64_t row_tiles, int* __restrict__ ea) {
  __shared__ unsigned long long part[kExpWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t w = blockIdx.x; w < row_tiles; w += gridDim.x) {
    const int64_t x0 = w * 32;  // padded rows of one problem come in multiples of 256
    const int q = find_desc(d, nd, x0, [](const SplitDesc& s) { return s.e_off; });
    const SplitDesc& s = d[q];
    const int64_t i = x0 - s.e_off + lane;
    unsigned long long mx = 0;
    if (i < s.m) {
      const double* a = s.A + i;
      const int64_t lda = s.lda;
      int p = warp;
      for (; p + 7 * kExpWarps < s.k; p += 8 * kExpWarps) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = a[(int64_t)(p + u * kExpWarps) * lda];
#pragma unroll
        for (int u = 0; u < 8; ++u) mx = max(mx, abs_bits(v[u]));
      }
      for (; p < s.k; p += kExpWarps) mx = max(mx, abs_bits(a[(int64_t)p * lda]));
    }
    part[warp][lane] = mx;
    __syncthreads();
    if (warp == 0) {
      unsigned long long v = part[0][lane];
#pragma unroll
      for (int u = 1; u < kExpWarps; ++u) v = max(v, part[u][lane]);
      ea[x0 + lane] = exponent_above(v);
    }
    __syncthreads();  // part is reused by the next row tile
  }
}

// Digits of 8 scaled values as 8 BF16 per slice, one 16-byte store each.
// d = rint(256 x) and the remainder 256 x - d come from the FP64 pipe:
// 256 x is exact and |256 x| < 2^51, so fma(x, 256, 1.5 * 2^52) rounds it to
// the nearest integer (ties to even, as rint does) and that integer is the
// low word of the sum.  |d| <= 256, so its BF16 pattern is the top half of
// the FP32 value (1.5 * 2^23 + d) - 1.5 * 2^23 (exact).  No conversion-unit
// instruction is involved.
// The FP32 value of a small integer d (|d| <= 2^22), whose top half is the
// BF16 pattern of d when d has at most 8 significant bits.
__device__ __forceinline__ uint32_t f32_bits_of_small_int(int d) {
  return __float_as_uint(__int_as_float(0x4B400000 + d) - 12582912.0f);
}

__device__ __forceinline__ void store_digits(double (&x)[8], int slices, __nv_bfloat16* dst, int64_t slice_stride) {
  const double kRound = 6755399441055744.0;  // 1.5 * 2^52
  for (int t = 0; t < slices; ++t) {
    uint32_t w[4];
#pragma unroll
    for (int c = 0; c < 8; c += 2) {
      const double y0 = fma(x[c], 256.0, kRound), y1 = fma(x[c + 1], 256.0, kRound);
      x[c] = fma(x[c], 256.0, -(y0 - kRound));
      x[c + 1] = fma(x[c + 1], 256.0, -(y1 - kRound));
      // top halves of the two FP32 values: one byte permute
      w[c / 2] = __byte_perm(f32_bits_of_small_int(__double2loint(y0)), f32_bits_of_small_int(__double2loint(y1)),
                             0x7632);
    }
    *reinterpret_cast<uint4*>(dst + t * slice_stride) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// INT8 digits of 8 scaled values, one 8-byte store per slice: d_0 = rint(64 x),
// then d_t = rint(128 r), by the same FP64-pipe rounding; |d_t| <= 64, and
// the low byte of the sum's low word is the digit's two's complement.
__device__ __forceinline__ void store_digits_i8(double (&x)[8], int slices, uint8_t* dst, int64_t slice_stride) {
  const double kRound = 6755399441055744.0;  // 1.5 * 2^52
  double radix = 64.0;
  for (int t = 0; t < slices; ++t) {
    uint32_t lo[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double y = fma(x[c], radix, kRound);
      x[c] = fma(x[c], radix, -(y - kRound));
      lo[c] = (uint32_t)__double2loint(y);
    }
    // the low bytes of lo[0..3] (lo[4..7]) in order: three byte permutes each
    const uint32_t w0 = __byte_perm(__byte_perm(lo[0], lo[1], 0x0040), __byte_perm(lo[2], lo[3], 0x0040), 0x5410);
    const uint32_t w1 = __byte_perm(__byte_perm(lo[4], lo[5], 0x0040), __byte_perm(lo[6], lo[7], 0x0040), 0x5410);
    *reinterpret_cast<uint2*>(dst + t * slice_stride) = make_uint2(w0, w1);
    radix = 128.0;
  }
}

// A slices: one work tile = 32 rows x 64 k (one BF16 k-block, half an INT8 one), read column-major
// (coalesced along rows) into shared memory, written as 128-byte k-block rows
// for every slice (8 threads per row, 16 bytes each).  The tile's row index
// is XOR-swizzled by k so that both the column-wise fill and the row-wise
// read-out touch every bank pair at most twice per warp.
// Position of an A-splitting work tile: its problem q, row tile rt (32
// rows) and 64-deep k-block kb.  A block's tiles advance by a fixed stride
// (the grid size), which within one problem is a fixed step in (rt, kb): no
// search and no division unless the tile enters another problem.  A
// problem's tiles number (padded rows / 32) * (64-deep k-blocks) < 2^32.
struct ATile {
  int q;
  int64_t end;              // first work tile after problem q
  uint32_t rows;            // row tiles of problem q
  uint32_t rt, kb;          // position within problem q
  uint32_t step_rt, step_kb;  // the stride in row tiles and k-blocks
};

__device__ __forceinline__ void atile_seek(const SplitDesc* __restrict__ d, int nd, int64_t total, int64_t w,
                                           uint32_t stride, ATile& t) {
  t.q = find_desc(d, nd, w, [](const SplitDesc& s) { return s.sa_begin; });
  const SplitDesc& s = d[t.q];
  t.end = t.q + 1 < nd ? d[t.q + 1].sa_begin : total;
  t.rows = (uint32_t)s.tiles_m * (kBM / 32);
  const uint32_t local = (uint32_t)(w - s.sa_begin);
  t.rt = local % t.rows;
  t.kb = local / t.rows;
  t.step_rt = stride % t.rows;
  t.step_kb = stride / t.rows;
}

__device__ __forceinline__ void atile_next(const SplitDesc* __restrict__ d, int nd, int64_t total, int64_t w,
                                           uint32_t stride, ATile& t) {
  if (w < t.end) {
    t.rt += t.step_rt;
    t.kb += t.step_kb;
    if (t.rt >= t.rows) {
      t.rt -= t.rows;
      ++t.kb;
    }
  } else {
    atile_seek(d, nd, total, w, stride, t);
  }
}

template <bool kInt8>
__global__ void __launch_bounds__(256) split_a(const SplitDesc* __restrict__ d, int nd, int64_t total, int slices,
                                               const int* __restrict__ ea, uint8_t* __restrict__ out) {
  __shared__ double tile[64 * 32];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int row = threadIdx.x >> 3, kc = (threadIdx.x & 7) * 8;
  const uint32_t stride = gridDim.x;
  auto at = [](int k, int r) { return k * 32 + (r ^ (((k >> 3) & 3) << 2)); };
  // The next tile's loads are issued before this tile's digits are computed
  // and stored, so each thread keeps a tile of loads in flight.
  auto load = [&](const ATile& t, double (&v)[8]) {
    const SplitDesc& s = d[t.q];
    const int64_t i = (int64_t)t.rt * 32 + tx, p0 = (int64_t)t.kb * kBK;
    const double* a = s.A + i + p0 * s.lda;
    if (i < s.m && p0 + kBK <= s.k) {
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = a[(int64_t)(ty + 8 * r) * s.lda];
    } else {
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int64_t p = p0 + ty + 8 * r;
        v[r] = (i < s.m && p < s.k) ? a[(int64_t)(ty + 8 * r) * s.lda] : 0.0;
      }
    }
  };
  double pre[8];
  ATile next;
  if ((int64_t)blockIdx.x < total) {
    atile_seek(d, nd, total, blockIdx.x, stride, next);
    load(next, pre);
  }
  for (int64_t w = blockIdx.x; w < total; w += stride) {
    const ATile cur = next;
    const SplitDesc& s = d[cur.q];
    const int64_t mp = (int64_t)s.tiles_m * kBM;
    const int64_t kb = cur.kb;
    const int64_t i0 = (int64_t)cur.rt * 32;
    __syncthreads();  // previous tile's readers are done
#pragma unroll
    for (int r = 0; r < 8; ++r) tile[at(ty + 8 * r, tx)] = pre[r];
    __syncthreads();
    if (w + stride < total) {
      atile_next(d, nd, total, w + stride, stride, next);
      load(next, pre);
    }
    const int e = ea[s.e_off + i0 + row];
    double x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = e == kSplitNonFinite ? 0.0 : scale_pow2(tile[at(kc + c, row)], e);
    const int64_t slice_bytes = (int64_t)s.kblocks * mp * 128;
    if constexpr (kInt8) {
      const int64_t orow = s.a_row + (kb >> 1) * mp + i0 + row;
      store_digits_i8(x, slices, out + orow * 128 + (kb & 1) * 64 + kc, slice_bytes);
    } else {
      const int64_t orow = s.a_row + kb * mp + i0 + row;
      store_digits(x, slices, reinterpret_cast<__nv_bfloat16*>(out + orow * 128) + kc, slice_bytes / 2);
    }
  }
}

// B: one warp per padded column: the column maximum (a warp butterfly), then
// the slices, 8 consecutive k per lane (B's columns are contiguous in k, so
// they are written as they are read; the second read hits L2).  A warp's
// columns advance by a fixed stride, so the problem search runs only when a
// column enters another problem, and no block barrier is involved.
constexpr int kSplitBWarps = 8;

template <bool kInt8>
__global__ void __launch_bounds__(32 * kSplitBWarps) split_b(const SplitDesc* __restrict__ d, int nd, int64_t total,
                                                             int slices, int* __restrict__ fb,
                                                             uint8_t* __restrict__ out) {
  constexpr int kRowValues = kInt8 ? kSplitI8KBlock : kBK;  // k values per 128-byte slice row
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * kSplitBWarps;
  int q = -1;
  int64_t q_end = 0;  // first column after problem q
  for (int64_t x = (int64_t)blockIdx.x * kSplitBWarps + (threadIdx.x >> 5); x < total; x += stride) {
    if (q < 0 || x >= q_end) {
      q = find_desc(d, nd, x, [](const SplitDesc& s) { return s.f_off; });
      q_end = q + 1 < nd ? d[q + 1].f_off : total;
    }
    const SplitDesc& s = d[q];
    const int64_t j = x - s.f_off;
    const int64_t np = (int64_t)s.tiles_n * kBN;
    const double* b = s.B + j * s.ldb;
    const bool live = j < s.n;
    const bool vec = (reinterpret_cast<uintptr_t>(b) & 15) == 0;
    const int k = s.k, kp = s.kblocks * kRowValues;
    auto load8 = [&](int p0, double (&v)[8]) {
      if (vec && p0 + 8 <= k) {
#pragma unroll
        for (int c = 0; c < 8; c += 2) {
          const double2 t2 = *reinterpret_cast<const double2*>(b + p0 + c);
          v[c] = t2.x;
          v[c + 1] = t2.y;
        }
      } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = p0 + c < k ? b[p0 + c] : 0.0;
      }
    };
    unsigned long long mx = 0;
    if (live) {
#pragma unroll 4
      for (int p0 = lane * 8; p0 < k; p0 += 256) {
        double v[8];
        load8(p0, v);
#pragma unroll
        for (int c = 0; c < 8; ++c) mx = max(mx, abs_bits(v[c]));
      }
    }
    for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    const int f = exponent_above(mx);
    if (lane == 0) fb[x] = f;
    const int64_t slice_bytes = (int64_t)s.kblocks * np * 128;
#pragma unroll 2
    for (int p0 = lane * 8; p0 < kp; p0 += 256) {
      double v[8];
      if (live) {
        load8(p0, v);
      } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = 0.0;
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) v[c] = f == kSplitNonFinite ? 0.0 : scale_pow2(v[c], f);
      const int64_t orow = s.b_row + (int64_t)(p0 / kRowValues) * np + j;
      if constexpr (kInt8)
        store_digits_i8(v, slices, out + orow * 128 + (p0 % kRowValues), slice_bytes);
      else
        store_digits(v, slices, reinterpret_cast<__nv_bfloat16*>(out + orow * 128) + (p0 % kRowValues),
                     slice_bytes / 2);
    }
  }
}

// ---------------------------------------------------------------------------
// tensor-core product of the slices

struct GemmParams {
  const SplitDesc* desc;
  const int* ea;
  const int* fb;
  int* err;
  int nd;
  int slices;
  int64_t tiles;
};

struct TileCoord {
  int q, tm, tn;
};

// Tiles of a problem (256 x 128, one per CTA pair; tm counts 256-row tiles)
// are walked in groups of kRasterRows tile rows, row index fastest within a
// group: the pairs of one wave share A slices across a group's columns and B
// slices down its rows, so both stay in L2 between them.  Measured on one
// B200 at 16384^3 and 8192^3 (5 and 3 slices, and Strassen's 49-leaf
// launches): groups of 1 and 2 pair rows within noise of each other, 4 about
// 1.5% and 8 about 3% slower, 16 slower still.
constexpr int kRasterRows = 2;

__device__ __forceinline__ TileCoord tile_coord(const GemmParams& g, int64_t tile) {
  TileCoord c;
  c.q = find_desc(g.desc, g.nd, tile, [](const SplitDesc& s) { return s.tile_begin; });
  const SplitDesc& s = g.desc[c.q];
  const int pair_rows = s.tiles_m / 2;
  const int64_t rem = tile - s.tile_begin;
  const int64_t per_group = (int64_t)kRasterRows * s.tiles_n;
  const int64_t group = rem / per_group;
  const int first = (int)(group * kRasterRows);
  const int rows = pair_rows - first < kRasterRows ? pair_rows - first : kRasterRows;
  const int64_t local = rem - group * per_group;
  c.tm = first + (int)(local % rows);
  c.tn = (int)(local / rows);
  return c;
}

// Calls fn(D, c0, c1) for the accumulation groups of a tile in order
// (split_group), until fn returns false; returns whether all ran.  With one
// chunk per group the loops are the plain chunk-then-diagonal order.  INT8
// digits: each diagonal over up to kSplitI8GroupChunks chunks (exact int32).
template <int kSpan, bool kInt8, class Fn>
__device__ __forceinline__ bool for_each_group(int chunks, int S, Fn&& fn) {
  if constexpr (kInt8) {
    for (int c0 = 0; c0 < chunks; c0 += kSplitI8GroupChunks) {
      const int c1 = min(c0 + kSplitI8GroupChunks, chunks);
      for (int D = 0; D < S; ++D)
        if (!fn(D, c0, c1)) return false;
    }
  } else if constexpr (kSpan == 1) {
    for (int c = 0; c < chunks; ++c)
      for (int D = 0; D < S; ++D)
        if (!fn(D, c, c + 1)) return false;
  } else {
    for (int cp = 0; cp < chunks; cp += kSpan) {
      const int nch = min(kSpan, chunks - cp);
      for (int gi = 0; gi < split_groups_in_pair(nch, S); ++gi) {
        const SplitGroup G = split_group(cp, nch, S, gi);
        if (!fn(G.D, G.c0, G.c1)) return false;
      }
    }
  }
  return true;
}

// A drained accumulator value as a double (exact either way) and the weight
// of diagonal D: FP32 sums of BF16 digits weigh 2^-8(D+2), int32 sums of
// INT8 digits 2^-(12+7D).
template <bool kInt8>
__device__ __forceinline__ double acc_value(uint32_t r) {
  if constexpr (kInt8)
    return (double)(int32_t)r;
  else
    return (double)__uint_as_float(r);
}

template <bool kInt8>
__device__ __forceinline__ double diagonal_weight(int D) {
  return kInt8 ? ldexp(1.0, -(12 + 7 * D)) : ldexp(1.0, -8 * (D + 2));
}

template <int kEpiGroups, bool kInt8>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(gemm_threads(kEpiGroups), 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const GemmParams g) {
  constexpr int kEpiCols = kBN / kEpiGroups;
  constexpr int kEpiWarps = 4 * kEpiGroups;
  // chunks per accumulation pair: the four-warpgroup form runs 3 slices or
  // fewer, where split_chunk_span pairs chunks (the launch checks this)
  constexpr int kSpan = kEpiGroups == 4 ? 2 : 1;
  static_assert(kEpiCols % 16 == 0, "drains move pairs of 8-column pieces");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  // full: the leader's count both CTAs' copies of a stage; empty, acc_full:
  // MMA commits multicast to both CTAs; acc_empty (leader's): 8 epilogue
  // warps of each CTA
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], acc_full[kAccBufs], acc_empty[kAccBufs], mma_done;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = g.slices;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int64_t pair = blockIdx.x >> 1, pairs = gridDim.x >> 1;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < kAccBufs; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 2 * kEpiWarps);
    }
    mbar_init(&mma_done, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc_pair(&tmem_slot, kAccBufs * kBN);
  tc_fence_before();
  cluster_sync();  // barriers of both CTAs initialised, tensor memory allocated
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  // the stage ring: 4 stages of one slice product (BF16), 3 of a diagonal pair (INT8)
  constexpr int kSt = kInt8 ? kI8Stages : kStages;
  constexpr int kStB = kInt8 ? kI8StageBytes : kStageBytes;

  if (warp == 0) {
    if (lane == 0) {
      // one stage = one slice product over one 128-deep chunk: this CTA's
      // 128 rows of A_t and 64 columns of B_u, two 64-deep k-blocks each
      prefetch_tensormap(&tmA);
      prefetch_tensormap(&tmB);
      uint32_t n = 0, st = 0, ph = 0;  // stages filled, current stage, its round parity
      bool ok = true;
      for (int64_t tile = pair; tile < g.tiles && ok; tile += pairs) {
        const TileCoord tc = tile_coord(g, tile);
        const SplitDesc& s = g.desc[tc.q];
        const int64_t mp = (int64_t)s.tiles_m * kBM, np = (int64_t)s.tiles_n * kBN;
        const int64_t ya_tile = s.a_row + (int64_t)tc.tm * kSplitPairRows + rank * kBM;
        const int64_t yb_tile = s.b_row + (int64_t)tc.tn * kBN + rank * kBHalf;
        const int chunks = s.kblocks / kChunkBlocks;
        if constexpr (kInt8) {
          // one stage: A_t with B_u1 and, for a paired product, B_u2, over
          // one 256-deep chunk starting at k-block blk
          auto load_stage = [&](int t, int u1, int u2, int64_t blk) -> bool {
            if (n >= (uint32_t)kSt && !mbar_wait(&empty[st], ph ^ 1u, g.err, 1)) return false;
            uint8_t* dst = base + st * kStB;
            const uint32_t bar = cluster_addr(&full[st], 0);  // the leader's
            const uint32_t bytes = kStageKBlocks * (kATileBytes + (u2 >= 0 ? 2 : 1) * kBTileBytes);
            if (leader) mbar_arrive_expect_tx(&full[st], 2 * bytes);
            const int64_t ya = ya_tile + ((int64_t)t * s.kblocks + blk) * mp;
            const int64_t yb1 = yb_tile + ((int64_t)u1 * s.kblocks + blk) * np;
#pragma unroll
            for (int b = 0; b < kStageKBlocks; ++b) {
              tma_load_2d_pair(dst + b * kATileBytes, &tmA, bar, 0, (int)(ya + b * mp));
              tma_load_2d_pair(dst + kStageKBlocks * kATileBytes + b * kBTileBytes, &tmB, bar, 0,
                               (int)(yb1 + b * np));
            }
            if (u2 >= 0) {
              const int64_t yb2 = yb_tile + ((int64_t)u2 * s.kblocks + blk) * np;
#pragma unroll
              for (int b = 0; b < kStageKBlocks; ++b)
                tma_load_2d_pair(dst + kStageKBlocks * (kATileBytes + kBTileBytes) + b * kBTileBytes, &tmB, bar, 0,
                                 (int)(yb2 + b * np));
            }
            ++n;
            if (++st == (uint32_t)kSt) {
              st = 0;
              ph ^= 1u;
            }
            return true;
          };
          // per group of chunks, the diagonal pairs (D0, D0 + 1) in order;
          // per chunk the stages t = 0..D0 (products (t, D0 - t) and
          // (t, D0 + 1 - t)) and the lone (D0 + 1, 0); an odd last diagonal
          // alone
          for (int cg = 0; cg < chunks && ok; cg += kSplitI8GroupChunks) {
            const int cend = min(cg + kSplitI8GroupChunks, chunks);
            for (int D0 = 0; D0 < S && ok; D0 += 2) {
              const bool two = D0 + 1 < S;
              for (int c = cg; c < cend && ok; ++c)
                for (int t = 0; t <= D0 + (two ? 1 : 0) && ok; ++t)
                  ok = load_stage(t, t <= D0 ? D0 - t : 0, (two && t <= D0) ? D0 + 1 - t : -1,
                                  (int64_t)c * kChunkBlocks);
            }
          }
          continue;
        }
        ok = for_each_group<kSpan, kInt8>(chunks, S, [&](int D, int c0, int c1) {
          for (int c = c0; c < c1; ++c)
            for (int t = 0; t <= D; ++t)
              for (int h = 0; h < kChunkBlocks; h += kStageKBlocks) {
                if (n >= (uint32_t)kStages && !mbar_wait(&empty[st], ph ^ 1u, g.err, 1)) return false;
                const int64_t blk = (int64_t)c * kChunkBlocks + h;
                const int64_t ya = ya_tile + ((int64_t)t * s.kblocks + blk) * mp;
                const int64_t yb = yb_tile + ((int64_t)(D - t) * s.kblocks + blk) * np;
                uint8_t* dst = base + st * kStageBytes;
                const uint32_t bar = cluster_addr(&full[st], 0);  // the leader's
                if (leader) mbar_arrive_expect_tx(&full[st], 2 * kStageBytes);
#pragma unroll
                for (int b = 0; b < kStageKBlocks; ++b) {
                  tma_load_2d_pair(dst + b * kATileBytes, &tmA, bar, 0, (int)(ya + b * mp));
                  tma_load_2d_pair(dst + kStageKBlocks * kATileBytes + b * kBTileBytes, &tmB, bar, 0,
                                   (int)(yb + b * np));
                }
                ++n;
                if (++st == (uint32_t)kStages) {
                  st = 0;
                  ph ^= 1u;
                }
              }
          return true;
        });
      }
      // Before the CTA can leave, its copies must have landed: each stage's
      // last round is released by the MMAs that read it, which waited for
      // the copies.  After an error the releases may never come; the wait
      // is then bounded and a short pause lets copies in flight land.
      bool drained = true;
      for (uint32_t sx = 0; sx < (uint32_t)kSt && sx < n; ++sx) {
        const uint32_t last = (n - 1 - sx) / kSt;  // round of stage sx
        drained = mbar_drain(&empty[sx], last & 1, 1000000ull) && drained;
      }
      if (!drained) spin_ns(100000ull);
    }
  } else if (warp == 1) {
    if (lane == 0 && leader) {
      const uint32_t idesc = kInt8 ? idesc_s8_s32(kSplitPairRows, kBN) : idesc_bf16_f32(kSplitPairRows, kBN);
      uint32_t st = 0, ph = 0, ai = 0;
      bool ok = true;
      for (int64_t tile = pair; tile < g.tiles && ok; tile += pairs) {
        const TileCoord tc = tile_coord(g, tile);
        const int chunks = g.desc[tc.q].kblocks / kChunkBlocks;
        if constexpr (kInt8) {
          // the producer's order: per group of chunks, per diagonal pair
          // (D0, D0 + 1) in accumulators b0, b1, per chunk the stages
          // t = 0..D0 (8 MMAs into b0 from B_{D0-t}, 8 into b1 from
          // B_{D0+1-t}) and the lone (D0 + 1, 0) into b1
          for (int cg = 0; cg < chunks && ok; cg += kSplitI8GroupChunks) {
            const int cend = min(cg + kSplitI8GroupChunks, chunks);
            for (int D0 = 0; D0 < S && ok; D0 += 2) {
              const bool two = D0 + 1 < S;
              const uint32_t b0 = ai % kAccBufs, b1 = (ai + 1) % kAccBufs;
              if (ai >= (uint32_t)kAccBufs && !mbar_wait(&acc_empty[b0], ((ai / kAccBufs) - 1) & 1, g.err, 2)) {
                ok = false;
                break;
              }
              if (two && ai + 1 >= (uint32_t)kAccBufs &&
                  !mbar_wait(&acc_empty[b1], (((ai + 1) / kAccBufs) - 1) & 1, g.err, 2)) {
                ok = false;
                break;
              }
              tc_fence_after();
              for (int c = cg; c < cend && ok; ++c)
                for (int t = 0; t <= D0 + (two ? 1 : 0); ++t) {
                  if (!mbar_wait(&full[st], ph, g.err, 3)) {
                    ok = false;
                    break;
                  }
                  tc_fence_after();
                  const bool paired = two && t <= D0;
                  const uint32_t d_first = tmem + ((two && t > D0) ? b1 : b0) * kBN;
                  const uint32_t a = smem_addr(base + st * kStB);
                  const uint32_t bb1 = a + kStageKBlocks * kATileBytes;
                  const uint32_t bb2 = bb1 + kStageKBlocks * kBTileBytes;
#pragma unroll
                  for (int kk = 0; kk < kStageKBlocks * kBK / 16; ++kk) {
                    const uint32_t koff = (kk & 3) * 32;
                    mma_s8_pair(d_first, smem_desc_sw128(a + (kk >> 2) * kATileBytes + koff),
                                smem_desc_sw128(bb1 + (kk >> 2) * kBTileBytes + koff), idesc,
                                c > cg || t > 0 || kk > 0);
                  }
                  if (paired) {
#pragma unroll
                    for (int kk = 0; kk < kStageKBlocks * kBK / 16; ++kk) {
                      const uint32_t koff = (kk & 3) * 32;
                      mma_s8_pair(tmem + b1 * kBN, smem_desc_sw128(a + (kk >> 2) * kATileBytes + koff),
                                  smem_desc_sw128(bb2 + (kk >> 2) * kBTileBytes + koff), idesc,
                                  c > cg || t > 0 || kk > 0);
                    }
                  }
                  mma_commit_pair(&empty[st], kPairMask);
                  if (++st == (uint32_t)kSt) {
                    st = 0;
                    ph ^= 1u;
                  }
                }
              if (!ok) break;
              mma_commit_pair(&acc_full[b0], kPairMask);
              if (two) mma_commit_pair(&acc_full[b1], kPairMask);
              ai += two ? 2 : 1;
            }
          }
          continue;
        }
        ok = for_each_group<kSpan, kInt8>(chunks, S, [&](int D, int c0, int c1) {
          const uint32_t buf = ai % kAccBufs;
          if (ai >= (uint32_t)kAccBufs && !mbar_wait(&acc_empty[buf], ((ai / kAccBufs) - 1) & 1, g.err, 2))
            return false;
          tc_fence_after();
          const uint32_t d_tmem = tmem + buf * kBN;
          for (int c = c0; c < c1; ++c)
            for (int t = 0; t <= D; ++t)
              for (int h = 0; h < kChunkBlocks; h += kStageKBlocks) {
                if (!mbar_wait(&full[st], ph, g.err, 3)) return false;
                tc_fence_after();
                const uint32_t a = smem_addr(base + st * kStageBytes);
                const uint32_t b = a + kStageKBlocks * kATileBytes;
#pragma unroll
                for (int kk = 0; kk < kStageKBlocks * kBK / 16; ++kk) {  // 32 bytes of each row per MMA
                  const uint32_t koff = (kk & 3) * 32;
                  const uint64_t ad = smem_desc_sw128(a + (kk >> 2) * kATileBytes + koff);
                  const uint64_t bd = smem_desc_sw128(b + (kk >> 2) * kBTileBytes + koff);
                  const bool accumulate = c > c0 || t > 0 || h > 0 || kk > 0;
                  if constexpr (kInt8)
                    mma_s8_pair(d_tmem, ad, bd, idesc, accumulate);
                  else
                    mma_bf16_pair(d_tmem, ad, bd, idesc, accumulate);
                }
                mma_commit_pair(&empty[st], kPairMask);
                if (++st == (uint32_t)kStages) {
                  st = 0;
                  ph ^= 1u;
                }
              }
          mma_commit_pair(&acc_full[buf], kPairMask);
          ++ai;
          return true;
        });
      }
      // every MMA issued by this thread completes before tensor memory is freed
      mma_commit_pair(&mma_done, 0x1);
      mbar_drain(&mma_done, 0, 1000000000ull);
    }
  } else {
    // warpgroup wg owns columns [kEpiCols wg, kEpiCols (wg + 1)) of the tile; warp
    // quadrant qd owns TMEM lanes (this CTA's tile rows) [32 qd, 32 qd + 32)
    const int wg = (warp - 2) >> 2, qd = warp & 3;
    const int row_in_tile = qd * 32 + lane;
    uint32_t ai = 0;
    bool ok = true;
    for (int64_t tile = pair; tile < g.tiles && ok; tile += pairs) {
      const TileCoord tc = tile_coord(g, tile);
      const SplitDesc& s = g.desc[tc.q];
      const int chunks = s.kblocks / kChunkBlocks;
      double acc[kEpiCols];
#pragma unroll
      for (int j = 0; j < kEpiCols; ++j) acc[j] = 0.0;
      ok = for_each_group<kSpan, kInt8>(chunks, S, [&](int D, int, int) {
          const int buf = ai % kAccBufs;
          if (!mbar_wait(&acc_full[buf], (ai / kAccBufs) & 1, g.err, 4)) return false;
          tc_fence_after();
          const double scale = diagonal_weight<kInt8>(D);
          const uint32_t taddr = tmem + ((uint32_t)(qd * 32) << 16) + buf * kBN + wg * kEpiCols;
          // eight pieces of 8 columns, software-pipelined: the load of piece
          // g + 1 is in flight while piece g is converted and accumulated
          uint32_t r0[8], r1[8];
          tmem_ld_32x32b_x8(taddr, r0);
          tmem_ld_wait();
#pragma unroll
          for (int g8 = 0; g8 < kEpiCols / 8; g8 += 2) {
            tmem_ld_32x32b_x8(taddr + (g8 + 1) * 8, r1);
#pragma unroll
            for (int j = 0; j < 8; ++j)
              acc[g8 * 8 + j] = fma(acc_value<kInt8>(r0[j]), scale, acc[g8 * 8 + j]);
            tmem_ld_wait();
            if (g8 + 2 < kEpiCols / 8) tmem_ld_32x32b_x8(taddr + (g8 + 2) * 8, r0);
            if (g8 + 2 == kEpiCols / 8) {  // the accumulator is free once the last piece is in registers
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive_cluster(cluster_addr(&acc_empty[buf], 0));  // the leader's
            }
#pragma unroll
            for (int j = 0; j < 8; ++j)
              acc[(g8 + 1) * 8 + j] = fma(acc_value<kInt8>(r1[j]), scale, acc[(g8 + 1) * 8 + j]);
            if (g8 + 2 < kEpiCols / 8) tmem_ld_wait();
          }
          ++ai;
          return true;
        });
      if (!ok) break;
      const int64_t row = (int64_t)tc.tm * kSplitPairRows + rank * kBM + row_in_tile;
      if (row < s.m) {
        const int er = g.ea[s.e_off + row];
        const int64_t col0 = (int64_t)tc.tn * kBN + wg * kEpiCols;
        const int* fcol = g.fb + s.f_off + col0;
        double* cp = s.C + row;
        const double alpha = s.alpha, beta = s.beta;
#pragma unroll
        for (int j = 0; j < kEpiCols; ++j) {
          const int64_t col = col0 + j;
          if (col < s.n) {
            double v = __dmul_rn(alpha, ldexp(acc[j], er + fcol[j]));
            if (beta != 0.0) v = __dadd_rn(v, __dmul_rn(beta, cp[col * s.ldc]));
            if (er == kSplitNonFinite || fcol[j] == kSplitNonFinite) v = __longlong_as_double(0x7ff8000000000000ll);
            cp[col * s.ldc] = v;
          }
        }
      }
    }
  }
  // no CTA of the pair leaves (or frees tensor memory) while the other may
  // still read its shared memory or arrive on its barriers
  tc_fence_before();
  cluster_sync();
  tc_fence_after();
  if (warp == 1) {
    __syncwarp();
    tmem_dealloc_pair(tmem, kAccBufs * kBN);
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// {64 BF16 or 128 INT8, rows} view of a slice buffer; boxes of `box_rows`
// 128-byte rows.
bool encode_slices(CUtensorMap* map, void* base, int64_t rows, int box_rows, bool int8) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t row_values = int8 ? 128 : 64;
  const cuuint64_t dims[2] = {row_values, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {128};
  const cuuint32_t box[2] = {(cuuint32_t)row_values, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  return enc(map, int8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box,
             es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

unsigned grid_for(int64_t work, int64_t cap) { return (unsigned)(work < cap ? (work > 0 ? work : 1) : cap); }

// One thread waits on an mbarrier that nothing arrives on: the bounded wait
// must give up after limit_ns and record `code` (a check of the timeout path
// that every kernel here relies on).
__global__ void wait_probe_kernel(int* err, uint64_t limit_ns, int code) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  fence_barrier_init();
  mbar_wait(&bar, 0, err, code, limit_ns);
}

}  // namespace

cudaError_t wait_probe_launch(int* d_err, uint64_t limit_ns, int code, cudaStream_t stream) {
  wait_probe_kernel<<<1, 32, 0, stream>>>(d_err, limit_ns, code);
  return cudaGetLastError();
}

cudaError_t split_gemm_launch(const SplitDesc* d_descs, int n, const SplitPlan& plan, void* scratch, int* d_err,
                              int num_sms, cudaStream_t stream, int64_t* launches, cudaEvent_t split_done) {
  if (plan.tiles == 0) return cudaSuccess;
  if (plan.slices < kSplitMinSlices || plan.slices > (plan.int8 ? kSplitI8MaxSlices : kSplitMaxSlices) || !d_err ||
      !scratch || reinterpret_cast<uintptr_t>(scratch) % 256 != 0)
    return cudaErrorInvalidValue;
  // tensor-map row coordinates are 32-bit
  if (plan.rows_a >= (int64_t(1) << 31) || plan.rows_b >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  char* base = static_cast<char*>(scratch);
  uint8_t* as = reinterpret_cast<uint8_t*>(base);
  uint8_t* bs = reinterpret_cast<uint8_t*>(base + plan.off_b);
  int* ea = reinterpret_cast<int*>(base + plan.off_e);
  int* fb = reinterpret_cast<int*>(base + plan.off_f);
  const int64_t cap = (int64_t)num_sms * 16;
  split_row_exponents<<<grid_for(plan.n_e / 32, (int64_t)num_sms * 4), kExpWarps * 32, 0, stream>>>(d_descs, n,
                                                                                             plan.n_e / 32, ea);
  if (plan.int8) {
    split_a<true><<<grid_for(plan.sa_work, cap), 256, 0, stream>>>(d_descs, n, plan.sa_work, plan.slices, ea, as);
    split_b<true><<<grid_for((plan.n_f + kSplitBWarps - 1) / kSplitBWarps, cap), 32 * kSplitBWarps, 0, stream>>>(
        d_descs, n, plan.n_f, plan.slices, fb, bs);
  } else {
    split_a<false><<<grid_for(plan.sa_work, cap), 256, 0, stream>>>(d_descs, n, plan.sa_work, plan.slices, ea, as);
    split_b<false><<<grid_for((plan.n_f + kSplitBWarps - 1) / kSplitBWarps, cap), 32 * kSplitBWarps, 0, stream>>>(
        d_descs, n, plan.n_f, plan.slices, fb, bs);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (split_done && (e = cudaEventRecord(split_done, stream)) != cudaSuccess) return e;
  CUtensorMap tA, tB;
  if (!encode_slices(&tA, as, plan.rows_a, kBM, plan.int8) || !encode_slices(&tB, bs, plan.rows_b, kBHalf, plan.int8))
    return cudaErrorInvalidValue;
  GemmParams gp;
  gp.desc = d_descs;
  gp.ea = ea;
  gp.fb = fb;
  gp.err = d_err;
  gp.nd = n;
  gp.slices = plan.slices;
  gp.tiles = plan.tiles;
  static bool opted_in[64] = {};
  static std::mutex mu;
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64 || !opted_in[dev]) {
      e = cudaFuncSetAttribute(split_gemm_kernel<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kGemmSmem);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(split_gemm_kernel<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kGemmSmem);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(split_gemm_kernel<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kGemmSmem);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) opted_in[dev] = true;
    }
  }
  // CTA pairs: the grid is even and a pair's CTAs are consecutive blocks
  const unsigned pairs = grid_for(plan.tiles, num_sms / 2 > 0 ? num_sms / 2 : 1);
  if (split_chunk_span(plan.slices) != (plan.slices <= 3 ? 2 : 1)) return cudaErrorInvalidValue;
  if (plan.int8)  // one drain per diagonal and tile: two epilogue warpgroups suffice
    split_gemm_kernel<2, true><<<2 * pairs, gemm_threads(2), kGemmSmem, stream>>>(tA, tB, gp);
  else if (plan.slices <= 3)
    split_gemm_kernel<4, false><<<2 * pairs, gemm_threads(4), kGemmSmem, stream>>>(tA, tB, gp);
  else
    split_gemm_kernel<2, false><<<2 * pairs, gemm_threads(2), kGemmSmem, stream>>>(tA, tB, gp);
  e = cudaGetLastError();
  if (e == cudaSuccess && launches) *launches += 4;
  return e;
}

}  // namespace fmm
