// FP64 products with at most kThinMax rows or columns: the fringe products of
// dynamic peeling (linalg/linalg.hpp:201-244), C = alpha * A * B + beta * C,
// where the peeled rows (or columns) of one level meet the whole inner
// dimension of its sub-problem.
//
// In the tensor-core GEMM such a product fills only 2-7 rows of every 128-row
// tile and walks the full k in one CTA, so a fringe launch is bound by a few
// long, nearly empty tiles.  Here the work is what the product needs: each
// element of the long operand is read once from memory, the short operand
// (at most kThinMax x k) comes from L1 / L2, FMAs run on the FP64 pipe, no
// barrier sits inside the k loop, and every output is summed in a fixed
// order:
//   * few rows (m <= kThinMax): a warp per column j of C; lane l adds the
//     products of k indices l, l + 32, ... of each 256-deep block, the block
//     sums go into a running sum per lane, and the 32 lane sums meet in a
//     fixed butterfly;
//   * few columns (n <= kThinMax): a thread per row in blocks of 64 rows and
//     four groups of threads per row block, group g taking the g-th quarter
//     of k in 256-deep blocks into a running sum; the four sums are added
//     (g0 + g1) + (g2 + g3).
//   * few inner indices (k <= kThinMax, the k fringe C_core += A(:, kx)
//     B(kx, :)): a 64 x 64 block of C per work item, a thread per pair of
//     rows and 8 columns; C is read and written once with 16-byte accesses
//     where it allows them, the short panels come from L1 / L2, and each
//     entry is the FMA chain over k in order plus +0 (what the tensor-core
//     GEMM's zero-padded MMA steps add), times alpha, plus beta C -- the
//     bits the tensor-core GEMM gives, at the cost of one pass over C.
// A work item is 8 columns (few rows), 64 rows (few columns) or a 64 x 64
// block (few inner indices) of one problem; tile_begin / tiles_m of the
// descriptors count work items (thin_prepare).

#include <cuda_runtime.h>

#include <cstdint>

#include "device_checks.cuh"
#include "fmm_internal.h"

namespace fmm {
namespace {

constexpr int kThreads = 256;
constexpr int kBlockK = 256;                       // k indices per block of the running sums
constexpr int kColsRows = kThinRowsPerItem;        // few columns: rows per work item
constexpr int kColsGroups = kThreads / kColsRows;  // few columns: k groups per row (4)
constexpr int kColumnsPerItem = kThinColumnsPerItem;  // few rows: one warp per column
static_assert(kColumnsPerItem * 32 == kThreads && kColsGroups == 4, "work items fill the CTA");

struct ThinSmem {
  double part[kColsGroups - 1][kColsRows][kThinMax + 1];  // few columns: sums of k groups 1..3
};

__device__ __forceinline__ int64_t item_count(const GemmDesc& d) { return thin_items(d.m, d.n, d.k); }

template <int MAXM>
__device__ void few_rows(const GemmDesc& d, int local) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int m = d.m, K = d.k;
  const int j = local * kColumnsPerItem + warp;
  if (j >= d.n) return;
  const double* __restrict__ A = d.A;
  const double* __restrict__ bcol = d.B + (int64_t)j * d.ldb;
  const int64_t lda = d.lda;
  double tot[MAXM];
#pragma unroll
  for (int i = 0; i < MAXM; ++i) tot[i] = 0.0;
  for (int p0 = 0; p0 < K; p0 += kBlockK) {
    const int pe = min(p0 + kBlockK, K);
    double acc[MAXM];
#pragma unroll
    for (int i = 0; i < MAXM; ++i) acc[i] = 0.0;
#pragma unroll 4
    for (int p = p0 + lane; p < pe; p += 32) {
      const double b = bcol[p];
      const double* ap = A + (int64_t)p * lda;
#pragma unroll
      for (int i = 0; i < MAXM; ++i)
        if (i < m) acc[i] = fma(ap[i], b, acc[i]);
    }
#pragma unroll
    for (int i = 0; i < MAXM; ++i) tot[i] += acc[i];
  }
#pragma unroll
  for (int i = 0; i < MAXM; ++i)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) tot[i] += __shfl_xor_sync(0xffffffffu, tot[i], off);
  if (lane == 0) {
    double* c = d.C + (int64_t)j * d.ldc;
#pragma unroll
    for (int i = 0; i < MAXM; ++i)
      if (i < m) {
        double v = d.alpha * tot[i];
        if (d.beta != 0.0) v += d.beta * c[i];
        c[i] = v;
      }
  }
}

template <int MAXN>
__device__ void few_columns(const GemmDesc& d, int local, ThinSmem& sm) {
  const int tid = threadIdx.x;
  const int r = tid % kColsRows, grp = tid / kColsRows;  // grp is uniform over a warp
  const int n = d.n, K = d.k;
  const int row = local * kColsRows + r;
  const bool live = row < d.m;
  const double* __restrict__ arow = d.A + (live ? row : 0);
  const double* __restrict__ B = d.B;
  const int64_t lda = d.lda, ldb = d.ldb;
  const int quarter = (K + kColsGroups - 1) / kColsGroups;
  const int pb = min(grp * quarter, K), pend = min(pb + quarter, K);
  double tot[MAXN];
#pragma unroll
  for (int j = 0; j < MAXN; ++j) tot[j] = 0.0;
  if (live) {
    for (int p0 = pb; p0 < pend; p0 += kBlockK) {
      const int pe = min(p0 + kBlockK, pend);
      double acc[MAXN];
#pragma unroll
      for (int j = 0; j < MAXN; ++j) acc[j] = 0.0;
#pragma unroll 8
      for (int p = p0; p < pe; ++p) {
        const double a = arow[(int64_t)p * lda];
#pragma unroll
        for (int j = 0; j < MAXN; ++j)
          if (j < n) acc[j] = fma(a, B[p + (int64_t)j * ldb], acc[j]);
      }
#pragma unroll
      for (int j = 0; j < MAXN; ++j) tot[j] += acc[j];
    }
  }
  if (grp > 0) {
#pragma unroll
    for (int j = 0; j < MAXN; ++j) sm.part[grp - 1][r][j] = tot[j];
  }
  __syncthreads();
  if (grp != 0 || !live) return;
  double* c = d.C + row;
#pragma unroll
  for (int j = 0; j < MAXN; ++j)
    if (j < n) {
      double* cp = c + (int64_t)j * d.ldc;
      double v = d.alpha * ((tot[j] + sm.part[0][r][j]) + (sm.part[1][r][j] + sm.part[2][r][j]));
      if (d.beta != 0.0) v += d.beta * *cp;
      *cp = v;
    }
}

// C(r..r+1, c0..c0+7) of a problem with few inner indices.
__device__ void few_inner(const GemmDesc& d, int local) {
  const int tid = threadIdx.x;
  const int rp = tid & 31, cg = tid >> 5;  // row pair, column group (a warp: 64 rows of 8 columns)
  const int blocks_m = (d.m + kThinBlock - 1) / kThinBlock;
  const int r = (local % blocks_m) * kThinBlock + 2 * rp;
  const int c0 = (local / blocks_m) * kThinBlock + cg * 8;
  if (r >= d.m || c0 >= d.n) return;
  const bool r1 = r + 1 < d.m;
  const int K = d.k;
  const double* __restrict__ A = d.A;
  const double* __restrict__ B = d.B;
  const int64_t lda = d.lda, ldb = d.ldb, ldc = d.ldc;
  double* const Cp = d.C;
  const bool pair = r1 && (reinterpret_cast<uintptr_t>(Cp) & 15) == 0 && (ldc & 1) == 0;  // r is even
  const double alpha = d.alpha, beta = d.beta;
  // C first: its loads are in flight while the short panels are multiplied
  double cin[8][2];
  if (beta != 0.0) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double* cp = Cp + r + (int64_t)(c0 + j) * ldc;
      if (c0 + j >= d.n) {
        cin[j][0] = cin[j][1] = 0.0;
      } else if (pair) {
        const double2 v = *reinterpret_cast<const double2*>(cp);
        cin[j][0] = v.x;
        cin[j][1] = v.y;
      } else {
        cin[j][0] = cp[0];
        cin[j][1] = r1 ? cp[1] : 0.0;
      }
    }
  }
  double acc[8][2];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = 0.0;
  for (int p = 0; p < K; ++p) {
    const double a0 = A[r + (int64_t)p * lda], a1 = r1 ? A[r + 1 + (int64_t)p * lda] : 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double b = c0 + j < d.n ? B[p + (int64_t)(c0 + j) * ldb] : 0.0;
      acc[j][0] = fma(a0, b, acc[j][0]);
      acc[j][1] = fma(a1, b, acc[j][1]);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if (c0 + j >= d.n) continue;
    double* cp = Cp + r + (int64_t)(c0 + j) * ldc;
    // the padded MMA steps of the tensor-core GEMM add +0 after the last k
    double v0 = alpha * (acc[j][0] + 0.0), v1 = alpha * (acc[j][1] + 0.0);
    if (beta != 0.0) {
      v0 += beta * cin[j][0];
      v1 += beta * cin[j][1];
    }
    if (pair) {
      *reinterpret_cast<double2*>(cp) = make_double2(v0, v1);
    } else {
      cp[0] = v0;
      if (r1) cp[1] = v1;
    }
  }
}

__global__ void __launch_bounds__(kThreads) thin_gemm_kernel(const GemmDesc* __restrict__ descs, int nprob,
                                                             int total) {
  __shared__ ThinSmem sm;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    int lo = 0, hi = nprob - 1;  // problem owning this item: last p with tile_begin <= item
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (descs[mid].tile_begin <= item)
        lo = mid;
      else
        hi = mid - 1;
    }
    const GemmDesc& d = descs[lo];
    const int local = item - d.tile_begin;
    // uniform over the CTA: a skipped item skips every barrier of it alike
    if (!FMM_CHECK(lo >= 0 && lo < nprob && local >= 0 && local < item_count(d) &&
                       (d.m <= kThinMax || d.n <= kThinMax),
                   kCheckGemmProblem))
      continue;
    // the widest fringe of a problem sizes its per-thread sums
    if (d.m <= kThinMax) {
      if (d.m <= 4)
        few_rows<4>(d, local);
      else if (d.m <= 8)
        few_rows<8>(d, local);
      else
        few_rows<kThinMax>(d, local);
    } else {
      if (d.n <= 4)
        few_columns<4>(d, local, sm);
      else if (d.n <= 8)
        few_columns<8>(d, local, sm);
      else
        few_columns<kThinMax>(d, local, sm);
    }
    __syncthreads();  // shared memory is refilled by the next item
  }
}

// Problems with few inner indices only (a launch of its own, so that its
// registers are its own).
__global__ void __launch_bounds__(kThreads, 2) thin_inner_kernel(const GemmDesc* __restrict__ descs, int nprob,
                                                              int total) {
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (descs[mid].tile_begin <= item)
        lo = mid;
      else
        hi = mid - 1;
    }
    const GemmDesc& d = descs[lo];
    const int local = item - d.tile_begin;
    if (!FMM_CHECK(lo >= 0 && lo < nprob && local >= 0 && local < item_count(d) && d.m > kThinMax &&
                       d.n > kThinMax && d.k <= kThinMax,
                   kCheckGemmProblem))
      continue;
    few_inner(d, local);
  }
}

}  // namespace

cudaError_t thin_checks_arm(const void* ws, size_t bytes, cudaStream_t stream) {
  const uintptr_t lo = reinterpret_cast<uintptr_t>(ws);
  return fmm_checks_arm_tu(CheckRange{lo, ws ? lo + bytes : 0}, stream);
}

cudaError_t thin_checks_take(unsigned* word) { return fmm_checks_take_tu(word); }

cudaError_t thin_launch(const GemmDesc* d_descs, int n, int64_t total_items, int num_sms, cudaStream_t stream,
                        bool inner) {
  if (total_items <= 0 || n <= 0) return cudaSuccess;
  if (total_items >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  const int64_t cap = (int64_t)num_sms * (inner ? 8 : 4);
  const int64_t grid = total_items < cap ? total_items : cap;
  if (inner)
    thin_inner_kernel<<<(unsigned)grid, kThreads, 0, stream>>>(d_descs, n, (int)total_items);
  else
    thin_gemm_kernel<<<(unsigned)grid, kThreads, 0, stream>>>(d_descs, n, (int)total_items);
  return cudaGetLastError();
}

}  // namespace fmm
