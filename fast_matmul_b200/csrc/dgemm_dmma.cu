// Grouped FP64 GEMM on the sm_100a FP64 tensor path (DMMA, mma.sync .f64).
//
// The reference's leaf product is one host-BLAS dgemm per recursion leaf
// (MatMul, linalg/linalg.hpp:261-269 -> blas::Gemm, linalg/blas_wrap.hpp:109-113).
// Here every leaf of a breadth-first level -- and every fringe product of
// dynamic peeling -- is one problem of a single persistent launch:
//   C_p = alpha_p * A_p * B_p + beta_p * C_p   (beta_p == 0: C_p is not read)
// for column-major operands with arbitrary leading dimensions, so sub-block
// views and workspace buffers are used in place.
//
// Tile: 128 x 128 per CTA, 16-deep k slices, 4-stage cp.async pipeline
// (16-byte copies where the operand's base and leading dimension allow it,
// 8-byte copies otherwise, zero fill outside the matrix), 8 warps each
// owning a 64 x 32 sub-tile as 4 x 4 m16n8k4 FP64 MMAs.  Shared-memory rows
// are padded so that every fragment load is two wavefronts (the minimum
// for 64-bit loads).  CTAs loop over the tiles of all problems.

#include <cuda_runtime.h>

#include <cstdint>

#include "fmm_internal.h"

namespace fmm {
namespace {

constexpr int BM = kGemmBM;
constexpr int BN = kGemmBN;
constexpr int BK = 16;
constexpr int STAGES = 4;
constexpr int THREADS = 256;
constexpr int A_LD = BM + 8;  // doubles per k-row of the A tile   [BK][A_LD]
constexpr int B_LD = BK + 4;  // doubles per column of the B tile  [BN][B_LD]
constexpr int A_STAGE = BK * A_LD;
constexpr int B_STAGE = BN * B_LD;
constexpr size_t SMEM_BYTES = (size_t)STAGES * (A_STAGE + B_STAGE) * sizeof(double);

static_assert(SMEM_BYTES <= 227 * 1024, "shared memory budget");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// D(16x8) += A(16x4, row) * B(4x8, col), FP64.
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void load_stage(const GemmDesc& d, int row0, int col0, int kt, double* sA, double* sB,
                                           int tid) {
  const int k0 = kt * BK;
  // A slice: BK columns of BM contiguous rows.
#pragma unroll
  for (int it = 0; it < 4; ++it) {
    const int c = tid + it * THREADS;  // 0..1023
    const int kk = c >> 6;             // 0..15
    const int r2 = (c & 63) * 2;       // 0..126
    const int gr = row0 + r2;
    const int gk = k0 + kk;
    const uint32_t dst = smem_u32(sA + kk * A_LD + r2);
    const double* src = d.A + gr + (int64_t)gk * d.lda;
    const bool kin = gk < d.k;
    if (d.flags & 1) {
      const int bytes = (kin && gr < d.m) ? ((gr + 1 < d.m) ? 16 : 8) : 0;
      cp_async16(dst, bytes ? src : d.A, bytes);
    } else {
      const int b0 = (kin && gr < d.m) ? 8 : 0;
      const int b1 = (kin && gr + 1 < d.m) ? 8 : 0;
      cp_async8(dst, b0 ? src : d.A, b0);
      cp_async8(dst + 8, b1 ? src + 1 : d.A, b1);
    }
  }
  // B slice: BN columns, each BK contiguous k values.
#pragma unroll
  for (int it = 0; it < 4; ++it) {
    const int c = tid + it * THREADS;  // 0..1023
    const int j = c >> 3;              // 0..127
    const int kk2 = (c & 7) * 2;       // 0..14
    const int gc = col0 + j;
    const int gk = k0 + kk2;
    const uint32_t dst = smem_u32(sB + j * B_LD + kk2);
    const double* src = d.B + gk + (int64_t)gc * d.ldb;
    const bool cin = gc < d.n;
    if (d.flags & 2) {
      const int bytes = (cin && gk < d.k) ? ((gk + 1 < d.k) ? 16 : 8) : 0;
      cp_async16(dst, bytes ? src : d.B, bytes);
    } else {
      const int b0 = (cin && gk < d.k) ? 8 : 0;
      const int b1 = (cin && gk + 1 < d.k) ? 8 : 0;
      cp_async8(dst, b0 ? src : d.B, b0);
      cp_async8(dst + 8, b1 ? src + 1 : d.B, b1);
    }
  }
}

__global__ void __launch_bounds__(THREADS, 1)
    grouped_dgemm_kernel(const GemmDesc* __restrict__ descs, int nprob, int total_tiles) {
  extern __shared__ __align__(128) double smem[];
  double* sA_all = smem;
  double* sB_all = smem + STAGES * A_STAGE;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane >> 2;
  const int tig = lane & 3;
  const int wm = warp & 1;   // 2 warps along M (64 rows each)
  const int wn = warp >> 1;  // 4 warps along N (32 columns each)

  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    // problem owning this tile: last p with tile_begin <= tile
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (descs[mid].tile_begin <= tile) lo = mid;
      else hi = mid - 1;
    }
    const GemmDesc d = descs[lo];
    const int local = tile - d.tile_begin;
    const int row0 = (local % d.tiles_m) * BM;
    const int col0 = (local / d.tiles_m) * BN;
    const int ktiles = (d.k + BK - 1) / BK;

    double acc[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < ktiles) load_stage(d, row0, col0, s, sA_all + s * A_STAGE, sB_all + s * B_STAGE, tid);
      cp_async_commit();
    }

    for (int kt = 0; kt < ktiles; ++kt) {
      cp_async_wait<STAGES - 2>();
      __syncthreads();
      {
        const int nk = kt + STAGES - 1;
        if (nk < ktiles) {
          const int ns = nk % STAGES;
          load_stage(d, row0, col0, nk, sA_all + ns * A_STAGE, sB_all + ns * B_STAGE, tid);
        }
        cp_async_commit();
      }
      const int st = kt % STAGES;
      const double* a_base = sA_all + st * A_STAGE + tig * A_LD + wm * 64 + g;
      const double* b_base = sB_all + st * B_STAGE + (wn * 32 + g) * B_LD + tig;
#pragma unroll
      for (int ks = 0; ks < BK / 4; ++ks) {
        double af[4][2];
        double bf[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
          af[mt][0] = a_base[ks * 4 * A_LD + mt * 16];
          af[mt][1] = a_base[ks * 4 * A_LD + mt * 16 + 8];
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) bf[nt] = b_base[nt * 8 * B_LD + ks * 4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma_16x8x4(acc[mt][nt], af[mt][0], af[mt][1], bf[nt]);
      }
    }
    cp_async_wait<0>();
    __syncthreads();  // shared buffers are refilled by the next tile

    // epilogue: C = alpha * acc + beta * C
    const double alpha = d.alpha;
    const double beta = d.beta;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = row0 + wm * 64 + mt * 16 + g + h * 8;
        if (r >= d.m) continue;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int cidx = col0 + wn * 32 + nt * 8 + tig * 2 + q;
            if (cidx < d.n) {
              double* cp = d.C + r + (int64_t)cidx * d.ldc;
              double v = alpha * acc[mt][nt][h * 2 + q];
              if (beta != 0.0) v += beta * *cp;
              *cp = v;
            }
          }
        }
      }
    }
  }
}

}  // namespace

cudaError_t gemm_launch(const GemmDesc* d_descs, int n, int64_t total_tiles, int num_sms, cudaStream_t stream) {
  if (total_tiles <= 0 || n <= 0) return cudaSuccess;
  cudaError_t err = cudaFuncSetAttribute(grouped_dgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)SMEM_BYTES);
  if (err != cudaSuccess) return err;
  const int64_t grid = total_tiles < num_sms ? total_tiles : num_sms;
  grouped_dgemm_kernel<<<(unsigned)grid, THREADS, SMEM_BYTES, stream>>>(d_descs, n, (int)total_tiles);
  return cudaGetLastError();
}

}  // namespace fmm
