// Diagonal scaling of the operands and of the product on the device: the
// reference's Scaling / PostProcessScaling (scaling/scaling.hpp:28-196).
//
// One kernel makes every pass over a matrix.  It applies an optional row
// factor and an optional column factor, X(i,j) = (X(i,j) * rowv[i]) *
// colv[j] (the order of PostProcessScaling, scaling.hpp:143-148), and it
// accumulates the maxima of |X| of the result along rows and along columns
// that the next scaling needs, with atomicMax on the bit patterns
// (non-negative doubles order like their bits; NaN entries are skipped, as
// the reference's `v > max` comparison skips them).  Fusing the next
// scaling's maxima into the pass that writes the matrix leaves one read and
// one write per matrix per scaling, after one read-only pass at the start.
//
// Every factor is the reference's own arithmetic: 1.0 / max (InverseVector,
// :52-58), sqrt(max_col(A) / max_row(B)) (InnerScaling, :129-138), products
// of two doubles (RowScale / ColScale / UpdateVals).  IEEE division, square
// root and multiplication are correctly rounded and a maximum is exact, so
// the device result equals the reference's bit for bit.

#include <algorithm>

#include "fmm_internal.h"

namespace fmm {

namespace {

constexpr int kRows = 256;   // rows of a tile = threads of a block
constexpr int kCols = 64;    // columns of a tile
constexpr int kUnroll = 8;   // loads in flight per thread

struct ScaleJob {
  double* X;
  int64_t ld;
  int rows, cols;
  const double* rowv;          // X(i,j) *= rowv[i] (null: none)
  const double* colv;          // then X(i,j) *= colv[j] (null: none)
  unsigned long long* rowmax;  // max_j |X(i,j)| of the result, as bits (null: not wanted)
  unsigned long long* colmax;  // max_i |X(i,j)| of the result, as bits (null: not wanted)
  int64_t tiles_r;             // ceil(rows / kRows)
  int64_t tiles;               // tiles_r * ceil(cols / kCols)
};

ScaleJob make_job(double* X, int64_t ld, int rows, int cols, const double* rowv, const double* colv,
                  unsigned long long* rowmax, unsigned long long* colmax) {
  ScaleJob j;
  j.X = X;
  j.ld = ld;
  j.rows = rows;
  j.cols = cols;
  j.rowv = rowv;
  j.colv = colv;
  j.rowmax = rowmax;
  j.colmax = colmax;
  j.tiles_r = rows > 0 ? (rows + kRows - 1) / kRows : 0;
  j.tiles = cols > 0 ? j.tiles_r * ((cols + kCols - 1) / kCols) : 0;
  return j;
}

// Maxima over the 32 lanes of a warp of 8 columns at once (a[u] = |X| of
// column u in this lane's row), by recursive halving: at lane distance 16
// each lane keeps 4 of the columns and trades the other 4, at 8 it keeps 2,
// at 4 one, then two plain steps.  9 shuffles instead of 8 x 5.  Returns the
// maximum of column column_of_lane(lane), valid in lanes with lane % 4 == 0.
__device__ __forceinline__ double warp_max8(const double (&a)[8], int lane) {
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
  double b4[4], b2[2];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const double keep = h16 ? a[j + 4] : a[j];
    const double send = h16 ? a[j] : a[j + 4];
    b4[j] = fmax(keep, __shfl_xor_sync(0xffffffffu, send, 16));
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const double keep = h8 ? b4[j + 2] : b4[j];
    const double send = h8 ? b4[j] : b4[j + 2];
    b2[j] = fmax(keep, __shfl_xor_sync(0xffffffffu, send, 8));
  }
  double b = fmax(h4 ? b2[1] : b2[0], __shfl_xor_sync(0xffffffffu, h4 ? b2[0] : b2[1], 4));
  b = fmax(b, __shfl_xor_sync(0xffffffffu, b, 2));
  return fmax(b, __shfl_xor_sync(0xffffffffu, b, 1));
}

__device__ __forceinline__ int column_of_lane(int lane) {
  return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}

// Blocks [0, j0.tiles) work on j0, the rest on j1.  A tile is kRows rows x
// kCols columns; thread t owns row t of the tile, so every column load of a
// warp is 32 consecutive doubles.
__global__ void __launch_bounds__(kRows) scale_reduce_kernel(ScaleJob j0, ScaleJob j1) {
  __shared__ double s_colv[kCols];
  __shared__ double s_part[kRows / 32][kCols];
  const bool second = (int64_t)blockIdx.x >= j0.tiles;
  const ScaleJob J = second ? j1 : j0;
  const int64_t t = second ? (int64_t)blockIdx.x - j0.tiles : (int64_t)blockIdx.x;
  const int64_t tr = t % J.tiles_r;
  const int c0 = (int)(t / J.tiles_r) * kCols;
  const int nc = min(kCols, J.cols - c0);
  const int64_t i = tr * kRows + threadIdx.x;
  const bool in = i < J.rows;
  const bool scales = J.rowv != nullptr || J.colv != nullptr;
  if (threadIdx.x < kCols) s_colv[threadIdx.x] = (J.colv && (int)threadIdx.x < nc) ? J.colv[c0 + threadIdx.x] : 1.0;
  __syncthreads();
  const double rv = (J.rowv && in) ? J.rowv[i] : 1.0;
  double* p = J.X + (in ? i : 0) + (int64_t)c0 * J.ld;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double rmax = 0.0;
  static_assert(kUnroll == 8, "warp_max8 reduces 8 columns");
  for (int cb = 0; cb < nc; cb += kUnroll) {
    double v[kUnroll], a[kUnroll];
    double* q = p + (int64_t)cb * J.ld;
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) v[u] = (in && cb + u < nc) ? q[(int64_t)u * J.ld] : 0.0;
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int c = cb + u;
      if (J.rowv) v[u] = v[u] * rv;
      if (J.colv) v[u] = v[u] * s_colv[c];
      if (scales && in && c < nc) q[(int64_t)u * J.ld] = v[u];
      a[u] = fabs(v[u]);
      rmax = fmax(rmax, a[u]);
    }
    if (J.colmax) {
      const double w = warp_max8(a, lane);
      if ((lane & 3) == 0) s_part[warp][cb + column_of_lane(lane)] = w;
    }
  }
  if (J.rowmax && in && rmax > 0.0) atomicMax(&J.rowmax[i], (unsigned long long)__double_as_longlong(rmax));
  if (J.colmax) {
    __syncthreads();
    if ((int)threadIdx.x < nc) {
      double mx = 0.0;
#pragma unroll
      for (int w = 0; w < kRows / 32; ++w) mx = fmax(mx, s_part[w][threadIdx.x]);
      if (mx > 0.0) atomicMax(&J.colmax[c0 + threadIdx.x], (unsigned long long)__double_as_longlong(mx));
    }
  }
}

struct Factors {
  int m, k, n;
  int inner;                    // 0: outer factors, 1: inner factors
  unsigned long long* row_a;    // max |A(i,:)|   (m)
  unsigned long long* col_a;    // max |A(:,l)|   (k)
  unsigned long long* row_b;    // max |B(l,:)|   (k)
  unsigned long long* col_b;    // max |B(:,j)|   (n)
  double* fa;                   // outer: 1 / x (m); inner: 1 / z (k)
  double* fb;                   // outer: 1 / y (n); inner: z (k)
  double* r;                    // outer: r *= x (m)
  double* s;                    // outer: s *= y (n)
};

// Turns the maxima into factors, then clears every maximum for the next
// pass.  Thread t alone reads and clears entry t of each array.
__global__ void scale_factors_kernel(Factors F) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (!F.inner) {
    // OuterScaling (:105-124) and UpdateVals (:93-98)
    if (t < F.m) {
      const double x = __longlong_as_double((long long)F.row_a[t]);
      F.fa[t] = 1.0 / x;
      F.r[t] = F.r[t] * x;
    }
    if (t < F.n) {
      const double y = __longlong_as_double((long long)F.col_b[t]);
      F.fb[t] = 1.0 / y;
      F.s[t] = F.s[t] * y;
    }
  } else if (t < F.k) {
    // InnerScaling (:129-138)
    const double z = sqrt(__longlong_as_double((long long)F.col_a[t]) / __longlong_as_double((long long)F.row_b[t]));
    F.fa[t] = 1.0 / z;
    F.fb[t] = z;
  }
  if (t < F.m) F.row_a[t] = 0ull;
  if (t < F.k) {
    F.col_a[t] = 0ull;
    F.row_b[t] = 0ull;
  }
  if (t < F.n) F.col_b[t] = 0ull;
}

// Every maximum cleared.  r and s keep the caller's starting values
// (Scaling's resize(m, 1.0), scaling.hpp:158-159, keeps the entries of
// vectors that arrive sized).
__global__ void scale_init_kernel(Factors F) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < F.m) F.row_a[t] = 0ull;
  if (t < F.n) F.col_b[t] = 0ull;
  if (t < F.k) {
    F.col_a[t] = 0ull;
    F.row_b[t] = 0ull;
  }
}

cudaError_t launch_jobs(const ScaleJob& j0, const ScaleJob& j1, cudaStream_t stream, int64_t* launches) {
  const int64_t blocks = j0.tiles + j1.tiles;
  if (blocks == 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  scale_reduce_kernel<<<(unsigned)blocks, kRows, 0, stream>>>(j0, j1);
  ++*launches;
  return cudaGetLastError();
}

// Array lengths padded to 32 entries (256 bytes).
int64_t pad32(int64_t v) { return (v + 31) / 32 * 32; }

}  // namespace

size_t scaling_scratch_bytes(int64_t m, int64_t k, int64_t n) {
  // four maxima arrays and two factor arrays, each rounded to 256 bytes
  return (size_t)8 * (size_t)(pad32(m) + 2 * pad32(k) + pad32(n) + pad32(std::max(m, k)) + pad32(std::max(n, k)));
}

cudaError_t scaling_launch(double* A, int64_t lda, double* B, int64_t ldb, int m, int k, int n, int num_steps,
                           int type, double* r, double* s, void* scratch, cudaStream_t stream, int64_t* launches) {
  Factors F;
  F.m = m;
  F.k = k;
  F.n = n;
  unsigned long long* base = static_cast<unsigned long long*>(scratch);
  F.row_a = base;
  F.col_a = F.row_a + pad32(m);
  F.row_b = F.col_a + pad32(k);
  F.col_b = F.row_b + pad32(k);
  F.fa = reinterpret_cast<double*>(F.col_b + pad32(n));
  F.fb = F.fa + pad32(std::max(m, k));
  F.r = r;
  F.s = s;
  F.inner = 0;
  const int64_t span = std::max<int64_t>(std::max(m, n), std::max(k, 1));
  const unsigned vec_blocks = (unsigned)((span + 255) / 256);
  scale_init_kernel<<<vec_blocks, 256, 0, stream>>>(F);
  ++*launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;

  // The reference's step sequence (Scaling, scaling.hpp:161-193): false = outer, true = inner.
  bool ops[2];
  int per_step = 0;
  switch (type) {
    case 0: ops[0] = false; ops[1] = true; per_step = 2; break;
    case 1: ops[0] = true; ops[1] = false; per_step = 2; break;
    case 2: ops[0] = true; per_step = 1; break;
    case 3: ops[0] = false; per_step = 1; break;
    default: return cudaErrorInvalidValue;
  }
  const int64_t total = (int64_t)num_steps * per_step;
  if (total == 0) return cudaSuccess;

  // Maxima for the first scaling, read-only over both operands.
  auto want = [&](bool inner, ScaleJob* ja, ScaleJob* jb) {
    ja->rowmax = inner ? nullptr : F.row_a;
    ja->colmax = inner ? F.col_a : nullptr;
    jb->rowmax = inner ? F.row_b : nullptr;
    jb->colmax = inner ? nullptr : F.col_b;
  };
  {
    ScaleJob ja = make_job(A, lda, m, k, nullptr, nullptr, nullptr, nullptr);
    ScaleJob jb = make_job(B, ldb, k, n, nullptr, nullptr, nullptr, nullptr);
    want(ops[0], &ja, &jb);
    e = launch_jobs(ja, jb, stream, launches);
    if (e != cudaSuccess) return e;
  }
  for (int64_t q = 0; q < total; ++q) {
    const bool inner = ops[q % per_step];
    F.inner = inner ? 1 : 0;
    scale_factors_kernel<<<vec_blocks, 256, 0, stream>>>(F);
    ++*launches;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // outer: rows of A by 1 / x, columns of B by 1 / y;
    // inner: columns of A by 1 / z, rows of B by z
    ScaleJob ja = make_job(A, lda, m, k, inner ? nullptr : F.fa, inner ? F.fa : nullptr, nullptr, nullptr);
    ScaleJob jb = make_job(B, ldb, k, n, inner ? F.fb : nullptr, inner ? nullptr : F.fb, nullptr, nullptr);
    if (q + 1 < total) want(ops[(q + 1) % per_step], &ja, &jb);
    e = launch_jobs(ja, jb, stream, launches);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t scaling_postprocess_launch(double* C, int64_t ldc, int m, int n, const double* r, const double* s,
                                       cudaStream_t stream, int64_t* launches) {
  const ScaleJob jc = make_job(C, ldc, m, n, r, s, nullptr, nullptr);
  const ScaleJob none = make_job(nullptr, 1, 0, 0, nullptr, nullptr, nullptr, nullptr);
  return launch_jobs(jc, none, stream, launches);
}

}  // namespace fmm
