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
// of two Scalars (RowScale / ColScale / UpdateVals).  IEEE division, square
// root and multiplication are correctly rounded and a maximum is exact, so
// the device result equals the reference's bit for bit.  With Scalar =
// float the reference divides and takes the square root in double (its 1.0
// is a double and MaxAbsRow / MaxAbsCol return double) and rounds the factor
// to float on assignment; the float kernels do the same.

#include <algorithm>

#include "fmm_internal.h"

namespace fmm {

namespace {

constexpr int kRows = 256;   // rows of a tile = threads of a block
constexpr int kCols = 64;    // columns of a tile
constexpr int kUnroll = 8;   // loads in flight per thread

// Non-negative values order like their bit patterns: maxima are kept as
// unsigned words of the same width and combined with atomicMax.
template <class T>
struct Bits;
template <>
struct Bits<double> {
  using U = unsigned long long;
};
template <>
struct Bits<float> {
  using U = unsigned int;
};

__device__ __forceinline__ unsigned long long to_bits(double x) { return (unsigned long long)__double_as_longlong(x); }
__device__ __forceinline__ unsigned int to_bits(float x) { return __float_as_uint(x); }
__device__ __forceinline__ double from_bits(unsigned long long b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ float from_bits(unsigned int b) { return __uint_as_float(b); }
__device__ __forceinline__ double vmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double vabs(double a) { return fabs(a); }
__device__ __forceinline__ float vabs(float a) { return fabsf(a); }

template <class T>
struct ScaleJob {
  using U = typename Bits<T>::U;
  T* X;
  int64_t ld;
  int rows, cols;
  const T* rowv;     // X(i,j) *= rowv[i] (null: none)
  const T* colv;     // then X(i,j) *= colv[j] (null: none)
  U* rowmax;         // max_j |X(i,j)| of the result, as bits (null: not wanted)
  U* colmax;         // max_i |X(i,j)| of the result, as bits (null: not wanted)
  int64_t tiles_r;   // ceil(rows / kRows)
  int64_t tiles;     // tiles_r * ceil(cols / kCols)
};

template <class T>
ScaleJob<T> make_job(T* X, int64_t ld, int rows, int cols, const T* rowv, const T* colv,
                     typename Bits<T>::U* rowmax, typename Bits<T>::U* colmax) {
  ScaleJob<T> j;
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
template <class T>
__device__ __forceinline__ T warp_max8(const T (&a)[8], int lane) {
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
  T b4[4], b2[2];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const T keep = h16 ? a[j + 4] : a[j];
    const T send = h16 ? a[j] : a[j + 4];
    b4[j] = vmax(keep, __shfl_xor_sync(0xffffffffu, send, 16));
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const T keep = h8 ? b4[j + 2] : b4[j];
    const T send = h8 ? b4[j] : b4[j + 2];
    b2[j] = vmax(keep, __shfl_xor_sync(0xffffffffu, send, 8));
  }
  T b = vmax(h4 ? b2[1] : b2[0], __shfl_xor_sync(0xffffffffu, h4 ? b2[0] : b2[1], 4));
  b = vmax(b, __shfl_xor_sync(0xffffffffu, b, 2));
  return vmax(b, __shfl_xor_sync(0xffffffffu, b, 1));
}

__device__ __forceinline__ int column_of_lane(int lane) {
  return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}

// Blocks [0, j0.tiles) work on j0, the rest on j1.  A tile is kRows rows x
// kCols columns; thread t owns row t of the tile, so every column load of a
// warp is 32 consecutive doubles.
template <class T>
__global__ void __launch_bounds__(kRows) scale_reduce_kernel(ScaleJob<T> j0, ScaleJob<T> j1) {
  __shared__ T s_colv[kCols];
  __shared__ T s_part[kRows / 32][kCols];
  const bool second = (int64_t)blockIdx.x >= j0.tiles;
  const ScaleJob<T> J = second ? j1 : j0;
  const int64_t t = second ? (int64_t)blockIdx.x - j0.tiles : (int64_t)blockIdx.x;
  const int64_t tr = t % J.tiles_r;
  const int c0 = (int)(t / J.tiles_r) * kCols;
  const int nc = min(kCols, J.cols - c0);
  const int64_t i = tr * kRows + threadIdx.x;
  const bool in = i < J.rows;
  const bool scales = J.rowv != nullptr || J.colv != nullptr;
  if (threadIdx.x < kCols) s_colv[threadIdx.x] = (J.colv && (int)threadIdx.x < nc) ? J.colv[c0 + threadIdx.x] : T(1);
  __syncthreads();
  const T rv = (J.rowv && in) ? J.rowv[i] : T(1);
  T* p = J.X + (in ? i : 0) + (int64_t)c0 * J.ld;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T rmax = T(0);
  static_assert(kUnroll == 8, "warp_max8 reduces 8 columns");
  for (int cb = 0; cb < nc; cb += kUnroll) {
    T v[kUnroll], a[kUnroll];
    T* q = p + (int64_t)cb * J.ld;
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) v[u] = (in && cb + u < nc) ? q[(int64_t)u * J.ld] : T(0);
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int c = cb + u;
      if (J.rowv) v[u] = v[u] * rv;
      if (J.colv) v[u] = v[u] * s_colv[c];
      if (scales && in && c < nc) q[(int64_t)u * J.ld] = v[u];
      a[u] = vabs(v[u]);
      rmax = vmax(rmax, a[u]);
    }
    if (J.colmax) {
      const T w = warp_max8(a, lane);
      if ((lane & 3) == 0) s_part[warp][cb + column_of_lane(lane)] = w;
    }
  }
  if (J.rowmax && in && rmax > T(0)) atomicMax(&J.rowmax[i], to_bits(rmax));
  if (J.colmax) {
    __syncthreads();
    if ((int)threadIdx.x < nc) {
      T mx = T(0);
#pragma unroll
      for (int w = 0; w < kRows / 32; ++w) mx = vmax(mx, s_part[w][threadIdx.x]);
      if (mx > T(0)) atomicMax(&J.colmax[c0 + threadIdx.x], to_bits(mx));
    }
  }
}

template <class T>
struct Factors {
  using U = typename Bits<T>::U;
  int m, k, n;
  int inner;  // 0: outer factors, 1: inner factors
  U* row_a;   // max |A(i,:)|   (m)
  U* col_a;   // max |A(:,l)|   (k)
  U* row_b;   // max |B(l,:)|   (k)
  U* col_b;   // max |B(:,j)|   (n)
  T* fa;      // outer: 1 / x (m); inner: 1 / z (k)
  T* fb;      // outer: 1 / y (n); inner: z (k)
  T* r;       // outer: r *= x (m)
  T* s;       // outer: s *= y (n)
};

// Turns the maxima into factors, then clears every maximum for the next
// pass.  Thread t alone reads and clears entry t of each array.  The
// quotient and the square root are taken in double and rounded to T, as
// the reference's 1.0 / vals[k] and sqrt(MaxAbsCol / MaxAbsRow) are.
template <class T>
__global__ void scale_factors_kernel(Factors<T> F) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (!F.inner) {
    // OuterScaling (:105-124) and UpdateVals (:93-98)
    if (t < F.m) {
      const T x = from_bits(F.row_a[t]);
      F.fa[t] = (T)(1.0 / (double)x);
      F.r[t] = F.r[t] * x;
    }
    if (t < F.n) {
      const T y = from_bits(F.col_b[t]);
      F.fb[t] = (T)(1.0 / (double)y);
      F.s[t] = F.s[t] * y;
    }
  } else if (t < F.k) {
    // InnerScaling (:129-138)
    const T z = (T)sqrt((double)from_bits(F.col_a[t]) / (double)from_bits(F.row_b[t]));
    F.fa[t] = (T)(1.0 / (double)z);
    F.fb[t] = z;
  }
  if (t < F.m) F.row_a[t] = 0;
  if (t < F.k) {
    F.col_a[t] = 0;
    F.row_b[t] = 0;
  }
  if (t < F.n) F.col_b[t] = 0;
}

// Every maximum cleared.  r and s keep the caller's starting values
// (Scaling's resize(m, 1.0), scaling.hpp:158-159, keeps the entries of
// vectors that arrive sized).
template <class T>
__global__ void scale_init_kernel(Factors<T> F) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < F.m) F.row_a[t] = 0;
  if (t < F.n) F.col_b[t] = 0;
  if (t < F.k) {
    F.col_a[t] = 0;
    F.row_b[t] = 0;
  }
}

template <class T>
cudaError_t launch_jobs(const ScaleJob<T>& j0, const ScaleJob<T>& j1, cudaStream_t stream, int64_t* launches) {
  const int64_t blocks = j0.tiles + j1.tiles;
  if (blocks == 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  scale_reduce_kernel<T><<<(unsigned)blocks, kRows, 0, stream>>>(j0, j1);
  ++*launches;
  return cudaGetLastError();
}

// Array lengths padded to 32 entries (256 bytes at 8 bytes an entry).
int64_t pad32(int64_t v) { return (v + 31) / 32 * 32; }

template <class T>
cudaError_t scaling_impl(T* A, int64_t lda, T* B, int64_t ldb, int m, int k, int n, int num_steps, int type, T* r,
                         T* s, void* scratch, cudaStream_t stream, int64_t* launches) {
  using U = typename Bits<T>::U;
  Factors<T> F;
  F.m = m;
  F.k = k;
  F.n = n;
  // entries of 8 bytes whatever T is: the layout of scaling_scratch_bytes
  char* base = static_cast<char*>(scratch);
  F.row_a = reinterpret_cast<U*>(base);
  F.col_a = reinterpret_cast<U*>(base + 8 * pad32(m));
  F.row_b = reinterpret_cast<U*>(base + 8 * (pad32(m) + pad32(k)));
  F.col_b = reinterpret_cast<U*>(base + 8 * (pad32(m) + 2 * pad32(k)));
  F.fa = reinterpret_cast<T*>(base + 8 * (pad32(m) + 2 * pad32(k) + pad32(n)));
  F.fb = reinterpret_cast<T*>(base + 8 * (pad32(m) + 2 * pad32(k) + pad32(n) + pad32(std::max(m, k))));
  F.r = r;
  F.s = s;
  F.inner = 0;
  const int64_t span = std::max<int64_t>(std::max(m, n), std::max(k, 1));
  const unsigned vec_blocks = (unsigned)((span + 255) / 256);
  scale_init_kernel<T><<<vec_blocks, 256, 0, stream>>>(F);
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
  auto want = [&](bool inner, ScaleJob<T>* ja, ScaleJob<T>* jb) {
    ja->rowmax = inner ? nullptr : F.row_a;
    ja->colmax = inner ? F.col_a : nullptr;
    jb->rowmax = inner ? F.row_b : nullptr;
    jb->colmax = inner ? nullptr : F.col_b;
  };
  {
    ScaleJob<T> ja = make_job<T>(A, lda, m, k, nullptr, nullptr, nullptr, nullptr);
    ScaleJob<T> jb = make_job<T>(B, ldb, k, n, nullptr, nullptr, nullptr, nullptr);
    want(ops[0], &ja, &jb);
    e = launch_jobs(ja, jb, stream, launches);
    if (e != cudaSuccess) return e;
  }
  for (int64_t q = 0; q < total; ++q) {
    const bool inner = ops[q % per_step];
    F.inner = inner ? 1 : 0;
    scale_factors_kernel<T><<<vec_blocks, 256, 0, stream>>>(F);
    ++*launches;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // outer: rows of A by 1 / x, columns of B by 1 / y;
    // inner: columns of A by 1 / z, rows of B by z
    ScaleJob<T> ja = make_job<T>(A, lda, m, k, inner ? nullptr : F.fa, inner ? F.fa : nullptr, nullptr, nullptr);
    ScaleJob<T> jb = make_job<T>(B, ldb, k, n, inner ? F.fb : nullptr, inner ? nullptr : F.fb, nullptr, nullptr);
    if (q + 1 < total) want(ops[(q + 1) % per_step], &ja, &jb);
    e = launch_jobs(ja, jb, stream, launches);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <class T>
cudaError_t postprocess_impl(T* C, int64_t ldc, int m, int n, const T* r, const T* s, cudaStream_t stream,
                             int64_t* launches) {
  const ScaleJob<T> jc = make_job<T>(C, ldc, m, n, r, s, nullptr, nullptr);
  const ScaleJob<T> none = make_job<T>(nullptr, 1, 0, 0, nullptr, nullptr, nullptr, nullptr);
  return launch_jobs(jc, none, stream, launches);
}

}  // namespace

size_t scaling_scratch_bytes(int64_t m, int64_t k, int64_t n) {
  // four maxima arrays and two factor arrays of 8-byte entries, each rounded to 256 bytes
  return (size_t)8 * (size_t)(pad32(m) + 2 * pad32(k) + pad32(n) + pad32(std::max(m, k)) + pad32(std::max(n, k)));
}

cudaError_t scaling_launch(double* A, int64_t lda, double* B, int64_t ldb, int m, int k, int n, int num_steps,
                           int type, double* r, double* s, void* scratch, cudaStream_t stream, int64_t* launches) {
  return scaling_impl<double>(A, lda, B, ldb, m, k, n, num_steps, type, r, s, scratch, stream, launches);
}

cudaError_t scaling_launch(float* A, int64_t lda, float* B, int64_t ldb, int m, int k, int n, int num_steps,
                           int type, float* r, float* s, void* scratch, cudaStream_t stream, int64_t* launches) {
  return scaling_impl<float>(A, lda, B, ldb, m, k, n, num_steps, type, r, s, scratch, stream, launches);
}

cudaError_t scaling_postprocess_launch(double* C, int64_t ldc, int m, int n, const double* r, const double* s,
                                       cudaStream_t stream, int64_t* launches) {
  return postprocess_impl<double>(C, ldc, m, n, r, s, stream, launches);
}

cudaError_t scaling_postprocess_launch(float* C, int64_t ldc, int m, int n, const float* r, const float* s,
                                       cudaStream_t stream, int64_t* launches) {
  return postprocess_impl<float>(C, ldc, m, n, r, s, stream, launches);
}

}  // namespace fmm
