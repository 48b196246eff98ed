// TEST INFRASTRUCTURE ONLY: a host interpreter for the engine's launch
// programs.
//
// It links the product planner (plan.cpp) unchanged, builds the program for
// a call with HOST pointers and a host workspace poisoned with NaN, and then
// executes every launch on the CPU: the generated operand-formation and
// combination code (fmm_alg_kernels.cuh, compiled here for the host with
// separately rounded adds and multiplies, as on the device) and a
// straightforward GEMM for the grouped products whose summation order
// matches the CPU oracle's.  The result must equal the oracle bit for bit,
// which checks the planner's views, multipliers, workspace layout,
// schedules and peeling on machines without a GPU.
//
// Split-BF16 leaf products are executed by a model of the device arithmetic
// (power-of-two scaling, 8-bit digit slices, exact integer sums per
// diagonal and accumulation group of k (SplitGroup), FP64 recombination in
// the device's order),
// so the device result must equal the model's bit for bit.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "plan.h"

namespace fmm {
// The device launchers are not used by the interpreter.
cudaError_t gemm_launch(const GemmDesc*, int, int64_t, int, cudaStream_t) { return cudaErrorNotSupported; }
void set_last_error(const std::string&) {}
cudaError_t form_launch(int, const FormLaunch&, const CoefSlots&, bool, int, cudaStream_t) {
  return cudaErrorNotSupported;
}
cudaError_t combine_launch(int, const CombineLaunch&, const CoefSlots&, bool, int, cudaStream_t) {
  return cudaErrorNotSupported;
}
cudaError_t split_gemm_launch(const SplitDesc*, int, const SplitPlan&, void*, int*, int, cudaStream_t, int64_t*) {
  return cudaErrorNotSupported;
}
}  // namespace fmm

namespace emu {

#define __device__
#define __forceinline__ inline

inline double fmm_add(double a, double b) { return a + b; }
inline double fmm_sub(double a, double b) { return a - b; }
inline double fmm_mul(double c, double a) { return c * a; }
inline double fmm_neg(double a) { return -a; }

#include "generated/fmm_alg_kernels.cuh"

#undef __device__
#undef __forceinline__

using fmm::CombineDesc;
using fmm::FormDesc;
using fmm::GemmDesc;

template <class ALG>
void run_form(const fmm::Op& op, const unsigned char* desc, const double* cf) {
  const FormDesc* d = reinterpret_cast<const FormDesc*>(desc + op.desc_off);
  for (int p = 0; p < op.n_s + op.n_t; ++p) {
    const bool s_side = p < op.n_s;
    const FormDesc& f = d[p];
    const int64_t rows = f.rows;
    const int64_t cols = f.cols;
    const int nbc = s_side ? ALG::kK0 : ALG::kN0;
    for (int64_t j = 0; j < cols; ++j)
      for (int64_t i = 0; i < rows; ++i) {
        auto ld = [&](int b) -> double {
          const int bi = b / nbc, bj = b % nbc;
          return f.in[(bi * rows + i) + (bj * cols + j) * f.ld_in];
        };
        auto st = [&](int o, double v) { f.out[o * f.out_stride + i + j * f.ld_out] = v; };
        if (s_side)
          ALG::template form_s<double>(cf, ld, st);
        else
          ALG::template form_t<double>(cf, ld, st);
      }
  }
}

template <class ALG>
void run_combine(const fmm::Op& op, const unsigned char* desc, const double* cf) {
  const CombineDesc* d = reinterpret_cast<const CombineDesc*>(desc + op.desc_off);
  for (int p = 0; p < op.n; ++p) {
    const CombineDesc& c = d[p];
    for (int64_t j = 0; j < c.cols; ++j)
      for (int64_t i = 0; i < c.rows; ++i) {
        auto ld = [&](int r) -> double { return c.m[r * c.m_stride + i + j * c.ld_m]; };
        auto ptr = [&](int b) -> double* {
          const int bi = b / ALG::kN0, bj = b % ALG::kN0;
          return c.c + (bi * c.rows + i) + (bj * c.cols + j) * c.ld_c;
        };
        auto ldc = [&](int b) -> double { return *ptr(b); };
        auto st = [&](int b, double v) { *ptr(b) = v; };
        if (c.beta != 0.0)
          ALG::template combine<double, true>(cf, c.beta, ld, ldc, st);
        else
          ALG::template combine<double, false>(cf, 0.0, ld, ldc, st);
      }
  }
}

// Same summation order as the CPU oracle's MatMul.
void run_gemm(const fmm::Op& op, const unsigned char* desc) {
  const GemmDesc* g = reinterpret_cast<const GemmDesc*>(desc + op.desc_off);
  std::vector<double> col;
  for (int p = 0; p < op.n; ++p) {
    const GemmDesc& d = g[p];
    col.assign((size_t)(d.m > 0 ? d.m : 1), 0.0);
    for (int j = 0; j < d.n; ++j) {
      for (int i = 0; i < d.m; ++i) col[i] = 0.0;
      for (int q = 0; q < d.k; ++q) {
        const double b = d.B[q + (int64_t)j * d.ldb];
        const double* a = d.A + (int64_t)q * d.lda;
        for (int i = 0; i < d.m; ++i) col[i] += a[i] * b;
      }
      for (int i = 0; i < d.m; ++i) {
        double v = d.alpha * col[i];
        if (d.beta != 0.0) v = v + d.beta * d.C[i + (int64_t)j * d.ldc];
        d.C[i + (int64_t)j * d.ldc] = v;
      }
    }
  }
}

int exponent_above(double maxabs) {
  if (!(maxabs > 0.0)) return 0;
  int e;
  std::frexp(maxabs, &e);
  return e;
}

// The split kernels' exponent of a row or column: kSplitNonFinite when it
// holds an Inf or a NaN, else exponent_above of its largest magnitude.
int split_exponent(const double* x, int64_t stride, int k) {
  double mx = 0.0;
  for (int p = 0; p < k; ++p) {
    const double v = x[(int64_t)p * stride];
    if (!std::isfinite(v)) return fmm::kSplitNonFinite;
    mx = std::fmax(mx, std::fabs(v));
  }
  return exponent_above(mx);
}

// Digits of x (|x| < 1): d_t = rint(256 r_{t-1}), r_t = 256 r_{t-1} - d_t.
void digits(double x, int slices, double* out) {
  for (int t = 0; t < slices; ++t) {
    const double y = x * 256.0;
    const double dg = std::rint(y);
    x = y - dg;
    out[t] = dg;
  }
}

// INT8 digits of x (|x| < 1): d_0 = rint(64 x), d_t = rint(128 r_{t-1}),
// |d_t| <= 64.
void digits_i8(double x, int slices, double* out) {
  double radix = 64.0;
  for (int t = 0; t < slices; ++t) {
    const double y = x * radix;
    const double dg = std::rint(y);
    x = y - dg;
    out[t] = dg;
    radix = 128.0;
  }
}

// One split product C = alpha * A * B + beta * C (split code `code`: BF16
// or INT8 digits), in the device's order.
void split_product(const fmm::SplitDesc& d, int code) {
  const int m = d.m, n = d.n, k = d.k;
  if (m <= 0 || n <= 0) return;
  const int S = fmm::split_code_slices(code);
  const bool int8 = fmm::split_code_int8(code);
  std::vector<int> ea((size_t)m), fb((size_t)n);
  for (int i = 0; i < m; ++i) ea[(size_t)i] = split_exponent(d.A + i, d.lda, k);
  for (int j = 0; j < n; ++j) fb[(size_t)j] = split_exponent(d.B + (int64_t)j * d.ldb, 1, k);
  auto scaled = [](double x, int e) { return e == fmm::kSplitNonFinite ? 0.0 : std::ldexp(x, -e); };
  // dA[(t * k + p) * m + i], dB[(t * k + p) * n + j]
  std::vector<double> dA((size_t)S * k * m), dB((size_t)S * k * n);
  double dg[8];
  for (int p = 0; p < k; ++p) {
    for (int i = 0; i < m; ++i) {
      (int8 ? digits_i8 : digits)(scaled(d.A[i + (int64_t)p * d.lda], ea[(size_t)i]), S, dg);
      for (int t = 0; t < S; ++t) dA[((size_t)t * k + p) * m + i] = dg[t];
    }
    for (int j = 0; j < n; ++j) {
      (int8 ? digits_i8 : digits)(scaled(d.B[p + (int64_t)j * d.ldb], fb[(size_t)j]), S, dg);
      for (int t = 0; t < S; ++t) dB[((size_t)t * k + p) * n + j] = dg[t];
    }
  }
  std::vector<double> acc((size_t)m * n, 0.0), part((size_t)m * n);
  // part[j * m + i] += sum over t <= D, p in [p0, p1) of dA_t[i, p] dB_{D-t}[p, j] (exact integers)
  auto diagonal_sum = [&](int D, int p0, int p1) {
    std::fill(part.begin(), part.end(), 0.0);
    for (int t = 0; t <= D; ++t)
      for (int p = p0; p < p1; ++p) {
        const double* a = &dA[((size_t)t * k + p) * m];
        const double* b = &dB[((size_t)(D - t) * k + p) * n];
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < m; ++i) part[(size_t)j * m + i] += a[i] * b[j];
      }
  };
  if (int8) {
    // each diagonal over groups of up to kSplitI8GroupChunks 256-deep chunks,
    // summed in int32 (exact: |sum| < 2^30), weighted 2^-(12 + 7D)
    const int chunks = std::max(1, (k + fmm::kSplitI8Chunk - 1) / fmm::kSplitI8Chunk);
    for (int c0 = 0; c0 < chunks; c0 += fmm::kSplitI8GroupChunks) {
      const int c1 = std::min(chunks, c0 + fmm::kSplitI8GroupChunks);
      for (int D = 0; D < S; ++D) {
        diagonal_sum(D, c0 * fmm::kSplitI8Chunk, std::min(k, c1 * fmm::kSplitI8Chunk));
        const double scale = std::ldexp(1.0, -(12 + 7 * D));
        for (size_t x = 0; x < part.size(); ++x) {
          const int32_t v = (int32_t)part[x];  // the int32 accumulator (exact)
          acc[x] = std::fma((double)v, scale, acc[x]);
        }
      }
    }
  }
  // C = alpha 2^(e_i + f_j) acc (+ beta C); NaN where a non-finite row or column reaches
  auto store = [&]() {
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) {
        double* c = &d.C[i + (int64_t)j * d.ldc];
        double v = d.alpha * std::ldexp(acc[(size_t)j * m + i], ea[(size_t)i] + fb[(size_t)j]);
        if (d.beta != 0.0) v = v + d.beta * *c;
        if (ea[(size_t)i] == fmm::kSplitNonFinite || fb[(size_t)j] == fmm::kSplitNonFinite)
          v = std::numeric_limits<double>::quiet_NaN();
        *c = v;
      }
  };
  if (int8) {
    store();
    return;
  }
  const int chunks = std::max(1, (k + fmm::kSplitChunk - 1) / fmm::kSplitChunk);
  for (int cp = 0; cp < chunks; cp += fmm::split_chunk_span(S)) {
    const int nch = std::min(fmm::split_chunk_span(S), chunks - cp);
    for (int gi = 0; gi < fmm::split_groups_in_pair(nch, S); ++gi) {
      const fmm::SplitGroup G = fmm::split_group(cp, nch, S, gi);
      const int D = G.D;
      diagonal_sum(D, G.c0 * fmm::kSplitChunk, std::min(k, G.c1 * fmm::kSplitChunk));
      const double scale = std::ldexp(1.0, -8 * (D + 2));
      for (size_t x = 0; x < part.size(); ++x) {
        const float f = (float)part[x];  // the FP32 accumulator (exact)
        acc[x] = std::fma((double)f, scale, acc[x]);
      }
    }
  }
  store();
}

void run_split(const fmm::Op& op, const unsigned char* desc) {
  const fmm::SplitDesc* g = reinterpret_cast<const fmm::SplitDesc*>(desc + op.desc_off);
  const int code = op.split.int8 ? fmm::kSplitInt8Code + op.split.slices : op.split.slices;
  for (int p = 0; p < op.n; ++p) split_product(g[p], code);
}

void run_ops(const fmm::Program& prog) {
  for (const fmm::Op& op : prog.ops) {
    const double* cf = prog.coefs[(size_t)op.cf].v;
    switch (op.kind) {
      case fmm::OpKind::kForm:
        switch (op.alg) {
#define EMU_FORM(idx, ALG) \
  case idx:                \
    run_form<ALG>(op, prog.desc.data(), cf); \
    break;
          FMM_FOR_EACH_ALGORITHM(EMU_FORM)
#undef EMU_FORM
        }
        break;
      case fmm::OpKind::kCombine:
        switch (op.alg) {
#define EMU_COMB(idx, ALG) \
  case idx:                \
    run_combine<ALG>(op, prog.desc.data(), cf); \
    break;
          FMM_FOR_EACH_ALGORITHM(EMU_COMB)
#undef EMU_COMB
        }
        break;
      case fmm::OpKind::kGemm:
        run_gemm(op, prog.desc.data());
        break;
      case fmm::OpKind::kSplitGemm:
        run_split(op, prog.desc.data());
        break;
    }
  }
}

}  // namespace emu

extern "C" {

size_t emu_workspace_bytes(int alg, int64_t m, int64_t k, int64_t n, int steps, int dfs_levels) {
  return fmm::workspace_bytes(fmm_algorithms[alg], m, k, n, steps, dfs_levels);
}

size_t emu_workspace_bytes_split(int alg, int64_t m, int64_t k, int64_t n, int steps, int dfs_levels, int slices) {
  return fmm::workspace_bytes(fmm_algorithms[alg], m, k, n, steps, dfs_levels, slices);
}

// The split-BF16 model for one classical product.
void emu_split_gemm(int m, int k, int n, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                    int64_t ldc, double alpha, double beta, int slices) {
  fmm::SplitDesc d{};
  d.A = A;
  d.B = B;
  d.C = C;
  d.lda = lda;
  d.ldb = ldb;
  d.ldc = ldc;
  d.m = m;
  d.n = n;
  d.k = k;
  d.alpha = alpha;
  d.beta = beta;
  emu::split_product(d, slices);
}

// Runs FastMatmul through the planner + interpreter (split_slices > 0: leaf
// products split-BF16).  stats (may be NULL) receives {#form, #gemm
// (FP64 or split), #combine launches, leaf products, workspace bytes}.
int emu_fast_matmul_split(int alg, double* A, int64_t lda, double* B, int64_t ldb, double* C, int64_t ldc, int m,
                          int k, int n, int steps, double x, double alpha, double beta, int dfs_levels, int slices,
                          int64_t* stats) {
  if (alg < 0 || alg >= FMM_NUM_ALGORITHMS) return -1;
  const size_t bytes = emu_workspace_bytes_split(alg, m, k, n, steps, dfs_levels, slices);
  std::vector<double> ws(bytes / sizeof(double) + 64, std::numeric_limits<double>::quiet_NaN());
  // 256-byte alignment like a device allocation
  double* base = ws.data();
  while (reinterpret_cast<uintptr_t>(base) % 256) ++base;
  fmm::Program prog;
  fmm::build_program(alg, m, k, n, steps, x, alpha, beta, dfs_levels, fmm::Operand{A, lda}, fmm::Operand{B, ldb},
                     fmm::Operand{C, ldc}, base, &prog, slices);
  if (prog.workspace_bytes > bytes) return -2;  // the query must cover the program
  emu::run_ops(prog);
  if (stats) {
    int64_t nf = 0, ng = 0, nc = 0;
    for (const fmm::Op& op : prog.ops) {
      nf += op.kind == fmm::OpKind::kForm;
      ng += op.kind == fmm::OpKind::kGemm || op.kind == fmm::OpKind::kSplitGemm;
      nc += op.kind == fmm::OpKind::kCombine;
    }
    stats[0] = nf;
    stats[1] = ng;
    stats[2] = nc;
    stats[3] = prog.leaf_count;
    stats[4] = (int64_t)prog.workspace_bytes;
  }
  return 0;
}

int emu_fast_matmul(int alg, double* A, int64_t lda, double* B, int64_t ldb, double* C, int64_t ldc, int m, int k,
                    int n, int steps, double x, double alpha, double beta, int dfs_levels, int64_t* stats) {
  return emu_fast_matmul_split(alg, A, lda, B, ldb, C, ldc, m, k, n, steps, x, alpha, beta, dfs_levels, 0, stats);
}

// A batch through the planner + interpreter: item i is
// (algs[i], steps[i], dims[3i..3i+2]) on A_i, B_i, C_i packed column-major
// (lda = m, ...) at the given offsets into A, B, C.
int emu_fast_matmul_batch_split(int count, const int* algs, const int* steps, const int64_t* dims, double* A,
                                const int64_t* a_off, double* B, const int64_t* b_off, double* C,
                                const int64_t* c_off, double x, double alpha, double beta, const int* slices,
                                int64_t* stats) {
  std::vector<fmm::BatchItem> items((size_t)count);
  for (int i = 0; i < count; ++i) {
    fmm::BatchItem& it = items[(size_t)i];
    it.alg = algs[i];
    it.steps = steps[i];
    it.m = dims[3 * i];
    it.k = dims[3 * i + 1];
    it.n = dims[3 * i + 2];
    it.A = fmm::Operand{A + a_off[i], it.m > 0 ? it.m : 1};
    it.B = fmm::Operand{B + b_off[i], it.k > 0 ? it.k : 1};
    it.C = fmm::Operand{C + c_off[i], it.m > 0 ? it.m : 1};
    it.x = x;
    it.alpha = alpha;
    it.beta = beta;
    it.classical = it.alg < 0;
    if (it.classical) it.alg = 0;
    it.split_slices = slices ? slices[i] : 0;
  }
  const size_t bytes = fmm::batch_workspace_bytes(items.data(), count);
  std::vector<double> ws(bytes / sizeof(double) + 64, std::numeric_limits<double>::quiet_NaN());
  double* base = ws.data();
  while (reinterpret_cast<uintptr_t>(base) % 256) ++base;
  fmm::Program prog;
  fmm::build_batch_program(items.data(), count, base, &prog);
  if (prog.workspace_bytes > bytes) return -2;
  emu::run_ops(prog);
  if (stats) {
    int64_t nf = 0, ng = 0, nc = 0;
    for (const fmm::Op& op : prog.ops) {
      nf += op.kind == fmm::OpKind::kForm;
      ng += (op.kind == fmm::OpKind::kGemm && !op.peel) || op.kind == fmm::OpKind::kSplitGemm;
      nc += op.kind == fmm::OpKind::kCombine;
    }
    stats[0] = nf;
    stats[1] = ng;
    stats[2] = nc;
    stats[3] = prog.leaf_count;
    stats[4] = (int64_t)prog.workspace_bytes;
  }
  return 0;
}

int emu_fast_matmul_batch(int count, const int* algs, const int* steps, const int64_t* dims, double* A,
                          const int64_t* a_off, double* B, const int64_t* b_off, double* C, const int64_t* c_off,
                          double x, double alpha, double beta, int64_t* stats) {
  return emu_fast_matmul_batch_split(count, algs, steps, dims, A, a_off, B, b_off, C, c_off, x, alpha, beta, nullptr,
                                     stats);
}

}  // extern "C"
