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
    }
  }
}

}  // namespace emu

extern "C" {

size_t emu_workspace_bytes(int alg, int64_t m, int64_t k, int64_t n, int steps, int dfs_levels) {
  return fmm::workspace_bytes(fmm_algorithms[alg], m, k, n, steps, dfs_levels);
}

// Runs FastMatmul through the planner + interpreter.  stats (may be NULL)
// receives {#form, #gemm, #combine launches, leaf products, workspace bytes}.
int emu_fast_matmul(int alg, double* A, int64_t lda, double* B, int64_t ldb, double* C, int64_t ldc, int m, int k,
                    int n, int steps, double x, double alpha, double beta, int dfs_levels, int64_t* stats) {
  if (alg < 0 || alg >= FMM_NUM_ALGORITHMS) return -1;
  const size_t bytes = emu_workspace_bytes(alg, m, k, n, steps, dfs_levels);
  std::vector<double> ws(bytes / sizeof(double) + 64, std::numeric_limits<double>::quiet_NaN());
  // 256-byte alignment like a device allocation
  double* base = ws.data();
  while (reinterpret_cast<uintptr_t>(base) % 256) ++base;
  fmm::Program prog;
  fmm::build_program(alg, m, k, n, steps, x, alpha, beta, dfs_levels, fmm::Operand{A, lda}, fmm::Operand{B, ldb},
                     fmm::Operand{C, ldc}, base, &prog);
  emu::run_ops(prog);
  if (stats) {
    int64_t nf = 0, ng = 0, nc = 0;
    for (const fmm::Op& op : prog.ops) {
      nf += op.kind == fmm::OpKind::kForm;
      ng += op.kind == fmm::OpKind::kGemm;
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

// A batch through the planner + interpreter: item i is
// (algs[i], steps[i], dims[3i..3i+2]) on A_i, B_i, C_i packed column-major
// (lda = m, ...) at the given offsets into A, B, C.
int emu_fast_matmul_batch(int count, const int* algs, const int* steps, const int64_t* dims, double* A,
                          const int64_t* a_off, double* B, const int64_t* b_off, double* C, const int64_t* c_off,
                          double x, double alpha, double beta, int64_t* stats) {
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
  }
  const size_t bytes = fmm::batch_workspace_bytes(items.data(), count);
  std::vector<double> ws(bytes / sizeof(double) + 64, std::numeric_limits<double>::quiet_NaN());
  double* base = ws.data();
  while (reinterpret_cast<uintptr_t>(base) % 256) ++base;
  fmm::Program prog;
  fmm::build_batch_program(items.data(), count, base, &prog);
  emu::run_ops(prog);
  if (stats) {
    int64_t nf = 0, ng = 0, nc = 0;
    for (const fmm::Op& op : prog.ops) {
      nf += op.kind == fmm::OpKind::kForm;
      ng += op.kind == fmm::OpKind::kGemm && !op.peel;
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

}  // extern "C"
