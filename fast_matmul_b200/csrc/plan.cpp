// Recursion planner and program runner.
//
// The reference recursion (FastMatmulRecursive, algorithms/strassen.hpp:377-659)
// visits sub-problems one at a time on the host.  Every sub-problem at one
// level has the same dimensions (floor splitting), so the recursion is
// planned here as a tree of *units*: a unit is a set of same-level
// sub-problems that are processed together -- one grouped formation launch,
// the children (recursively), one grouped combination launch, one grouped
// peeling launch.  Depth-first levels use units of one sub-problem (the
// reference's DFS order); breadth-first levels take all children of the
// unit above (the reference's BFS task tree, util/par_util.hpp, as single
// launches).  The R^steps leaf products of a unit go out as one grouped GEMM.
//
// Workspace (MemoryManager, util/MemoryManager.hpp:65-118, allocates S, T and M
// for every product of every level up front): here each level owns exactly
// one region sized for ONE unit of that level, which sibling units reuse in
// turn, so depth-first levels cost one sub-problem's temporaries and only
// the breadth-first levels scale with R^l.  Leading dimensions are padded to
// even and blocks to 256-byte multiples so every workspace block allows
// 16-byte vector access.

#include "plan.h"

#include <algorithm>
#include <cstring>
#include <stdexcept>

namespace fmm {

namespace {

constexpr int64_t kAlignDoubles = 32;  // 256 bytes

int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

struct LevelLayout {
  int64_t cm, ck, cn;         // child block dims (level l+1)
  int64_t ldS, ldT, ldM;      // padded leading dimensions
  int64_t sizeS, sizeT, sizeM;  // doubles per block
  int64_t unit;               // sub-problems per unit at this level
  size_t off_S, off_T, off_M;   // byte offsets
  size_t bytes;
};

int64_t unit_size(int l, int dfs_levels, int R) {
  if (l < dfs_levels) return 1;
  int64_t u = (dfs_levels == 0) ? 1 : R;
  const int start = (dfs_levels == 0) ? 0 : dfs_levels;
  for (int i = start; i < l; ++i) u *= R;
  return u;
}

std::vector<LevelLayout> layout(const fmm_alg_table& t, const std::vector<LevelDims>& dims, int steps,
                                int dfs_levels, size_t* total) {
  std::vector<LevelLayout> lay(steps);
  size_t off = 0;
  for (int l = 0; l < steps; ++l) {
    LevelLayout& L = lay[l];
    L.cm = dims[l + 1].m;
    L.ck = dims[l + 1].k;
    L.cn = dims[l + 1].n;
    L.ldS = std::max<int64_t>(2, round_up(L.cm, 2));
    L.ldT = std::max<int64_t>(2, round_up(L.ck, 2));
    L.ldM = std::max<int64_t>(2, round_up(L.cm, 2));
    L.sizeS = round_up(L.ldS * L.ck, kAlignDoubles);
    L.sizeT = round_up(L.ldT * L.cn, kAlignDoubles);
    L.sizeM = round_up(L.ldM * L.cn, kAlignDoubles);
    L.unit = unit_size(l, dfs_levels, t.rank);
    L.off_S = off;
    off += (size_t)(L.unit * t.n_a_out * L.sizeS) * sizeof(double);
    L.off_T = off;
    off += (size_t)(L.unit * t.n_b_out * L.sizeT) * sizeof(double);
    L.off_M = off;
    off += (size_t)(L.unit * t.rank * L.sizeM) * sizeof(double);
    L.bytes = off - L.off_S;
  }
  *total = off;
  return lay;
}

struct SubProblem {
  Operand A, B, C;
  double mult;  // the product's multiplier: alpha of its leaf GEMMs and fringes
  double beta;
};

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

class Builder {
 public:
  Builder(int alg, int steps, int dfs_levels, const std::vector<LevelDims>& dims, const std::vector<LevelLayout>& lay,
          const double* slots, char* ws, Program* prog)
      : t_(fmm_algorithms[alg]), steps_(steps), d_(dfs_levels), dims_(dims), lay_(lay), slots_(slots), ws_(ws),
        prog_(prog) {}

  void level(int l, const std::vector<SubProblem>& F) {
    if (F.empty()) return;
    if (l == steps_) {
      emit_leaves(l, F);
      return;
    }
    if (l < d_) {
      for (const SubProblem& p : F) unit(l, &p, 1);
    } else {
      unit(l, F.data(), (int64_t)F.size());
    }
  }

 private:
  template <class D>
  size_t append(const std::vector<D>& v) {
    std::vector<unsigned char>& b = prog_->desc;
    size_t off = round_up((int64_t)b.size(), 64);
    b.resize(off + v.size() * sizeof(D));
    std::memcpy(b.data() + off, v.data(), v.size() * sizeof(D));
    return off;
  }

  void emit_gemm(int l, std::vector<GemmDesc>& g, bool leaves) {
    // (tile counts and copy widths are filled in by gemm_prepare)
    if (g.empty()) return;
    const int64_t tiles = gemm_prepare(g.data(), (int)g.size());
    double flops = 0.0;
    for (const GemmDesc& d : g) flops += 2.0 * d.m * d.n * (double)d.k;
    if (leaves) {
      prog_->leaf_flops += flops;
      prog_->leaf_count += (int64_t)g.size();
    } else {
      prog_->peel_flops += flops;
    }
    if (tiles == 0) return;
    Op op;
    op.kind = OpKind::kGemm;
    op.n = (int)g.size();
    op.total_tiles = tiles;
    op.level = l;
    op.peel = !leaves;
    op.flops = flops;
    op.desc_off = append(g);
    prog_->ops.push_back(op);
  }

  void emit_leaves(int l, const std::vector<SubProblem>& F) {
    const LevelDims& D = dims_[l];
    std::vector<GemmDesc> g;
    g.reserve(F.size());
    for (const SubProblem& p : F) {
      GemmDesc d{};
      d.A = p.A.ptr;
      d.B = p.B.ptr;
      d.C = p.C.ptr;
      d.lda = p.A.ld;
      d.ldb = p.B.ld;
      d.ldc = p.C.ld;
      d.m = (int)D.m;
      d.n = (int)D.n;
      d.k = (int)D.k;
      d.alpha = p.mult;
      d.beta = 0.0;  // the base case calls MatMul(A, B, C) with its default beta
      g.push_back(d);
    }
    emit_gemm(l, g, true);
  }

  Operand block(const Operand& X, int64_t rows, int64_t cols, int nbc, int b) const {
    const int bi = b / nbc, bj = b % nbc;
    return Operand{X.ptr + bi * rows + bj * cols * X.ld, X.ld};
  }

  void unit(int l, const SubProblem* F, int64_t nf) {
    const LevelLayout& L = lay_[l];
    const int R = t_.rank;
    double* S = reinterpret_cast<double*>(ws_ + L.off_S);
    double* T = reinterpret_cast<double*>(ws_ + L.off_T);
    double* M = reinterpret_cast<double*>(ws_ + L.off_M);

    // 1. form the materialised S and T operands of every product
    const bool s_work = t_.n_a_out > 0 && L.cm > 0 && L.ck > 0;
    const bool t_work = t_.n_b_out > 0 && L.ck > 0 && L.cn > 0;
    if (s_work || t_work) {
      std::vector<FormDesc> fd;
      bool vec2 = true;
      if (s_work) {
        for (int64_t q = 0; q < nf; ++q) {
          FormDesc d{F[q].A.ptr, F[q].A.ld, S + q * t_.n_a_out * L.sizeS, L.ldS, L.sizeS};
          vec2 = vec2 && aligned16(d.in) && d.ld_in % 2 == 0 && L.cm % 2 == 0;
          fd.push_back(d);
        }
      }
      if (t_work) {
        for (int64_t q = 0; q < nf; ++q) {
          FormDesc d{F[q].B.ptr, F[q].B.ld, T + q * t_.n_b_out * L.sizeT, L.ldT, L.sizeT};
          vec2 = vec2 && aligned16(d.in) && d.ld_in % 2 == 0 && L.ck % 2 == 0;
          fd.push_back(d);
        }
      }
      Op op;
      op.kind = OpKind::kForm;
      op.n = (int)fd.size();
      op.n_s = s_work ? (int)nf : 0;
      op.n_t = t_work ? (int)nf : 0;
      op.a_rows = L.cm;
      op.a_cols = L.ck;
      op.b_rows = L.ck;
      op.b_cols = L.cn;
      op.vec2 = vec2;
      op.level = l;
      op.bytes = 8.0 * nf *
                 ((s_work ? (double)L.cm * L.ck * (t_.m0 * t_.k0 + t_.n_a_out) : 0.0) +
                  (t_work ? (double)L.ck * L.cn * (t_.k0 * t_.n0 + t_.n_b_out) : 0.0));
      op.desc_off = append(fd);
      prog_->ops.push_back(op);
    }

    // 2. the children (codegen/gen.py:574-657): operands are materialised
    //    outputs or views; single coefficients fold into the multiplier
    std::vector<SubProblem> ch((size_t)(nf * R));
    for (int64_t q = 0; q < nf; ++q) {
      const SubProblem& p = F[q];
      for (int r = 0; r < R; ++r) {
        SubProblem& c = ch[(size_t)(q * R + r)];
        const short* as = t_.a_src + 3 * r;
        const short* bs = t_.b_src + 3 * r;
        c.mult = p.mult;
        if (as[0] == 0) {
          c.A = block(p.A, L.cm, L.ck, t_.k0, as[1]);
        } else {
          c.A = Operand{S + (q * t_.n_a_out + as[1]) * L.sizeS, L.ldS};
        }
        if (as[2]) c.mult *= slots_[as[2] - 1];
        if (bs[0] == 0) {
          c.B = block(p.B, L.ck, L.cn, t_.n0, bs[1]);
        } else {
          c.B = Operand{T + (q * t_.n_b_out + bs[1]) * L.sizeT, L.ldT};
        }
        if (bs[2]) c.mult *= slots_[bs[2] - 1];
        c.C = Operand{M + (q * R + r) * L.sizeM, L.ldM};
        c.beta = 0.0;
      }
    }
    level(l + 1, ch);

    // 3. C blocks = sum of gamma * M (+ beta * C)  (strassen.hpp:646-649)
    if (L.cm > 0 && L.cn > 0) {
      std::vector<CombineDesc> cd;
      bool vec2 = (L.cm % 2 == 0);
      for (int64_t q = 0; q < nf; ++q) {
        CombineDesc d{M + q * R * L.sizeM, L.ldM, L.sizeM, F[q].C.ptr, F[q].C.ld};
        vec2 = vec2 && aligned16(d.c) && d.ld_c % 2 == 0;
        cd.push_back(d);
      }
      Op op;
      op.kind = OpKind::kCombine;
      op.n = (int)cd.size();
      op.rows = L.cm;
      op.cols = L.cn;
      op.beta = F[0].beta;
      op.vec2 = vec2;
      op.level = l;
      op.bytes = 8.0 * nf * (double)L.cm * L.cn * (R + t_.m0 * t_.n0 * (F[0].beta != 0.0 ? 2 : 1));
      op.desc_off = append(cd);
      prog_->ops.push_back(op);
    }

    // 4. dynamic peeling of the fringes (linalg/linalg.hpp:201-244)
    const LevelDims& D = dims_[l];
    const int64_t xr = D.m - (D.m / t_.m0) * t_.m0;
    const int64_t xk = D.k - (D.k / t_.k0) * t_.k0;
    const int64_t xc = D.n - (D.n / t_.n0) * t_.n0;
    if (xr || xk || xc) {
      std::vector<GemmDesc> g;
      for (int64_t q = 0; q < nf; ++q) {
        const SubProblem& p = F[q];
        if (xk > 0) {  // C(core, core) += A(core, kx) * B(kx, core)
          const int64_t rd = D.m - xr, cdim = D.n - xc, inner = D.k - xk;
          GemmDesc d{};
          d.A = p.A.ptr + inner * p.A.ld;
          d.lda = p.A.ld;
          d.B = p.B.ptr + inner;
          d.ldb = p.B.ld;
          d.C = p.C.ptr;
          d.ldc = p.C.ld;
          d.m = (int)rd;
          d.n = (int)cdim;
          d.k = (int)xk;
          d.alpha = p.mult;
          d.beta = 1.0;
          g.push_back(d);
        }
        if (xc > 0) {  // C(:, nx) = A * B(:, nx) + beta * C(:, nx)
          const int64_t s = D.n - xc;
          GemmDesc d{};
          d.A = p.A.ptr;
          d.lda = p.A.ld;
          d.B = p.B.ptr + s * p.B.ld;
          d.ldb = p.B.ld;
          d.C = p.C.ptr + s * p.C.ld;
          d.ldc = p.C.ld;
          d.m = (int)D.m;
          d.n = (int)xc;
          d.k = (int)D.k;
          d.alpha = p.mult;
          d.beta = p.beta;
          g.push_back(d);
        }
        if (xr > 0) {  // C(mx, core) = A(mx, :) * B(:, core) + beta * C(mx, core)
          const int64_t s = D.m - xr, nc = D.n - xc;
          GemmDesc d{};
          d.A = p.A.ptr + s;
          d.lda = p.A.ld;
          d.B = p.B.ptr;
          d.ldb = p.B.ld;
          d.C = p.C.ptr + s;
          d.ldc = p.C.ld;
          d.m = (int)xr;
          d.n = (int)nc;
          d.k = (int)D.k;
          d.alpha = p.mult;
          d.beta = p.beta;
          g.push_back(d);
        }
      }
      emit_gemm(l, g, false);
    }
  }

  const fmm_alg_table& t_;
  int steps_;
  int d_;
  const std::vector<LevelDims>& dims_;
  const std::vector<LevelLayout>& lay_;
  const double* slots_;
  char* ws_;
  Program* prog_;
};

}  // namespace

int64_t gemm_prepare(GemmDesc* descs, int n, int tile_n, int tile_m) {
  int64_t total = 0;
  for (int i = 0; i < n; ++i) {
    GemmDesc& d = descs[i];
    const int tm = (d.m + tile_m - 1) / tile_m;
    const int tn = (d.n + tile_n - 1) / tile_n;
    d.tiles_m = tm > 0 ? tm : 1;
    d.tile_begin = (int)total;
    int flags = 0;
    if ((reinterpret_cast<uintptr_t>(d.A) % 16 == 0) && (d.lda % 2 == 0)) flags |= 1;
    if ((reinterpret_cast<uintptr_t>(d.B) % 16 == 0) && (d.ldb % 2 == 0)) flags |= 2;
    d.flags = flags;
    if (d.m > 0 && d.n > 0) total += (int64_t)tm * tn;
  }
  return total;
}

std::vector<LevelDims> level_dims(const fmm_alg_table& t, int64_t m, int64_t k, int64_t n, int steps) {
  std::vector<LevelDims> d((size_t)steps + 1);
  d[0] = LevelDims{m, k, n};
  for (int l = 1; l <= steps; ++l) d[l] = LevelDims{d[l - 1].m / t.m0, d[l - 1].k / t.k0, d[l - 1].n / t.n0};
  return d;
}

size_t workspace_bytes(const fmm_alg_table& t, int64_t m, int64_t k, int64_t n, int steps, int dfs_levels) {
  size_t total = 0;
  layout(t, level_dims(t, m, k, n, steps), steps, dfs_levels, &total);
  return total;
}

void build_program(int alg, int64_t m, int64_t k, int64_t n, int steps, double x, double alpha, double beta,
                   int dfs_levels, Operand A, Operand B, Operand C, void* ws, Program* out) {
  const fmm_alg_table& t = fmm_algorithms[alg];
  const std::vector<LevelDims> dims = level_dims(t, m, k, n, steps);
  size_t total = 0;
  const std::vector<LevelLayout> lay = layout(t, dims, steps, dfs_levels, &total);
  double slots[FMM_MAX_SLOTS > 0 ? FMM_MAX_SLOTS : 1];
  t.eval(x, slots);
  out->ops.clear();
  out->desc.clear();
  out->workspace_bytes = total;
  out->dfs_levels = dfs_levels;
  out->leaf_flops = 0.0;
  out->peel_flops = 0.0;
  out->leaf_count = 0;
  // FastMatmul (strassen.hpp:661-722): A's multiplier is alpha; the first
  // recursion folds it into C's (C.mult = 1 * alpha * 1).
  SubProblem root{A, B, C, 1.0 * alpha * 1.0, beta};
  Builder b(alg, steps, dfs_levels, dims, lay, slots, static_cast<char*>(ws), out);
  b.level(0, std::vector<SubProblem>{root});
}

}  // namespace fmm
