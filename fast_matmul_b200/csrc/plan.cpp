// Recursion planner.
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
//
// A batch of independent products is planned breadth-first per item, with
// the launches of all items merged: one formation launch per (algorithm,
// level), one GEMM launch for every leaf of every item, then the
// combinations and fringe products level by level upwards.

#include "plan.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <stdexcept>
#include <utility>

namespace fmm {

namespace {

constexpr int64_t kAlignDoubles = 32;  // 256 bytes

int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

struct LevelLayout {
  int64_t cm, ck, cn;           // child block dims (level l+1)
  int64_t ldS, ldT, ldM;        // padded leading dimensions
  int64_t sizeS, sizeT, sizeM;  // doubles per block
  int64_t unit;                 // sub-problems per unit at this level
  size_t off_S, off_T, off_M;   // byte offsets
};

int64_t unit_size(int l, int dfs_levels, int R) {
  if (l < dfs_levels) return 1;
  int64_t u = (dfs_levels == 0) ? 1 : R;
  const int start = (dfs_levels == 0) ? 0 : dfs_levels;
  for (int i = start; i < l; ++i) u *= R;
  return u;
}

std::vector<LevelLayout> layout(const fmm_alg_table& t, const std::vector<LevelDims>& dims, int steps,
                                int dfs_levels, size_t base, size_t* end) {
  std::vector<LevelLayout> lay(steps);
  size_t off = base;
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
  }
  *end = off;
  return lay;
}

struct SubProblem {
  Operand A, B, C;
  double mult;  // the product's multiplier: alpha of its leaf GEMMs and fringes
  double beta;
};

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <class D>
size_t append_desc(Program* prog, const std::vector<D>& v) {
  std::vector<unsigned char>& b = prog->desc;
  const size_t off = (size_t)round_up((int64_t)b.size(), 64);
  b.resize(off + v.size() * sizeof(D));
  std::memcpy(b.data() + off, v.data(), v.size() * sizeof(D));
  return off;
}

// ---- per-level building blocks shared by the single and batched builders

// Formation descriptors of one sub-problem (A side into sd, B side into td).
void add_form_descs(const fmm_alg_table& t, const LevelLayout& L, const SubProblem& p, double* S, double* T,
                    std::vector<FormDesc>* sd, std::vector<FormDesc>* td, bool* vec2, int64_t* max_items,
                    double* bytes) {
  if (t.n_a_out > 0 && L.cm > 0 && L.ck > 0) {
    FormDesc d{p.A.ptr, p.A.ld, S, L.ldS, L.sizeS, L.cm, L.ck};
    *vec2 = *vec2 && aligned16(d.in) && d.ld_in % 2 == 0 && L.cm % 2 == 0;
    sd->push_back(d);
    *max_items = std::max(*max_items, add_work_items(L.cm, L.ck, 1));
    *bytes += 8.0 * (double)L.cm * L.ck * (t.m0 * t.k0 + t.n_a_out);
  }
  if (t.n_b_out > 0 && L.ck > 0 && L.cn > 0) {
    FormDesc d{p.B.ptr, p.B.ld, T, L.ldT, L.sizeT, L.ck, L.cn};
    *vec2 = *vec2 && aligned16(d.in) && d.ld_in % 2 == 0 && L.ck % 2 == 0;
    td->push_back(d);
    *max_items = std::max(*max_items, add_work_items(L.ck, L.cn, 1));
    *bytes += 8.0 * (double)L.ck * L.cn * (t.k0 * t.n0 + t.n_b_out);
  }
}

Operand block_of(const Operand& X, int64_t rows, int64_t cols, int nbc, int b) {
  const int bi = b / nbc, bj = b % nbc;
  return Operand{X.ptr + bi * rows + bj * cols * X.ld, X.ld};
}

// The R children of p (codegen/gen.py:574-657): operands are materialised
// outputs or views; single coefficients fold into the multiplier.
void add_children(const fmm_alg_table& t, const double* slots, const LevelLayout& L, const SubProblem& p, double* S,
                  double* T, double* M, std::vector<SubProblem>* out) {
  const int R = t.rank;
  for (int r = 0; r < R; ++r) {
    SubProblem c;
    const short* as = t.a_src + 3 * r;
    const short* bs = t.b_src + 3 * r;
    c.mult = p.mult;
    if (as[0] == 0)
      c.A = block_of(p.A, L.cm, L.ck, t.k0, as[1]);
    else
      c.A = Operand{S + as[1] * L.sizeS, L.ldS};
    if (as[2]) c.mult *= slots[as[2] - 1];
    if (bs[0] == 0)
      c.B = block_of(p.B, L.ck, L.cn, t.n0, bs[1]);
    else
      c.B = Operand{T + bs[1] * L.sizeT, L.ldT};
    if (bs[2]) c.mult *= slots[bs[2] - 1];
    c.C = Operand{M + r * L.sizeM, L.ldM};
    c.beta = 0.0;
    out->push_back(c);
  }
}

// C blocks = sum of gamma * M (+ beta * C)  (strassen.hpp:646-649)
void add_combine_desc(const fmm_alg_table& t, const LevelLayout& L, const SubProblem& p, double* M,
                      std::vector<CombineDesc>* cd, bool* vec2, int64_t* max_items, double* bytes) {
  if (L.cm <= 0 || L.cn <= 0) return;
  CombineDesc d{M, L.ldM, L.sizeM, p.C.ptr, p.C.ld, L.cm, L.cn, p.beta};
  *vec2 = *vec2 && L.cm % 2 == 0 && aligned16(d.c) && d.ld_c % 2 == 0;
  cd->push_back(d);
  *max_items = std::max(*max_items, add_work_items(L.cm, L.cn, 1));
  *bytes += 8.0 * (double)L.cm * L.cn * (t.rank + t.m0 * t.n0 * (p.beta != 0.0 ? 2 : 1));
}

// Dynamic peeling of the fringes of p (linalg/linalg.hpp:201-244).
// D: p's dimensions, Ch: its children's (level_dims); the fringes are what the
// m0 x k0 x n0 blocks of Ch leave over.
void add_peel_descs(const fmm_alg_table& t, const LevelDims& D, const LevelDims& Ch, const SubProblem& p,
                    std::vector<GemmDesc>* g) {
  const int64_t xr = D.m - Ch.m * t.m0;
  const int64_t xk = D.k - Ch.k * t.k0;
  const int64_t xc = D.n - Ch.n * t.n0;
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
    g->push_back(d);
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
    g->push_back(d);
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
    g->push_back(d);
  }
}

GemmDesc leaf_desc(const LevelDims& D, const SubProblem& p) {
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
  return d;
}

// ---- op emission

void emit_form(Program* prog, int alg, int cf, int level, const std::vector<FormDesc>& sd,
               const std::vector<FormDesc>& td, bool vec2, int64_t max_items, double bytes) {
  if (sd.empty() && td.empty()) return;
  std::vector<FormDesc> all(sd);
  all.insert(all.end(), td.begin(), td.end());
  Op op;
  op.kind = OpKind::kForm;
  op.alg = alg;
  op.cf = cf;
  op.n = (int)all.size();
  op.n_s = (int)sd.size();
  op.n_t = (int)td.size();
  op.max_items = vec2 ? (max_items + 1) / 2 : max_items;
  op.vec2 = vec2;
  op.level = level;
  op.bytes = bytes;
  op.desc_off = append_desc(prog, all);
  prog->ops.push_back(op);
}

void emit_combine(Program* prog, int alg, int cf, int level, const std::vector<CombineDesc>& cd, bool vec2,
                  int64_t max_items, double bytes) {
  if (cd.empty()) return;
  Op op;
  op.kind = OpKind::kCombine;
  op.alg = alg;
  op.cf = cf;
  op.n = (int)cd.size();
  op.max_items = vec2 ? (max_items + 1) / 2 : max_items;
  op.vec2 = vec2;
  op.level = level;
  op.bytes = bytes;
  op.desc_off = append_desc(prog, cd);
  prog->ops.push_back(op);
}

// One grouped GEMM launch per tile configuration in use: problem i of g
// runs with tiles[i]; tiles may be null (every problem Auto) or hold one
// entry (all problems alike).  The Auto problems of a launch share one
// configuration, the one gemm_tile_rule favours over their rows in total,
// so a launch splits in two only where problems ask for different ones.
void emit_gemm(Program* prog, int level, std::vector<GemmDesc>& g, bool leaves, const std::vector<int>* tiles) {
  if (g.empty()) return;
  double flops = 0.0;
  for (const GemmDesc& d : g) flops += 2.0 * d.m * d.n * (double)d.k;
  if (leaves) {
    prog->leaf_flops += flops;
    prog->leaf_count += (int64_t)g.size();
  } else {
    prog->peel_flops += flops;
  }
  auto asked = [&](size_t i) {
    const int c = (tiles && !tiles->empty()) ? (*tiles)[tiles->size() == 1 ? 0 : i] : kGemmTileAuto;
    return (c == kGemmTileLarge || c == kGemmTileSmall) ? c : kGemmTileAuto;
  };
  // padded tile area of the Auto problems under each configuration
  double area_large = 0.0, area_small = 0.0;
  for (size_t i = 0; i < g.size(); ++i) {
    if (asked(i) != kGemmTileAuto) continue;
    const double cols = (double)((g[i].n + kGemmBN - 1) / kGemmBN) * kGemmBN;
    area_large += cols * (double)((g[i].m + kGemmBM - 1) / kGemmBM) * kGemmBM;
    area_small += cols * (double)((g[i].m + kGemmBMSmall - 1) / kGemmBMSmall) * kGemmBMSmall;
  }
  const int auto_cfg = area_large > 1.07 * area_small ? kGemmTileSmall : kGemmTileLarge;
  // fringe products with few rows, columns or inner indices go to the thin kernel whatever
  // the tile configuration (which changes no result), so results stay the
  // same under every configuration
  // parts: 0 large tiles, 1 small tiles, 2 few rows or columns, 3 few inner indices
  auto part_of = [&](const GemmDesc& d, int cfg) {
    if (!leaves && (d.m <= kThinMax || d.n <= kThinMax)) return 2;
    if (!leaves && d.k <= kThinMax) return 3;
    return cfg == kGemmTileSmall ? 1 : 0;
  };
  std::vector<GemmDesc> part[4];
  double part_flops[4] = {0.0, 0.0, 0.0, 0.0};
  for (size_t i = 0; i < g.size(); ++i) {
    int cfg = asked(i);
    if (cfg == kGemmTileAuto) cfg = auto_cfg;
    const int c = part_of(g[i], cfg);
    part[c].push_back(g[i]);
    part_flops[c] += 2.0 * g[i].m * g[i].n * (double)g[i].k;
  }
  for (int c = 0; c < 4; ++c) {
    if (part[c].empty()) continue;
    const int cfg = c == 3 ? kGemmTileThinInner : c == 2 ? kGemmTileThin : c ? kGemmTileSmall : kGemmTileLarge;
    const int64_t ntiles = c >= 2 ? thin_prepare(part[c].data(), (int)part[c].size())
                                  : gemm_prepare(part[c].data(), (int)part[c].size(), kGemmBN, gemm_tile_rows(cfg));
    if (ntiles == 0) continue;
    Op op;
    op.kind = OpKind::kGemm;
    op.n = (int)part[c].size();
    op.total_tiles = ntiles;
    op.gemm_tile = cfg;
    op.level = level;
    op.peel = !leaves;
    op.flops = part_flops[c];
    op.desc_off = append_desc(prog, part[c]);
    prog->ops.push_back(op);
  }
}

// Leaf products of one launch as split products of split code `slices`
// (BF16 or INT8 digits, fmm_internal.h).
// All split launches of a program run in order on one stream, so they share
// one scratch region sized for the largest (Program::split_bytes).
void emit_split_gemm(Program* prog, int level, const std::vector<GemmDesc>& g, int slices) {
  if (g.empty()) return;
  std::vector<SplitDesc> sd;
  sd.reserve(g.size());
  double flops = 0.0;
  for (const GemmDesc& d : g) {
    SplitDesc s{};
    s.A = d.A;
    s.B = d.B;
    s.C = d.C;
    s.lda = d.lda;
    s.ldb = d.ldb;
    s.ldc = d.ldc;
    s.alpha = d.alpha;
    s.beta = d.beta;
    s.m = d.m;
    s.n = d.n;
    s.k = d.k;
    sd.push_back(s);
    flops += 2.0 * d.m * d.n * (double)d.k;
  }
  prog->leaf_flops += flops;
  prog->leaf_count += (int64_t)g.size();
  const SplitPlan plan = split_prepare(sd.data(), (int)sd.size(), slices);
  if (plan.tiles == 0) return;
  Op op;
  op.kind = OpKind::kSplitGemm;
  op.n = (int)sd.size();
  op.total_tiles = plan.tiles;
  op.level = level;
  op.flops = flops;
  op.split = plan;
  op.desc_off = append_desc(prog, sd);
  prog->ops.push_back(op);
  prog->split_bytes = std::max(prog->split_bytes, plan.bytes);
}

// Places the split scratch after the recursion's workspace.
void place_split_scratch(Program* prog, char* ws) {
  if (prog->split_bytes == 0) return;
  const size_t off = (size_t)round_up((int64_t)prog->workspace_bytes, 1024);
  prog->split_scratch = ws + off;
  prog->workspace_bytes = off + prog->split_bytes;
}

// ---- single call, any schedule

class Builder {
 public:
  Builder(int alg, int steps, int dfs_levels, const std::vector<LevelDims>& dims, const std::vector<LevelLayout>& lay,
          const double* slots, char* ws, Program* prog, int gemm_tile)
      : alg_(alg), t_(fmm_algorithms[alg]), steps_(steps), d_(dfs_levels), dims_(dims), lay_(lay), slots_(slots),
        ws_(ws), prog_(prog), tile_(1, gemm_tile) {}

  void level(int l, const std::vector<SubProblem>& F) {
    if (F.empty()) return;
    if (l == steps_) {
      std::vector<GemmDesc> g;
      g.reserve(F.size());
      for (const SubProblem& p : F) g.push_back(leaf_desc(dims_[l], p));
      if (prog_->split_slices > 0)
        emit_split_gemm(prog_, l, g, prog_->split_slices);
      else
        emit_gemm(prog_, l, g, true, &tile_);
      return;
    }
    // depth-first: one unit per sub-problem, and the fringe products of all
    // of them in one launch after the last (they touch only their own
    // operands and C, which live until the parent's combination reads them)
    std::vector<GemmDesc> peel;
    if (l < d_) {
      for (const SubProblem& p : F) unit(l, &p, 1, &peel);
    } else {
      unit(l, F.data(), (int64_t)F.size(), &peel);
    }
    emit_gemm(prog_, l, peel, false, &tile_);
  }

 private:
  // Forms, recurses and combines F[0..nf) as one unit; appends its fringe
  // products to *peel.
  void unit(int l, const SubProblem* F, int64_t nf, std::vector<GemmDesc>* peel) {
    const LevelLayout& L = lay_[l];
    const int R = t_.rank;
    double* S = reinterpret_cast<double*>(ws_ + L.off_S);
    double* T = reinterpret_cast<double*>(ws_ + L.off_T);
    double* M = reinterpret_cast<double*>(ws_ + L.off_M);
    {
      std::vector<FormDesc> sd, td;
      bool vec2 = true;
      int64_t items = 0;
      double bytes = 0.0;
      for (int64_t q = 0; q < nf; ++q)
        add_form_descs(t_, L, F[q], S + q * t_.n_a_out * L.sizeS, T + q * t_.n_b_out * L.sizeT, &sd, &td, &vec2,
                       &items, &bytes);
      emit_form(prog_, alg_, 0, l, sd, td, vec2, items, bytes);
    }
    std::vector<SubProblem> ch;
    ch.reserve((size_t)(nf * R));
    for (int64_t q = 0; q < nf; ++q)
      add_children(t_, slots_, L, F[q], S + q * t_.n_a_out * L.sizeS, T + q * t_.n_b_out * L.sizeT,
                   M + q * R * L.sizeM, &ch);
    level(l + 1, ch);
    {
      std::vector<CombineDesc> cd;
      bool vec2 = true;
      int64_t items = 0;
      double bytes = 0.0;
      for (int64_t q = 0; q < nf; ++q) add_combine_desc(t_, L, F[q], M + q * R * L.sizeM, &cd, &vec2, &items, &bytes);
      emit_combine(prog_, alg_, 0, l, cd, vec2, items, bytes);
    }
    for (int64_t q = 0; q < nf; ++q) add_peel_descs(t_, dims_[l], dims_[l + 1], F[q], peel);
  }

  int alg_;
  const fmm_alg_table& t_;
  int steps_;
  int d_;
  const std::vector<LevelDims>& dims_;
  const std::vector<LevelLayout>& lay_;
  const double* slots_;
  char* ws_;
  Program* prog_;
  std::vector<int> tile_;  // the program's tile configuration (one entry)
};

struct ItemState {
  std::vector<LevelDims> dims;
  std::vector<LevelLayout> lay;
  std::vector<std::vector<SubProblem>> frontier;  // sub-problems per level
  int cf = 0;
};

}  // namespace

void Program::clear() {
  ops.clear();
  desc.clear();
  coefs.clear();
  workspace_bytes = 0;
  dfs_levels = 0;
  leaf_flops = 0.0;
  peel_flops = 0.0;
  leaf_count = 0;
  split_slices = 0;
  split_scratch = nullptr;
  split_bytes = 0;
  ws_base = nullptr;
}

// Rows and inner dimension of a block: floor(x / b), one less when that is
// odd and at least kEvenBlockMin, so that every block of an operand with an
// even leading dimension starts on a 16-byte boundary (the leaf GEMM's and
// the formation kernels' 16-byte copies) at the cost of peeling up to
// 2b - 1 instead of b - 1 rows; the fringe products that take them are
// padded to whole GEMM tiles either way.
int64_t block_dim(int64_t x, int b) {
  const int64_t c = x / b;
  return (c >= kEvenBlockMin && (c & 1)) ? c - 1 : c;
}

std::vector<LevelDims> level_dims(const fmm_alg_table& t, int64_t m, int64_t k, int64_t n, int steps) {
  std::vector<LevelDims> d((size_t)steps + 1);
  d[0] = LevelDims{m, k, n};
  for (int l = 1; l <= steps; ++l)
    d[l] = LevelDims{block_dim(d[l - 1].m, t.m0), block_dim(d[l - 1].k, t.k0), d[l - 1].n / t.n0};
  return d;
}

int64_t thin_prepare(GemmDesc* descs, int n) {
  int64_t total = 0;
  for (int i = 0; i < n; ++i) {
    GemmDesc& d = descs[i];
    const int64_t items = thin_items(d.m, d.n, d.k);
    d.tiles_m = (int)items;
    d.tile_begin = (int)total;
    d.flags = 0;
    total += items;
  }
  return total;
}

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

size_t workspace_bytes(const fmm_alg_table& t, int64_t m, int64_t k, int64_t n, int steps, int dfs_levels,
                       int split_slices) {
  size_t total = 0;
  const std::vector<LevelDims> dims = level_dims(t, m, k, n, steps);
  layout(t, dims, steps, dfs_levels, 0, &total);
  if (split_slices > 0) {
    // leaf products per launch: R^steps breadth-first; below depth-first
    // levels, the R^(steps - d + 1) leaves of one unit at level d - 1
    int64_t leaves = 1;
    if (steps > 0) {
      const int d = std::max(1, std::min(dfs_levels, steps));
      for (int i = 0; i < steps - d + 1; ++i) leaves *= t.rank;
    }
    const LevelDims& L = dims[(size_t)steps];
    const size_t sb = split_scratch_bytes(L.m, L.k, L.n, leaves, split_slices);
    if (sb > 0) total = (size_t)round_up((int64_t)total, 1024) + sb;
  }
  return total;
}

void build_program(int alg, int64_t m, int64_t k, int64_t n, int steps, double x, double alpha, double beta,
                   int dfs_levels, Operand A, Operand B, Operand C, void* ws, Program* out, int split_slices,
                   int gemm_tile) {
  const fmm_alg_table& t = fmm_algorithms[alg];
  const std::vector<LevelDims> dims = level_dims(t, m, k, n, steps);
  size_t total = 0;
  const std::vector<LevelLayout> lay = layout(t, dims, steps, dfs_levels, 0, &total);
  out->clear();
  CoefSlots cf{};
  t.eval(x, cf.v);
  out->coefs.push_back(cf);
  out->workspace_bytes = total;
  out->dfs_levels = dfs_levels;
  out->split_slices = split_slices;
  // FastMatmul (strassen.hpp:661-722): A's multiplier is alpha; the first
  // recursion folds it into C's (C.mult = 1 * alpha * 1).
  SubProblem root{A, B, C, 1.0 * alpha * 1.0, beta};
  Builder b(alg, steps, dfs_levels, dims, lay, out->coefs[0].v, static_cast<char*>(ws), out, gemm_tile);
  b.level(0, std::vector<SubProblem>{root});
  place_split_scratch(out, static_cast<char*>(ws));
  out->ws_base = ws;
}

// Split scratch of a batch: one split launch per distinct slice count, all
// sharing one region sized for the largest.
void BatchFootprint::add(const BatchItem& it) {
  if (!it.classical) {
    const fmm_alg_table& t = fmm_algorithms[it.alg];
    size_t end = 0;
    layout(t, level_dims(t, it.m, it.k, it.n, it.steps), it.steps, 0, 0, &end);
    fp64_ += (size_t)round_up((int64_t)end, 256);  // items are laid out back to back, 256-byte aligned
  }
  if (it.split_slices <= 0) return;
  auto f = split_.find(it.split_slices);
  if (f == split_.end()) f = split_.emplace(it.split_slices, split_plan_for(it.split_slices)).first;
  SplitPlan& p = f->second;
  if (it.classical) {
    split_accumulate(&p, it.m, it.k, it.n, 1);
    return;
  }
  const fmm_alg_table& t = fmm_algorithms[it.alg];
  const std::vector<LevelDims> dims = level_dims(t, it.m, it.k, it.n, it.steps);
  int64_t leaves = 1;
  for (int l = 0; l < it.steps; ++l) leaves *= t.rank;
  split_accumulate(&p, dims[(size_t)it.steps].m, dims[(size_t)it.steps].k, dims[(size_t)it.steps].n, leaves);
}

size_t BatchFootprint::bytes() const {
  size_t mx = 0;
  for (const auto& kv : split_) {
    SplitPlan p = kv.second;
    split_finish(&p);
    if (p.tiles > 0) mx = std::max(mx, p.bytes);
  }
  return mx > 0 ? (size_t)round_up((int64_t)fp64_, 1024) + mx : fp64_;
}

size_t batch_workspace_bytes(const BatchItem* items, int count) {
  BatchFootprint f;
  for (int i = 0; i < count; ++i) f.add(items[i]);
  return f.bytes();
}

void build_batch_program(const BatchItem* items, int count, void* ws, Program* out) {
  out->clear();
  out->dfs_levels = 0;
  char* base = static_cast<char*>(ws);
  std::vector<ItemState> st((size_t)count);
  std::map<std::pair<int, double>, int> coef_index;  // (alg, x) -> coefficient set
  int max_steps = 0;
  size_t off = 0;
  for (int i = 0; i < count; ++i) {
    const BatchItem& it = items[i];
    const fmm_alg_table& t = fmm_algorithms[it.classical ? 0 : it.alg];
    ItemState& s = st[(size_t)i];
    const int isteps = it.classical ? 0 : it.steps;
    s.dims = level_dims(t, it.m, it.k, it.n, isteps);
    size_t end = 0;
    s.lay = layout(t, s.dims, isteps, 0, off, &end);
    off = (size_t)round_up((int64_t)end, 256);
    const std::pair<int, double> key(it.alg, it.x);
    auto found = coef_index.find(key);
    if (found == coef_index.end()) {
      CoefSlots cf{};
      t.eval(it.x, cf.v);
      out->coefs.push_back(cf);
      found = coef_index.emplace(key, (int)out->coefs.size() - 1).first;
    }
    s.cf = found->second;
    s.frontier.resize((size_t)isteps + 1);
    s.frontier[0].push_back(SubProblem{it.A, it.B, it.C, 1.0 * it.alpha * 1.0, it.beta});
    for (int l = 0; l < isteps; ++l) {
      const LevelLayout& L = s.lay[(size_t)l];
      double* S = reinterpret_cast<double*>(base + L.off_S);
      double* T = reinterpret_cast<double*>(base + L.off_T);
      double* M = reinterpret_cast<double*>(base + L.off_M);
      const std::vector<SubProblem>& F = s.frontier[(size_t)l];
      for (size_t q = 0; q < F.size(); ++q)
        add_children(t, out->coefs[(size_t)s.cf].v, L, F[q], S + q * t.n_a_out * L.sizeS,
                     T + q * t.n_b_out * L.sizeT, M + q * t.rank * L.sizeM, &s.frontier[(size_t)l + 1]);
    }
    max_steps = std::max(max_steps, isteps);
  }
  out->workspace_bytes = off;
  auto steps_of = [&](int i) { return items[i].classical ? 0 : items[i].steps; };

  // formations, top-down: one launch per (algorithm, coefficient set, level)
  for (int l = 0; l < max_steps; ++l) {
    std::map<std::pair<int, int>, std::vector<int>> groups;
    for (int i = 0; i < count; ++i)
      if (steps_of(i) > l) groups[{items[i].alg, st[(size_t)i].cf}].push_back(i);
    for (const auto& g : groups) {
      const fmm_alg_table& t = fmm_algorithms[g.first.first];
      std::vector<FormDesc> sd, td;
      bool vec2 = true;
      int64_t mx = 0;
      double bytes = 0.0;
      for (int i : g.second) {
        const ItemState& s = st[(size_t)i];
        const LevelLayout& L = s.lay[(size_t)l];
        double* S = reinterpret_cast<double*>(base + L.off_S);
        double* T = reinterpret_cast<double*>(base + L.off_T);
        const std::vector<SubProblem>& F = s.frontier[(size_t)l];
        for (size_t q = 0; q < F.size(); ++q)
          add_form_descs(t, L, F[q], S + q * t.n_a_out * L.sizeS, T + q * t.n_b_out * L.sizeT, &sd, &td, &vec2,
                         &mx, &bytes);
      }
      emit_form(out, g.first.first, g.first.second, l, sd, td, vec2, mx, bytes);
    }
  }
  // every leaf of every item: one grouped GEMM (FP64), one split launch per
  // distinct slice count
  {
    std::map<int, std::vector<GemmDesc>> g;
    std::vector<int> fp64_tiles;  // tile configuration of each FP64 leaf (g[0])
    for (int i = 0; i < count; ++i) {
      const ItemState& s = st[(size_t)i];
      const size_t steps = (size_t)steps_of(i);
      const int code = std::max(0, items[i].split_slices);
      std::vector<GemmDesc>& dst = g[code];
      for (const SubProblem& p : s.frontier[steps]) {
        GemmDesc d = leaf_desc(s.dims[steps], p);
        if (items[i].classical) d.beta = items[i].beta;
        dst.push_back(d);
        if (code == 0) fp64_tiles.push_back(items[i].gemm_tile);
      }
    }
    for (auto& kv : g) {
      if (kv.first == 0)
        emit_gemm(out, max_steps, kv.second, true, &fp64_tiles);
      else
        emit_split_gemm(out, max_steps, kv.second, kv.first);
    }
  }
  // combinations and fringes, bottom-up
  for (int l = max_steps - 1; l >= 0; --l) {
    std::map<std::pair<int, int>, std::vector<int>> groups;
    for (int i = 0; i < count; ++i)
      if (steps_of(i) > l) groups[{items[i].alg, st[(size_t)i].cf}].push_back(i);
    for (const auto& g : groups) {
      const fmm_alg_table& t = fmm_algorithms[g.first.first];
      std::vector<CombineDesc> cd;
      bool vec2 = true;
      int64_t mx = 0;
      double bytes = 0.0;
      for (int i : g.second) {
        const ItemState& s = st[(size_t)i];
        const LevelLayout& L = s.lay[(size_t)l];
        double* M = reinterpret_cast<double*>(base + L.off_M);
        const std::vector<SubProblem>& F = s.frontier[(size_t)l];
        for (size_t q = 0; q < F.size(); ++q)
          add_combine_desc(t, L, F[q], M + q * t.rank * L.sizeM, &cd, &vec2, &mx, &bytes);
      }
      emit_combine(out, g.first.first, g.first.second, l, cd, vec2, mx, bytes);
    }
    std::vector<GemmDesc> peel;
    std::vector<int> peel_tiles;
    for (int i = 0; i < count; ++i) {
      if (steps_of(i) <= l) continue;
      const fmm_alg_table& t = fmm_algorithms[items[i].alg];
      const ItemState& s = st[(size_t)i];
      for (const SubProblem& p : s.frontier[(size_t)l])
        add_peel_descs(t, s.dims[(size_t)l], s.dims[(size_t)l + 1], p, &peel);
      peel_tiles.resize(peel.size(), items[i].gemm_tile);
    }
    emit_gemm(out, l, peel, false, &peel_tiles);
  }
  place_split_scratch(out, base);
  out->ws_base = ws;
}

}  // namespace fmm
