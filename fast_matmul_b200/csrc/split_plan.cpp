// Scratch layout of split-BF16 and split-INT8 leaf products (host arithmetic
// only, so the planner and its CPU emulator share it).
//
// Slices are stored "k-block major": for problem p, slice t, k-block b, the
// padded rows (or columns) of that block form consecutive 128-byte rows (64
// BF16 or 128 INT8 values).  One 2-D tensor map of 128-byte rows then covers
// every slice of every problem, whatever the shapes: a 128-row operand tile
// is the box at x = 0, y = a_row + (t * kblocks + b) * padded_rows +
// tile_row.  Rows of A are padded to a multiple of 256, the rows of the
// output tile of one CTA pair; output tiles are counted per pair (256 x 128).
// k is padded to whole chunks (two k-blocks: 128 values BF16, 256 INT8).

#include <algorithm>

#include "fmm_internal.h"

namespace fmm {

namespace {

int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

struct Geometry {
  int64_t tiles_m, tiles_n, kblocks;
};

Geometry geometry(int64_t m, int64_t k, int64_t n, bool int8) {
  const int64_t chunk = int8 ? kSplitI8Chunk : kSplitChunk;
  Geometry g;
  g.tiles_m = (m + kSplitPairRows - 1) / kSplitPairRows * (kSplitPairRows / kSplitTile);
  g.tiles_n = (n + kSplitTile - 1) / kSplitTile;
  g.kblocks = std::max<int64_t>(1, (k + chunk - 1) / chunk) * 2;
  return g;
}

// A-splitting work tiles (32 rows x 64 k) of one problem.
int64_t a_work(const Geometry& g, bool int8) { return (g.tiles_m * kSplitTile / 32) * g.kblocks * (int8 ? 2 : 1); }

}  // namespace

SplitPlan split_plan_for(int code) {
  SplitPlan p;
  p.slices = split_code_slices(code);
  p.int8 = split_code_int8(code);
  return p;
}

SplitPlan split_prepare(SplitDesc* descs, int n, int code) {
  SplitPlan p = split_plan_for(code);
  const int slices = p.slices;
  for (int i = 0; i < n; ++i) {
    SplitDesc& d = descs[i];
    const bool empty = d.m <= 0 || d.n <= 0;
    const Geometry g = geometry(empty ? 0 : d.m, d.k, empty ? 0 : d.n, p.int8);
    d.kblocks = (int)g.kblocks;
    d.tiles_m = (int)g.tiles_m;
    d.tiles_n = (int)g.tiles_n;
    d.tile_begin = p.tiles;
    d.sa_begin = p.sa_work;
    d.a_row = p.rows_a;
    d.b_row = p.rows_b;
    d.e_off = p.n_e;
    d.f_off = p.n_f;
    if (empty) continue;
    const int64_t mp = g.tiles_m * kSplitTile, np = g.tiles_n * kSplitTile;
    p.tiles += g.tiles_m / 2 * g.tiles_n;
    p.sa_work += a_work(g, p.int8);
    p.rows_a += (int64_t)slices * g.kblocks * mp;
    p.rows_b += (int64_t)slices * g.kblocks * np;
    p.n_e += mp;
    p.n_f += np;
  }
  split_finish(&p);
  return p;
}

void split_accumulate(SplitPlan* p, int64_t m, int64_t k, int64_t n, int64_t count) {
  if (m <= 0 || n <= 0 || count <= 0) return;
  const Geometry g = geometry(m, k, n, p->int8);
  const int64_t mp = g.tiles_m * kSplitTile, np = g.tiles_n * kSplitTile;
  p->tiles += count * (g.tiles_m / 2) * g.tiles_n;
  p->sa_work += count * a_work(g, p->int8);
  p->rows_a += count * p->slices * g.kblocks * mp;
  p->rows_b += count * p->slices * g.kblocks * np;
  p->n_e += count * mp;
  p->n_f += count * np;
}

void split_finish(SplitPlan* p) {
  p->off_b = (size_t)round_up(p->rows_a * 128, 1024);
  p->off_e = p->off_b + (size_t)round_up(p->rows_b * 128, 1024);
  p->off_f = p->off_e + (size_t)round_up(p->n_e * 4, 1024);
  p->bytes = p->off_f + (size_t)round_up(p->n_f * 4, 1024);
}

size_t split_scratch_bytes(int64_t m, int64_t k, int64_t n, int64_t count, int code) {
  SplitPlan p = split_plan_for(code);
  split_accumulate(&p, m, k, n, count);
  split_finish(&p);
  return p.bytes;
}

}  // namespace fmm
