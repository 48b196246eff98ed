// Batches of independent products, the shape-bucket autotuner and CUDA-graph
// plans (include/fmm.h).  No counterpart in the reference: its FastMatmul
// multiplies one pair per call, with the algorithm and depth fixed when the
// header is chosen.

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "api_internal.h"

using namespace fmm::api;

namespace {

int ceil_log2(int64_t v) {
  int b = 0;
  while (b < 62 && ((int64_t)1 << b) < v) ++b;
  return b;
}

std::tuple<int, int, int> bucket_of(int64_t m, int64_t k, int64_t n) {
  return std::make_tuple(ceil_log2(m), ceil_log2(k), ceil_log2(n));
}

// Size rule used for shapes the autotuner has not measured; from the
// fast-vs-classical sweep on B200 (FP64): fast algorithms pay off only when
// every dimension is large.
void rule_choice(int64_t m, int64_t k, int64_t n, int* alg, int* steps) {
  const int64_t lo = std::min(m, std::min(k, n));
  if (lo >= 12000) {
    *alg = fmm_algorithm_lookup("grey424_26_206");
    *steps = 2;
  } else if (lo >= 4000) {
    *alg = fmm_algorithm_lookup("strassen");
    *steps = 2;
  } else {
    *alg = FMM_ALG_CLASSICAL;
    *steps = 0;
  }
}

void choice_for(fmm_handle h, int64_t m, int64_t k, int64_t n, int* alg, int* steps, int* tile = nullptr) {
  auto it = h->tuned.find(bucket_of(m, k, n));
  if (tile) *tile = FMM_GEMM_TILE_AUTO;
  if (it != h->tuned.end()) {
    *alg = it->second.alg;
    *steps = it->second.steps;
    if (tile) *tile = it->second.tile;
    return;
  }
  rule_choice(m, k, n, alg, steps);
}

}  // namespace

namespace fmm {
namespace api {

fmm_status resolve_items(fmm_handle h, const fmm_batch_item* items, int count, std::vector<fmm::BatchItem>* out) {
  out->clear();
  out->reserve((size_t)count);
  for (int i = 0; i < count; ++i) {
    const fmm_batch_item& it = items[i];
    fmm_status s = check_dims(it.m, it.k, it.n, it.lda, it.ldb, it.ldc);
    if (s != FMM_OK) return fail(s, "batch item " + std::to_string(i) + ": " + fmm_last_error());
    if (it.m == 0 || it.n == 0) continue;
    if (!it.C || (it.k > 0 && (!it.A || !it.B)))
      return fail(FMM_ERR_INVALID_ARGUMENT, "batch item " + std::to_string(i) + ": null matrix pointer");
    fmm::BatchItem b{};
    int alg = it.alg, steps = it.num_steps, tuned_tile = FMM_GEMM_TILE_AUTO;
    if (alg == FMM_ALG_AUTO) choice_for(h, it.m, it.k, it.n, &alg, &steps, &tuned_tile);
    if (it.gemm_tile < FMM_GEMM_TILE_AUTO || it.gemm_tile > FMM_GEMM_TILE_SMALL)
      return fail(FMM_ERR_INVALID_ARGUMENT, "batch item " + std::to_string(i) + ": unknown gemm_tile");
    b.gemm_tile = it.gemm_tile != FMM_GEMM_TILE_AUTO ? it.gemm_tile : tuned_tile;
    if (alg == FMM_ALG_CLASSICAL) {
      b.classical = true;
      b.alg = 0;
      b.steps = 0;
    } else {
      if ((s = check_alg(alg)) != FMM_OK) return s;
      if (steps < 0 || steps > 16)
        return fail(FMM_ERR_INVALID_ARGUMENT, "batch item " + std::to_string(i) + ": num_steps out of range");
      b.classical = false;
      b.alg = alg;
      b.steps = steps;
    }
    b.m = it.m;
    b.k = it.k;
    b.n = it.n;
    b.A = fmm::Operand{const_cast<double*>(it.A), it.lda};
    b.B = fmm::Operand{const_cast<double*>(it.B), it.ldb};
    b.C = fmm::Operand{it.C, it.ldc};
    b.x = it.x;
    b.alpha = it.alpha;
    b.beta = it.beta;
    if ((s = split_slices_for(it.precision, it.split_slices, &b.split_slices)) != FMM_OK)
      return fail(s, "batch item " + std::to_string(i) + ": " + fmm_last_error());
    out->push_back(b);
  }
  return FMM_OK;
}

}  // namespace api
}  // namespace fmm

namespace {

// Splits resolved items into consecutive groups whose workspace fits `limit`.
std::vector<std::pair<int, int>> chunk_items(const std::vector<fmm::BatchItem>& items, size_t limit) {
  std::vector<std::pair<int, int>> chunks;
  int start = 0;
  size_t acc = 0;
  for (int i = 0; i < (int)items.size(); ++i) {
    const size_t need = fmm::batch_workspace_bytes(&items[(size_t)i], 1);
    if (i > start && acc + need > limit) {
      chunks.emplace_back(start, i);
      start = i;
      acc = 0;
    }
    acc += need;
  }
  if (start < (int)items.size()) chunks.emplace_back(start, (int)items.size());
  return chunks;
}

}  // namespace

struct fmm_plan_s {
  fmm_handle h = nullptr;
  fmm::Program prog;
  void* ws = nullptr;
  size_t ws_cap = 0;
  void* d_desc = nullptr;
  size_t d_desc_cap = 0;
  void* h_desc = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t kernels = 0;
};

namespace {

void plan_free(fmm_plan p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->ws) cudaFree(p->ws);
  if (p->d_desc) cudaFree(p->d_desc);
  if (p->h_desc) cudaFreeHost(p->h_desc);
  delete p;
}

// Captures the plan's program (descriptor upload + launches) into a graph.
fmm_status plan_capture(fmm_plan p) {
  fmm_handle h = p->h;
  const size_t nd = p->prog.desc.size();
  if (nd) {
    FMM_CUDA_TRY(cudaMallocHost(&p->h_desc, nd), "cudaMallocHost(plan descriptors)");
    std::memcpy(p->h_desc, p->prog.desc.data(), nd);
    FMM_CUDA_TRY(cudaMalloc(&p->d_desc, nd), "cudaMalloc(plan descriptors)");
  }
  cudaStream_t cap = nullptr;
  FMM_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "cudaStreamCreate");
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    int64_t n = 0;
    e = fmm::run_program(p->prog, p->h_desc, p->d_desc, h->num_sms, cap, &n, nullptr, h->d_err);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cap, &g);
    if (e == cudaSuccess) e = e2;
    p->graph = g;
    p->kernels = n;
  }
  cudaStreamDestroy(cap);
  if (e != cudaSuccess) return cuda_fail(e, "graph capture");
  FMM_CUDA_TRY(cudaGraphInstantiate(&p->exec, p->graph, 0), "cudaGraphInstantiate");
  return FMM_OK;
}

}  // namespace

extern "C" {

fmm_status fmm_fast_matmul_batched(fmm_handle h, const fmm_batch_item* items, int count) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  if (count < 0 || (count > 0 && !items)) return fail(FMM_ERR_INVALID_ARGUMENT, "bad batch");
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  std::vector<fmm::BatchItem> resolved;
  fmm_status s = resolve_items(h, items, count, &resolved);
  if (s != FMM_OK) return s;
  for (const std::pair<int, int>& c : chunk_items(resolved, h->ws_limit)) {
    const int n = c.second - c.first;
    const size_t need = fmm::batch_workspace_bytes(&resolved[(size_t)c.first], n);
    if (need > h->ws_limit)
      return fail(FMM_ERR_OUT_OF_MEMORY, "batch item needs " + std::to_string(need) +
                                             " bytes of workspace, above the handle's limit");
    if ((s = ensure_device_buffer(h, &h->ws, &h->ws_cap, need ? need : 256, "workspace")) != FMM_OK) return s;
    try {
      fmm::build_batch_program(&resolved[(size_t)c.first], n, h->ws, &h->prog);
    } catch (const std::exception& ex) {
      return fail(FMM_ERR_OUT_OF_MEMORY, std::string("planning failed: ") + ex.what());
    }
    if ((s = stage_descriptors(h, h->prog)) != FMM_OK) return s;
    if ((s = run_staged(h, h->prog)) != FMM_OK) return s;
  }
  return FMM_OK;
}

fmm_status fmm_autotune_choice(fmm_handle h, int64_t m, int64_t k, int64_t n, int* alg, int* num_steps) {
  if (!h || !alg || !num_steps) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  if (m <= 0 || k <= 0 || n <= 0) return fail(FMM_ERR_INVALID_ARGUMENT, "dimensions must be positive");
  choice_for(h, m, k, n, alg, num_steps);
  return FMM_OK;
}

fmm_status fmm_autotune_tile(fmm_handle h, int64_t m, int64_t k, int64_t n, int* tile) {
  if (!h || !tile) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  if (m <= 0 || k <= 0 || n <= 0) return fail(FMM_ERR_INVALID_ARGUMENT, "dimensions must be positive");
  int alg = 0, steps = 0;
  choice_for(h, m, k, n, &alg, &steps, tile);
  return FMM_OK;
}

fmm_status fmm_autotune(fmm_handle h, const int64_t* shapes, int count, const int* candidates, int n_candidates,
                        int max_steps) {
  if (!h || (count > 0 && !shapes)) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  if (max_steps < 0 || max_steps > 4) return fail(FMM_ERR_INVALID_ARGUMENT, "max_steps must be in [0, 4]");
  std::vector<int> cands;
  if (candidates && n_candidates > 0) {
    for (int i = 0; i < n_candidates; ++i) {
      fmm_status s = check_alg(candidates[i]);
      if (s != FMM_OK) return s;
      cands.push_back(candidates[i]);
    }
  } else {
    for (const char* nm : {"strassen", "grey424_26_206", "grey333_23_125", "smirnov333_23_128"})
      cands.push_back(fmm_algorithm_lookup(nm));
  }
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  // one representative (the first) shape per bucket
  std::map<std::tuple<int, int, int>, std::array<int64_t, 3>> reps;
  for (int i = 0; i < count; ++i) {
    const int64_t m = shapes[3 * i], k = shapes[3 * i + 1], n = shapes[3 * i + 2];
    if (m <= 0 || k <= 0 || n <= 0) return fail(FMM_ERR_INVALID_ARGUMENT, "shapes must be positive");
    reps.emplace(bucket_of(m, k, n), std::array<int64_t, 3>{m, k, n});
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FMM_CUDA_TRY(cudaEventCreate(&e0), "cudaEventCreate");
  FMM_CUDA_TRY(cudaEventCreate(&e1), "cudaEventCreate");
  fmm_status result = FMM_OK;
  for (const auto& kv : reps) {
    const int64_t m = kv.second[0], k = kv.second[1], n = kv.second[2];
    double *A = nullptr, *B = nullptr, *C = nullptr;
    if (cudaMalloc(&A, sizeof(double) * (size_t)(m * k)) != cudaSuccess ||
        cudaMalloc(&B, sizeof(double) * (size_t)(k * n)) != cudaSuccess ||
        cudaMalloc(&C, sizeof(double) * (size_t)(m * n)) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(A);
      cudaFree(B);
      result = fail(FMM_ERR_OUT_OF_MEMORY, "autotune: cannot allocate a representative shape");
      break;
    }
    fmm_fill_uniform(h, A, m, k, m, 5, 1, -1.0, 1.0);
    fmm_fill_uniform(h, B, k, n, k, 5, 2, -1.0, 1.0);
    auto time_it = [&](auto&& fn) -> float {
      if (fn() != FMM_OK) return -1.f;
      cudaEventRecord(e0, h->stream);
      for (int r = 0; r < 3; ++r)
        if (fn() != FMM_OK) return -1.f;
      cudaEventRecord(e1, h->stream);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      return ms / 3.f;
    };
    // every candidate with each tile configuration of the FP64 GEMM
    int best_alg = FMM_ALG_CLASSICAL, best_steps = 0, best_tile = FMM_GEMM_TILE_LARGE;
    float best = -1.f;
    for (int tile : {FMM_GEMM_TILE_LARGE, FMM_GEMM_TILE_SMALL}) {
      const float ms = time_it([&] { return dgemm_tiled(h, A, m, B, k, C, m, m, k, n, 1.0, 0.0, tile); });
      if (ms > 0.f && (best < 0.f || ms < best)) {
        best = ms;
        best_tile = tile;
      }
    }
    for (int alg : cands) {
      const fmm_alg_table& t = fmm_algorithms[alg];
      int64_t mm = m, kk = k, nn = n;
      for (int steps = 1; steps <= max_steps; ++steps) {
        mm /= t.m0;
        kk /= t.k0;
        nn /= t.n0;
        if (mm < 64 || kk < 64 || nn < 64) break;
        for (int tile : {FMM_GEMM_TILE_LARGE, FMM_GEMM_TILE_SMALL}) {
          fmm_options o;
          fmm_options_init(&o);
          o.gemm_tile = tile;
          const float ms = time_it(
              [&] { return fmm_fast_matmul(h, alg, A, m, B, k, C, m, m, k, n, steps, 1e-8, 1.0, 0.0, &o); });
          if (ms > 0.f && (best < 0.f || ms < best)) {
            best = ms;
            best_alg = alg;
            best_steps = steps;
            best_tile = tile;
          }
        }
      }
    }
    h->tuned[kv.first] = fmm_handle_s::Tuned{best_alg, best_steps, best_tile};
    cudaFree(A);
    cudaFree(B);
    cudaFree(C);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return result;
}

fmm_status fmm_autotune_export(fmm_handle h, char* buf, size_t cap, size_t* len) {
  if (!h) return fail(FMM_ERR_INVALID_ARGUMENT, "null handle");
  std::ostringstream os;
  for (const auto& kv : h->tuned)
    os << std::get<0>(kv.first) << ' ' << std::get<1>(kv.first) << ' ' << std::get<2>(kv.first) << ' '
       << kv.second.alg << ' ' << kv.second.steps << ' ' << kv.second.tile << '\n';
  const std::string text = os.str();
  if (len) *len = text.size() + 1;
  if (buf) {
    if (cap < text.size() + 1) return fail(FMM_ERR_INVALID_ARGUMENT, "buffer too small");
    std::memcpy(buf, text.c_str(), text.size() + 1);
  }
  return FMM_OK;
}

fmm_status fmm_autotune_import(fmm_handle h, const char* text) {
  if (!h || !text) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  // one bucket per line: "mb kb nb alg steps [tile]" (tables without the
  // tile column load with the tile chosen per problem)
  std::istringstream is(text);
  std::string line;
  while (std::getline(is, line)) {
    std::istringstream ls(line);
    int mb, kb, nb, alg, steps, tile = FMM_GEMM_TILE_AUTO;
    if (!(ls >> mb >> kb >> nb >> alg >> steps)) continue;
    if (!(ls >> tile)) tile = FMM_GEMM_TILE_AUTO;
    if (alg != FMM_ALG_CLASSICAL && (alg < 0 || alg >= FMM_NUM_ALGORITHMS))
      return fail(FMM_ERR_UNKNOWN_ALGORITHM, "tuning table names an unknown algorithm");
    if (tile < FMM_GEMM_TILE_AUTO || tile > FMM_GEMM_TILE_SMALL)
      return fail(FMM_ERR_INVALID_ARGUMENT, "tuning table names an unknown gemm tile");
    h->tuned[std::make_tuple(mb, kb, nb)] = fmm_handle_s::Tuned{alg, steps, tile};
  }
  return FMM_OK;
}

fmm_status fmm_plan_create(fmm_handle h, int alg, const double* A, int64_t lda, const double* B, int64_t ldb,
                           double* C, int64_t ldc, int64_t m, int64_t k, int64_t n, int num_steps, double x,
                           double alpha, double beta, const fmm_options* opts, fmm_plan* out) {
  if (!h || !out) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  fmm_status s = check_alg(alg);
  if (s != FMM_OK) return s;
  if ((s = check_dims(m, k, n, lda, ldb, ldc)) != FMM_OK) return s;
  if (num_steps < 0 || num_steps > 16) return fail(FMM_ERR_INVALID_ARGUMENT, "num_steps must be in [0, 16]");
  if (!C || (k > 0 && (!A || !B))) return fail(FMM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  fmm_options o;
  resolve_options(opts, &o);
  int slices = 0;
  if ((s = split_slices_for(o.precision, o.split_slices, &slices)) != FMM_OK) return s;
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  int d = 0;
  size_t bytes = 0;
  if ((s = choose_dfs_levels(h, alg, m, k, n, num_steps, o, &d, &bytes)) != FMM_OK) return s;
  fmm_plan p = new fmm_plan_s();
  p->h = h;
  if (cudaMalloc(&p->ws, bytes ? bytes : 256) != cudaSuccess) {
    cudaGetLastError();
    plan_free(p);
    return fail(FMM_ERR_OUT_OF_MEMORY, "cannot allocate the plan's workspace");
  }
  fmm::build_program(alg, m, k, n, num_steps, x, alpha, beta, d, fmm::Operand{const_cast<double*>(A), lda},
                     fmm::Operand{const_cast<double*>(B), ldb}, fmm::Operand{C, ldc}, p->ws, &p->prog, slices,
                     o.gemm_tile);
  if ((s = plan_capture(p)) != FMM_OK) {
    plan_free(p);
    return s;
  }
  *out = p;
  return FMM_OK;
}

fmm_status fmm_plan_create_batched(fmm_handle h, const fmm_batch_item* items, int count, fmm_plan* out) {
  if (!h || !out) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  DeviceGuard g(h->device);
  if (!g.ok()) return fail(FMM_ERR_CUDA, "cudaSetDevice failed");
  std::vector<fmm::BatchItem> resolved;
  fmm_status s = resolve_items(h, items, count, &resolved);
  if (s != FMM_OK) return s;
  const size_t need = fmm::batch_workspace_bytes(resolved.data(), (int)resolved.size());
  if (need > h->ws_limit)
    return fail(FMM_ERR_OUT_OF_MEMORY, "batch workspace of " + std::to_string(need) + " bytes exceeds the limit");
  fmm_plan p = new fmm_plan_s();
  p->h = h;
  if (cudaMalloc(&p->ws, need ? need : 256) != cudaSuccess) {
    cudaGetLastError();
    plan_free(p);
    return fail(FMM_ERR_OUT_OF_MEMORY, "cannot allocate the plan's workspace");
  }
  fmm::build_batch_program(resolved.data(), (int)resolved.size(), p->ws, &p->prog);
  if ((s = plan_capture(p)) != FMM_OK) {
    plan_free(p);
    return s;
  }
  *out = p;
  return FMM_OK;
}

fmm_status fmm_plan_execute(fmm_plan p) {
  if (!p) return fail(FMM_ERR_INVALID_ARGUMENT, "null plan");
  DeviceGuard g(p->h->device);
  FMM_CUDA_TRY(cudaGraphLaunch(p->exec, p->h->stream), "cudaGraphLaunch");
  p->h->launches += p->kernels;
  return FMM_OK;
}

fmm_status fmm_plan_destroy(fmm_plan p) {
  if (!p) return FMM_OK;
  DeviceGuard g(p->h->device);
  cudaStreamSynchronize(p->h->stream);
  plan_free(p);
  return FMM_OK;
}

int64_t fmm_plan_kernel_count(fmm_plan p) { return p ? p->kernels : 0; }

}  // extern "C"
