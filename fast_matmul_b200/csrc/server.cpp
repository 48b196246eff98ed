// Serving: a continuous-batching request loop (fmm_server_* in include/fmm.h).
//
// A background thread owns `max_inflight` launch slots, each with its own
// stream, completion event and descriptor buffers, and a device workspace
// pool managed by a first-fit free list.  On every turn it
//   1. retires slots whose event has completed (their requests are done,
//      their workspace block returns to the pool), and
//   2. for every idle slot, admits queued requests in arrival order while the
//      summed S/T/M workspace of the requests fits one free block of the pool
//      (and at most max_batch requests), plans them as one batch program
//      (breadth-first per request, all FP64 leaf products in one grouped GEMM,
//      all split-BF16 leaf products in one tensor-core launch per slice
//      count) and launches it on the slot's stream.
// Requests that arrive while earlier batches run are admitted as soon as a
// slot and memory free up; batches of different slots overlap on the device.

#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "api_internal.h"

using namespace fmm::api;

namespace {

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  void* h_desc = nullptr;
  size_t h_cap = 0;
  void* d_desc = nullptr;
  size_t d_cap = 0;
  bool busy = false;
  std::vector<uint64_t> tickets;
  size_t ws_off = 0, ws_size = 0;
  fmm::Program prog;
  int* d_err = nullptr;  // error word of the slot's split-BF16 kernels
  int* h_err = nullptr;  // pinned copy, valid once `done` has completed
};

struct Pending {
  fmm_request req;
  uint64_t ticket;
};

}  // namespace

struct fmm_server_s {
  fmm_handle h = nullptr;  // device, SM count, tuning table
  char* pool = nullptr;
  size_t pool_size = 0;
  std::map<size_t, size_t> free_blocks;  // offset -> size
  size_t in_use = 0;
  std::vector<Slot> slots;
  int max_batch = 64;
  std::deque<Pending> pending;
  std::unordered_map<uint64_t, fmm_request_info> info;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
  uint64_t next_ticket = 1;
  fmm_server_stats stats{};
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

bool pool_alloc(fmm_server s, size_t bytes, size_t* off) {
  bytes = (bytes + 255) & ~(size_t)255;
  if (bytes == 0) bytes = 256;
  for (auto it = s->free_blocks.begin(); it != s->free_blocks.end(); ++it) {
    if (it->second >= bytes) {
      *off = it->first;
      const size_t rest = it->second - bytes;
      const size_t next = it->first + bytes;
      s->free_blocks.erase(it);
      if (rest) s->free_blocks[next] = rest;
      s->in_use += bytes;
      if (s->in_use > s->stats.workspace_peak) s->stats.workspace_peak = s->in_use;
      return true;
    }
  }
  return false;
}

void pool_free(fmm_server s, size_t off, size_t bytes) {
  bytes = (bytes + 255) & ~(size_t)255;
  if (bytes == 0) bytes = 256;
  s->in_use -= bytes;
  auto it = s->free_blocks.emplace(off, bytes).first;
  auto next = std::next(it);
  if (next != s->free_blocks.end() && it->first + it->second == next->first) {
    it->second += next->second;
    s->free_blocks.erase(next);
  }
  if (it != s->free_blocks.begin()) {
    auto prev = std::prev(it);
    if (prev->first + prev->second == it->first) {
      prev->second += it->second;
      s->free_blocks.erase(it);
    }
  }
}

size_t largest_free(fmm_server s) {
  size_t best = 0;
  for (const auto& kv : s->free_blocks) best = kv.second > best ? kv.second : best;
  return best;
}

fmm_batch_item as_item(const fmm_request& r) {
  fmm_batch_item it{};
  it.alg = r.alg;
  it.num_steps = r.num_steps;
  it.A = r.A;
  it.lda = r.lda;
  it.B = r.B;
  it.ldb = r.ldb;
  it.C = r.C;
  it.ldc = r.ldc;
  it.m = r.m;
  it.k = r.k;
  it.n = r.n;
  it.x = r.x;
  it.alpha = r.alpha;
  it.beta = r.beta;
  it.precision = r.precision;
  it.split_slices = r.split_slices;
  return it;
}

void finish(fmm_server s, uint64_t ticket, fmm_status st) {
  fmm_request_info& inf = s->info[ticket];
  inf.done = 1;
  inf.status = st;
  inf.done_ms = s->now_ms();
  s->stats.completed++;
}

bool ensure_slot_buffers(Slot& sl, size_t need) {
  if (need > sl.h_cap) {
    if (sl.h_desc) cudaFreeHost(sl.h_desc);
    sl.h_desc = nullptr;
    sl.h_cap = 0;
    const size_t cap = need * 2;
    if (cudaMallocHost(&sl.h_desc, cap) != cudaSuccess) return false;
    sl.h_cap = cap;
  }
  if (need > sl.d_cap) {
    if (sl.d_desc) cudaFree(sl.d_desc);
    sl.d_desc = nullptr;
    sl.d_cap = 0;
    const size_t cap = need * 2;
    if (cudaMalloc(&sl.d_desc, cap) != cudaSuccess) return false;
    sl.d_cap = cap;
  }
  return true;
}

// One turn of the loop; returns whether anything changed.  Called with s->mu held.
bool turn(fmm_server s) {
  bool progressed = false;
  for (Slot& sl : s->slots) {
    if (!sl.busy) continue;
    const cudaError_t q = cudaEventQuery(sl.done);
    if (q == cudaErrorNotReady) continue;
    fmm_status st = q == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
    if (st == FMM_OK && *sl.h_err != 0) st = FMM_ERR_TIMEOUT;  // a bounded device wait gave up
    for (uint64_t t : sl.tickets) finish(s, t, st);
    sl.tickets.clear();
    pool_free(s, sl.ws_off, sl.ws_size);
    sl.busy = false;
    progressed = true;
  }
  if (progressed) s->cv_done.notify_all();
  if (s->stop) return progressed;
  for (Slot& sl : s->slots) {
    if (sl.busy || s->pending.empty()) continue;
    std::vector<fmm::BatchItem> batch;
    std::vector<uint64_t> tickets;
    fmm::BatchFootprint footprint;
    size_t need = 0;
    const size_t avail = largest_free(s);
    while (!s->pending.empty() && (int)batch.size() < s->max_batch) {
      const Pending& p = s->pending.front();
      const fmm_batch_item it = as_item(p.req);
      std::vector<fmm::BatchItem> one;
      fmm_status st = resolve_items(s->h, &it, 1, &one);
      if (st != FMM_OK) {
        finish(s, p.ticket, st);
        s->pending.pop_front();
        progressed = true;
        continue;
      }
      const size_t bytes = one.empty() ? 0 : fmm::batch_workspace_bytes(one.data(), 1);
      if (bytes > s->pool_size) {
        finish(s, p.ticket, FMM_ERR_OUT_OF_MEMORY);
        s->pending.pop_front();
        progressed = true;
        continue;
      }
      // the footprint of the batch with this request, laid out as the batch
      // program lays it out (alignment between items included)
      fmm::BatchFootprint trial = footprint;
      for (const fmm::BatchItem& b : one) trial.add(b);
      const size_t total = trial.bytes();
      if (total + 256 > avail) break;  // admit in order: wait for memory
      need = (total + 255) & ~(size_t)255;
      footprint = trial;
      batch.insert(batch.end(), one.begin(), one.end());
      tickets.push_back(p.ticket);
      s->pending.pop_front();
    }
    if (tickets.empty()) break;
    size_t off = 0;
    if (!pool_alloc(s, need, &off)) {  // cannot happen: need <= largest free block
      for (uint64_t t : tickets) finish(s, t, FMM_ERR_OUT_OF_MEMORY);
      continue;
    }
    const double launch = s->now_ms();
    for (uint64_t t : tickets) s->info[t].launch_ms = launch;
    fmm_status st = FMM_OK;
    if (!batch.empty()) {
      try {
        fmm::build_batch_program(batch.data(), (int)batch.size(), s->pool + off, &sl.prog);
      } catch (const std::exception&) {
        st = FMM_ERR_OUT_OF_MEMORY;
      }
      // the program lays the batch out exactly as batch_workspace_bytes does
      if (st == FMM_OK && sl.prog.workspace_bytes > need) st = FMM_ERR_OUT_OF_MEMORY;
      if (st == FMM_OK && !ensure_slot_buffers(sl, sl.prog.desc.size() + 64)) st = FMM_ERR_OUT_OF_MEMORY;
      if (st == FMM_OK) {
        std::memcpy(sl.h_desc, sl.prog.desc.data(), sl.prog.desc.size());
        int64_t n = 0;
        *sl.h_err = 0;
        cudaError_t e = cudaMemsetAsync(sl.d_err, 0, sizeof(int), sl.stream);
        if (e == cudaSuccess)
          e = fmm::run_program(sl.prog, sl.h_desc, sl.d_desc, s->h->num_sms, sl.stream, &n, nullptr, sl.d_err);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.h_err, sl.d_err, sizeof(int), cudaMemcpyDeviceToHost, sl.stream);
        if (e != cudaSuccess) st = FMM_ERR_CUDA;
        s->stats.launches += n;
      }
    }
    if (st != FMM_OK || cudaEventRecord(sl.done, sl.stream) != cudaSuccess) {
      for (uint64_t t : tickets) finish(s, t, st == FMM_OK ? FMM_ERR_CUDA : st);
      pool_free(s, off, need);
      continue;
    }
    sl.busy = true;
    sl.tickets = tickets;
    sl.ws_off = off;
    sl.ws_size = need;
    s->stats.batches++;
    if ((int64_t)tickets.size() > s->stats.max_batch_seen) s->stats.max_batch_seen = (int64_t)tickets.size();
    progressed = true;
  }
  return progressed;
}

void worker_main(fmm_server s) {
  cudaSetDevice(s->h->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    const bool progressed = turn(s);
    bool idle = true;
    for (const Slot& sl : s->slots) idle = idle && !sl.busy;
    if (s->stop && idle) break;
    if (!progressed) s->cv_work.wait_for(lk, std::chrono::microseconds(20));
  }
  for (const Pending& p : s->pending) finish(s, p.ticket, FMM_ERR_TIMEOUT);
  s->pending.clear();
  s->cv_done.notify_all();
}

}  // namespace

extern "C" {

fmm_status fmm_server_create(const fmm_server_config* cfg, fmm_server* out) {
  if (!cfg || !out) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  fmm_handle h = nullptr;
  fmm_status st = fmm_handle_create(&h, cfg->device);
  if (st != FMM_OK) return st;
  DeviceGuard g(cfg->device);
  fmm_server s = new fmm_server_s();
  s->h = h;
  s->max_batch = cfg->max_batch > 0 ? cfg->max_batch : 64;
  size_t bytes = cfg->workspace_bytes;
  if (bytes == 0) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    bytes = (size_t)(0.4 * (double)free_b);
  }
  if (cudaMalloc(&s->pool, bytes) != cudaSuccess) {
    cudaGetLastError();
    fmm_handle_destroy(h);
    delete s;
    return fail(FMM_ERR_OUT_OF_MEMORY, "cannot allocate the server's workspace pool");
  }
  s->pool_size = bytes;
  s->free_blocks[0] = bytes;
  const int nslots = cfg->max_inflight > 0 ? cfg->max_inflight : 4;
  s->slots.resize((size_t)nslots);
  for (Slot& sl : s->slots) {
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess || !ensure_slot_buffers(sl, 1 << 20) ||
        cudaMalloc(&sl.d_err, 256) != cudaSuccess || cudaMallocHost(&sl.h_err, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      s->stop = true;
      fmm_server_destroy(s);
      return fail(FMM_ERR_CUDA, "cannot create the server's streams");
    }
  }
  s->worker = std::thread(worker_main, s);
  *out = s;
  return FMM_OK;
}

fmm_status fmm_server_submit(fmm_server s, const fmm_request* req, uint64_t* ticket) {
  if (!s || !req) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return fail(FMM_ERR_INVALID_ARGUMENT, "server is stopping");
  const uint64_t t = s->next_ticket++;
  fmm_request_info inf{};
  inf.submit_ms = s->now_ms();
  s->info[t] = inf;
  s->pending.push_back(Pending{*req, t});
  s->stats.submitted++;
  if (ticket) *ticket = t;
  s->cv_work.notify_one();
  return FMM_OK;
}

fmm_status fmm_server_wait(fmm_server s, uint64_t ticket, double timeout_ms, fmm_request_info* info) {
  if (!s) return fail(FMM_ERR_INVALID_ARGUMENT, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->info.find(ticket);
  if (it == s->info.end()) return fail(FMM_ERR_INVALID_ARGUMENT, "unknown ticket");
  auto ready = [&] { return s->info[ticket].done != 0; };
  if (timeout_ms < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready))
    return fail(FMM_ERR_TIMEOUT, "request not done within the timeout");
  if (info) *info = s->info[ticket];
  return FMM_OK;
}

fmm_status fmm_server_drain(fmm_server s, double timeout_ms) {
  if (!s) return fail(FMM_ERR_INVALID_ARGUMENT, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto ready = [&] { return s->stats.completed == s->stats.submitted; };
  if (timeout_ms < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready))
    return fail(FMM_ERR_TIMEOUT, "requests still pending after the timeout");
  return FMM_OK;
}

fmm_status fmm_server_get_stats(fmm_server s, fmm_server_stats* out) {
  if (!s || !out) return fail(FMM_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return FMM_OK;
}

fmm_status fmm_server_destroy(fmm_server s) {
  if (!s) return FMM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  DeviceGuard g(s->h->device);
  for (Slot& sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.h_desc) cudaFreeHost(sl.h_desc);
    if (sl.d_desc) cudaFree(sl.d_desc);
    if (sl.d_err) cudaFree(sl.d_err);
    if (sl.h_err) cudaFreeHost(sl.h_err);
  }
  if (s->pool) cudaFree(s->pool);
  fmm_handle_destroy(s->h);
  delete s;
  return FMM_OK;
}

}  // extern "C"
