// Runs a planned launch program on a stream (kept apart from the planner so
// the planner also builds for host-only checking).

#include "plan.h"

namespace fmm {

cudaEvent_t Profiler::get() {
  if (used == pool.size()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    pool.push_back(e);
  }
  return pool[used++];
}

void Profiler::reset() {
  recs.clear();
  used = 0;
}

Profiler::~Profiler() {
  for (cudaEvent_t e : pool) cudaEventDestroy(e);
}

cudaError_t run_program(const Program& prog, const void* h_desc, void* d_desc, int num_sms, cudaStream_t stream,
                        int64_t* launches, Profiler* prof, int* d_err, cudaEvent_t desc_copied) {
  if (device_checks_built()) {
    // debug builds: register the program's workspace for the kernels'
    // checks (not while a graph is captured: the range would be read at
    // every replay from a host buffer the next program reuses)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
      cudaError_t e = device_checks_arm(prog.ws_base, prog.workspace_bytes, stream);
      if (e != cudaSuccess) return e;
    }
  }
  if (!prog.desc.empty()) {
    cudaError_t e = cudaMemcpyAsync(d_desc, h_desc, prog.desc.size(), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    if (desc_copied && (e = cudaEventRecord(desc_copied, stream)) != cudaSuccess) return e;
  }
  const unsigned char* base = static_cast<const unsigned char*>(d_desc);
  int64_t count = 0;
  for (const Op& op : prog.ops) {
    cudaError_t e = cudaSuccess;
    Profiler::Rec rec{op.kind, op.peel, op.flops, op.bytes, nullptr, nullptr};
    if (prof) {
      rec.start = prof->get();
      rec.stop = prof->get();
      if (!rec.start || !rec.stop) return cudaErrorMemoryAllocation;
      cudaEventRecord(rec.start, stream);
    }
    switch (op.kind) {
      case OpKind::kForm: {
        FormLaunch L;
        L.s_desc = reinterpret_cast<const FormDesc*>(base + op.desc_off);
        L.t_desc = L.s_desc + op.n_s;
        L.n_s = op.n_s;
        L.n_t = op.n_t;
        L.max_items = op.max_items;
        e = form_launch(op.alg, L, prog.coefs[(size_t)op.cf], op.vec2, num_sms, stream);
        break;
      }
      case OpKind::kGemm:
        e = gemm_launch(reinterpret_cast<const GemmDesc*>(base + op.desc_off), op.n, op.total_tiles, num_sms,
                        stream, op.gemm_tile);
        break;
      case OpKind::kSplitGemm: {
        int64_t n_launched = 0;
        if (prof) {
          rec.mid = prof->get();
          if (!rec.mid) return cudaErrorMemoryAllocation;
          const double products = op.split.slices * (op.split.slices + 1) / 2.0;
          rec.bf16_flops = op.flops * products;
        }
        e = split_gemm_launch(reinterpret_cast<const SplitDesc*>(base + op.desc_off), op.n, op.split,
                              prog.split_scratch, d_err, num_sms, stream, &n_launched, rec.mid);
        count += n_launched - 1;  // the op itself is counted below
        break;
      }
      case OpKind::kCombine: {
        CombineLaunch L;
        L.desc = reinterpret_cast<const CombineDesc*>(base + op.desc_off);
        L.n = op.n;
        L.max_items = op.max_items;
        e = combine_launch(op.alg, L, prog.coefs[(size_t)op.cf], op.vec2, num_sms, stream);
        break;
      }
    }
    if (e != cudaSuccess) return e;
    if (prof) {
      cudaEventRecord(rec.stop, stream);
      prof->recs.push_back(rec);
    }
    ++count;
  }
  if (launches) *launches += count;
  return cudaSuccess;
}

}  // namespace fmm
