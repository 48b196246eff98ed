#!/usr/bin/env python
"""Benchmark: effective TFLOP/s (2MNK/t) of a fast algorithm vs classical GEMM on B200.

Default workload: fast424_26_206 (<4,2,4;26> with common-subexpression
elimination, namespace grey424_26_206), 16384 x 16384 x 16384, 2 recursive
steps, FP64, seeded uniform [0, 1) inputs (A: stream 1, B: stream 2), alpha 1,
beta 0.  One step = one FastMatmul of the whole product.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (launched by torch.distributed.run): independent replicas, one per GPU
(the product does not shard across GPUs); the only collectives are the
barrier and the max over ranks of the timed region.

Reported beside the headline: the engine's own classical FP64 GEMM and
cuBLAS DGEMM on the same matrices, the error of the result against the
classical product, per-phase kernel times with their roofline, an end-to-end
number through the host-memory C entry point, clocks sampled during the
timed region, and the reference's CPU path on a bounded sample.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "effective TFLOP/s (2MNK/t) fast vs classical GEMM, same B200, at stated error"
NOMINAL_FP64_TFLOPS = 40.0


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--alg", default="grey424_26_206")
    ap.add_argument("--num-steps", type=int, default=2)
    ap.add_argument("--m", type=int, default=16384)
    ap.add_argument("--k", type=int, default=16384)
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--schedule", default="auto", choices=["auto", "dfs", "bfs", "hybrid"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the precision, batch and serve sub-records of the headline line")
    ap.add_argument("--cpu-sample", type=int, default=4096, help="edge of the CPU baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU work budget of the baseline sample")
    ap.add_argument("--workload", default="product",
                    choices=["product", "batch", "serve", "precision", "scaling", "fp32", "int8", "profile"],
                    help="product: one large FastMatmul (the headline); batch: 4096 independent products "
                         "with log-uniform dimensions in [64, 1024] in one CUDA-graph plan; serve: a Poisson "
                         "request stream through the continuous-batching server; precision: split-BF16 leaf "
                         "products (Strassen, Bini) against the FP64 oracle; scaling: diagonal scaling "
                         "(Scaling + FastMatmul + PostProcessScaling) on skewed operands; fp32: "
                         "FastMatmul<float> against cuBLAS SGEMM; int8: split-INT8 leaf products beside "
                         "split-BF16 and FP64; profile: one product configuration (--alg or classical, --m/--k/--n, "
                         "--num-steps, --precision, --split-slices) called --steps times untimed, as a profiler "
                         "target (each call launches the same kernels, so a capture skips the first call's "
                         "launches with ncu -s)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split_bf16", "split_int8"],
                    help="leaf products of the profile workload")
    ap.add_argument("--split-slices", type=int, default=5, help="slices of the profile workload's split leaves")
    ap.add_argument("--fp32-size", type=int, default=16384, help="square size of the fp32 workload")
    ap.add_argument("--int8-size", type=int, default=16384, help="square size of the int8 workload")
    ap.add_argument("--scaling-size", type=int, default=16384, help="square size of the scaling workload")
    ap.add_argument("--precision-sizes", default="8192,16384",
                    help="square sizes of the precision workload")
    ap.add_argument("--batch-precision", default="fp64", choices=["fp64", "split_bf16", "split_int8"])
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--batch-tile", default="auto", choices=["auto", "large", "small"],
                    help="FP64 GEMM tile configuration of the batch items (auto: the autotuned one per bucket)")
    ap.add_argument("--serve-requests", type=int, default=300)
    ap.add_argument("--serve-slots", type=int, default=6)
    ap.add_argument("--sweep", action="store_true",
                    help="time every configuration of the fast-vs-classical study (one JSON line each) "
                         "instead of the single headline line")
    a = ap.parse_args(argv)
    if a.warmup < 3 and a.impl == "ours":
        a.warmup = 3
    return a


def workload_name(a):
    return "%s %dx%dx%d, %d recursive steps, FP64, uniform[0,1)" % (a.alg, a.m, a.k, a.n, a.num_steps)


# ---------------------------------------------------------------------------
# reference CPU path (the oracle/_ref build of the reference's own headers)


def cpu_reference_sample(alg, num_steps, edge, seconds, max_runs=None):
    """Times the reference's FastMatmul on an edge^3 sample with all host
    threads; returns (median ms, runs, threads)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # the CPU baseline leg may load the reference build

    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libfmm_ref.so is not built")
    threads = os.cpu_count() or 1
    oracle.ref_lib().fmmref_set_threads(threads)
    A = oracle.uniform(edge, edge, 7, 1)
    B = oracle.uniform(edge, edge, 7, 2)
    C = oracle.uniform(edge, edge, 7, 3)
    times = []
    t_end = time.time() + seconds
    oracle.ref_fast_matmul(alg, A, B, C, num_steps)  # warm (page faults, thread pool)
    while time.time() < t_end or len(times) < 2:
        t0 = time.perf_counter()
        oracle.ref_fast_matmul(alg, A, B, C, num_steps)
        times.append((time.perf_counter() - t0) * 1e3)
        if max_runs and len(times) >= max_runs:
            break
    return statistics.median(times), len(times), threads


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    edge = a.cpu_sample
    sample = "%s %d^3, %d recursive steps, uniform[0,1), median of timed runs" % (a.alg, edge, a.num_steps)
    flops = 2.0 * edge ** 3
    try:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle

        if not oracle.ref_available():
            raise RuntimeError("reference build oracle/_ref is missing")
        threads = os.cpu_count() or 1
        oracle.ref_lib().fmmref_set_threads(threads)
        A = oracle.uniform(edge, edge, 7, 1)
        B = oracle.uniform(edge, edge, 7, 2)
        C = oracle.uniform(edge, edge, 7, 3)
        for _ in range(a.warmup):
            oracle.ref_fast_matmul(a.alg, A, B, C, a.num_steps)
        times = []
        for _ in range(a.steps):
            t0 = time.perf_counter()
            oracle.ref_fast_matmul(a.alg, A, B, C, a.num_steps)
            times.append((time.perf_counter() - t0) * 1e3)
    except Exception as ex:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": str(ex)}))
        return 0
    ms = sum(times) / len(times)
    value = flops / (ms * 1e-3) / 1e12
    out = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(a), "sample": sample, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------------------
# clocks


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        # samples under load: the upper part of the distribution (the
        # sampler also sees the idle moments around the region)
        busy = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our engine


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return json.load(fh), "measured"
    except Exception:  # noqa: BLE001
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def committed_traffic(name="roofline_traffic.json"):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary."""
    path = os.path.join(REPO, "profiles", name)
    try:
        with open(path) as fh:
            return json.load(fh)
    except Exception:  # noqa: BLE001
        return None


class Replicas:
    """N independent replicas, one process per GPU (torch.distributed.run):
    the only collectives are a barrier around the timed region and the
    maximum over ranks of a measured time.  `backend` is "nccl" on GPUs
    ("gloo" lets the same logic run on host processes); with WORLD_SIZE 1
    nothing is initialised.  Every rank calls the same methods in the same
    order."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 600.0):
        import datetime

        import torch
        import torch.distributed as dist

        self.dist = dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device if device is not None else torch.device("cpu")
        if self.world > 1:
            kw = {"device_id": self.device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)

    def barrier(self) -> None:
        if self.world > 1:
            self.dist.barrier()

    def max(self, value: float) -> float:
        """The maximum of `value` over the ranks (every rank gets it)."""
        import torch

        t = torch.tensor([value], dtype=torch.float64, device=self.device)
        if self.world > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def whole_job_rate(self, units_per_rank: float, seconds_max: float) -> float:
        """Units all ranks processed per second of the slowest rank."""
        return self.world * units_per_rank / seconds_max

    def close(self) -> None:
        if self.world > 1:
            self.barrier()
            self.dist.destroy_process_group()


def reference_digest_diff(alg, m, k, n, steps, seed, C):
    """Max relative difference of C from the reference's own result for this
    product, over the committed digest of that result (sampled entries, fringe
    rows and columns included, and band sums; tests/golden/reference_baseline.json,
    written by tests/golden/make_reference_digests.py), or None without one."""
    gold = os.path.join(REPO, "tests", "golden")
    path = os.path.join(gold, "reference_baseline.json")
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        cases = json.load(fh)["cases"]
    hit = [c for c in cases if (c["alg"], c["m"], c["k"], c["n"], c["steps"], c["seed"]) == (alg, m, k, n, steps, seed)]
    if not hit:
        return None
    c = hit[0]
    sys.path.insert(0, gold)
    import digest as dg

    import fast_matmul_b200 as fmm

    info = fmm.algorithm_info(alg)
    rows, cols = dg.positions(m, n, info["m0"], info["n0"], steps, c["samples_count"], seed)
    got = dg.digest_torch(C, rows, cols, c["groups"])
    diff = dg.rel_diffs({key: dg.dec(c[key]) for key in ("samples", "rowsum", "colsum")}, got)
    return {"max": diff["max"], "sampled_entries": diff["samples"], "row_band_sums": diff["rowsum"],
            "column_band_sums": diff["colsum"], "entries": c["samples_count"], "bands": c["groups"],
            "reference_max_rel_diff_vs_its_classical": c["ref_err"],
            "source": "digest of the reference's own FastMatmul result on the same seeded inputs "
                      "(tests/golden/reference_baseline.json)"}


def precision_record(a, fmm, h, A, B, ref, classical_tf, cublas_tf, slices=5, steps=2):
    """The split-BF16 precision target on the headline's operands: Strassen
    with `steps` steps, leaf products split into `slices` BF16 slices (FP64 in
    and out), timed with CUDA events (3 calls after one warm-up, clocks
    sampled meanwhile), its error against the engine's FP64 classical product
    `ref` of the same inputs, and the ratios to the engine's DGEMM and to
    cuBLAS DGEMM measured in the same run."""
    import torch

    m, k = A.shape
    n = B.shape[1]
    flops = 2.0 * m * n * k
    C = fmm.colmajor_empty(m, n, A.device)

    def call():
        fmm.fast_matmul("strassen", A, B, C, steps, precision="split_bf16", split_slices=slices, handle=h)

    call()
    torch.cuda.synchronize()
    reps = 3
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.2)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        call()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / reps
    h.profile(True)
    h.profile_reset()
    call()
    prof = h.profile_read()
    h.profile(False)
    fmm.synchronize(h)
    rel, absd = fmm.max_relative_diff(ref, C, handle=h)
    ex_rel, ex_scaled = exact_sample_errors(A, B, C, count=16)
    leaf_ms = prof["gemm_ms"] - prof["split_ms"]
    tf = flops / (ms * 1e-3) / 1e12
    peaks, peak_src = measured_peaks()
    pk = peaks.get("bf16_tflops_sustained", 1400.0)
    prod_tf = prof["split_bf16_flops"] / (leaf_ms * 1e-3) / 1e12 if leaf_ms > 0 else None
    del C
    return {
        "workload": "strassen %dx%dx%d, %d recursive steps, split-BF16 leaf products (%d slices), FP64 in and out, "
                    "uniform[0,1) (the headline's operands)" % (m, k, n, steps, slices),
        "value": tf, "unit": "TFLOP/s", "ms_per_call": ms, "calls": reps,
        "error": {"max_rel_elementwise_vs_fp64_classical": rel,
                  "max_rel_normwise_vs_fp64_classical": absd / float(ref.abs().max()),
                  "max_rel_vs_exact_16_sampled_entries": ex_rel,
                  "max_vs_exact_over_absAB_16_sampled_entries": ex_scaled, "target": 1e-12},
        "speedup_vs_engine_dgemm": tf / classical_tf, "speedup_vs_cublas_dgemm": tf / cublas_tf,
        "phases_ms": {"splitting": prof["split_ms"], "slice_products": leaf_ms, "form": prof["form_ms"],
                      "combine": prof["combine_ms"], "peel": prof["peel_ms"]},
        "roofline": {"kernel": "split_gemm_kernel (tcgen05 BF16 slice products)", "bound": "tensor",
                     "achieved": prod_tf, "peak": pk, "unit": "TFLOP/s", "frac": prod_tf / pk if prod_tf else None,
                     "peak_source": "bf16_tflops_sustained (%s)" % peak_src},
        "clocks": clk,
    }


def run_ours(a):
    import torch

    import fast_matmul_b200 as fmm

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rep = Replicas("nccl", torch.device("cuda", local))
    world, rank = rep.world, rep.rank
    barrier = rep.barrier

    m, k, n = a.m, a.k, a.n
    h = fmm.default_handle(local)
    A = fmm.random_matrix(m, k, 1234 + rank, 1, device=local)
    B = fmm.random_matrix(k, n, 1234 + rank, 2, device=local)
    C = fmm.colmajor_empty(m, n, torch.device("cuda", local))
    flops = 2.0 * m * n * k

    def step():
        fmm.fast_matmul(a.alg, A, B, C, a.num_steps, schedule=a.schedule, handle=h)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    h.profile(True)
    h.profile_reset()
    launches0 = h.launches()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(a.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    elapsed_ms = ev0.elapsed_time(ev1)
    launches = h.launches() - launches0
    prof = h.profile_read()
    h.profile(False)
    clk = clocks.stop()

    t_max = rep.max(elapsed_ms)
    ms_step = t_max / a.steps
    value = rep.whole_job_rate(flops * a.steps, t_max * 1e-3) / 1e12

    # ---- classical comparators and error (outside the timed region)
    Cc = fmm.colmajor_empty(m, n, torch.device("cuda", local))
    fmm.matmul(A, B, Cc, handle=h)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 2
    e0.record()
    for _ in range(reps):
        fmm.matmul(A, B, Cc, handle=h)
    e1.record()
    torch.cuda.synchronize()
    classical_tf = flops * reps / (e0.elapsed_time(e1) * 1e-3) / 1e12
    rel, absd = fmm.max_relative_diff(Cc, C, handle=h)
    ex_rel, ex_scaled = exact_sample_errors(A, B, C, count=32)
    Ct = torch.matmul(A, B)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        torch.matmul(A, B, out=Ct)
    e1.record()
    torch.cuda.synchronize()
    cublas_tf = flops * reps / (e0.elapsed_time(e1) * 1e-3) / 1e12
    Ct_cm = fmm.colmajor_empty(m, n, torch.device("cuda", local))
    Ct_cm.copy_(Ct)
    rel_cublas, _ = fmm.max_relative_diff(Ct_cm, C, handle=h)
    del Ct_cm
    del Ct
    vs_ref = reference_digest_diff(a.alg, m, k, n, a.num_steps, 1234 + rank, C) if world == 1 else None

    # ---- end to end through the host-memory C entry points: every step copies
    # its A and B from pinned host memory to the device and its C back.  The
    # pipelined entry point (fmm_fast_matmul_host_async) overlaps one step's
    # copies with the neighbouring steps' products; the synchronous one
    # (fmm_fast_matmul_host) runs them strictly one after the other.
    e2e = None
    if not a.no_e2e:
        Ah = torch.empty((k, m), dtype=torch.float64, pin_memory=True).t()
        Bh = torch.empty((n, k), dtype=torch.float64, pin_memory=True).t()
        Ch = torch.empty((n, m), dtype=torch.float64, pin_memory=True).t()
        Ah.copy_(A)
        Bh.copy_(B)
        fmm.fast_matmul_host(a.alg, Ah, Bh, Ch, a.num_steps, schedule=a.schedule, handle=h)  # warm
        for _ in range(2):
            fmm.fast_matmul_host_async(a.alg, Ah, Bh, Ch, a.num_steps, schedule=a.schedule, handle=h)
        fmm.host_sync(h)
        e2e_steps = max(3, a.steps)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            fmm.fast_matmul_host_async(a.alg, Ah, Bh, Ch, a.num_steps, schedule=a.schedule, handle=h)
        fmm.host_sync(h)
        e2e_s = rep.max(time.perf_counter() - t0)
        e2e_ok = bool(torch.equal(Ch.to(C.device), C))
        sync_steps = max(2, min(a.steps, 3))
        barrier()
        t0 = time.perf_counter()
        for _ in range(sync_steps):
            fmm.fast_matmul_host(a.alg, Ah, Bh, Ch, a.num_steps, schedule=a.schedule, handle=h)
        sync_s = rep.max(time.perf_counter() - t0)
        e2e = {"value": rep.whole_job_rate(flops * e2e_steps, e2e_s) / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": 8 * (m * k + k * n), "d2h_bytes_per_step": 8 * m * n,
               "ms_per_step": e2e_s * 1e3 / e2e_steps, "steps": e2e_steps,
               "api": "fmm_fast_matmul_host_async + fmm_host_sync (include/fmm.h), pinned host buffers",
               "result_equals_device_call": e2e_ok,
               "one_call_at_a_time": {"value": rep.whole_job_rate(flops * sync_steps, sync_s) / 1e12,
                                      "ms_per_step": sync_s * 1e3 / sync_steps, "steps": sync_steps,
                                      "api": "fmm_fast_matmul_host (include/fmm.h)"}}
        del Ah, Bh, Ch

    # ---- roofline of the dominant kernel (grouped leaf FP64 GEMM)
    peaks, peak_src = measured_peaks()
    gemm_launches = max(prof["gemm_launches"], 1)
    gemm_tf = prof["gemm_flops"] / (prof["gemm_ms"] * 1e-3) / 1e12 if prof["gemm_ms"] else 0.0
    traffic = committed_traffic()
    roofline = {
        "kernel": "grouped_dgemm_kernel (leaf products)",
        "bound": "tensor", "achieved": gemm_tf, "peak": cublas_tf, "unit": "TFLOP/s",
        "frac": gemm_tf / cublas_tf if cublas_tf else None,
        "peak_source": "cuBLAS DGEMM %dx%dx%d measured in this run (no FP64 figure in MEASURED_PEAKS.json); "
                       "nominal B200 FP64 %.0f TFLOP/s" % (m, k, n, NOMINAL_FP64_TFLOPS),
        "frac_of_nominal": gemm_tf / NOMINAL_FP64_TFLOPS,
        "flops_per_launch": prof["gemm_flops"] / gemm_launches,
        "ms_per_launch": prof["gemm_ms"] / gemm_launches,
        "traffic": (traffic or {}).get("bytes_per_launch"),
        "traffic_source": (traffic or {}).get("source"),
    }
    hbm = peaks.get("hbm_gbs", 6650.0)
    phases = {
        "form": {"launches": prof["form_launches"], "ms": prof["form_ms"],
                 "GB/s": prof["form_bytes"] / (prof["form_ms"] * 1e-3) / 1e9 if prof["form_ms"] else None},
        "combine": {"launches": prof["combine_launches"], "ms": prof["combine_ms"],
                    "GB/s": prof["combine_bytes"] / (prof["combine_ms"] * 1e-3) / 1e9 if prof["combine_ms"] else None},
        "leaf_gemm": {"launches": prof["gemm_launches"], "ms": prof["gemm_ms"], "TFLOP/s": gemm_tf},
        "peel_gemm": {"launches": prof["peel_launches"], "ms": prof["peel_ms"]},
        "hbm_peak_gbs": hbm, "hbm_peak_source": peak_src,
    }

    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not a.no_cpu_baseline:
            try:
                ms_cpu, runs, threads = cpu_reference_sample(a.alg, a.num_steps, a.cpu_sample, a.cpu_seconds)
                cpu = {"value": 2.0 * a.cpu_sample ** 3 / (ms_cpu * 1e-3) / 1e12, "unit": "TFLOP/s",
                       "cores": threads, "kind": "reference",
                       "sample": "%s %d^3, %d recursive steps, median of %d runs, host BLAS with %d threads"
                                 % (a.alg, a.cpu_sample, a.num_steps, runs, threads)}
            except Exception as ex:  # noqa: BLE001
                cpu = {"value": None, "unit": "TFLOP/s", "cores": None, "kind": "reference",
                       "sample": "unavailable: %s" % ex}
        info = fmm.algorithm_info(a.alg)
        out = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(a), "algorithm": info["name"],
                       "base_case": "<%d,%d,%d;%d>" % (info["m0"], info["k0"], info["n0"], info["rank"]),
                       "m": m, "k": k, "n": n, "num_steps": a.num_steps, "schedule": a.schedule,
                       "precision": "fp64", "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (each operand %.1f GiB > 126 MB)" % (8.0 * m * k / 2**30)},
            "error": {"max_rel_diff_vs_reference": vs_ref["max"] if vs_ref else None,
                      "vs_reference": vs_ref,
                      "max_rel_diff_vs_classical": rel, "max_abs_diff_vs_classical": absd,
                      "max_rel_diff_vs_cublas": rel_cublas,
                      "max_rel_vs_exact_32_sampled_entries": ex_rel,
                      "max_vs_exact_over_absAB_32_sampled_entries": ex_scaled},
            "classical": {"engine_dgemm_tflops": classical_tf, "cublas_dgemm_tflops": cublas_tf,
                          "speedup_vs_engine_classical": value / world / classical_tf,
                          "speedup_vs_cublas": value / world / cublas_tf},
            "roofline": roofline,
            "phases": phases,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": launches,
            "workspace_bytes": fmm.workspace_bytes(a.alg, m, k, n, a.num_steps, a.schedule, handle=h),
        }
        if world == 1 and not a.no_extras:
            # the precision, batch and serving records, each with its own clock record
            out["precision"] = precision_record(a, fmm, h, A, B, Cc, classical_tf, cublas_tf)
            del A, B, C, Cc
            h.release_workspace()
            torch.cuda.empty_cache()
            out["batch"] = {"fp64": batch_record(a, "fp64"), "split_bf16": batch_record(a, "split_bf16")}
            out["serve"] = serve_record(a)
        print(json.dumps(out))
    rep.close()
    return 0


# ---------------------------------------------------------------------------
# sweep over the study's configurations


SWEEP_SHAPES = [
    ("square 4096^3", 4096, 4096, 4096, [("strassen", (1, 2))]),
    ("square 16384^3", 16384, 16384, 16384,
     [("strassen", (1, 2, 3)), ("grey424_26_206", (1, 2, 3)), ("grey333_23_125", (1, 2, 3)),
      ("smirnov333_23_128", (1, 2, 3))]),
    ("outer-product-like 16384x1600x16384", 16384, 1600, 16384,
     [("grey424_26_206", (1, 2, 3)), ("grey333_23_125", (1, 2, 3)), ("smirnov333_23_128", (1, 2, 3))]),
    ("tall-skinny 65536x2400x2400", 65536, 2400, 2400,
     [("grey424_26_206", (1, 2, 3)), ("grey333_23_125", (1, 2, 3)), ("smirnov333_23_128", (1, 2, 3))]),
]


def run_sweep(a):
    import torch

    import fast_matmul_b200 as fmm

    torch.cuda.set_device(0)
    h = fmm.default_handle(0)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    for label, m, k, n, algs in SWEEP_SHAPES:
        A = fmm.random_matrix(m, k, 11, 1)
        B = fmm.random_matrix(k, n, 11, 2)
        C = fmm.colmajor_empty(m, n)
        Cc = fmm.colmajor_empty(m, n)
        flops = 2.0 * m * n * k
        ms_cls = timed(lambda: fmm.matmul(A, B, Cc, handle=h), 2)
        Ct = torch.matmul(A, B)
        ms_cub = timed(lambda: torch.matmul(A, B, out=Ct), 2)
        del Ct
        print(json.dumps({"sweep": label, "alg": "classical", "engine_dgemm_tflops": flops / ms_cls / 1e9,
                          "cublas_dgemm_tflops": flops / ms_cub / 1e9}), flush=True)
        for alg, steps_list in algs:
            for steps in steps_list:
                for sched in ("bfs", "hybrid", "dfs"):
                    if sched == "hybrid" and steps < 3:
                        continue
                    rec = {"sweep": label, "alg": alg, "num_steps": steps, "schedule": sched}
                    try:
                        ws = fmm.workspace_bytes(alg, m, k, n, steps, sched, handle=h)
                        ms = timed(lambda: fmm.fast_matmul(alg, A, B, C, steps, schedule=sched, handle=h), 2)
                        rel, _ = fmm.max_relative_diff(Cc, C, handle=h)
                        rec.update({"tflops_effective": flops / ms / 1e9, "ms": ms,
                                    "speedup_vs_engine_classical": ms_cls / ms, "speedup_vs_cublas": ms_cub / ms,
                                    "max_rel_diff_vs_classical": rel, "workspace_gib": ws / 2**30})
                    except fmm.FmmError as ex:
                        rec["skipped"] = str(ex)[:160]
                    print(json.dumps(rec), flush=True)
        del A, B, C, Cc
        torch.cuda.empty_cache()
    return 0


def run_batch_workload(a):
    """4096 independent products, M, K, N each floor(exp(U(ln 64, ln 1024))) from
    a seed, entries uniform [-1, 1); the autotuner picks algorithm and depth
    per shape bucket; the whole batch is one CUDA-graph plan (all leaf
    products in one persistent grouped GEMM launch).  Compared with the same
    products launched one call at a time."""
    import torch

    torch.cuda.set_device(0)
    print(json.dumps(batch_record(a, a.batch_precision)))
    return 0


def batch_record(a, precision):
    """The batch workload's JSON record for leaf products of `precision`."""
    import numpy as np
    import torch

    import fast_matmul_b200 as fmm

    h = fmm.default_handle(torch.cuda.current_device())
    rng = np.random.default_rng(2024)
    dims = np.floor(np.exp(rng.uniform(np.log(64), np.log(1024), size=(a.batch_count, 3)))).astype(int)
    probs = []
    for i, (m, k, n) in enumerate(dims):
        probs.append({"A": fmm.random_matrix(int(m), int(k), 7000 + i, 1, -1.0, 1.0, handle=h),
                      "B": fmm.random_matrix(int(k), int(n), 7000 + i, 2, -1.0, 1.0, handle=h),
                      "C": fmm.colmajor_empty(int(m), int(n)), "alg": fmm.AUTO,
                      "precision": precision, "split_slices": 6, "gemm_tile": a.batch_tile})
    flops = float(sum(2.0 * m * n * k for m, k, n in dims))
    t0 = time.perf_counter()
    fmm.autotune([tuple(int(v) for v in d) for d in dims], max_steps=1, handle=h)
    tune_s = time.perf_counter() - t0
    choices = {}
    tiles = {}
    for m, k, n in dims:
        c = fmm.autotune_choice(int(m), int(k), int(n), handle=h)
        choices[c] = choices.get(c, 0) + 1
        t = a.batch_tile if a.batch_tile != "auto" else fmm.autotune_tile(int(m), int(k), int(n), handle=h)
        tiles[t] = tiles.get(t, 0) + 1
    plan = fmm.Plan.for_batch(probs, handle=h)

    def timed(fn, reps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    for _ in range(a.warmup):
        plan.execute()
    launches0 = h.launches()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ms = timed(plan.execute, a.steps)
    clk = clocks.stop()
    launches = (h.launches() - launches0) // max(a.steps, 1)

    def one_at_a_time():
        for p, (m, k, n) in zip(probs, dims):
            alg, steps = fmm.autotune_choice(int(m), int(k), int(n), handle=h)
            if alg == fmm.CLASSICAL:
                if precision == "split_bf16":
                    fmm.matmul_split_bf16(p["A"], p["B"], p["C"], slices=6, handle=h)
                elif precision == "split_int8":
                    fmm.matmul_split_int8(p["A"], p["B"], p["C"], slices=6, handle=h)
                else:
                    fmm.matmul(p["A"], p["B"], p["C"], handle=h)
            else:
                fmm.fast_matmul(alg, p["A"], p["B"], p["C"], steps, precision=precision, split_slices=6,
                                handle=h)

    one_at_a_time()
    ms_single = timed(one_at_a_time, 1)
    out = {
        "metric": METRIC, "value": flops / (ms * 1e-3) / 1e12, "unit": "TFLOP/s", "n_gpus": 1, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp64": "f64", "split_bf16": "bf16 slices (FP64 in and out)",
                  "split_int8": "int8 slices (FP64 in and out)"}[precision], "data": "synthetic",
        "config": {"workload": "batch of %d independent %s products, M,K,N log-uniform in [64,1024], "
                               "uniform[-1,1), autotuned per shape bucket, one CUDA-graph plan"
                               % (a.batch_count, {"fp64": "FP64", "split_bf16": "split-BF16 (6 slices)",
                                                  "split_int8": "split-INT8 (6 slices)"}[precision]),
                   "total_gflop": flops / 1e9, "autotune_seconds": tune_s,
                   "choices": {("classical" if k[0] == fmm.CLASSICAL else "%s/%d" % (fmm.algorithm_names()[k[0]], k[1])): v
                               for k, v in choices.items()},
                   "gemm_tiles": tiles, "batch_tile": a.batch_tile},
        "one_at_a_time": {"value": flops / (ms_single * 1e-3) / 1e12, "ms": ms_single,
                          "speedup_of_batched": ms_single / ms},
        "clocks": clk,
        "gpu_launches": launches,
    }
    plan.close()
    return out


def run_serve_workload(a):
    """Poisson stream of products (70% FP64, 30% split-BF16 with 6 slices),
    M, K, N each log-uniform in [256, 8192], uniform [-1, 1) entries, operands
    resident in device memory, offered at
    twice the rate that one-at-a-time launches sustain; the server admits
    requests by workspace footprint into concurrent batches (--serve-slots).  Reports
    throughput, p50/p99 latency (submission to completion) and the
    one-at-a-time throughput on the same requests."""
    import torch

    torch.cuda.set_device(0)
    print(json.dumps(serve_record(a)))
    return 0


def serve_record(a):
    """The serving workload's JSON record (on the current device)."""
    import threading

    import numpy as np
    import torch

    import fast_matmul_b200 as fmm

    dev = torch.cuda.current_device()
    h = fmm.default_handle(dev)
    rng = np.random.default_rng(77)
    N = a.serve_requests
    dims = np.floor(np.exp(rng.uniform(np.log(256), np.log(8192), size=(N, 3)))).astype(int)
    split_share = 0.3
    wants_split = rng.uniform(size=N) < split_share
    reqs = []
    for i, (m, k, n) in enumerate(dims):
        reqs.append((fmm.random_matrix(int(m), int(k), 9000 + i, 1, -1.0, 1.0, handle=h),
                     fmm.random_matrix(int(k), int(n), 9000 + i, 2, -1.0, 1.0, handle=h),
                     fmm.colmajor_empty(int(m), int(n))))
    flops = float(sum(2.0 * m * n * k for m, k, n in dims))

    split_slices = 6  # the 1e-12 target of the split-BF16 share

    def alone(i):
        A, B, C = reqs[i]
        alg, steps = fmm.autotune_choice(*(int(v) for v in dims[i]), handle=h)
        if alg == fmm.CLASSICAL:
            if wants_split[i]:
                fmm.matmul_split_bf16(A, B, C, slices=split_slices, handle=h)
            else:
                fmm.matmul(A, B, C, handle=h)
        else:
            fmm.fast_matmul(alg, A, B, C, steps, precision="split_bf16" if wants_split[i] else "fp64",
                            split_slices=split_slices, handle=h)

    for i in range(min(N, 8)):  # warm
        alone(i)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(N):
        alone(i)
        torch.cuda.synchronize()
    t_single = time.perf_counter() - t0
    reference = [reqs[i][2].clone() for i in range(0, N, max(1, N // 16))]
    # one-at-a-time plain launches: the classical FP64 GEMM per request
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for A, B, C in reqs:
        fmm.matmul(A, B, C, handle=h)
        torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    for _, _, C in reqs:
        C.zero_()
    torch.cuda.synchronize()

    rate = 2.0 * N / t_single  # requests per second offered
    gaps = rng.exponential(1.0 / rate, size=N)
    srv = fmm.Server(dev, workspace_bytes=0, max_inflight=a.serve_slots, max_batch=64)
    tickets = [None] * N

    def client():
        t_next = time.perf_counter()
        for i in range(N):
            t_next += gaps[i]
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            A, B, C = reqs[i]
            tickets[i] = srv.submit(A, B, C, fmm.AUTO, precision="split_bf16" if wants_split[i] else "fp64",
                                    split_slices=split_slices)

    clocks = ClockSampler(dev)
    clocks.start()
    th = threading.Thread(target=client)
    th.start()
    th.join()
    srv.drain()
    clk = clocks.stop()
    infos = [srv.wait(t) for t in tickets]
    stats = srv.stats()
    srv.close()
    t_first = min(x["submit_ms"] for x in infos)
    t_last = max(x["done_ms"] for x in infos)
    t_serve = (t_last - t_first) * 1e-3
    lat = np.array([x["done_ms"] - x["submit_ms"] for x in infos])
    same = all(torch.equal(ref, reqs[i][2]) for ref, i in zip(reference, range(0, N, max(1, N // 16))))
    out = {
        "metric": METRIC, "value": flops / t_serve / 1e12, "unit": "TFLOP/s", "n_gpus": 1, "steps": N,
        "warmup": 8, "ms_per_step": t_serve * 1e3 / N, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "serving: %d Poisson requests, M,K,N log-uniform in [256,8192], uniform[-1,1), "
                               "offered at 2x the one-at-a-time rate (%.1f req/s), %.0f%% FP64 / %.0f%% split-BF16 "
                               "(%d slices)" % (N, rate, 100 - 100 * split_share, 100 * split_share, split_slices),
                   "total_tflop": flops / 1e12, "requests_split_bf16": int(wants_split.sum())},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max())},
        "one_at_a_time": {"value": flops / t_single / 1e12, "seconds": t_single,
                          "throughput_ratio_of_server": t_single / t_serve,
                          "what": "same algorithm and precision per request, one launch set + synchronize each"},
        "one_at_a_time_plain": {"value": flops / t_plain / 1e12, "seconds": t_plain,
                                "throughput_ratio_of_server": t_plain / t_serve,
                                "what": "classical FP64 GEMM per request, launch + synchronize each"},
        "server": stats,
        "results_identical_to_alone": bool(same),
        "clocks": clk,
        "gpu_launches": stats["launches"],
    }
    del reqs, reference
    torch.cuda.empty_cache()
    return out


def scaled_normal(m, n, seed, per, device):
    """Column-major m x n FP64 matrix: N(0, 1) entries times 2^e, e an integer
    uniform in [-16, 16] drawn per row (per="row") or per column."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    X = torch.randn((n, m), generator=g, device=device, dtype=torch.float64).t()
    cnt = m if per == "row" else n
    e = torch.randint(-16, 17, (cnt,), generator=g, device=device).to(torch.float64)
    s = torch.exp2(e)
    if per == "row":
        X.mul_(s[:, None])
    else:
        X.mul_(s[None, :])
    return X


def exact_sample_errors(A, B, C, count=32, seed=0):
    """Errors of C against the exact product on `count` sampled entries:
    (max |c - q| / |q|, max |c - q| / (|A||B|)_ij) with q the exact rational
    value of the dot product (every double is an integer times a power of two,
    so the sum is formed in Python integers over a common power-of-two
    denominator)."""
    from fractions import Fraction

    import numpy as np
    import torch

    m, k = A.shape
    n = B.shape[1]
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, m, count)
    cols = rng.integers(0, n, count)
    ri = torch.as_tensor(rows, device=A.device)
    ci = torch.as_tensor(cols, device=B.device)
    ar = A.index_select(0, ri).cpu().numpy()
    bc = B.index_select(1, ci).t().cpu().numpy()
    cv = C[ri, ci].cpu().numpy()
    worst_rel = worst_scaled = 0.0
    for s in range(count):
        nums, dens, anums = [], [], []
        for x, y in zip(ar[s].tolist(), bc[s].tolist()):
            nx, dx = x.as_integer_ratio()
            ny, dy = y.as_integer_ratio()
            nums.append(nx * ny)
            dens.append(dx * dy)
        den = max(dens)
        q_num = sum(nv * (den // dv) for nv, dv in zip(nums, dens))
        aq_num = sum(abs(nv) * (den // dv) for nv, dv in zip(nums, dens))
        diff = abs(Fraction(float(cv[s])) - Fraction(q_num, den))
        if q_num:
            worst_rel = max(worst_rel, float(diff / abs(Fraction(q_num, den))))
        if aq_num:
            worst_scaled = max(worst_scaled, float(diff / Fraction(aq_num, den)))
    return worst_rel, worst_scaled


def precision_errors(fmm, A, B, C, ref, absAB, h):
    """Errors of C against the FP64 classical product ref: elementwise
    max |C - D| / |D| (the reference's MaxRelativeDiff), normwise
    max |C - D| / max |D|, and max |C - D| / (|A| |B|)."""
    import torch

    rel, absd = fmm.max_relative_diff(ref, C, handle=h)
    norm = absd / float(ref.abs().max())
    d = (C - ref).abs_().div_(absAB.clamp_min(1e-300))
    scaled = float(d.max())
    del d
    ex_rel, ex_scaled = exact_sample_errors(A, B, C, count=16)
    return {"max_rel_elementwise": rel, "max_rel_normwise": norm, "max_abs_over_absAB": scaled,
            "max_rel_vs_exact_16_sampled_entries": ex_rel, "max_vs_exact_over_absAB_16_sampled_entries": ex_scaled}


def run_precision_workload(a):
    """Split-BF16 leaf products against the FP64 oracle.  For each size and
    input distribution (uniform [0, 1); N(0, 1) with per-row (A) / per-column
    (B) scales 2^U{-16..16}): Strassen with 2 and 3 steps and bini322 with
    lambda swept over 2^-10 .. 2^-26 (1 step), leaf products split into 3..6
    BF16 slices, each timed (CUDA events, inputs resident) and checked
    against the engine's FP64 classical product of the same inputs.  The
    headline is the fastest Strassen configuration at 16384^3 whose
    elementwise error on uniform inputs stays within 1e-12."""
    import numpy as np
    import torch

    import fast_matmul_b200 as fmm

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    h = fmm.default_handle(0)
    sizes = [int(x) for x in a.precision_sizes.split(",") if x]

    def timed(fn, reps=2):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    rows = []
    classical = {}
    head = None
    clocks = ClockSampler(0)
    clocks.start()
    for n in sizes:
        flops = 2.0 * n ** 3
        for dist in ("uniform[0,1)", "N(0,1)*2^U(-16,16)"):
            if dist.startswith("uniform"):
                A = fmm.random_matrix(n, n, 31, 1, handle=h)
                B = fmm.random_matrix(n, n, 31, 2, handle=h)
            else:
                A = scaled_normal(n, n, 41, "row", dev)
                B = scaled_normal(n, n, 42, "col", dev)
            ref = fmm.colmajor_empty(n, n, dev)
            ms = timed(lambda: fmm.matmul(A, B, ref, handle=h))
            if dist.startswith("uniform"):
                classical[n] = {"engine_dgemm_tflops": flops / (ms * 1e-3) / 1e12}
                Ct = torch.matmul(A, B)
                msb = timed(lambda: torch.matmul(A, B, out=Ct))
                classical[n]["cublas_dgemm_tflops"] = flops / (msb * 1e-3) / 1e12
                del Ct
            absAB = fmm.colmajor_empty(n, n, dev)
            fmm.matmul(A.abs(), B.abs(), absAB, handle=h)
            C = fmm.colmajor_empty(n, n, dev)
            runs = [("strassen", s, 1e-8, sl) for s in (2, 3) for sl in (4, 5, 6)]
            runs += [("fp64 strassen", s, 1e-8, 0) for s in (2,)]
            if n == sizes[0]:
                runs += [("split classical", 0, 0.0, sl) for sl in (3, 4, 5, 6)]
                runs += [("bini322_10_52_approx", 1, 2.0 ** -lg, sl) for lg in (10, 14, 18, 22, 26) for sl in (0, 6)]
            for alg, steps, x, sl in runs:
                if alg == "split classical":
                    fn = lambda: fmm.matmul_split_bf16(A, B, C, slices=sl, handle=h)  # noqa: E731
                    name = "classical"
                elif alg == "fp64 strassen":
                    fn = lambda: fmm.fast_matmul("strassen", A, B, C, steps, handle=h)  # noqa: E731
                    name = "strassen"
                else:
                    prec = "split_bf16" if sl else "fp64"
                    fn = lambda: fmm.fast_matmul(alg, A, B, C, steps, x, precision=prec, split_slices=sl,  # noqa: E731
                                                 handle=h)
                    name = alg
                ms = timed(fn)
                h.profile(True)
                h.profile_reset()
                fn()
                prof = h.profile_read()
                h.profile(False)
                fmm.synchronize(h)
                err = precision_errors(fmm, A, B, C, ref, absAB, h)
                leaf_ms = prof["gemm_ms"] - prof["split_ms"]
                row = {"n": n, "inputs": dist, "algorithm": name, "num_steps": steps,
                       "lambda": x if "approx" in name else None,
                       "precision": "split_bf16 x%d" % sl if sl else "fp64", "ms": ms,
                       "effective_tflops": flops / (ms * 1e-3) / 1e12, "error": err,
                       "split_kernel_ms": prof["split_ms"] if sl else None,
                       "slice_product_bf16_tflops": (prof["split_bf16_flops"] / (leaf_ms * 1e-3) / 1e12
                                                     if sl and leaf_ms > 0 else None)}
                rows.append(row)
                print(json.dumps({"precision_row": row}), file=sys.stderr, flush=True)
                if (n == max(sizes) and dist.startswith("uniform") and name == "strassen" and sl
                        and err["max_rel_elementwise"] <= 1e-12
                        and (head is None or row["effective_tflops"] > head["effective_tflops"])):
                    head = row
            del A, B, C, ref, absAB
            torch.cuda.empty_cache()

    clk = clocks.stop()
    peaks, peak_src = measured_peaks()
    n_head = max(sizes)
    base = classical[n_head]
    value = head["effective_tflops"] if head else None
    roofline = None
    if head and head["slice_product_bf16_tflops"]:
        # the product kernel runs for ~0.1 s inside a multi-second sweep: the
        # sustained (power-capped) cuBLAS figure is its denominator
        pk = peaks.get("bf16_tflops_sustained", 1400.0)
        burst = peaks.get("bf16_tflops", 1590.0)
        traffic = committed_traffic("roofline_traffic_split.json")
        ach = head["slice_product_bf16_tflops"]
        roofline = {"kernel": "split_gemm_kernel (tcgen05 BF16 slice products)", "bound": "tensor",
                    "achieved": ach, "peak": pk, "unit": "TFLOP/s", "frac": ach / pk,
                    "peak_source": "bf16_tflops_sustained of MEASURED_PEAKS.json (%s; cuBLAS bf16 8192^3 looped "
                                   "for 4 s under the power cap)" % peak_src,
                    "frac_of_burst_peak": ach / burst,
                    "traffic": (traffic or {}).get("bytes_per_launch"),
                    "traffic_source": (traffic or {}).get("source")}
    out = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": 1, "steps": 2, "warmup": 1,
        "ms_per_step": head["ms"] if head else None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 slices (FP64 in and out)", "data": "synthetic",
        "config": {"workload": "precision: split-BF16 leaf products; headline = fastest Strassen at %d^3 "
                               "within 1e-12 (elementwise, uniform inputs) of the FP64 classical product"
                               % n_head,
                   "headline": head, "l2": "inputs larger than L2"},
        "classical": {str(k): v for k, v in classical.items()},
        "speedup_vs_engine_classical": value / base["engine_dgemm_tflops"] if value else None,
        "speedup_vs_cublas": value / base["cublas_dgemm_tflops"] if value else None,
        "roofline": roofline,
        "clocks": clk,
        "rows": rows,
    }
    print(json.dumps(out))
    return 0


def skewed_pair(fmm, n, seed, dev):
    """Seeded uniform [0, 1) operands with rows of A, columns of B and the
    inner dimension scaled by powers of two 2^U{-20..20}: A = D_r U_A D_t,
    B = D_t^-1 U_B D_c (the product is as well conditioned as U_A U_B)."""
    import numpy as np
    import torch

    rng = np.random.default_rng(seed)
    er, ec, et = (rng.integers(-20, 21, n) for _ in range(3))
    A = fmm.random_matrix(n, n, 41, 1, device=dev.index)
    B = fmm.random_matrix(n, n, 41, 2, device=dev.index)
    p2 = lambda e: torch.from_numpy(np.ldexp(1.0, e)).to(dev)  # noqa: E731
    A.mul_(p2(er)[:, None]).mul_(p2(et)[None, :])
    B.mul_(p2(-et)[:, None]).mul_(p2(ec)[None, :])
    return A, B


def cpu_scaling_sample(edge, scaling_steps, seconds):
    """Times the reference's Scaling<double> (scaling/scaling.hpp, single
    host thread: the header has no parallel loop) on an edge x edge pair;
    returns (median ms, runs)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # the CPU baseline leg may load the reference build

    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libfmm_ref.so is not built")
    A = oracle.uniform(edge, edge, 7, 1)
    B = oracle.uniform(edge, edge, 7, 2)
    times = []
    t_end = time.time() + seconds
    while time.time() < t_end or len(times) < 2:
        t0 = time.perf_counter()
        oracle.scaling(A, B, scaling_steps, 0, ref=True)
        times.append((time.perf_counter() - t0) * 1e3)
    return statistics.median(times), len(times)


def run_scaling_workload(a):
    """Diagonal scaling (scaling/scaling.hpp) as the reference's
    strassen_scaling_perf driver runs it: Scaling with 5 outside-inside
    steps, Strassen with one step, PostProcessScaling, at n^3 on operands
    skewed by powers of two.  Reported: the scaling's bandwidth against the
    measured HBM copy peak (algorithmic bytes: one read of A and B, then one
    read + write of both per outer or inner scaling), the time of the whole
    scaled product against the unscaled one, the errors of both against the
    classical FP64 product, and the reference's own Scaling on the host."""
    import torch

    import fast_matmul_b200 as fmm

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    h = fmm.default_handle(0)
    n, sc_steps = a.scaling_size, 5
    A, B = skewed_pair(fmm, n, 5, dev)
    As, Bs = fmm.colmajor_empty(n, n, dev), fmm.colmajor_empty(n, n, dev)
    C, ref = fmm.colmajor_empty(n, n, dev), fmm.colmajor_empty(n, n, dev)
    fmm.matmul(A, B, ref, handle=h)

    def timed(fn, reps):
        for _ in range(max(a.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # kernel bandwidth: inputs (2 x 2 GiB at 16384) are far larger than L2
    As.copy_(A)
    Bs.copy_(B)
    launches0 = h.launches()
    r, s = fmm.diagonal_scaling(As, Bs, sc_steps, fmm.OUTSIDE_INSIDE, handle=h)
    launches_per_call = h.launches() - launches0
    clocks = ClockSampler(0)
    clocks.start()
    ms_scale = timed(lambda: fmm.diagonal_scaling(As, Bs, sc_steps, fmm.OUTSIDE_INSIDE, handle=h), a.steps)
    ms_post = timed(lambda: fmm.scaling_postprocess(C, r, s, handle=h), a.steps)
    clk = clocks.stop()
    passes = 1 + 2 * (2 * sc_steps)
    bytes_scale = 8.0 * (2 * n * n) * passes
    bytes_post = 16.0 * n * n
    gbs_scale = bytes_scale / (ms_scale * 1e-3) / 1e9
    gbs_post = bytes_post / (ms_post * 1e-3) / 1e9

    def pipeline(kind, steps, **kw):
        As.copy_(A)
        Bs.copy_(B)
        rr, ss = fmm.diagonal_scaling(As, Bs, sc_steps, kind, handle=h)
        fmm.fast_matmul("strassen", As, Bs, C, steps, handle=h, **kw)
        fmm.scaling_postprocess(C, rr, ss, handle=h)

    rows = []
    for label, steps, kw in [("fp64 strassen", 1, {}), ("fp64 strassen", 2, {}),
                             ("split_bf16 x5 strassen", 1, {"precision": "split_bf16", "split_slices": 5}),
                             ("split_bf16 x6 strassen", 1, {"precision": "split_bf16", "split_slices": 6})]:
        ms_plain = timed(lambda: fmm.fast_matmul("strassen", A, B, C, steps, handle=h, **kw), 2)
        e_plain, _ = fmm.max_relative_diff(ref, C, handle=h)
        kind = fmm.OUTSIDE_INSIDE
        # the copies of A and B are the caller's (the reference's driver
        # copies too); they are timed apart and not charged to the scaling
        ms_copy = timed(lambda: (As.copy_(A), Bs.copy_(B)), 2)
        ms_scaled = timed(lambda: pipeline(kind, steps, **kw), 2) - ms_copy
        e_scaled, _ = fmm.max_relative_diff(ref, C, handle=h)
        row = {"product": label, "num_steps": steps, "scaling": ["outside_inside", "inside_outside", "inside",
                                                                 "outside"][kind],
               "scaling_steps": sc_steps, "ms_unscaled": ms_plain, "ms_scaled_pipeline": ms_scaled,
               "overhead": ms_scaled / ms_plain - 1.0, "max_rel_err_unscaled": e_plain,
               "max_rel_err_scaled": e_scaled}
        rows.append(row)
        print(json.dumps({"scaling_row": row}), file=sys.stderr, flush=True)

    peaks, peak_src = measured_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    traffic = committed_traffic("roofline_traffic_scaling.json")
    cpu = None
    if not a.no_cpu_baseline:
        edge = 4096
        cms, runs = cpu_scaling_sample(edge, sc_steps, a.cpu_seconds)
        cpu = {"value": 8.0 * (2 * edge * edge) * passes / (cms * 1e-3) / 1e9, "unit": "GB/s", "cores": 1,
               "kind": "reference",
               "sample": "Scaling<double>(A, B, 5, r, s, OUTSIDE_INSIDE) of scaling/scaling.hpp, %d x %d "
                         "uniform pair, median of %d runs, %.1f ms each" % (edge, edge, runs, cms)}
    out = {
        "metric": "diagonal scaling bandwidth (algorithmic bytes / time)", "value": gbs_scale, "unit": "GB/s",
        "n_gpus": 1, "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": ms_scale,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "diagonal scaling: Scaling(A, B, 5, r, s, OUTSIDE_INSIDE) at %d x %d, "
                               "strassen_scaling_perf's pipeline beside it" % (n, n),
                   "l2": "inputs larger than L2"},
        "gpu_launches": launches_per_call * a.steps,
        "clocks": clk,
        "roofline": {"kernel": "scale_reduce_kernel (+ factor kernels)", "bound": "hbm", "achieved": gbs_scale,
                     "peak": hbm, "unit": "GB/s", "frac": gbs_scale / hbm,
                     "peak_source": "hbm_gbs of MEASURED_PEAKS.json (%s)" % peak_src,
                     "algorithmic_bytes_per_call": bytes_scale,
                     "traffic": (traffic or {}).get("bytes_per_call"),
                     "traffic_source": (traffic or {}).get("source")},
        "postprocess": {"ms": ms_post, "achieved_gbs": gbs_post, "frac": gbs_post / hbm},
        "cpu_baseline": cpu,
        "pipelines": rows,
    }
    print(json.dumps(out))
    return 0


def run_int8_workload(a):
    """Split-INT8 leaf products (7-bit digits on the INT8 tensor cores, exact
    int32 sums) beside split-BF16 and FP64 at n^3 on seeded uniform [0, 1)
    inputs: Strassen with 2 and 3 steps, fast424 with 2 steps and the
    classical split product, each timed (CUDA events, inputs resident, L2
    flushed by the inputs' size) and checked against the engine's FP64
    classical product; the engine's DGEMM and cuBLAS DGEMM give the ratios.
    The headline is the fastest configuration within 1e-12 (elementwise)."""
    import torch

    import fast_matmul_b200 as fmm

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    h = fmm.default_handle(0)
    n = a.int8_size
    flops = 2.0 * n ** 3
    A = fmm.random_matrix(n, n, 31, 1, handle=h)
    B = fmm.random_matrix(n, n, 31, 2, handle=h)

    def timed(fn, reps):
        for _ in range(max(a.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ref = fmm.colmajor_empty(n, n, dev)
    ms = timed(lambda: fmm.matmul(A, B, ref, handle=h), 2)
    engine = flops / (ms * 1e-3) / 1e12
    Ct = torch.matmul(A, B)
    msb = timed(lambda: torch.matmul(A, B, out=Ct), 2)
    cublas = flops / (msb * 1e-3) / 1e12
    del Ct
    absAB = fmm.colmajor_empty(n, n, dev)
    fmm.matmul(A.abs(), B.abs(), absAB, handle=h)
    C = fmm.colmajor_empty(n, n, dev)
    clocks = ClockSampler(0)
    clocks.start()
    configs = [("strassen", 2, "split_bf16", 5), ("strassen", 2, "split_int8", 6), ("strassen", 2, "split_int8", 7),
               ("strassen", 3, "split_int8", 6), ("grey424_26_206", 2, "split_int8", 6),
               ("classical", 0, "split_int8", 6), ("classical", 0, "split_bf16", 5)]
    rows = []
    for alg, steps, prec, sl in configs:
        if alg == "classical":
            mm = fmm.matmul_split_int8 if prec == "split_int8" else fmm.matmul_split_bf16
            fn = lambda: mm(A, B, C, slices=sl, handle=h)  # noqa: E731
        else:
            fn = lambda: fmm.fast_matmul(alg, A, B, C, steps, precision=prec, split_slices=sl,  # noqa: E731
                                         handle=h)
        ms = timed(fn, a.steps)
        h.profile(True)
        h.profile_reset()
        fn()
        prof = h.profile_read()
        h.profile(False)
        fmm.synchronize(h)
        err = precision_errors(fmm, A, B, C, ref, absAB, h)
        leaf_ms = prof["gemm_ms"] - prof["split_ms"]
        rows.append({"algorithm": alg, "num_steps": steps, "precision": "%s x%d" % (prec, sl), "ms": ms,
                     "effective_tflops": flops / (ms * 1e-3) / 1e12, "error": err,
                     "split_kernel_ms": prof["split_ms"], "product_kernel_ms": leaf_ms,
                     "slice_product_tensor_tops": (prof["split_bf16_flops"] / (leaf_ms * 1e-3) / 1e12
                                                   if leaf_ms > 0 else None)})
        print(json.dumps({"int8_row": rows[-1]}), file=sys.stderr, flush=True)
    clk = clocks.stop()
    ok = [r for r in rows if r["error"]["max_rel_elementwise"] <= 1e-12]
    head = max(ok, key=lambda r: r["effective_tflops"]) if ok else None
    # N(0, 1) entries with per-row (A) / per-column (B) scales 2^U{-16..16}:
    # errors only (elementwise relative errors are unbounded there for every
    # Strassen variant, FP64 included; normwise ones are comparable)
    del A, B, ref, absAB
    torch.cuda.empty_cache()
    A = scaled_normal(n, n, 41, "row", dev)
    B = scaled_normal(n, n, 42, "col", dev)
    ref = fmm.colmajor_empty(n, n, dev)
    fmm.matmul(A, B, ref, handle=h)
    absAB = fmm.colmajor_empty(n, n, dev)
    fmm.matmul(A.abs(), B.abs(), absAB, handle=h)
    scaled_rows = []
    for prec, sl in (("fp64", 0), ("split_bf16", 6), ("split_int8", 6), ("split_int8", 7)):
        fmm.fast_matmul("strassen", A, B, C, 2, precision=prec, split_slices=sl, handle=h)
        fmm.synchronize(h)
        scaled_rows.append({"algorithm": "strassen", "num_steps": 2, "precision": "%s x%d" % (prec, sl) if sl else prec,
                            "error": precision_errors(fmm, A, B, C, ref, absAB, h)})
        print(json.dumps({"int8_scaled_row": scaled_rows[-1]}), file=sys.stderr, flush=True)
    peaks, peak_src = measured_peaks()
    roofline = None
    if head and head["slice_product_tensor_tops"] and "int8" in head["precision"]:
        # no INT8 figure is measured: the INT8 tensor rate is twice the BF16 one on
        # B200 (4.5 against 2.25 dense POPS nominal), so twice the sustained cuBLAS
        # BF16 figure stands in as the denominator
        pk = 2.0 * peaks.get("bf16_tflops_sustained", 1400.0)
        ach = head["slice_product_tensor_tops"]
        roofline = {"kernel": "split_gemm_kernel<2, true> (tcgen05 kind::i8 slice products)", "bound": "tensor",
                    "achieved": ach, "peak": pk, "unit": "TOP/s", "frac": ach / pk,
                    "peak_source": "2 x bf16_tflops_sustained of MEASURED_PEAKS.json (%s): INT8 dense is twice "
                                   "BF16 dense on B200" % peak_src, "traffic": None}
    out = {
        "metric": "effective TFLOP/s (2MNK/t) fast vs classical GEMM, same B200, at stated error",
        "value": head["effective_tflops"] if head else None, "unit": "TFLOP/s", "n_gpus": 1, "steps": a.steps,
        "warmup": max(a.warmup, 3), "ms_per_step": head["ms"] if head else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8 slices (FP64 in and out)", "data": "synthetic",
        "config": {"workload": "int8: split-INT8 leaf products at %d^3, uniform [0, 1); headline = fastest "
                               "configuration within 1e-12 (elementwise) of the FP64 classical product" % n,
                   "headline": head, "l2": "inputs larger than L2"},
        "classical": {"engine_dgemm_tflops": engine, "cublas_dgemm_tflops": cublas},
        "speedup_vs_engine_classical": head["effective_tflops"] / engine if head else None,
        "speedup_vs_cublas": head["effective_tflops"] / cublas if head else None,
        "roofline": roofline, "clocks": clk, "rows": rows,
        "scaled_normal_inputs": scaled_rows,
    }
    print(json.dumps(out))
    return 0


def run_fp32_workload(a):
    """FastMatmul<float> (fmm_fast_matmul_f32): FP32 operands widened to FP64
    on the device, split leaf products (5 INT8 slices by default; BF16 and
    other INT8 slice counts as rows), rounded to FP32 once.  At n^3: Strassen with 1 and 2 steps and the classical
    product (fmm_sgemm) against cuBLAS SGEMM (torch.matmul in float32, TF32
    off) on the same inputs, errors against the exact product of the FP32
    inputs on sampled entries, and the reference's own FastMatmul<float>
    (sgemm leaves, all host threads) on a bounded sample."""
    import numpy as np
    import torch

    import fast_matmul_b200 as fmm

    torch.cuda.set_device(0)
    torch.backends.cuda.matmul.allow_tf32 = False
    dev = torch.device("cuda", 0)
    h = fmm.default_handle(0)
    n = a.fp32_size
    flops = 2.0 * n ** 3
    A64 = fmm.random_matrix(n, n, 51, 1, handle=h)
    B64 = fmm.random_matrix(n, n, 51, 2, handle=h)
    A = A64.float()
    B = B64.float()
    A64 = A.double()  # the exact values of the FP32 operands
    B64 = B.double()
    C = torch.empty((n, n), dtype=torch.float32, device=dev).t()

    def timed(fn, reps):
        for _ in range(max(a.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def errors(Cf):
        rel, _ = exact_sample_errors(A64, B64, Cf.double(), count=32)
        return rel

    rows = []
    Cb = torch.matmul(A, B)
    ms_cublas = timed(lambda: torch.matmul(A, B, out=Cb), a.steps)
    rows.append({"product": "cuBLAS SGEMM (torch.matmul, float32, TF32 off)", "ms": ms_cublas,
                 "tflops": flops / (ms_cublas * 1e-3) / 1e12, "max_rel_vs_exact_32_sampled": errors(Cb)})
    del Cb
    clocks = ClockSampler(0)
    clocks.start()
    # split-INT8 with 4 slices (27 bits) is as accurate as split-BF16 with 3-4
    # once the result is rounded to FP32
    configs = [("classical (fmm_sgemm)", None, 0, "split_int8", 5), ("strassen", "strassen", 1, "split_bf16", 4),
               ("strassen", "strassen", 2, "split_bf16", 4), ("strassen", "strassen", 2, "split_bf16", 3),
               ("strassen", "strassen", 3, "split_bf16", 3), ("grey424_26_206", "grey424_26_206", 2, "split_bf16", 4),
               ("grey424_26_206", "grey424_26_206", 2, "split_bf16", 3), ("strassen", "strassen", 2, "split_int8", 4),
               ("strassen", "strassen", 3, "split_int8", 4), ("grey424_26_206", "grey424_26_206", 2, "split_int8", 4),
               ("strassen", "strassen", 2, "split_int8", 5)]
    for label, alg, steps, prec, sl in configs:
        if alg is None:
            fn = lambda: fmm.matmul(A, B, C, handle=h)  # noqa: E731
        else:
            fn = lambda: fmm.fast_matmul(alg, A, B, C, steps, precision=prec, split_slices=sl,  # noqa: E731
                                         handle=h)
        ms = timed(fn, a.steps)
        fmm.synchronize(h)
        rows.append({"product": label, "num_steps": steps, "precision": "%s x%d" % (prec, sl), "ms": ms,
                     "tflops": flops / (ms * 1e-3) / 1e12, "max_rel_vs_exact_32_sampled": errors(C)})
        print(json.dumps({"fp32_row": rows[-1]}), file=sys.stderr, flush=True)
    clk = clocks.stop()
    best = max((r for r in rows[1:] if r["max_rel_vs_exact_32_sampled"] <= rows[0]["max_rel_vs_exact_32_sampled"]
                or r["max_rel_vs_exact_32_sampled"] <= 2.0 ** -23), key=lambda r: r["tflops"])
    cpu = None
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle  # the CPU baseline leg may load the reference build

        if oracle.ref_available():
            edge = 4096
            threads = os.cpu_count() or 1
            oracle.ref_lib().fmmref_set_threads(threads)
            Ah = np.asfortranarray(oracle.uniform(edge, edge, 7, 1).astype(np.float32))
            Bh = np.asfortranarray(oracle.uniform(edge, edge, 7, 2).astype(np.float32))
            Ch = np.zeros((edge, edge), dtype=np.float32, order="F")
            oracle.ref_fast_matmul_f32("strassen", Ah, Bh, Ch, 2)
            ts = []
            t_end = time.time() + a.cpu_seconds
            while time.time() < t_end or len(ts) < 2:
                t0 = time.perf_counter()
                oracle.ref_fast_matmul_f32("strassen", Ah, Bh, Ch, 2)
                ts.append((time.perf_counter() - t0) * 1e3)
            cms = statistics.median(ts)
            cpu = {"value": 2.0 * edge ** 3 / (cms * 1e-3) / 1e12, "unit": "TFLOP/s", "cores": threads,
                   "kind": "reference",
                   "sample": "strassen::FastMatmul<float>(A, B, C, 2) of the reference (sgemm leaves), %d^3, "
                             "median of %d runs, %.0f ms each" % (edge, len(ts), cms)}
    peaks, peak_src = measured_peaks()
    out = {
        "metric": "effective TFLOP/s (2MNK/t), FP32 operands, vs cuBLAS SGEMM", "value": best["tflops"],
        "unit": "TFLOP/s", "n_gpus": 1, "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": best["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 in/out (bf16 slices, f64 accumulation)", "data": "synthetic",
        "config": {"workload": "FastMatmul<float> at %d^3, seeded uniform [0,1) rounded to FP32; headline = fastest "
                               "configuration whose sampled error is within cuBLAS SGEMM's or 2^-23" % n,
                   "headline": best, "l2": "inputs larger than L2"},
        "speedup_vs_cublas_sgemm": best["tflops"] / rows[0]["tflops"],
        "clocks": clk, "cpu_baseline": cpu, "peak_source": peak_src, "rows": rows,
    }
    print(json.dumps(out))
    return 0


def run_profile_workload(a):
    """One product configuration called a.steps times, untimed (a profiler target)."""
    import fast_matmul_b200 as fmm

    A = fmm.random_matrix(a.m, a.k, 1, 1)
    B = fmm.random_matrix(a.k, a.n, 1, 2)
    C = fmm.colmajor_empty(a.m, a.n, A.device)
    for _ in range(a.steps):
        if a.alg == "classical":
            if a.precision == "split_int8":
                fmm.matmul_split_int8(A, B, C, slices=a.split_slices)
            elif a.precision == "split_bf16":
                fmm.matmul_split_bf16(A, B, C, slices=a.split_slices)
            else:
                fmm.matmul(A, B, C)
        else:
            fmm.fast_matmul(a.alg, A, B, C, a.num_steps, schedule=a.schedule, precision=a.precision,
                            split_slices=a.split_slices)
    fmm.synchronize()
    print(json.dumps({"workload": "profile", "alg": a.alg, "m": a.m, "k": a.k, "n": a.n, "num_steps": a.num_steps,
                      "precision": a.precision, "split_slices": a.split_slices, "calls": a.steps,
                      "c00": float(C[0, 0])}))
    return 0


def main(argv=None):
    a = parse_args(argv)
    if a.impl == "reference":
        return run_reference(a)
    if a.sweep:
        return run_sweep(a)
    if a.workload == "batch":
        return run_batch_workload(a)
    if a.workload == "serve":
        return run_serve_workload(a)
    if a.workload == "precision":
        return run_precision_workload(a)
    if a.workload == "scaling":
        return run_scaling_workload(a)
    if a.workload == "int8":
        return run_int8_workload(a)
    if a.workload == "fp32":
        return run_fp32_workload(a)
    if a.workload == "profile":
        return run_profile_workload(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
