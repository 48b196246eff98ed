"""Batches of independent products, CUDA-graph plans and the autotuner.

Each item of a batch must give exactly (bit for bit) the result of the same
product computed alone; a plan replays the same work; the autotuner records
a valid choice per shape bucket."""

import numpy as np
import pytest

from helpers import colmajor_copy, gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import fast_matmul_b200 as fmm


def make_problems(count, seed, lo=48, hi=700):
    rng = np.random.default_rng(seed)
    specs = ["strassen", "grey424_26_206", "grey333_23_125", fmm.CLASSICAL if gpu_available() else -2, "auto"]
    probs = []
    for i in range(count):
        m, k, n = (int(v) for v in rng.integers(lo, hi, size=3))
        A = fmm.random_matrix(m, k, seed * 1000 + i, 1, -1.0, 1.0)
        B = fmm.random_matrix(k, n, seed * 1000 + i, 2, -1.0, 1.0)
        C = fmm.random_matrix(m, n, seed * 1000 + i, 3, -1.0, 1.0)
        alg = specs[i % len(specs)]
        p = {"A": A, "B": B, "C": C, "alpha": 1.5, "beta": 0.5 if i % 2 else 0.0}
        if alg == "auto":
            p["alg"] = fmm.AUTO
        elif alg == fmm.CLASSICAL:
            p["alg"] = fmm.CLASSICAL
        else:
            p["alg"] = alg
            p["num_steps"] = 1 + i % 2
        probs.append(p)
    return probs


def run_alone(p):
    C = colmajor_copy(p["C"])
    alg = p["alg"]
    if alg == fmm.AUTO:
        m, k = p["A"].shape
        alg, steps = fmm.autotune_choice(m, k, p["B"].shape[1])
    else:
        steps = p.get("num_steps", 1)
    if alg == fmm.CLASSICAL:
        fmm.matmul(p["A"], p["B"], C, p["alpha"], p["beta"])
    else:
        fmm.fast_matmul(alg, p["A"], p["B"], C, steps, 1e-8, p["alpha"], p["beta"])
    return C


def test_batch_items_equal_their_single_calls():
    probs = make_problems(40, 1)
    want = [run_alone(p) for p in probs]
    batch = [dict(p, C=colmajor_copy(p["C"])) for p in probs]
    fmm.fast_matmul_batched(batch)
    torch.cuda.synchronize()
    for i, (w, b) in enumerate(zip(want, batch)):
        assert torch.equal(w, b["C"]), i


def test_batch_plan_replays_and_sees_new_data():
    probs = make_problems(24, 2)
    batch = [dict(p, C=colmajor_copy(p["C"])) for p in probs]
    C0 = [colmajor_copy(b["C"]) for b in batch]
    plan = fmm.Plan.for_batch(batch)
    assert plan.kernels >= 1
    plan.execute()
    first = [colmajor_copy(b["C"]) for b in batch]
    for b, c0 in zip(batch, C0):  # restore C (beta reads it) and replay
        b["C"].copy_(c0)
    plan.execute()
    torch.cuda.synchronize()
    for f, b in zip(first, batch):
        assert torch.equal(f, b["C"])
    want = [run_alone(p) for p in probs]
    for w, f in zip(want, first):
        assert torch.equal(w, f)
    # new data in the same buffers is picked up by the replay
    for b in batch:
        b["A"].mul_(2.0)
    for b, c0 in zip(batch, C0):
        b["C"].copy_(c0)
    plan.execute()
    torch.cuda.synchronize()
    for p, b in zip(probs, batch):
        assert torch.equal(run_alone(dict(p)), b["C"])
    plan.close()


def test_product_plan_equals_direct_call():
    A = fmm.random_matrix(1030, 900, 3, 1)
    B = fmm.random_matrix(900, 1100, 3, 2)
    C1 = fmm.colmajor_empty(1030, 1100)
    C2 = fmm.colmajor_empty(1030, 1100)
    fmm.fast_matmul("grey424_26_206", A, B, C1, 2)
    plan = fmm.Plan.for_product("grey424_26_206", A, B, C2, 2)
    plan.execute()
    plan.execute()
    torch.cuda.synchronize()
    assert torch.equal(C1, C2)
    plan.close()


def test_autotune_records_valid_choices_and_roundtrips():
    h = fmm.Handle(0)
    h.bind_current_stream()
    fmm.autotune([(256, 256, 256), (2048, 2048, 2048)], max_steps=2, handle=h)
    table = fmm.autotune_table(handle=h)
    lines = [l.split() for l in table.strip().splitlines()]
    assert len(lines) == 2
    for mb, kb, nb, alg, steps, tile in lines:
        assert int(alg) == fmm.CLASSICAL or 0 <= int(alg) < fmm.num_algorithms()
        assert int(tile) in (1, 2)  # the measured FP64 GEMM tile configuration
    alg, steps = fmm.autotune_choice(256, 256, 256, handle=h)
    tile = fmm.autotune_tile(256, 256, 256, handle=h)
    h2 = fmm.Handle(0)
    fmm.autotune_load(table, handle=h2)
    assert fmm.autotune_choice(256, 256, 256, handle=h2) == (alg, steps)
    assert fmm.autotune_tile(256, 256, 256, handle=h2) == tile
    h.close()
    h2.close()
