"""The N > 1 path of bench.py on host processes (gloo, world size 2).

bench.py runs one replica per GPU under torch.distributed.run: the product
does not shard, so the only collectives are a barrier around the timed
region and the maximum over ranks of the measured time.  The same
coordination (bench.Replicas) runs here on the gloo backend; the reference
arm's rank handling (rank 0 measures and prints, the others exit 0 without
work) is checked in-process.
"""

import contextlib
import io
import json
import os
import socket

import pytest
import torch.multiprocessing as mp

from helpers import REPO


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def replica(rank, world, port, out):
    import sys

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, REPO)
    import bench

    rep = bench.Replicas("gloo", timeout_s=60.0)
    rep.barrier()
    elapsed = 1.0 + 2.0 * rank  # the slower rank sets the job's time
    t_max = rep.max(elapsed)
    rate = rep.whole_job_rate(10.0, t_max)
    rep.close()
    out.put((rank, rep.world, t_max, rate))


def test_replicas_take_the_max_over_ranks_and_count_every_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=replica, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, w, t_max, rate in got:
        assert w == world
        assert t_max == 3.0
        assert rate == pytest.approx(world * 10.0 / 3.0)


def test_single_process_needs_no_process_group(monkeypatch):
    import bench

    for var in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(var, raising=False)
    rep = bench.Replicas("gloo")
    assert rep.world == 1 and rep.max(2.5) == 2.5 and rep.whole_job_rate(4.0, 2.0) == 2.0
    rep.barrier()
    rep.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import oracle

    import bench

    monkeypatch.setenv("RANK", "1")
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.main(["--impl", "reference", "--cpu-sample", "128", "--steps", "1", "--warmup", "0"]) == 0
    assert buf.getvalue() == ""
    if not oracle.ref_available():
        pytest.skip("reference build oracle/_ref not present")
    monkeypatch.setenv("RANK", "0")
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.main(["--impl", "reference", "--cpu-sample", "128", "--steps", "1", "--warmup", "0"]) == 0
    line = json.loads(buf.getvalue().strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
