"""The multi-process path of bench.py on CPU (gloo, world size 2).

The hot path does not shard: N GPUs run N independent replicas of the
workload, and the bench's only cross-rank steps are a barrier around the timed
region and the maximum of the ranks' times. These tests run those steps as two
gloo ranks, and the reference arm under torchrun, where rank 0 alone measures
and prints one JSON line and the other rank exits 0 without work."""
import contextlib
import io
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        impl = "reference"
        steps, warmup = 2, 0
        ref_n = 8

    w, r, _ = bench.dist_init(Args)
    try:
        bench.barrier(w)
        t = bench.max_over_ranks(w, 0.5 + r)  # rank 1 is the slower one
        # replicas: the units all ranks processed over the slowest rank's time
        value = w * Args.steps / t
        # the reference arm with a stand-in sample: only rank 0 measures and prints
        bench.cpu_simple = lambda n, warm=1, timed=1: ([0.25], "reference")
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            bench.run_reference(Args, w, r)
        q.put((r, w, t, value, out.getvalue()))
    finally:
        import torch.distributed as dist
        dist.destroy_process_group()


def test_barrier_and_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, t, value, printed in got:
        assert w == 2
        assert t == 1.5  # the maximum over ranks, on every rank
        assert value == pytest.approx(2 * 2 / 1.5)
    lines = [json.loads(line) for _, _, _, _, printed in got for line in printed.splitlines() if line.strip()]
    assert len(lines) == 1 and got[1][4] == ""  # rank 1 printed nothing
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2


def test_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-n", "16"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["cells"] == 1448 * 1448 and d["config"]["sample_cells"] == 16 * 16
    # the sample's measured time per step, its it/s scaled to the stated cavity by the cell ratio
    assert d["value"] == pytest.approx(1000.0 / d["ms_per_step"] * (16 * 16) / (1448 * 1448))
