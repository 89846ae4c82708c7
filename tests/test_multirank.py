"""The multi-rank path of bench.py on the CPU: world size 2 with the gloo backend.

`bench.py --gpus N` runs one independent replica per rank (the batched ensemble, the
adjoint and the plain engine are replicas-only here) and reports the whole-job rate
over the slowest rank's device time. These tests run the same helpers on gloo ranks
(every rank takes the same collectives in the same order), and the reference arm under
torchrun, where rank 0 alone runs and prints one line and the other ranks exit 0.
"""
import datetime
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


def _rank_main(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # the timed region's device milliseconds differ per rank; the job takes the slowest
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        ms_e2e = bench.max_over_ranks(30.0 - 7.0 * rank, world)
        rate = bench.job_rate(world, 1000, 10, ms)
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"ms": ms, "ms_e2e": ms_e2e, "rate": rate}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_on_gloo(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        d = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert d["ms"] == 15.0  # the slower rank's time on every rank
        assert d["ms_e2e"] == 30.0
        # two replicas of 1000 particles, 10 steps each, in 15 ms
        assert d["rate"] == pytest.approx(2 * 1000 * 10 / 0.015)


def test_single_rank_helpers_need_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(4.5, 1) == 4.5
    assert bench.job_rate(1, 200000, 100, 28.0) == pytest.approx(200000 * 100 / 0.028)


def test_reference_arm_under_torchrun_prints_once():
    sys.path.insert(0, ROOT)
    from oracle import refengine
    if not refengine.available():
        pytest.skip("reference engine library not built")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
