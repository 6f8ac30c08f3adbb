"""Multi-rank bench bookkeeping on CPU (gloo, two ranks): the replica job's
time is the slowest rank's and its work the sum of the ranks' work, the same
combination bench.py makes over NCCL when launched with torchrun."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        # rank r took (1 + r) ms of device time, (2 + r) ms of wall time and
        # did (10 + r) units of work
        res = bench.combine_over_ranks(1e-3 * (1 + rank), 1e-3 * (2 + rank), 10.0 + rank, "cpu")
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_replicas_combine_max_time_and_sum_work():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        for r in range(world):
            dev_s, wall_s, work = out[r]
            assert dev_s == pytest.approx(2e-3)
            assert wall_s == pytest.approx(3e-3)
            assert work == 21.0


def test_reference_arm_prints_one_json_line():
    """``bench.py --impl reference`` runs the CPU restatement of the path on
    the default workload and prints the contract's JSON line (no GPU)."""
    import json
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    out = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "3"], cwd=root, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "cell-substeps/s"
    assert d["config"]["workload"] == "config1_plain_path_701"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
