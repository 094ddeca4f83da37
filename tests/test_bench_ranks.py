"""The replicas path of bench.py on CPU: two gloo ranks (127.0.0.1), each with
its own seed set, combined into whole-job figures (slowest rank's time, all
ranks' particle-steps); and the reference arm under two ranks, where only
rank 0 runs and prints."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    from dpa_b200 import fields
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grid = fields.abc(16)
        seeds = bench.rank_seeds(grid, 64, 10, rank).position
        # Rank r pretends its step took 10 + r ms and took 1000 (r + 1) steps.
        ms, steps = bench.combine_over_ranks(10.0 + rank, 1000.0 * (rank + 1), "cpu")
        np.save(out / f"seeds_{rank}.npy", seeds)
        (out / f"combined_{rank}.json").write_text(json.dumps([ms, steps]))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replicas_combine_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, tmp_path)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        ms, steps = json.loads((tmp_path / f"combined_{r}.json").read_text())
        assert ms == 11.0 and steps == 3000.0  # max of the times, sum of the steps
    a, b = np.load(tmp_path / "seeds_0.npy"), np.load(tmp_path / "seeds_1.npy")
    assert a.shape == b.shape == (64, 3) and not np.array_equal(a, b)


def test_single_process_combination_is_the_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.combine_over_ranks(12.5, 77.0, "cpu") == (12.5, 77.0)


@pytest.mark.timeout(600)
def test_reference_arm_under_two_ranks_prints_once(tmp_path):
    # Only rank 0 runs the CPU baseline; rank 1 exits 0 without work. A small
    # workload keeps the oracle sample to seconds.
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--grid", "32", "--seeds", "4096", "--iterations", "50"]
    r = subprocess.run(cmd, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["cpu_baseline"]["kind"] == "port"
