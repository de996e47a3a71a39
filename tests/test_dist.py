"""The multi-rank plumbing of bench.py (one process per GPU, replicas) on CPU
with the gloo backend, world size 2: process-group setup from the launcher's
environment, max-over-ranks timing and the replica rate; and the reference
arm under torchrun (rank 0 alone runs and prints, the other ranks exit 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    w, r, local = bench.dist_setup()
    dist = bench.init_dist(w, local, use_cuda=False, timeout_s=60)
    mx = bench.max_over_ranks(1.5 + r, dist)
    dist.barrier()
    rate = bench.replica_rate(w, 1000.0, mx)
    with open(os.path.join(out_dir, f"r{r}.json"), "w") as f:
        json.dump({"world": w, "rank": r, "max": mx, "rate": rate}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_rate_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    for r in res:
        assert r["world"] == 2 and r["max"] == 2.5
        assert r["rate"] == pytest.approx(2 * 1000.0 / 2.5)


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.init_dist(1, 0) is None
    assert bench.max_over_ranks(3.0, None) == 3.0


def test_reference_arm_under_torchrun_two_ranks():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--scale", "10"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    # the keys the reference arm's line carries besides the value
    assert line["metric"] == "pagerank_gteps_rmat24" and line["unit"] == "GTEPS"
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 3
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] >= 1 and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == "GTEPS"
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"].startswith("pagerank_rmat10")
