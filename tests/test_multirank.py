"""CPU tests of the multi-rank path (world size 2, gloo).

The LD path shards by independent regions with no data exchange: under
torchrun each rank of bench.py runs its own region (replicas, weak scaling)
and the only collectives are a barrier and the maximum of the ranks' times.
These tests run that plumbing on the host: the max-over-ranks reduction,
per-rank regions that differ, and the launch contract of the reference arm
(rank 0 prints the one JSON line, every rank exits 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mx = bench.max_over_ranks(1.5 + rank, world, "cpu")
        T, S = bench.make_table("all_pairs", "cpu", seed_offset=rank)
        chk = torch.tensor([int(T.sum()), S], dtype=torch.int64)
        got = [torch.zeros_like(chk) for _ in range(world)]
        dist.all_gather(got, chk)
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": mx, "sums": [int(g[0]) for g in got],
                       "S": [int(g[1]) for g in got]}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_and_own_regions(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["max"] == 2.5                      # max over ranks, seen by every rank
        assert r["sums"] == res[0]["sums"]
        assert r["S"] == res[0]["S"]
    assert res[0]["sums"][0] != res[0]["sums"][1]   # each replica has its own region


def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--workload", "all_pairs", "--gpus", "2", "--steps", "1",
           "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference"


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
