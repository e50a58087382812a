"""CPU tests of the multi-GPU split of one task (qld_cuda_split_rows, the
partition qld_cuda_ld_device_part uses): the parts are consecutive whole tile
rows covering every B row once, with (nearly) equal numbers of output tiles,
and two gloo ranks that each take their own part cover the task between
them."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from qld_b200 import api

TILE_ROWS = {api.KERNEL_POPC: (128, 128), api.KERNEL_MMA: (128, 256), api.KERNEL_FP4: (256, 240)}


def _tiles(m, n, bm, bn, symmetric, b0, b1):
    """Output tiles of B rows [b0, b1): every A tile of the rectangle; of the
    triangle, the tiles holding an entry with a >= b."""
    count = 0
    for tb in range(b0 // bn, -(-b1 // bn)):
        for ta in range(-(-m // bm)):
            if not symmetric or (ta + 1) * bm - 1 >= tb * bn:
                count += 1
    return count


@pytest.mark.parametrize("kernel", sorted(TILE_ROWS))
@pytest.mark.parametrize("m,n,K,sym", [(29_817, 29_817, 260, True), (3000, 2000, 70, False),
                                        (700, 700, 5, True), (100, 100, 2, True)])
@pytest.mark.parametrize("nparts", [1, 2, 3, 8])
def test_parts_cover_the_task_in_balanced_tile_rows(kernel, m, n, K, sym, nparts):
    bm, bn = TILE_ROWS[kernel]
    n = m if sym else n
    parts = [api.split_rows(m, n, K, sym, kernel, p, nparts) for p in range(nparts)]
    assert parts[0][0] == 0 and parts[-1][1] == n
    for (a0, a1), (b0, _) in zip(parts, parts[1:]):
        assert a1 == b0 and a0 <= a1
    for r0, r1 in parts:
        assert (r0 % bn == 0 or r0 == n) and (r1 % bn == 0 or r1 == n)
    total = _tiles(m, n, bm, bn, sym, 0, n)
    row_max = max(_tiles(m, n, bm, bn, sym, tb * bn, min(n, tb * bn + bn))
                  for tb in range(-(-n // bn)))
    for r0, r1 in parts:
        if r0 < r1 or -(-n // bn) >= nparts:
            assert abs(_tiles(m, n, bm, bn, sym, r0, r1) - total / nparts) <= row_max + 1


def test_bad_arguments():
    with pytest.raises(api.QldError):
        api.split_rows(100, 100, 2, True, api.KERNEL_FP4, 3, 3)
    with pytest.raises(api.QldError):
        api.split_rows(100, 100, 2, True, 9, 0, 1)


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r0, r1 = api.split_rows(29_817, 29_817, 260, True, api.KERNEL_AUTO, rank, world)
        got = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(got, torch.tensor([r0, r1], dtype=torch.int64))
        if rank == 0:
            with open(out, "w") as f:
                f.write(" ".join(f"{int(g[0])},{int(g[1])}" for g in got))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_consecutive_parts(tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "parts.txt")
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    parts = [tuple(int(x) for x in p.split(",")) for p in open(out).read().split()]
    assert parts[0][0] == 0 and parts[0][1] == parts[1][0] and parts[1][1] == 29_817
    assert 0 < parts[0][1] < 29_817
