"""Multi-rank plumbing of the replica runs on CPU: a world_size-2 gloo group
checks the partition of an ensemble and the MAX / SUM reductions that turn
per-rank device times into whole-job throughput (no GPU involved)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import mpcf.replicas as rp


def test_partition_balanced_and_complete():
    cells = [32 ** 3, 48 ** 3, 64 ** 3, 96 ** 3, 128 ** 3, 32 * 64 * 128, 96 * 48 * 32, 64 ** 3]
    for world in (1, 2, 3, 4, 8):
        g = rp.partition_domains(cells, world)
        assert len(g) == world
        flat = [i for grp in g for i in grp]
        assert flat == list(range(len(cells)))                 # contiguous, complete, ordered
        if world <= len(cells):
            assert all(grp for grp in g)                        # every rank gets work
    g = rp.partition_domains([1] * 64, 4)
    assert [len(x) for x in g] == [16, 16, 16, 16]
    with pytest.raises(ValueError):
        rp.partition_domains([1, 2], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        cells = [64 ** 3, 96 ** 3, 32 ** 3, 128 ** 3]
        mine = rp.partition_domains(cells, world)[rank]
        my_cells = sum(cells[i] for i in mine)
        ms = 10.0 + 5.0 * rank                       # rank 1 is the slower one
        dist.barrier()
        value, ms_max = rp.throughput(dist, my_cells, 3 * 4, ms)
        out[rank] = (value, ms_max, my_cells)
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions_gloo():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    total = 64 ** 3 + 96 ** 3 + 32 ** 3 + 128 ** 3
    for r in range(world):
        value, ms_max, _ = out[r]
        assert ms_max == 15.0                                   # MAX over ranks
        assert abs(value - total * 12 / 15e-3) < 1e-6 * value   # SUM of work / slowest time
    assert out[0][2] + out[1][2] == total
