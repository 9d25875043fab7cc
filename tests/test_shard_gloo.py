"""Multi-process (gloo, world size 2) check of the frame sharding used by
multi-GPU runs: every output frame is produced by exactly one rank and each
rank's source range covers its windows."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from zb3d import shard


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = []
        for nf, r, v2 in ((64, 0, False), (7, 2, True), (3, 1, False), (1, 0, False)):
            a, b = shard.output_range(nf, world, rank)
            sa, sb = shard.source_range(nf, world, rank, r, v2)
            t = torch.tensor([a, b, sa, sb], dtype=torch.int64)
            out = [torch.zeros(4, dtype=torch.int64) for _ in range(world)]
            dist.all_gather(out, t)
            res.append((nf, r, v2, [o.tolist() for o in out]))
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_frame_sharding_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == got[1]
    for nf, r, v2, ranges in got[0]:
        covered = []
        halo = 2 * r if v2 and r else r
        for a, b, sa, sb in ranges:
            covered += list(range(a, b))
            if a < b:
                assert sa == max(a - halo, 0) and sb == min(b + halo, nf)
        assert covered == list(range(nf))
