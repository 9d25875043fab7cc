"""Multi-process (gloo, world size 2) checks of the frame sharding used by
multi-GPU runs: every output frame is produced by exactly one rank and each
rank's source range covers its windows; and the two ranks' outputs of a temporal
BM3Dv2 clip (radius 1, CPU oracle), gathered and concatenated, equal the outputs
of one process filtering the whole clip."""
import os
import sys

import numpy as np

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


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle_v2_clip(frames, radius, sigma, bs=4, rng=6):
    """Temporal BM3Dv2 (step 1) of a gray clip on the CPU oracle: the accumulator stack of
    every centre's window, then the temporal aggregation of the stacks around each frame."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import ref_configs as rc
    nf = len(frames)
    h, w = frames[0].shape
    tw = 2 * radius + 1
    cfg = orc.make_cfg(w, h, w, [rc.scaled_sigma(sigma, False)], bs, rng, radius, nthreads=2)
    clamp = lambda i: min(max(i, 0), nf - 1)  # noqa: E731
    stacks = {}

    def stack(c):
        if c not in stacks:
            win = np.stack([frames[clamp(c - radius + t)] for t in range(tw)])
            num, den, _ = orc.bm3d_pass(cfg, win[None, None], want_matches=False)
            st = np.zeros((tw, 2, h, w), np.float32)
            st[:, 0], st[:, 1] = num[0], den[0]
            stacks[c] = st.reshape(tw * 2 * h, w)
        return stacks[c]

    def out(n):
        return orc.vaggregate_plane([stack(clamp(n - radius + i)) for i in range(tw)], w, h, w, radius, n, nf)
    return out


def _clip_frame(g):
    from zb3d import synth
    return synth.noisy_plane(40, 32, 12.0, clip=5, frame=g, motion=True)


def _sharded_worker(rank, world, port, q, nframes, radius):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard.run_rank(nframes, world, rank, _clip_frame,
                              lambda frames: _oracle_v2_clip(frames, radius, 12.0), radius=radius, v2=True)
        got = [None] * world
        dist.all_gather_object(got, [np.asarray(f).tolist() for f in mine])
        if rank == 0:
            q.put([np.array(f, np.float32) for part in got for f in part])
    finally:
        dist.destroy_process_group()


def test_sharded_temporal_outputs_equal_the_single_process_run():
    nframes, radius = 7, 1
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q, nframes, radius)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    single = _oracle_v2_clip([_clip_frame(g) for g in range(nframes)], radius, 12.0)
    assert len(gathered) == nframes
    for n in range(nframes):
        assert np.array_equal(gathered[n], single(n)), n
    # a halo one frame short changes the rank boundary's outputs: the check has teeth
    a, b = shard.output_range(nframes, 2, 1)
    short = _oracle_v2_clip([_clip_frame(g) for g in range(a - 1, nframes)], radius, 12.0)
    assert not np.array_equal(short(0 + 1), single(a))
