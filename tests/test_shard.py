"""Frame sharding across ranks (CPU): plans, halos and a world-size-2 run.

The per-rank compute is the oracle here (the sharding logic is what is
tested: which outputs each rank owns, which source frames it reads, and that
the shards reproduce the whole clip bit for bit); the GPU path runs the same
plan with the CUDA denoiser in test_gpu_parity.py.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from oracle import Oracle, Params
from vsfeel import shard
from vsfeel.synthetic import make_clip

PARAMS = dict(sigma=6.0, block_step=4, bm_range=5, radius=2, ps_num=2, ps_range=2)


def _oracle_denoise(params):
    o = Oracle()
    p = Params(**params)
    return lambda sub, first, count: o.bm3d(sub, p, out_first=first, out_count=count, nthreads=2)


@pytest.mark.parametrize("n,world,r", [(1, 1, 0), (7, 2, 1), (9, 3, 2), (5, 4, 2), (3, 5, 1),
                                       (24, 8, 4), (10, 3, 0)])
def test_plan_covers_every_output_once(n, world, r):
    plans = shard.plan(n, world, r)
    assert [s.rank for s in plans] == list(range(world))
    outs = [f for s in plans for f in range(s.out_first, s.out_first + s.out_count)]
    assert outs == list(range(n))
    counts = [s.out_count for s in plans]
    assert max(counts) - min(counts) <= 1
    for s in plans:
        if s.out_count:
            assert s.in_first == max(s.out_first - 2 * r, 0)
            assert s.in_last == min(s.out_first + s.out_count - 1 + 2 * r, n - 1)
            assert 0 <= s.local_first <= 2 * r


def test_plan_rejects_bad_arguments():
    with pytest.raises(ValueError):
        shard.plan(0, 2, 1)
    with pytest.raises(ValueError):
        shard.plan(4, 2, 5)


@pytest.mark.parametrize("n,world,params", [
    (7, 2, PARAMS),
    (6, 3, dict(PARAMS, radius=1)),
    (5, 2, dict(PARAMS, radius=0)),
    (9, 4, dict(PARAMS, radius=2, extractor_exp=2)),
])
def test_shards_reproduce_the_whole_clip(n, world, params):
    frames = make_clip(n, 40, 48, sigma=params["sigma"], shift=2, seed=n * 10 + world)
    whole = Oracle().bm3d(frames, Params(**params), nthreads=2)
    parts = [shard.denoise_shard(frames, s, _oracle_denoise(params))
             for s in shard.plan(n, world, params["radius"])]
    assert np.array_equal(np.concatenate(parts, axis=0), whole)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        n = 7
        frames = make_clip(n, 40, 48, sigma=PARAMS["sigma"], shift=2, seed=5)
        plans = shard.plan(n, world, PARAMS["radius"])
        local = shard.denoise_shard(frames, plans[rank], _oracle_denoise(PARAMS))
        full = shard.gather(local, plans, rank)
        if rank == 0:
            np.save(out_path, full)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_world_size_two_gloo(tmp_path):
    import torch.multiprocessing as mp

    out = tmp_path / "full.npy"
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True,
                       start_method="spawn")
    full = np.load(out)
    frames = make_clip(7, 40, 48, sigma=PARAMS["sigma"], shift=2, seed=5)
    assert np.array_equal(full, Oracle().bm3d(frames, Params(**PARAMS), nthreads=2))


def test_frame_ranges_generate_alone_and_agree_with_the_whole_clip():
    """The multi-GPU bench builds each rank's sub-clip alone
    (make_clip_range); every range must equal the same frames of the whole
    clip, and its clean frames make_clip's."""
    from vsfeel.synthetic import make_clip_range

    total = 12
    whole = make_clip_range(total, 0, total, 40, 56, sigma=3.0, shift=4, seed=2000)
    for sh in shard.plan(total, 3, 2):
        part = make_clip_range(total, sh.in_first, sh.in_count, 40, 56, sigma=3.0, shift=4,
                               seed=2000)
        assert np.array_equal(part, whole[sh.in_first:sh.in_last + 1])
    clean = make_clip(total, 40, 56, sigma=0.0, shift=4, seed=2000)
    assert np.array_equal(make_clip_range(total, 0, total, 40, 56, sigma=0.0, shift=4, seed=2000),
                          clean)
    with pytest.raises(ValueError):
        make_clip_range(total, 10, 5, 40, 56)


@pytest.mark.parametrize("world,r", [(1, 2), (2, 2), (4, 2), (8, 2), (8, 4)])
def test_halo_recompute_fraction_of_the_sharded_bench(world, r):
    """Stacks a sharded run computes beyond one per output frame: each
    interior side of a shard adds r stacks (its halo outputs' stacks), so
    for 32 outputs per rank the fraction is 2r(N-1)/(32N)."""
    nfr = 32
    plans = shard.plan(nfr * world, world, r)

    def stacks(s):
        lo = max(s.local_first - r, 0)
        hi = min(s.local_first + s.out_count - 1 + r, s.in_count - 1)
        return hi - lo + 1

    frac = sum(stacks(s) for s in plans) / (nfr * world) - 1.0
    assert abs(frac - 2 * r * (world - 1) / (nfr * world)) < 1e-12
