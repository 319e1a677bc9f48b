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


# ---------------------------------------------------------------------------
# Many clips across ranks (the batched form): whole clips, longest processing
# time first.

@pytest.mark.parametrize("world", [1, 2, 3, 5, 8, 70])
def test_assign_clips_gives_every_clip_to_one_rank_and_balances(world):
    rng = np.random.default_rng(world)
    costs = list(rng.uniform(0.5, 40.0, size=64))
    plan = shard.assign_clips(costs, world)
    assert len(plan) == world
    flat = sorted(i for part in plan for i in part)
    assert flat == list(range(64))
    loads = [sum(costs[i] for i in part) for part in plan]
    # greedy by falling cost: no rank ends more than one clip above the mean
    assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
    assert plan == shard.assign_clips(costs, world)   # the same plan on every rank
    for part in plan:
        assert part == sorted(part)


def test_assign_clips_takes_the_largest_first_and_breaks_ties_by_index():
    assert shard.assign_clips([1.0, 5.0, 1.0, 3.0], 2) == [[1], [0, 2, 3]]
    assert shard.assign_clips([2.0, 2.0, 2.0, 2.0], 2) == [[0, 2], [1, 3]]
    assert shard.assign_clips([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard.assign_clips([1.0], 0)
    with pytest.raises(ValueError):
        shard.assign_clips([-1.0], 1)


def test_clip_cost_follows_the_work():
    p2 = dict(sigma=3.0, block_step=4, bm_range=16, radius=2, ps_num=2, ps_range=7)
    c1080 = shard.clip_cost(32, 1080, 1920, p2)
    assert abs(c1080 - 32 * (1.609 + 0.175)) / c1080 < 0.01   # the measured 1080p r2 stack
    assert shard.clip_cost(32, 2160, 3840, p2) > 3.9 * c1080
    assert shard.clip_cost(32, 1080, 1920, dict(p2, radius=1)) < c1080
    assert shard.clip_cost(32, 1080, 1920, dict(p2, block_step=8)) < c1080 / 3
    # the exact search (radius >= 3) costs more per candidate
    p4 = dict(p2, radius=4, ps_num=4)
    cand4 = 33 ** 2 + 2 * 4 * 4 * 15 ** 2
    assert shard.clip_cost(1, 1080, 1920, p4) > 128851 * cand4 * shard.MS_PER_SLIDING_CANDIDATE
    assert shard.clip_cost(0, 1080, 1920, p2) == 0.0


def test_assign_the_batched_workload():
    """The 64-clip workload's plan: even at 2 and 4 ranks; at 8 the largest
    clip (a 3840x2160 radius-2 clip) bounds the largest load."""
    spec = []
    rng = np.random.default_rng(3000)
    sizes = [(640, 360)] * 16 + [(1280, 720)] * 24 + [(1920, 1080)] * 16 + [(3840, 2160)] * 8
    for w, h in sizes:
        spec.append((16, h, w, dict(sigma=float(rng.uniform(1.0, 10.0)),
                                    block_step=int(rng.choice([4, 8])), bm_range=16,
                                    radius=int(rng.choice([0, 1, 2])), ps_num=2, ps_range=7)))
    costs = [shard.clip_cost(*s) for s in spec]
    for world in (2, 4, 8):
        loads = [sum(costs[i] for i in part) for part in shard.assign_clips(costs, world)]
        assert max(loads) <= max(1.01 * sum(costs) / world, max(costs) + 1e-9), world


SMALL_CLIPS = [
    (4, 40, 48, dict(sigma=6.0, block_step=4, bm_range=5, radius=1, ps_num=2, ps_range=2)),
    (3, 32, 40, dict(sigma=4.0, block_step=4, bm_range=4, radius=0)),
    (5, 36, 44, dict(sigma=7.0, block_step=3, bm_range=4, radius=2, ps_num=2, ps_range=2)),
    (3, 24, 32, dict(sigma=5.0, block_step=4, bm_range=4, radius=1, ps_num=1, ps_range=2,
                     extractor_exp=2)),
    (2, 48, 40, dict(sigma=3.0, block_step=8, bm_range=6, radius=0)),
]


def _small_clip(i):
    n, h, w, p = SMALL_CLIPS[i]
    return make_clip(n, h, w, sigma=p["sigma"], shift=2, seed=600 + i)


def _clips_rank_main(rank, world, port, out_path):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        costs = [shard.clip_cost(*c) for c in SMALL_CLIPS]
        mine = shard.assign_clips(costs, world)[rank]
        o = Oracle()
        local = {i: o.bm3d(_small_clip(i), Params(**SMALL_CLIPS[i][3]), nthreads=2) for i in mine}
        parts = [None] * world if rank == 0 else None
        dist.gather_object(local, parts, dst=0)
        if rank == 0:
            merged = {}
            for part in parts:
                assert not set(part) & set(merged)   # no clip on two ranks
                merged.update(part)
            np.savez(out_path, **{str(i): merged[i] for i in sorted(merged)})
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_clips_across_two_gloo_ranks(tmp_path):
    """Each rank denoises the clips the plan gives it (the oracle stands in
    for the per-rank batch); gathered on rank 0, every clip is there once and
    equals the single-process result."""
    import torch.multiprocessing as mp

    out = tmp_path / "clips.npz"
    mp.start_processes(_clips_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    assert sorted(int(k) for k in got.files) == list(range(len(SMALL_CLIPS)))
    o = Oracle()
    for i, (_, _, _, p) in enumerate(SMALL_CLIPS):
        assert np.array_equal(got[str(i)], o.bm3d(_small_clip(i), Params(**p), nthreads=2)), i
