"""Frame sharding of one clip across ranks (one process per GPU), and the
assignment of a batch's clips to ranks.

BM3Dv2 output frame n reads source frames n-2r .. n+2r only (the filter's
frame request, src/bm3d.cpp:704-712), so a clip splits into contiguous
output ranges with no exchange step: each rank denoises the sub-clip of its
range plus a 2r-frame halo on either side (clamped to the clip), keeping
only its own outputs. With the halo, every output's stacks, windows and
aggregation slices are the same as in the whole clip -- an output at least
2r frames inside the sub-clip sees no clamping there, and near a real clip
end the sub-clip ends there too -- so the shards reproduce the whole-clip
result. Ranks need no collective to compute; ``gather`` is the optional step
that brings the outputs to one rank.

Many clips (the batched form) need no split at all: ``assign_clips`` gives
whole clips to ranks, longest processing time first, by ``clip_cost``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Shard:
    rank: int
    out_first: int     # first output frame of this rank
    out_count: int     # number of output frames (may be 0)
    in_first: int      # first source frame the rank needs
    in_last: int       # last source frame the rank needs

    @property
    def in_count(self) -> int:
        return self.in_last - self.in_first + 1 if self.out_count else 0

    @property
    def local_first(self) -> int:
        """Index of out_first within the rank's sub-clip."""
        return self.out_first - self.in_first


def plan(num_frames: int, world: int, radius: int) -> list[Shard]:
    """Contiguous, balanced output ranges (sizes differ by at most one) and
    the source range each rank reads."""
    if num_frames <= 0 or world <= 0:
        raise ValueError("num_frames and world must be positive")
    if not 0 <= radius <= 4:
        raise ValueError("radius must be in range [0, 4]")
    base, extra = divmod(num_frames, world)
    out, first = [], 0
    for r in range(world):
        count = base + (1 if r < extra else 0)
        if count:
            lo = max(first - 2 * radius, 0)
            hi = min(first + count - 1 + 2 * radius, num_frames - 1)
        else:
            lo, hi = first, first - 1
        out.append(Shard(r, first, count, lo, hi))
        first += count
    return out


def denoise_shard(frames: np.ndarray, shard: Shard, denoise) -> np.ndarray:
    """Runs `denoise(subclip, local_first, count)` on the rank's sub-clip and
    returns its output frames (count, H, W)."""
    if shard.out_count == 0:
        return np.empty((0,) + frames.shape[1:], dtype=np.float32)
    sub = np.ascontiguousarray(frames[shard.in_first:shard.in_last + 1])
    return denoise(sub, shard.local_first, shard.out_count)


def cuda_denoiser(params: dict, device: int = 0):
    """The library's denoiser as a `denoise` callable for denoise_shard."""
    from . import BM3Dv2, clip_from_array

    def run(sub, first, count):
        return BM3Dv2(clip_from_array(sub), device=device, **params).output(first, count)

    return run


def gather(local: np.ndarray, shards: list[Shard], rank: int, group=None, dst: int = 0):
    """Collects every rank's output frames on rank `dst` (torch.distributed,
    any backend); returns the whole clip there and None elsewhere."""
    import torch
    import torch.distributed as dist

    parts = [None] * len(shards) if rank == dst else None
    dist.gather_object(np.ascontiguousarray(local), parts, dst=dst, group=group)
    if rank != dst:
        return None
    return np.concatenate([p for p in parts if p is not None and len(p)], axis=0)


# Measured on one B200 (CUDA events): the sliding matcher (radius < 3) at
# 1.609 ms per 1080p radius-2 stack of 368.5 M candidates (the autotuner's
# tile); the exact matcher (radius >= 3) at 46.6 ms per 3840x2160
# radius-4 stack of 4.28 G candidates; the filter and normalisation at
# 0.175 ms per 128,851 blocks.
MS_PER_SLIDING_CANDIDATE = 1.609 / 368.5e6
MS_PER_EXACT_CANDIDATE = 46.6 / 4.28e9
MS_PER_BLOCK = 0.175 / 128851


def _blocks(extent: int, step: int) -> int:
    # block positions x0 = b*step < extent - 8 + step (src/bm3d.comp:451-458)
    return max((extent - 9 + 2 * step) // step, 0)


def clip_cost(num_frames: int, height: int, width: int, params: dict) -> float:
    """Estimated milliseconds of one clip on one B200: per stack, every
    block's candidates (the spatial window plus ps_num temporal windows per
    searched frame, unclamped) at the matcher's measured cost per candidate,
    plus the filter's and normaliser's cost per block."""
    step = int(params.get("block_step", 8))
    R = int(params.get("bm_range", 9))
    r = int(params.get("radius", 0))
    P = int(params.get("ps_num", 2))
    Q = int(params.get("ps_range", 4))
    cand = (2 * R + 1) ** 2 + 2 * r * P * (2 * Q + 1) ** 2
    per = MS_PER_EXACT_CANDIDATE if r >= 3 else MS_PER_SLIDING_CANDIDATE
    blocks = _blocks(width, step) * _blocks(height, step)
    return num_frames * blocks * (cand * per + MS_PER_BLOCK)


def assign_clips(costs, world: int) -> list[list[int]]:
    """Longest processing time first: clips in falling cost (ties by index)
    each go to the rank with the least assigned cost so far (ties to the
    lower rank). Returns each rank's clip indices in ascending order. The
    largest load is at most 4/3 of the optimum plus nothing more than one
    clip can add, and the plan is the same on every rank."""
    if world <= 0:
        raise ValueError("world must be positive")
    costs = [float(c) for c in costs]
    if any(c < 0 for c in costs):
        raise ValueError("clip costs must be non-negative")
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        rk = min(range(world), key=lambda q: (load[q], q))
        out[rk].append(i)
        load[rk] += costs[i]
    return [sorted(x) for x in out]
