"""Batched form on B200: every clip of a mixed batch equals the plain path.

The batch groups clips by shape class and runs each class as one persistent
match-and-filter launch plus one normalise launch, captured in a CUDA graph.
Each clip's output must equal what the plain path gives for that clip alone
(within the float-atomic reordering bar of the other GPU tests), for every
tile shape, with and without the autotuner, across repeated runs and after
new input is written into the bound buffers.
"""

from __future__ import annotations

import numpy as np
import pytest

import vsfeel
from oracle import Params
from vsfeel.batch import Batch
from vsfeel.synthetic import make_clip

pytestmark = pytest.mark.gpu

TOL = 2e-5

# (frames, height, width, params): several classes, uneven sizes, two clips
# sharing a class, a radius-3 class and a tiny clip that take the
# direct-read kernels, an extractor
CLIPS = [
    (3, 96, 128, dict(sigma=5.0, block_step=4, bm_range=8, radius=1, ps_num=2, ps_range=3)),
    (5, 72, 88, dict(sigma=8.0, block_step=8, bm_range=12, radius=2, ps_num=2, ps_range=4)),
    (4, 64, 64, dict(sigma=3.0, block_step=4, bm_range=9, radius=0)),
    (6, 80, 96, dict(sigma=6.0, block_step=4, bm_range=8, radius=2, ps_num=2, ps_range=3)),
    (4, 48, 56, dict(sigma=9.0, block_step=4, bm_range=6, radius=3, ps_num=2, ps_range=2)),
    (3, 40, 48, dict(sigma=4.0, block_step=4, bm_range=8, radius=1, ps_num=2, ps_range=3,
                     extractor_exp=2)),
    (3, 9, 8, dict(sigma=7.0, block_step=4, bm_range=8, radius=1, ps_num=3, ps_range=3)),
]


def _inputs(seed=0):
    import torch

    src, dst = [], []
    for i, (n, h, w, p) in enumerate(CLIPS):
        frames = make_clip(n, h, w, sigma=p["sigma"], shift=3, seed=seed * 100 + i)
        src.append(torch.from_numpy(frames).cuda())
        dst.append(torch.full((n, h, w), float("nan"), device="cuda"))
    return src, dst


def _plain(src):
    import torch

    outs = []
    for t, (n, h, w, p) in zip(src, CLIPS):
        out = torch.empty_like(t)
        vsfeel.BM3Dv2(vsfeel.clip_from_array(t.cpu().numpy()), **p).output_device(t, out)
        outs.append(out)
    torch.cuda.synchronize()
    return outs


def _run(batch):
    import torch

    batch.run()
    torch.cuda.synchronize()
    batch.finish()


@pytest.mark.parametrize("mode", ["autotune", "default", "8x4", "16x2", "4x8", "8x2", "4x4",
                                  "8x4/16", "16x2/16", "4x4/16"])
def test_batch_equals_plain_path_per_clip(mode):
    """Every tile shape, with 8 lanes per reference block and (the /16
    cases) 16 lanes per block in 512-thread CTAs."""
    src, dst = _inputs()
    kw = dict(autotune=mode == "autotune")
    if mode not in ("autotune", "default"):
        shape, _, lanes = mode.partition("/")
        kw["tile_shape"] = shape
        if lanes:
            kw["lanes"] = int(lanes)
    batch = Batch([(s, d, p) for s, d, (_, _, _, p) in zip(src, dst, CLIPS)], **kw)
    _run(batch)
    for i, (out, ref) in enumerate(zip(dst, _plain(src))):
        assert bool(out.isfinite().all()), i
        err = float((out - ref).abs().max())
        assert err <= TOL, (i, err)


def test_batch_classes_and_direct_read_fallback():
    src, dst = _inputs()
    batch = Batch([(s, d, p) for s, d, (_, _, _, p) in zip(src, dst, CLIPS)], autotune=True)
    classes = batch.classes()
    keyed = {(c["radius"], c["block_step"], c["bm_range"], c["ps_num"], c["ps_range"]): c
             for c in classes}
    assert len(keyed) == len(classes) == 6
    assert keyed[(1, 4, 8, 2, 3)]["clips"] == 2           # clips 0 and 5 share a class
    assert keyed[(3, 4, 6, 2, 2)]["tile_shape"] == "direct"  # radius 3
    assert keyed[(1, 4, 8, 3, 3)]["tile_shape"] == "direct"  # seeds at (0, 0)
    # the autotuner times every fitting shape with 8 and 16 lanes per block
    # and keeps the fastest pair
    tuned = keyed[(2, 8, 12, 2, 4)]
    assert tuned["tile_shape"] in tuned["tuned_ms"]
    assert set(tuned["tuned_ms"]) == set(tuned["tuned_ms_16"])
    chosen = (tuned["tuned_ms"] if tuned["lanes"] == 8 else tuned["tuned_ms_16"])[tuned["tile_shape"]]
    assert chosen == min(list(tuned["tuned_ms"].values()) + list(tuned["tuned_ms_16"].values()))
    assert keyed[(3, 4, 6, 2, 2)]["lanes"] == 8   # direct-read classes report 8
    assert sum(c["stacks"] for c in classes) == sum(n for n, _, _, _ in CLIPS)
    assert batch.device_bytes > 0


def test_batch_merged_and_per_stack_output_slots_agree(monkeypatch):
    """Interior outputs of clips without the extractor keep one merged
    accumulator pair (the default) instead of one per stack
    (VSFEEL_MERGED_SLOTS=0): the same outputs within the bar, in less
    device memory. Longer clips than CLIPS' so that most outputs are
    interior."""
    import torch

    kws = [dict(sigma=5.0, block_step=4, bm_range=8, radius=2, ps_num=2, ps_range=3),
           dict(sigma=6.0, block_step=4, bm_range=8, radius=1, ps_num=2, ps_range=3),
           dict(sigma=4.0, block_step=4, bm_range=8, radius=1, ps_num=2, ps_range=3,
                extractor_exp=2)]
    src = [torch.from_numpy(make_clip(10, 64, 80, sigma=p["sigma"], shift=3, seed=40 + i)).cuda()
           for i, p in enumerate(kws)]
    outs, sizes = {}, {}
    for merged in ("0", "1"):
        monkeypatch.setenv("VSFEEL_MERGED_SLOTS", merged)
        dst = [torch.full_like(s, float("nan")) for s in src]
        batch = Batch(list(zip(src, dst, kws)), autotune=False)
        _run(batch)
        outs[merged], sizes[merged] = dst, batch.device_bytes
    for i, (a, b) in enumerate(zip(outs["0"], outs["1"])):
        assert bool(b.isfinite().all()), i
        assert float((a - b).abs().max()) <= TOL, i
    assert torch.equal(outs["0"][2], outs["1"][2])   # the extractor clip keeps its slices
    assert sizes["1"] < sizes["0"]


def test_batch_reruns_and_new_input():
    import torch

    src, dst = _inputs(seed=1)
    batch = Batch([(s, d, p) for s, d, (_, _, _, p) in zip(src, dst, CLIPS)], autotune=False)
    _run(batch)
    first = [d.clone() for d in dst]
    _run(batch)
    for a, b in zip(first, dst):
        assert float((a - b).abs().max()) <= 1e-5
    # new frames into the bound inputs, then run again
    new_src, _ = _inputs(seed=2)
    for s, n in zip(src, new_src):
        s.copy_(n)
    torch.cuda.synchronize()
    _run(batch)
    for i, (out, ref) in enumerate(zip(dst, _plain(src))):
        assert float((out - ref).abs().max()) <= TOL, i


def test_batch_matches_oracle_on_a_clip(oracle_lib):
    import torch

    src, dst = _inputs(seed=3)
    batch = Batch([(s, d, p) for s, d, (_, _, _, p) in zip(src, dst, CLIPS)])
    _run(batch)
    for i in (1, 3):
        n, h, w, p = CLIPS[i]
        expected = oracle_lib.bm3d(src[i].cpu().numpy(), Params(**p))
        assert float(np.abs(dst[i].cpu().numpy() - expected).max()) <= 1e-4


def test_batch_rejects_bad_clips():
    import torch

    x = torch.zeros((3, 32, 32), device="cuda")
    y = torch.zeros((3, 32, 32), device="cuda")
    with pytest.raises(vsfeel.Error, match="clip 1: \"radius\" must be in range"):
        Batch([(x, y, dict(radius=1)), (x, y, dict(radius=5))])
    with pytest.raises(vsfeel.Error, match="src and dst shapes differ"):
        Batch([(x, y[:, :16], dict(radius=1))])
