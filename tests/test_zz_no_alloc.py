"""The allocation-free entry point (vsfeel_bm3d_process_device_noalloc).

It exists for callers that cannot let the library allocate device memory --
processes that reserve the GPU in their own fixed pools, and pipelines that
must not take cudaMalloc/cudaFree's implicit device synchronisation -- and
keeps all its scratch in one static device array. Called through the C ABI
twice in a row, it must give what the allocating entry point gives, within
the tolerance of the other GPU tests (the two differ only in the order of
float atomic adds). The file is named so that pytest collects it last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import vsfeel
from vsfeel import _lib
from vsfeel.synthetic import make_clip

pytestmark = pytest.mark.gpu

TOL = 2e-5


def _args(**kw):
    args, _ = vsfeel._make_args(None, kw.get("sigma"), kw.get("block_step"), kw.get("bm_range"),
                                kw.get("radius"), kw.get("ps_num"), kw.get("ps_range"), None,
                                kw.get("extractor_exp"))
    return args


@pytest.mark.parametrize("kw", [
    dict(sigma=5.0, block_step=4, bm_range=12, radius=1, ps_num=2, ps_range=5),
    dict(sigma=3.0, block_step=8, bm_range=9, radius=0),
    dict(sigma=8.0, block_step=4, bm_range=16, radius=2, ps_num=2, ps_range=7, extractor_exp=2),
])
def test_noalloc_matches_allocating_entry_point_twice(kw):
    import torch

    lib = _lib.load()
    frames = make_clip(6, 96, 128, sigma=kw["sigma"], shift=4, seed=31)
    n, h, w = frames.shape
    src = torch.from_numpy(frames).cuda()
    expected = torch.empty_like(src)
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **kw)
    node.output_device(src, expected)
    torch.cuda.synchronize()

    args = _args(**kw)
    vi = _lib.VideoInfo(w, h, n, _lib.CF_GRAY, _lib.ST_FLOAT, 32, 0, 0)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out = torch.full_like(src, float("nan"))
        rc = lib.vsfeel_bm3d_process_device_noalloc(
            ctypes.byref(args), ctypes.byref(vi), src.data_ptr(), src.stride(0), src.stride(1),
            out.data_ptr(), out.stride(0), out.stride(1), 0, n, stream)
        assert rc == _lib.OK, _lib.last_error(lib)
        torch.cuda.synchronize()
        diff = (out - expected).abs().max().item()
        assert diff <= TOL, diff


@pytest.mark.parametrize("first,count,kw", [
    (2, 2, dict(sigma=5.0, block_step=4, bm_range=12, radius=2, ps_num=2, ps_range=5)),
    (5, 2, dict(sigma=5.0, block_step=4, bm_range=12, radius=2, ps_num=2, ps_range=5)),
    (0, 3, dict(sigma=6.0, block_step=4, bm_range=10, radius=3, ps_num=4, ps_range=4)),
    (3, 4, dict(sigma=8.0, block_step=4, bm_range=16, radius=3, ps_num=4, ps_range=7,
                extractor_exp=2)),
])
def test_noalloc_sub_ranges_and_radius3(first, count, kw):
    """Output ranges that start inside the clip (dst indexed from n - first,
    the slot ring starting mid-clip) or end before it does, and the radius-3
    exact matcher, against the allocating entry point on the same range."""
    import torch

    lib = _lib.load()
    frames = make_clip(7, 96, 128, sigma=kw["sigma"], shift=4, seed=32)
    n, h, w = frames.shape
    src = torch.from_numpy(frames).cuda()
    expected = torch.empty((count, h, w), device="cuda")
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **kw)
    node.output_device(src, expected, first=first, count=count)
    torch.cuda.synchronize()

    args = _args(**kw)
    vi = _lib.VideoInfo(w, h, n, _lib.CF_GRAY, _lib.ST_FLOAT, 32, 0, 0)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out = torch.full((count, h, w), float("nan"), device="cuda")
        rc = lib.vsfeel_bm3d_process_device_noalloc(
            ctypes.byref(args), ctypes.byref(vi), src.data_ptr(), src.stride(0), src.stride(1),
            out.data_ptr(), out.stride(0), out.stride(1), first, count, stream)
        assert rc == _lib.OK, _lib.last_error(lib)
        torch.cuda.synchronize()
        diff = (out - expected).abs().max().item()
        assert diff <= TOL, diff


def test_noalloc_rejects_clips_beyond_its_scratch():
    import torch

    lib = _lib.load()
    limit = lib.vsfeel_bm3d_noalloc_scratch_bytes()
    assert limit == 32 << 20
    # 4K at radius 2 needs 25 pairs of 33 MB accumulator planes
    w, h, n = 3840, 2160, 3
    src = torch.zeros((n, h, w), dtype=torch.float32, device="cuda")
    out = torch.empty_like(src)
    args = _args(radius=2)
    vi = _lib.VideoInfo(w, h, n, _lib.CF_GRAY, _lib.ST_FLOAT, 32, 0, 0)
    rc = lib.vsfeel_bm3d_process_device_noalloc(
        ctypes.byref(args), ctypes.byref(vi), src.data_ptr(), src.stride(0), src.stride(1),
        out.data_ptr(), out.stride(0), out.stride(1), 0, n, None)
    assert rc == _lib.E_ARG
    assert "too large for the allocation-free entry point" in _lib.last_error(lib)
