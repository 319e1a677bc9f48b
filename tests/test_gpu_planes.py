"""Per-plane denoising (the ``planes`` extension) vs the oracle (B200).

The reference parses sigma, block_step, bm_range, ps_num and ps_range per
plane and applies element [0] to luma only (src/bm3d.cpp:1090-1167,
1265-1272). With ``planes`` every listed plane is denoised with its own
element; the oracle restates the same algorithm on that plane, so each
plane must agree with the oracle run on the plane alone, match tables
bit-exact and outputs within the parity bar.
"""

from __future__ import annotations

import numpy as np
import pytest

import vsfeel
from oracle import Params
from vsfeel.synthetic import make_clip

pytestmark = pytest.mark.gpu

OUT_TOL = 1e-4        # parity bar, max abs error on the [0, 1] scale
TYPICAL_TOL = 2e-5    # what float-atomic reordering costs in the basic pass

PLANE_ARGS = dict(sigma=[3.0, 6.0, 9.0], block_step=[4, 3, 2], bm_range=[12, 6],
                  radius=1, ps_num=[2, 3, 1], ps_range=[5, 4, 3])


def _plane_params(p: int) -> Params:
    def pick(v):
        return v[min(p, len(v) - 1)] if isinstance(v, list) else v
    return Params(**{k: pick(v) for k, v in PLANE_ARGS.items()})


def _yuv420(n=6, h=64, w=96, seed=40):
    luma = make_clip(n, h, w, sigma=3.0, shift=3, seed=seed)
    u = make_clip(n, h // 2, w // 2, sigma=6.0, shift=2, seed=seed + 1)
    v = make_clip(n, h // 2, w // 2, sigma=9.0, shift=2, seed=seed + 2)
    return vsfeel.clip_from_array(luma, u, v)


def test_every_plane_matches_the_oracle_on_that_plane(oracle_lib):
    clip = _yuv420()
    node = vsfeel.BM3Dv2(clip, planes=[0, 1, 2], **PLANE_ARGS)
    assert node.planes == [0, 1, 2]
    expected = [oracle_lib.bm3d(clip.plane_array(p), _plane_params(p)) for p in range(3)]
    for p in range(3):
        inf = node.plane_info(p)
        assert (inf.width, inf.height) == clip.plane_array(p).shape[:0:-1]
        assert inf.block_step == _plane_params(p).block_step
        out = node.output(plane=p)
        assert np.abs(out.astype(np.float64) - expected[p]).max() <= TYPICAL_TOL, p
    for n in (0, 3, 5):
        f = node.get_frame(n)
        for p in range(3):
            assert np.abs(f[p].astype(np.float64) - expected[p][n]).max() <= TYPICAL_TOL, (n, p)


def test_chroma_match_tables_identical(oracle_lib):
    import torch
    clip = _yuv420(n=4, seed=50)
    node = vsfeel.BM3Dv2(clip, planes=[1, 2], **PLANE_ARGS)
    for p in (1, 2):
        ctx = node._ctxs[p]
        inf = node.plane_info(p)
        frames = clip.plane_array(p)
        dev = torch.from_numpy(np.ascontiguousarray(frames)).cuda()
        table = np.empty((inf.blocks_x * inf.blocks_y, 8, 3), dtype=np.int32)
        for m in (0, 2, 3):
            ctx.check(ctx.lib.vsfeel_bm3d_match_table_device(
                ctx.handle, dev.data_ptr(), dev.stride(0), dev.stride(1), m, table.ctypes.data))
            assert np.array_equal(table, oracle_lib.matches(frames, _plane_params(p), m)), (p, m)


def test_unlisted_planes_pass_through():
    clip = _yuv420(n=4, seed=60)
    node = vsfeel.BM3Dv2(clip, planes=[2], **PLANE_ARGS)
    f = node.get_frame(1)
    assert np.array_equal(f[0], clip.plane_array(0)[1])
    assert np.array_equal(f[1], clip.plane_array(1)[1])
    assert not np.array_equal(f[2], clip.plane_array(2)[1])


def test_default_planes_keep_reference_behaviour():
    clip = _yuv420(n=4, seed=70)
    node = vsfeel.BM3Dv2(clip, **PLANE_ARGS)
    assert node.planes == [0]
    f = node.get_frame(2)
    assert np.array_equal(f[1], clip.plane_array(1)[2])
    assert np.array_equal(f[2], clip.plane_array(2)[2])


def test_device_entry_point_per_plane():
    import torch
    clip = _yuv420(n=5, seed=80)
    node = vsfeel.BM3Dv2(clip, planes=[0, 1], **PLANE_ARGS)
    host = node.output(plane=1)
    src = torch.from_numpy(np.ascontiguousarray(clip.plane_array(1))).cuda()
    out = torch.empty_like(src)
    node.output_device(src, out, plane=1)
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy() - host).max() < 1e-5


def test_final_pass_per_plane_vs_oracle(oracle_lib):
    clip = _yuv420(n=5, seed=90)
    basic = vsfeel.BM3Dv2(clip, planes=[0, 1, 2], **PLANE_ARGS)
    est = [basic.output(plane=p) for p in range(3)]
    ref = vsfeel.clip_from_array(est[0], est[1], est[2])
    final = vsfeel.BM3Dv2(clip, ref=ref, planes=[1, 2], **PLANE_ARGS)
    assert final.final_pass
    for p in (1, 2):
        expected = oracle_lib.bm3d(clip.plane_array(p), _plane_params(p), ref=est[p])
        out = final.output(plane=p)
        assert np.abs(out.astype(np.float64) - expected).max() <= OUT_TOL, p


def test_node_as_ref_uses_its_denoised_planes(oracle_lib):
    """A BM3DNode stands in for a clip: as ``ref`` it supplies its output."""
    clip = _yuv420(n=4, seed=95)
    basic = vsfeel.BM3Dv2(clip, planes=[0, 2], **PLANE_ARGS)
    assert np.array_equal(basic.plane_array(1), clip.plane_array(1))
    est2 = basic.output(plane=2)
    assert np.abs(basic.plane_array(2) - est2).max() <= TYPICAL_TOL
    final = vsfeel.BM3Dv2(clip, ref=basic, planes=[2], **PLANE_ARGS)
    expected = oracle_lib.bm3d(clip.plane_array(2), _plane_params(2), ref=basic.plane_array(2))
    assert np.abs(final.output(plane=2).astype(np.float64) - expected).max() <= OUT_TOL
