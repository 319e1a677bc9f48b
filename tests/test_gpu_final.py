"""The final (Wiener) pass on B200: BM3Dv2(clip, ref=basic_estimate).

Bars as for the basic estimate: match tables (block matching runs on ref)
identical to the oracle's, outputs within OUT_TOL of the reference's golden
vectors (bit-exact with an extractor), every entry point (host, device,
per-frame) agreeing, and the reference's own checks of the ref pass
(tests/test_bm3dv2.py:165-181): finite, deterministic, different from the
basic estimate.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import vsfeel
from vsfeel import _lib
from oracle import Params
from vsfeel.synthetic import make_chroma, make_clip

pytestmark = pytest.mark.gpu

OUT_TOL = 1e-4
TYPICAL_TOL = 2e-5

PARAMS = dict(sigma=6.0, block_step=4, bm_range=8, radius=1, ps_num=2, ps_range=3)


def _final(frames, ref, **params):
    return vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), ref=vsfeel.clip_from_array(ref), **params)


def test_golden_final_vectors(golden_final):
    worst = 0.0
    for name, params, frames, ref, expected in golden_final:
        out = _final(frames, ref, **params).output()
        err = float(np.abs(out.astype(np.float64) - expected).max())
        worst = max(worst, err)
        assert np.isfinite(out).all(), name
        assert err <= OUT_TOL, f"{name}: max abs err {err}"
        if params.get("extractor_exp"):
            assert np.array_equal(out, expected), name
    assert worst <= TYPICAL_TOL, worst


def test_final_pass_matches_on_ref(oracle_lib):
    import torch

    frames = make_clip(4, 48, 64, sigma=6.0, seed=21)
    basic = oracle_lib.bm3d(frames, Params(**PARAMS))
    node = _final(frames, basic, **PARAMS)
    ctx = node._ctx
    inf = node.info
    dev = torch.from_numpy(basic).cuda()
    for m in (0, 2, 3):
        table = np.empty((inf.blocks_x * inf.blocks_y, 8, 3), dtype=np.int32)
        ctx.check(ctx.lib.vsfeel_bm3d_match_table_device(ctx.handle, dev.data_ptr(), dev.stride(0),
                                                         dev.stride(1), m, table.ctypes.data))
        assert np.array_equal(table, oracle_lib.matches(basic, Params(**PARAMS), m)), m


@pytest.mark.parametrize("params", [PARAMS,
                                    dict(sigma=10.0, block_step=8, bm_range=9, radius=0),
                                    dict(sigma=8.0, block_step=4, bm_range=6, radius=3, ps_num=2,
                                         ps_range=2),
                                    dict(sigma=5.0, block_step=4, bm_range=16, radius=2, ps_num=2,
                                         ps_range=7)])
def test_final_pass_vs_oracle_and_entry_points(params, oracle_lib):
    import torch

    p = Params(**params)
    frames = make_clip(5, 64, 80, sigma=p.sigma, shift=3, seed=22)
    basic = oracle_lib.bm3d(frames, p)
    expected = oracle_lib.bm3d(frames, p, ref=basic)
    node = _final(frames, basic, **params)
    host = node.output()
    assert float(np.abs(host - expected).max()) <= OUT_TOL
    dev_out = torch.empty((5, 64, 80), device="cuda")
    node.output_device(torch.from_numpy(frames).cuda(), dev_out, ref=torch.from_numpy(basic).cuda())
    torch.cuda.synchronize()
    assert float(np.abs(dev_out.cpu().numpy() - host).max()) <= TYPICAL_TOL
    for n in (0, 2, 4):
        assert float(np.abs(node.get_frame(n)[0] - host[n]).max()) <= TYPICAL_TOL


def test_final_pass_properties():
    frames = make_clip(5, 64, 80, sigma=8.0, seed=23)
    basic = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **PARAMS).output()
    a = _final(frames, basic, **PARAMS).output()
    b = _final(frames, basic, **PARAMS).output()
    assert np.isfinite(a).all()
    assert float(np.abs(a - b).max()) <= 1e-5
    assert float(np.abs(a - basic).max()) > 1e-4


def test_final_pass_yuv_passthrough():
    n, h, w = 3, 48, 64
    luma = make_clip(n, h, w, sigma=6.0, seed=24)
    u = make_chroma(n, h // 2, w // 2, seed=1)
    v = make_chroma(n, h // 2, w // 2, seed=2)
    clip = vsfeel.clip_from_array(luma, u, v)
    basic = vsfeel.BM3Dv2(clip, **PARAMS)
    ref = vsfeel.clip_from_array(basic.output(), u, v)
    node = vsfeel.BM3Dv2(clip, ref=ref, **PARAMS)
    f = node.get_frame(1)
    assert np.array_equal(f[1], u[1]) and np.array_equal(f[2], v[1])
    gray = _final(luma, basic.output(), **PARAMS).get_frame(1)[0]
    assert float(np.abs(f[0] - gray).max()) <= 1e-5


def test_pass_and_entry_point_must_agree():
    import torch

    frames = make_clip(3, 32, 32, sigma=5.0, seed=25)
    final = _final(frames, frames, **PARAMS)
    basic = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **PARAMS)
    x = torch.from_numpy(frames).cuda()
    out = torch.empty_like(x)
    lib = final._ctx.lib
    rc = lib.vsfeel_bm3d_process_device(final._ctx.handle, x.data_ptr(), x.stride(0), x.stride(1),
                                        out.data_ptr(), out.stride(0), out.stride(1), 0, 3, None)
    assert rc == _lib.E_ARG and "runs the final pass" in _lib.last_error(lib)
    rc = lib.vsfeel_bm3d_process_device_ref(basic._ctx.handle, x.data_ptr(), x.stride(0),
                                            x.stride(1), x.data_ptr(), x.stride(0), x.stride(1),
                                            out.data_ptr(), out.stride(0), out.stride(1), 0, 3, None)
    assert rc == _lib.E_ARG and "no \"ref\" clip" in _lib.last_error(lib)
