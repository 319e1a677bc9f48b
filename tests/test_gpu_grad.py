"""Differentiable form: the CUDA adjoint against FP64 references (B200).

The forward pass records the match table, the keep masks and the
denominators; with those frozen the denoiser is a linear map A of its input
and the adjoint kernel computes A^T g. The checks:

* the recorded forward equals the plain path, and the recorded match tables
  equal the plain path's;
* the FP64 frozen operator (oracle/frozen_operator.py) rebuilt from the
  recorded state reproduces the CUDA output (so the state is complete);
* dL/dx for L = sum(W * out), W ~ N(0, 1) seeded, against the FP64 PyTorch
  gradient of the frozen operator (relative error <= GRAD_TOL) and against
  FP64 central differences with h = 1e-6 on seeded pixels.

GRAD_TOL is the relative error bar: ||g - g_ref|| / ||g_ref|| over all
pixels, and max |g - g_ref| / max |g_ref| per element.
"""

from __future__ import annotations

import numpy as np
import pytest

import vsfeel
from vsfeel import _lib
from vsfeel.autograd import BM3DFunction, Denoiser, bm3d
from vsfeel.synthetic import make_clip
from oracle.frozen_operator import SavedState

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-5
OUT_TOL_FP64 = 2e-5   # FP64 frozen operator vs the FP32 CUDA output

C4 = dict(sigma=5.0, block_step=4, bm_range=12, radius=1, ps_num=2, ps_range=5)


def _setup(n, h, w, seed, shift=3, **params):
    import torch

    frames = make_clip(n, h, w, sigma=params.get("sigma", 3.0), shift=shift, seed=seed)
    x = torch.from_numpy(frames).cuda()
    den = Denoiser(x.shape, 0, **params)
    return frames, x, den


def _state(den, saved):
    n, h, w = den.shape
    return SavedState(saved, den.layout, n, h, w, den.info.radius, device="cuda")


def _rel(g, ref):
    g, ref = g.double(), ref.double()
    norm = float((g - ref).norm() / ref.norm())
    elem = float((g - ref).abs().max() / ref.abs().max())
    return norm, elem


CASES = [
    ("r1_small", 6, 96, 128, dict(C4)),
    ("r0", 4, 80, 96, dict(sigma=8.0, block_step=4, bm_range=9, radius=0)),
    ("r2_clip_ends", 3, 64, 80, dict(sigma=6.0, block_step=4, bm_range=8, radius=2, ps_num=2,
                                     ps_range=3)),
    ("r4_step8", 10, 72, 88, dict(sigma=10.0, block_step=8, bm_range=10, radius=4, ps_num=3,
                                  ps_range=4)),
    ("extractor", 5, 64, 96, dict(sigma=8.0, block_step=4, bm_range=8, radius=1, ps_num=2,
                                  ps_range=4, extractor_exp=2)),
]


@pytest.mark.parametrize("name,n,h,w,params", CASES, ids=[c[0] for c in CASES])
def test_recorded_forward_equals_plain_path(name, n, h, w, params):
    import torch

    frames, x, den = _setup(n, h, w, seed=71, **params)
    out, saved = den.forward_saved(x)
    plain = torch.empty_like(x)
    vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **params).output_device(x, plain)
    torch.cuda.synchronize()
    assert float((out - plain).abs().max()) <= 2e-5
    # recorded match tables are the plain path's
    st = _state(den, saved)
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **params)
    ctx = node._ctx
    nb = st.nblocks
    for m in sorted({0, n // 2, n - 1}):
        table = np.empty((nb, 8, 3), dtype=np.int32)
        ctx.check(ctx.lib.vsfeel_bm3d_match_table_device(ctx.handle, x.data_ptr(), x.stride(0),
                                                         x.stride(1), m, table.ctypes.data))
        assert np.array_equal(table[:, :, 0], st.x[m].cpu().numpy())
        assert np.array_equal(table[:, :, 1], st.y[m].cpu().numpy())
        assert np.array_equal(table[:, :, 2], st.z[m].cpu().numpy())


@pytest.mark.parametrize("name,n,h,w,params", CASES, ids=[c[0] for c in CASES])
def test_fp64_frozen_operator_reproduces_forward(name, n, h, w, params):
    import torch

    frames, x, den = _setup(n, h, w, seed=72, **params)
    out, saved = den.forward_saved(x)
    torch.cuda.synchronize()
    st = _state(den, saved)
    # the recorded denominators are the weights' sums; with an extractor
    # every scattered weight is rounded to a multiple of ulp(2^exp)
    dref = st.denominators()
    den_tol = 1e-6 if not params.get("extractor_exp") else 2e-4
    assert float(((dref - st.den) / dref).abs().max()) <= den_tol
    ref = st.apply(x.double())
    tol = OUT_TOL_FP64 if not params.get("extractor_exp") else 1e-4
    assert float((ref - out.double()).abs().max()) <= tol


@pytest.mark.parametrize("name,n,h,w,params", [CASES[0], CASES[4]], ids=["r1_small", "extractor"])
def test_fused_tiles_record_the_same_state(name, n, h, w, params, monkeypatch):
    """The fused match-and-filter tiles (VSFEEL_FUSED_FILTER=1, shared-memory
    accumulation of the reference slice) record keep bits and denominators
    from which the FP64 frozen operator reproduces their output, and give
    the plain path's output."""
    import torch

    monkeypatch.setenv("VSFEEL_FUSED_FILTER", "1")
    frames, x, den = _setup(n, h, w, seed=74, **params)
    out, saved = den.forward_saved(x)
    torch.cuda.synchronize()
    st = _state(den, saved)
    dref = st.denominators()
    den_tol = 1e-6 if not params.get("extractor_exp") else 2e-4
    assert float(((dref - st.den) / dref).abs().max()) <= den_tol
    tol = OUT_TOL_FP64 if not params.get("extractor_exp") else 1e-4
    assert float((st.apply(x.double()) - out.double()).abs().max()) <= tol
    monkeypatch.delenv("VSFEEL_FUSED_FILTER")
    plain = torch.empty_like(x)
    vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **params).output_device(x, plain)
    torch.cuda.synchronize()
    assert float((out - plain).abs().max()) <= 2e-5


@pytest.mark.parametrize("name,n,h,w,params", CASES, ids=[c[0] for c in CASES])
def test_gradient_vs_fp64_reference(name, n, h, w, params):
    import torch

    frames, x, den = _setup(n, h, w, seed=73, **params)
    weights = torch.from_numpy(np.random.default_rng(5).standard_normal((n, h, w))).cuda()
    xr = x.clone().requires_grad_(True)
    out = den(xr)
    (out.double() * weights).sum().backward()
    g = xr.grad.detach()

    _, saved = den.forward_saved(x)
    st = _state(den, saved)
    x64 = x.double().requires_grad_(True)
    (st.apply(x64) * weights).sum().backward()
    norm, elem = _rel(g, x64.grad)
    assert norm <= GRAD_TOL and elem <= GRAD_TOL, (norm, elem)


def test_gradient_vs_central_differences_512x512_r1():
    """The differentiable workload: 16 frames 512x512, radius 1, sigma 5,
    block_step 4, bm_range 12, ps_num 2, ps_range 5; 256 seeded pixels."""
    import torch

    frames, x, den = _setup(16, 512, 512, seed=4, **C4)
    weights = torch.from_numpy(np.random.default_rng(6).standard_normal((16, 512, 512))).cuda()
    xr = x.clone().requires_grad_(True)
    (den(xr).double() * weights).sum().backward()
    g = xr.grad.detach()

    _, saved = den.forward_saved(x)
    st = _state(den, saved)
    rng = np.random.default_rng(7)
    pix = np.stack([rng.integers(0, 16, 256), rng.integers(0, 512, 256),
                    rng.integers(0, 512, 256)], axis=1)
    fd = st.central_differences(x.double(), weights, pix, h=1e-6)
    gs = g[pix[:, 0], pix[:, 1], pix[:, 2]].double().cpu()
    norm, elem = _rel(gs, fd)
    assert norm <= GRAD_TOL and elem <= GRAD_TOL, (norm, elem)

    # and the whole gradient against the FP64 autograd reference
    x64 = x.double().requires_grad_(True)
    (st.apply(x64) * weights).sum().backward()
    norm, elem = _rel(g, x64.grad)
    assert norm <= GRAD_TOL and elem <= GRAD_TOL, (norm, elem)


def test_functional_form_and_gradient_flow():
    import torch

    frames, x, _ = _setup(4, 64, 64, seed=9, sigma=5.0, block_step=4, bm_range=8, radius=1)
    xr = x.clone().requires_grad_(True)
    y = bm3d(xr, sigma=5.0, block_step=4, bm_range=8, radius=1)
    assert y.requires_grad
    y.sum().backward()
    assert xr.grad is not None and torch.isfinite(xr.grad).all()
    # the frozen operator maps a constant clip to itself (only the DC, which
    # is always kept, survives), so sum(A^T 1) = sum(A 1) = N*H*W
    assert abs(float(xr.grad.double().sum()) - 4 * 64 * 64) <= 1e-4 * 4 * 64 * 64


def test_rejects_misaligned_saved_state_and_wrong_shapes():
    import torch

    frames, x, den = _setup(3, 64, 64, seed=10, sigma=5.0, radius=1)
    out = torch.empty_like(x)
    buf = torch.empty(int(den.layout.bytes) + 512, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = den.lib.vsfeel_bm3d_forward_saved(den.handle, x.data_ptr(), x.stride(0), x.stride(1),
                                           out.data_ptr(), out.stride(0), out.stride(1),
                                           buf.data_ptr() + 16, stream)
    assert rc == _lib.E_ARG
    assert "256-byte aligned" in _lib.last_error(den.lib)
    with pytest.raises(vsfeel.Error):
        den.forward_saved(x[:, :32])
