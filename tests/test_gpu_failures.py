"""Failure handling on B200, injected on the host (no GPU fault is made).

* a frame callback that returns no frame -> VSFEEL_E_FETCH, and the context
  stays usable;
* a callback stride below the width -> VSFEEL_E_ARG;
* a bounded wait that runs out (VSFEEL_TIMEOUT_MS = 1 ms against ~15 ms of
  GPU work, pinned buffers so that the copies do not block the host) ->
  VSFEEL_E_TIMEOUT, after which the context still works once the limit is
  back to normal;
* the kernels' status word: a test hook (VSFEEL_TEST_PROBE_TILE) makes one
  tile's staged-region check report a window outside the region. The tile
  sets the word and skips its scan -- no out-of-range access is made -- and
  the host must turn the word into VSFEEL_E_CUDA "internal error", through
  the whole-clip path and the per-frame path, after which the same context
  denoises correctly again.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import vsfeel
from vsfeel import _lib
from vsfeel.synthetic import make_clip

pytestmark = pytest.mark.gpu

PARAMS = dict(sigma=5.0, block_step=4, bm_range=8, radius=1, ps_num=2, ps_range=3)


def _get_frame(node, n, fetch, release=None):
    ctx = node._ctx
    out = np.empty((node.height, node.width), dtype=np.float32)
    rel = release or _lib.RELEASE_FN(lambda user, f: None)
    rc = ctx.lib.vsfeel_bm3d_get_frame(ctx.handle, n, fetch, rel, None, out.ctypes.data,
                                       out.strides[0])
    return rc, out


def test_fetch_failure_is_reported_and_the_context_recovers():
    frames = make_clip(4, 48, 64, sigma=5.0, seed=3)
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **PARAMS)
    released = []

    @_lib.FETCH_FN
    def failing(user, f, stride):
        if f == 2:
            return None
        stride[0] = frames.strides[1]
        return frames[f].ctypes.data

    @_lib.RELEASE_FN
    def release(user, f):
        released.append(f)

    # output 1 at radius 1 reads frames 0..3; frame 2 fails after 0 and 1
    rc, _ = _get_frame(node, 1, failing, release)
    assert rc == _lib.E_FETCH
    assert _lib.last_error(node._ctx.lib) == "BM3D: could not fetch source frame 2"
    assert released == [0, 1]
    # the context still denoises
    ref = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **PARAMS).get_frame(1)[0]
    assert float(np.abs(node.get_frame(1)[0] - ref).max()) <= 2e-5


def test_callback_stride_below_width_is_rejected():
    frames = make_clip(3, 48, 64, sigma=5.0, seed=4)
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **PARAMS)

    @_lib.FETCH_FN
    def short_stride(user, f, stride):
        stride[0] = 16
        return frames[f].ctypes.data

    rc, _ = _get_frame(node, 0, short_stride)
    assert rc == _lib.E_ARG
    assert "stride smaller than the width" in _lib.last_error(node._ctx.lib)


def test_bounded_wait_times_out_and_the_context_recovers(monkeypatch):
    import torch

    # pinned host buffers: the copies are asynchronous, so the bounded wait
    # runs while the GPU still works on the clip (~15 ms at 1080p radius 2)
    frames = make_clip(5, 1080, 1920, sigma=3.0, seed=5)
    params = dict(sigma=3.0, block_step=4, bm_range=16, radius=2, ps_num=2, ps_range=7)
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **params)
    src = torch.from_numpy(frames).pin_memory()
    out = torch.empty(frames.shape, dtype=torch.float32).pin_memory()
    ctx = node._ctx

    def run():
        return ctx.lib.vsfeel_bm3d_process_host(
            ctx.handle, src.data_ptr(), src.stride(0) * 4, src.stride(1) * 4, out.data_ptr(),
            out.stride(0) * 4, out.stride(1) * 4, 0, 5)

    monkeypatch.setenv("VSFEEL_TIMEOUT_MS", "1")
    rc = run()
    assert rc == _lib.E_TIMEOUT
    assert "timed out after" in _lib.last_error(ctx.lib)
    monkeypatch.delenv("VSFEEL_TIMEOUT_MS")
    assert run() == _lib.OK
    ref = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **params).output(2, 1)
    assert float(np.abs(out.numpy()[2] - ref[0]).max()) <= 2e-5


def test_status_word_reaches_the_caller_and_the_context_recovers(monkeypatch):
    frames = make_clip(3, 64, 80, sigma=5.0, seed=9)
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **PARAMS)
    expected = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **PARAMS).output()
    msg = "internal error: a search window left the staged region"
    monkeypatch.setenv("VSFEEL_TEST_PROBE_TILE", "1")
    with pytest.raises(vsfeel.Error, match=msg):
        node.output()
    with pytest.raises(vsfeel.Error, match=msg):
        node.get_frame(1)
    monkeypatch.delenv("VSFEEL_TEST_PROBE_TILE")
    # the word was cleared when it was reported: the same context is clean
    assert float(np.abs(node.output() - expected).max()) <= 2e-5
    fresh = vsfeel.BM3Dv2(vsfeel.clip_from_array(frames), **PARAMS)
    assert float(np.abs(node.get_frame(2)[0] - fresh.get_frame(2)[0]).max()) <= 2e-5
