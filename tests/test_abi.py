"""The C ABI library: loads, exports every declared symbol, and validates
arguments like the reference's BM3DCreate (CPU only; no kernel runs)."""

from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT
import vsfeel
from vsfeel import _lib


def _declared_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"VSFEEL_API\s+[\w\s\*]+?\b(vsfeel_\w+)\s*\(", text))
    return names


def test_header_declares_the_binding_exports():
    assert _declared_symbols() == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in _declared_symbols():
        assert hasattr(lib, name), name
    assert lib.vsfeel_bm3d_abi_version() == _lib.ABI_VERSION


def test_library_exports_nothing_else():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.split()[-1].startswith("vsfeel")}
    assert exported == _declared_symbols()


def _create(clip_shape=(4, 32, 48), fmt=vsfeel.GRAYS, **kw):
    clip = vsfeel.clip_from_array(np.zeros(clip_shape, np.float32), fmt=fmt)
    return vsfeel.BM3Dv2(clip, **kw)


@pytest.mark.parametrize("kwargs,message", [
    (dict(sigma=-1.0), '"sigma" must be non-negative'),
    (dict(sigma=[1.0, -0.5]), '"sigma" must be non-negative'),
    (dict(block_step=0), '"block_step" must be in range [1, 8]'),
    (dict(block_step=9), '"block_step" must be in range [1, 8]'),
    (dict(bm_range=0), '"bm_range" must be positive'),
    (dict(radius=5), '"radius" must be in range [0, 4]'),
    (dict(radius=-1), '"radius" must be in range [0, 4]'),
    (dict(ps_num=0), '"ps_num" must be in range [1, 8]'),
    (dict(ps_num=9), '"ps_num" must be in range [1, 8]'),
    (dict(ps_range=0), '"ps_range" must be positive'),
    (dict(num_streams=0), '"num_streams" must be positive'),
])
def test_argument_validation_messages(kwargs, message):
    # src/bm3d.cpp:1090-1190 (the reference's tests: test_bm3dv2_rejects_radius5)
    with pytest.raises(vsfeel.Error, match=re.escape("BM3D: " + message)):
        _create(**kwargs)


def test_rejects_integer_formats():
    # test_bm3dv2_rejects_gray8: only 32-bit float input
    gray8 = vsfeel.VideoFormat(_lib.CF_GRAY, _lib.ST_INTEGER, 8, 0, 0)
    with pytest.raises(vsfeel.Error, match="only constant format 32 bit float input supported"):
        _create(fmt=gray8)


def test_rejects_bad_ref_format():
    # test_bm3dv2_rejects_bad_ref_format: a ref of other dimensions
    clip = vsfeel.clip_from_array(np.zeros((4, 32, 48), np.float32))
    bad = vsfeel.clip_from_array(np.zeros((4, 32, 49), np.float32))
    with pytest.raises(vsfeel.Error, match='"ref" must be of the same dimensions as "clip"'):
        vsfeel.BM3Dv2(clip, ref=bad)
    shorter = vsfeel.clip_from_array(np.zeros((3, 32, 48), np.float32))
    with pytest.raises(vsfeel.Error, match='"ref" must be of the same number of frames'):
        vsfeel.BM3Dv2(clip, ref=shorter)
    yuv = vsfeel.clip_from_array(np.zeros((4, 32, 48), np.float32), np.zeros((4, 16, 24), np.float32),
                                 np.zeros((4, 16, 24), np.float32))
    with pytest.raises(vsfeel.Error, match='"ref" must be of the same format as "clip"'):
        vsfeel.BM3Dv2(clip, ref=yuv)


def test_rejects_rgb():
    rgb = vsfeel.VideoFormat(2, _lib.ST_FLOAT, 32, 0, 0)
    with pytest.raises(vsfeel.Error, match="only Gray and YUV input"):
        _create(fmt=rgb)


def test_rejects_frames_below_block_size():
    with pytest.raises(vsfeel.Error, match="at least 8x8"):
        _create(clip_shape=(2, 7, 32))


def test_valid_arguments_reach_the_device_check_without_a_gpu():
    """On a machine without a GPU, valid arguments fail only at the device
    probe: the whole validation passed."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(vsfeel.Error, match="no CUDA device"):
        _create(sigma=[3.0], block_step=4, bm_range=16, radius=2, ps_num=2, ps_range=7,
                num_streams=4, extractor_exp=2)


def test_errors_are_per_thread_and_prefixed():
    lib = _lib.load()
    with pytest.raises(vsfeel.Error):
        _create(radius=7)
    assert _lib.last_error(lib).startswith("BM3D: ")


def test_null_context_is_rejected():
    lib = _lib.load()
    lo, hi = ctypes.c_int(), ctypes.c_int()
    assert lib.vsfeel_bm3d_frame_range(None, 0, ctypes.byref(lo), ctypes.byref(hi)) == _lib.E_ARG
    lib.vsfeel_bm3d_free(None)
    assert lib.vsfeel_bm3d_launch_count(None) == 0


def _yuv420_clip(h=32, w=48, n=4):
    z = np.zeros
    return vsfeel.clip_from_array(z((n, h, w), np.float32), z((n, h // 2, w // 2), np.float32),
                                  z((n, h // 2, w // 2), np.float32))


def test_plane_params_follow_the_reference_fill_rule():
    """Element [p] of each per-plane array, a missing element copying the
    previous one (src/bm3d.cpp:1090-1167), on the plane's own dimensions."""
    clip = _yuv420_clip()
    kw = dict(sigma=[2.0, 4.0], block_step=[8, 4, 2], bm_range=[16], ps_num=[3, 1],
              ps_range=[7, 5, 3], radius=1)
    want = {0: (2.0, 8, 16, 3, 7, 48, 32), 1: (4.0, 4, 16, 1, 5, 24, 16),
            2: (4.0, 2, 16, 1, 3, 24, 16)}
    for p, (sigma, step, bmr, psn, psr, w, h) in want.items():
        inf = vsfeel.plane_params(clip, p, **kw)
        assert (inf.sigma, inf.block_step, inf.bm_range, inf.ps_num, inf.ps_range) == (
            sigma, step, bmr, psn, psr), p
        assert (inf.width, inf.height, inf.num_frames, inf.radius) == (w, h, 4, 1), p
        assert inf.device_bytes == 0
    # the threshold scales the plane's own sigma by the pass factor
    basic = vsfeel.plane_params(clip, 1, **kw).threshold
    assert basic == np.float32(np.float32(4.0) * np.frombuffer(
        np.uint32(0x3f021bb6).tobytes(), np.float32)[0])
    ref = vsfeel.plane_params(clip, 2, ref=clip, **kw).threshold
    assert ref == np.float32(np.float32(4.0) * np.frombuffer(
        np.uint32(0x3e40c0c1).tobytes(), np.float32)[0])


def test_plane_params_plane_zero_equals_create():
    """Plane 0 of the extension is the reference's (luma) configuration."""
    clip = vsfeel.clip_from_array(np.zeros((3, 40, 56), np.float32))
    inf = vsfeel.plane_params(clip, 0, sigma=[5.0, 1.0], block_step=[4, 8])
    assert (inf.sigma, inf.block_step, inf.bm_range, inf.width, inf.height) == (5.0, 4, 9, 56, 40)
    assert (inf.blocks_x, inf.blocks_y) == (13, 9)


def test_plane_params_report_the_matcher_configuration():
    """Before any autotuning the matcher uses the largest tile shape whose
    shared-memory plan fits (8x4 blocks at the radius-2, step-4, range-16
    settings) with 8 lanes per block; windows too large for every staged tile
    go to the direct-read matcher (-1)."""
    clip = vsfeel.clip_from_array(np.zeros((3, 270, 480), np.float32))
    inf = vsfeel.plane_params(clip, 0, sigma=3.0, block_step=4, bm_range=16, radius=2,
                              ps_num=2, ps_range=7)
    assert (inf.match_tile_shape, inf.match_lanes, inf.autotuned) == (0, 8, 0)
    big = vsfeel.plane_params(clip, 0, block_step=4, bm_range=60, radius=1)
    assert big.match_tile_shape == -1


@pytest.mark.parametrize("plane,fmt_yuv", [(1, False), (3, True), (-1, True)])
def test_plane_outside_the_clip_is_rejected(plane, fmt_yuv):
    clip = _yuv420_clip() if fmt_yuv else vsfeel.clip_from_array(np.zeros((2, 16, 16), np.float32))
    with pytest.raises(vsfeel.Error, match='"planes" must name planes of the clip'):
        vsfeel.plane_params(clip, plane)


def test_small_chroma_planes_are_rejected():
    clip = _yuv420_clip(h=14, w=48)
    vsfeel.plane_params(clip, 0)
    with pytest.raises(vsfeel.Error, match="chroma planes must be at least 8x8"):
        vsfeel.plane_params(clip, 1)


def test_plane_params_validate_every_argument():
    clip = _yuv420_clip()
    with pytest.raises(vsfeel.Error, match='"block_step" must be in range'):
        vsfeel.plane_params(clip, 2, block_step=[4, 4, 9])


@pytest.mark.parametrize("planes,message", [
    ([], '"planes" must name at least one plane'),
    ([0, 0], '"planes" must not repeat a plane'),
    ([0, 3], '"planes" must name planes of the clip'),
])
def test_planes_keyword_validation(planes, message):
    with pytest.raises(vsfeel.Error, match=re.escape("BM3D: " + message)):
        vsfeel.BM3Dv2(_yuv420_clip(), planes=planes)


def test_all_planes_reach_the_device_check_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(vsfeel.Error, match="no CUDA device"):
        vsfeel.BM3Dv2(_yuv420_clip(), planes=[0, 1, 2], sigma=[3.0, 5.0], block_step=[4, 2])


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """Every struct the ctypes stub mirrors has the header's size and member
    offsets (gcc compiles the header and prints them), so a member added on
    one side only fails here instead of corrupting a call."""
    import ctypes
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("gcc is not installed")
    pairs = [("vsfeel_bm3d_video_info", _lib.VideoInfo), ("vsfeel_bm3d_args", _lib.Args),
             ("vsfeel_bm3d_info", _lib.Info), ("vsfeel_bm3d_saved_info", _lib.SavedInfo),
             ("vsfeel_bm3d_batch_clip", _lib.BatchClip),
             ("vsfeel_bm3d_batch_class_info", _lib.BatchClassInfo)]
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "vsfeel_bm3d.h"',
           "int main(void) {"]
    want = []
    for cname, cls in pairs:
        src.append(f'printf("%zu\\n", sizeof({cname}));')
        want.append(ctypes.sizeof(cls))
        for name, *_ in cls._fields_:
            src.append(f'printf("%zu\\n", offsetof({cname}, {name}));')
            want.append(getattr(cls, name).offset)
    src.append("return 0; }")
    (tmp_path / "layout.c").write_text("\n".join(src))
    include = ROOT / "include"
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(include), str(tmp_path / "layout.c"), "-o", str(exe)],
                   check=True, capture_output=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got == want
