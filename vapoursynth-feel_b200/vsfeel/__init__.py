"""vsfeel (B200): BM3Dv2 basic estimate behind the reference's plugin API.

``BM3Dv2(clip, ref=None, sigma=..., block_step=..., bm_range=..., radius=...,
ps_num=..., ps_range=..., num_streams=..., extractor_exp=...)`` takes and
returns the same arguments as ``core.vsfeel.BM3Dv2`` (README.md:44-77,
src/bm3d.cpp:1558-1574). Clips are ``VideoNode`` objects holding float32
planes; ``clip_from_array`` builds one from numpy arrays. Errors raise
``vsfeel.Error`` with the reference's messages.

One keyword goes past the reference: ``planes`` (default ``[0]``, the
reference's behaviour of denoising luma and passing chroma through) lists
the planes to denoise, each with its own element of the per-plane argument
arrays, which the reference parses but does not apply
(src/bm3d.cpp:1090-1167).

All denoising runs in libvsfeel_bm3d.so on the GPU through the C ABI of
include/vsfeel_bm3d.h; there is no CPU path.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib

__all__ = ["Error", "VideoFormat", "GRAYS", "YUV420PS", "YUV444PS", "VideoNode", "VideoFrame",
           "clip_from_array", "BM3Dv2", "bm3d_device", "plane_params", "get_include",
           "library_path"]

__version__ = "1.0.0"


def get_include() -> str:
    """The directory holding vsfeel_bm3d.h: inside an installed wheel, or the
    checkout's include/ when the package runs from the source tree."""
    from pathlib import Path

    here = Path(__file__).resolve().parent
    packaged = here / "include"
    return str(packaged if (packaged / "vsfeel_bm3d.h").exists() else here.parent.parent / "include")


def library_path() -> str:
    """The C-ABI library (libvsfeel_bm3d.so) that other languages link or load."""
    return str(_lib.LIB_PATH)


class Error(Exception):
    """Raised for invalid arguments or GPU failures (mirrors vapoursynth.Error)."""


@dataclass(frozen=True)
class VideoFormat:
    color_family: int
    sample_type: int
    bits_per_sample: int
    subsampling_w: int
    subsampling_h: int

    @property
    def num_planes(self) -> int:
        return 1 if self.color_family == _lib.CF_GRAY else 3


GRAYS = VideoFormat(_lib.CF_GRAY, _lib.ST_FLOAT, 32, 0, 0)
YUV420PS = VideoFormat(_lib.CF_YUV, _lib.ST_FLOAT, 32, 1, 1)
YUV444PS = VideoFormat(_lib.CF_YUV, _lib.ST_FLOAT, 32, 0, 0)


class VideoFrame:
    def __init__(self, planes: Sequence[np.ndarray], fmt: VideoFormat):
        self.planes = list(planes)
        self.format = fmt

    def __getitem__(self, p: int) -> np.ndarray:
        return self.planes[p]

    @property
    def width(self) -> int:
        return self.planes[0].shape[1]

    @property
    def height(self) -> int:
        return self.planes[0].shape[0]


class VideoNode:
    """A clip of ``num_frames`` frames; plane p is an array (N, h_p, w_p)."""

    def __init__(self, planes: Sequence[np.ndarray], fmt: VideoFormat):
        self._planes = list(planes)
        self.format = fmt
        self.num_frames = int(self._planes[0].shape[0])
        self.height = int(self._planes[0].shape[1])
        self.width = int(self._planes[0].shape[2])

    def get_frame(self, n: int) -> VideoFrame:
        if not 0 <= n < self.num_frames:
            raise Error("frame index out of range")
        return VideoFrame([p[n] for p in self._planes], self.format)

    def plane_array(self, p: int = 0) -> np.ndarray:
        return self._planes[p]

    def video_info(self) -> _lib.VideoInfo:
        f = self.format
        return _lib.VideoInfo(self.width, self.height, self.num_frames, f.color_family,
                              f.sample_type, f.bits_per_sample, f.subsampling_w, f.subsampling_h)


def clip_from_array(luma: np.ndarray, u: np.ndarray | None = None, v: np.ndarray | None = None,
                    fmt: VideoFormat | None = None) -> VideoNode:
    """A GRAYS clip from (N, H, W) luma, or a YUV clip when u and v are given."""
    luma = np.asarray(luma)
    if luma.ndim == 2:
        luma = luma[None]
    if u is None:
        return VideoNode([luma], fmt or GRAYS)
    if fmt is None:
        sw = int(round(np.log2(luma.shape[2] / u.shape[2]))) if u.shape[2] else 0
        sh = int(round(np.log2(luma.shape[1] / u.shape[1]))) if u.shape[1] else 0
        fmt = VideoFormat(_lib.CF_YUV, _lib.ST_FLOAT, 32, sw, sh)
    return VideoNode([luma, np.asarray(u), np.asarray(v)], fmt)


def _array_arg(value, name: str, cast):
    if value is None:
        return [], 0
    vals = list(value) if isinstance(value, (list, tuple, np.ndarray)) else [value]
    if len(vals) > 3:
        raise Error(f"BM3D: \"{name}\" has more than 3 elements")
    return [cast(v) for v in vals], len(vals)


def _make_args(ref, sigma, block_step, bm_range, radius, ps_num, ps_range, num_streams,
               extractor_exp) -> tuple[_lib.Args, object]:
    a = _lib.Args()
    for name, value, cast in (("sigma", sigma, float), ("block_step", block_step, int),
                              ("bm_range", bm_range, int), ("ps_num", ps_num, int),
                              ("ps_range", ps_range, int)):
        vals, n = _array_arg(value, name, cast)
        arr = getattr(a, name)
        for i, v in enumerate(vals):
            arr[i] = v
        setattr(a, f"{name}_count", n)
    for name, value in (("radius", radius), ("num_streams", num_streams),
                        ("extractor_exp", extractor_exp)):
        if value is not None:
            setattr(a, name, int(value))
            setattr(a, f"{name}_set", 1)
    keep = None
    if ref is not None:
        keep = ref.video_info()
        a.has_ref = 1
        a.ref_info = ctypes.pointer(keep)
    return a, keep


class _Context:
    """Owns one vsfeel_bm3d context, bound to one plane of the clip."""

    def __init__(self, clip: VideoNode, args: _lib.Args, device: int, plane: int = 0):
        self.lib = _lib.load()
        self.vi = clip.video_info()
        self.plane = plane
        h = ctypes.c_void_p()
        rc = self.lib.vsfeel_bm3d_create_plane(ctypes.byref(args), ctypes.byref(self.vi), plane,
                                               device, ctypes.byref(h))
        if rc != _lib.OK:
            raise Error(_lib.last_error(self.lib))
        self.handle = h

    def check(self, rc: int) -> None:
        if rc != _lib.OK:
            raise Error(_lib.last_error(self.lib))

    def info(self) -> _lib.Info:
        inf = _lib.Info()
        self.check(self.lib.vsfeel_bm3d_get_info(self.handle, ctypes.byref(inf)))
        return inf

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self.lib.vsfeel_bm3d_free(h)
            self.handle = None


class BM3DNode(VideoNode):
    """The filter's output clip. Frames are denoised on demand (``get_frame``,
    the VapourSynth request path) or all at once (``output``). Each denoised
    plane has its own context; the others pass through."""

    def __init__(self, clip: VideoNode, ctxs: Sequence[_Context], ref: VideoNode | None = None):
        super().__init__([clip.plane_array(p) for p in range(clip.format.num_planes)], clip.format)
        self._src = clip
        self._ctxs = {c.plane: c for c in ctxs}
        self._ctx = ctxs[0]
        self._whole: dict[int, np.ndarray] = {}
        self._plane_src = {p: np.ascontiguousarray(clip.plane_array(p), dtype=np.float32)
                           for p in self._ctxs}
        # the final (Wiener) pass: the basic estimate that matching runs on
        self._plane_ref = (None if ref is None else
                           {p: np.ascontiguousarray(ref.plane_array(p), dtype=np.float32)
                            for p in self._ctxs})

    @property
    def planes(self) -> list[int]:
        """The denoised planes, in the order given."""
        return list(self._ctxs)

    def plane_array(self, p: int = 0) -> np.ndarray:
        """Plane p of every output frame, (N, h, w): denoised planes are
        computed once on first use, the others are the source's. This makes
        the node usable wherever a clip is, e.g. as ``ref`` of the final
        pass."""
        if p not in self._ctxs:
            return self._src.plane_array(p)
        if p not in self._whole:
            self._whole[p] = self.output(plane=p)
        return self._whole[p]

    @property
    def final_pass(self) -> bool:
        return self._plane_ref is not None

    @property
    def info(self) -> _lib.Info:
        return self._ctx.info()

    def plane_info(self, plane: int) -> _lib.Info:
        return self._plane_ctx(plane).info()

    def _plane_ctx(self, plane: int | None) -> _Context:
        if plane is None:
            return self._ctx
        if plane not in self._ctxs:
            raise Error(f"BM3D: plane {plane} is not denoised by this node")
        return self._ctxs[plane]

    def frame_range(self, n: int) -> tuple[int, int]:
        lo, hi = ctypes.c_int(), ctypes.c_int()
        self._ctx.check(self._ctx.lib.vsfeel_bm3d_frame_range(self._ctx.handle, n,
                                                               ctypes.byref(lo), ctypes.byref(hi)))
        return lo.value, hi.value

    def get_frame(self, n: int) -> VideoFrame:
        if not 0 <= n < self.num_frames:
            raise Error("frame index out of range")
        planes = [self._denoise_plane(n, p) if p in self._ctxs else self._src.plane_array(p)[n]
                  for p in range(self.format.num_planes)]
        return VideoFrame(planes, self.format)

    def _denoise_plane(self, n: int, plane: int) -> np.ndarray:
        ctx = self._ctxs[plane]
        src = self._plane_src[plane]
        out = np.empty(src.shape[1:], dtype=np.float32)
        if self.final_pass:
            clips = (src, self._plane_ref[plane])

            @_lib.FETCH2_FN
            def fetch2(user, clip, f, stride):
                stride[0] = clips[clip].strides[1]
                return clips[clip][f].ctypes.data

            @_lib.RELEASE2_FN
            def release2(user, clip, f):
                pass

            ctx.check(ctx.lib.vsfeel_bm3d_get_frame_ref(
                ctx.handle, n, fetch2, release2, None, out.ctypes.data, out.strides[0]))
        else:
            @_lib.FETCH_FN
            def fetch(user, f, stride):
                stride[0] = src.strides[1]
                return src[f].ctypes.data

            @_lib.RELEASE_FN
            def release(user, f):
                pass

            ctx.check(ctx.lib.vsfeel_bm3d_get_frame(
                ctx.handle, n, fetch, release, None, out.ctypes.data, out.strides[0]))
        return out

    def output_device(self, src, out, first: int = 0, count: int | None = None,
                      ref=None, plane: int | None = None) -> None:
        """Denoises from device memory: src is a CUDA float32 tensor
        (num_frames, h, w) holding one plane of the clip (the first denoised
        plane, or ``plane``), out receives frames first..first+count-1 as
        (count, h, w); in the final pass ref holds the basic estimate's
        plane like src. Enqueued on torch's current stream; no host copies."""
        import torch

        ctx = self._plane_ctx(plane)
        count = self.num_frames - first if count is None else count
        for t in (src, out) + ((ref,) if ref is not None else ()):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32
                    and t.dim() == 3 and t.stride(2) == 1):
                raise Error("BM3D: device buffers must be CUDA float32 (N, H, W) tensors")
        stream = torch.cuda.current_stream(src.device).cuda_stream
        if ref is None:
            ctx.check(ctx.lib.vsfeel_bm3d_process_device(
                ctx.handle, src.data_ptr(), src.stride(0), src.stride(1), out.data_ptr(),
                out.stride(0), out.stride(1), first, count, stream))
        else:
            ctx.check(ctx.lib.vsfeel_bm3d_process_device_ref(
                ctx.handle, src.data_ptr(), src.stride(0), src.stride(1), ref.data_ptr(),
                ref.stride(0), ref.stride(1), out.data_ptr(), out.stride(0), out.stride(1), first,
                count, stream))

    def launch_count(self) -> int:
        return int(self._ctx.lib.vsfeel_bm3d_launch_count(self._ctx.handle))

    def trace(self, enable: bool) -> None:
        """Per-kernel CUDA-event timing of the launches that follow."""
        self._ctx.check(self._ctx.lib.vsfeel_bm3d_trace(self._ctx.handle, 1 if enable else 0))

    def trace_read(self) -> dict[str, tuple[float, int]]:
        """{kernel name: (summed device ms, launches)} of the traced launches."""
        ms = (ctypes.c_double * _lib.KERNEL_KINDS)()
        n = (ctypes.c_int64 * _lib.KERNEL_KINDS)()
        self._ctx.check(self._ctx.lib.vsfeel_bm3d_trace_read(self._ctx.handle, ms, n))
        return {name: (ms[k], n[k]) for k, name in enumerate(_lib.KERNEL_NAMES)}

    def output(self, first: int = 0, count: int | None = None,
               out: np.ndarray | None = None, plane: int | None = None) -> np.ndarray:
        """Denoised frames first..first+count-1 of the first denoised plane
        (luma by default), or of ``plane``, as (count, h, w)."""
        ctx = self._plane_ctx(plane)
        count = self.num_frames - first if count is None else count
        src = self._plane_src[ctx.plane]
        if out is None:
            out = np.empty((count,) + src.shape[1:], dtype=np.float32)
        if self.final_pass:
            ref = self._plane_ref[ctx.plane]
            ctx.check(ctx.lib.vsfeel_bm3d_process_host_ref(
                ctx.handle, src.ctypes.data, src.strides[0], src.strides[1], ref.ctypes.data,
                ref.strides[0], ref.strides[1], out.ctypes.data, out.strides[0], out.strides[1],
                first, count))
        else:
            ctx.check(ctx.lib.vsfeel_bm3d_process_host(
                ctx.handle, src.ctypes.data, src.strides[0], src.strides[1],
                out.ctypes.data, out.strides[0], out.strides[1], first, count))
        return out


def _plane_list(planes) -> list[int]:
    if planes is None:
        return [0]
    vals = [int(p) for p in (planes if isinstance(planes, (list, tuple, np.ndarray)) else [planes])]
    if not vals:
        raise Error('BM3D: "planes" must name at least one plane')
    if len(set(vals)) != len(vals):
        raise Error('BM3D: "planes" must not repeat a plane')
    return vals


def BM3Dv2(clip: VideoNode, ref: VideoNode | None = None, sigma=None, block_step=None,
           bm_range=None, radius=None, ps_num=None, ps_range=None, num_streams=None,
           extractor_exp=None, planes=None, device: int = 0) -> BM3DNode:
    """core.vsfeel.BM3Dv2: the BM3D basic estimate (hard thresholding), or
    with ``ref`` (a basic estimate of the same clip) the final Wiener pass.
    ``planes`` (an extension) lists the planes to denoise; plane p uses
    element [p] of sigma, block_step, bm_range, ps_num and ps_range."""
    if not isinstance(clip, VideoNode):
        clip = clip_from_array(np.asarray(clip))
    if ref is not None and not isinstance(ref, VideoNode):
        ref = clip_from_array(np.asarray(ref))
    args, keep = _make_args(ref, sigma, block_step, bm_range, radius, ps_num, ps_range,
                            num_streams, extractor_exp)
    plane_list = _plane_list(planes)
    # every plane's arguments are checked before any context takes the device
    lib = _lib.load()
    vi = clip.video_info()
    for p in plane_list[1:]:
        if lib.vsfeel_bm3d_plane_params(ctypes.byref(args), ctypes.byref(vi), p,
                                        ctypes.byref(_lib.Info())) != _lib.OK:
            raise Error(_lib.last_error(lib))
    ctxs = [_Context(clip, args, device, p) for p in plane_list]
    del keep
    return BM3DNode(clip, ctxs, ref)


def plane_params(clip: VideoNode, plane: int = 0, ref: VideoNode | None = None, sigma=None,
                 block_step=None, bm_range=None, radius=None, ps_num=None, ps_range=None,
                 num_streams=None, extractor_exp=None) -> _lib.Info:
    """The parameters ``BM3Dv2(..., planes=[plane])`` applies to ``plane``,
    validated like BM3DCreate; needs no GPU."""
    args, keep = _make_args(ref, sigma, block_step, bm_range, radius, ps_num, ps_range,
                            num_streams, extractor_exp)
    lib = _lib.load()
    vi = clip.video_info()
    inf = _lib.Info()
    rc = lib.vsfeel_bm3d_plane_params(ctypes.byref(args), ctypes.byref(vi), plane,
                                      ctypes.byref(inf))
    del keep
    if rc != _lib.OK:
        raise Error(_lib.last_error(lib))
    return inf


def bm3d_device(frames, sigma=None, block_step=None, bm_range=None, radius=None, ps_num=None,
                ps_range=None, extractor_exp=None, out=None):
    """Denoises a CUDA float32 tensor (N, H, W) in place on torch's current
    stream and returns the output tensor (N, H, W)."""
    import torch

    if not (isinstance(frames, torch.Tensor) and frames.is_cuda and frames.dtype == torch.float32):
        raise Error("BM3D: frames must be a CUDA float32 tensor")
    if frames.dim() != 3 or frames.stride(2) != 1:
        raise Error("BM3D: frames must be (N, H, W) with contiguous rows")
    n, h, w = frames.shape
    fmt = GRAYS
    vi = _lib.VideoInfo(w, h, n, fmt.color_family, fmt.sample_type, 32, 0, 0)
    args, _ = _make_args(None, sigma, block_step, bm_range, radius, ps_num, ps_range, None,
                         extractor_exp)
    lib = _lib.load()
    handle = ctypes.c_void_p()
    if lib.vsfeel_bm3d_create(ctypes.byref(args), ctypes.byref(vi), frames.device.index or 0,
                              ctypes.byref(handle)) != _lib.OK:
        raise Error(_lib.last_error(lib))
    try:
        if out is None:
            out = torch.empty((n, h, w), dtype=torch.float32, device=frames.device)
        stream = torch.cuda.current_stream(frames.device).cuda_stream
        rc = lib.vsfeel_bm3d_process_device(handle, frames.data_ptr(), frames.stride(0),
                                            frames.stride(1), out.data_ptr(), out.stride(0),
                                            out.stride(1), 0, n, stream)
        if rc != _lib.OK:
            raise Error(_lib.last_error(lib))
        # the context's scratch buffers are freed by vsfeel_bm3d_free, which
        # waits for its own stream only: finish this stream first
        torch.cuda.current_stream(frames.device).synchronize()
    finally:
        lib.vsfeel_bm3d_free(handle)
    return out
