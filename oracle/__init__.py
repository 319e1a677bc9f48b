"""TEST INFRASTRUCTURE: ctypes access to the CPU checkers.

``Oracle`` wraps libbm3d_oracle.so, the C++ restatement of the reference's
BM3Dv2 basic estimate (bm3d_oracle.cpp cites the reference line by line).
``ReferenceShaders`` wraps oracle/_ref/libvsfeel_ref.so, the reference's own
shaders compiled for the CPU. Only tests/, __graft_entry__.smoke() and the
benchmark's CPU legs use this package; the product path never does.

Frames are float32 arrays of shape (nframes, height, width).
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

_f = ctypes.c_float
_i = ctypes.c_int
_p = ctypes.c_void_p


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _frames(frames: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(frames, dtype=np.float32)
    if a.ndim == 2:
        a = a[None]
    if a.ndim != 3:
        raise ValueError("frames must be (nframes, height, width)")
    return a


class Params:
    """The BM3Dv2 arguments (reference defaults, src/bm3d.cpp:1090-1190)."""

    def __init__(self, sigma=3.0, block_step=8, bm_range=9, radius=0, ps_num=2, ps_range=4,
                 extractor_exp=0):
        self.sigma = float(sigma)
        self.block_step = int(block_step)
        self.bm_range = int(bm_range)
        self.radius = int(radius)
        self.ps_num = int(ps_num)
        self.ps_range = int(ps_range)
        self.extractor_exp = int(extractor_exp)

    def args(self):
        return (_f(self.sigma), self.block_step, self.bm_range, self.radius, self.ps_num,
                self.ps_range)

    def as_dict(self):
        return dict(sigma=self.sigma, block_step=self.block_step, bm_range=self.bm_range,
                    radius=self.radius, ps_num=self.ps_num, ps_range=self.ps_range,
                    extractor_exp=self.extractor_exp)


def _default_threads() -> int:
    return max(1, os.cpu_count() or 1)


class Oracle:
    """The C++ restatement (FP32 faithful and FP64)."""

    def __init__(self, path: str | os.PathLike | None = None):
        path = Path(path) if path else HERE / "libbm3d_oracle.so"
        if not path.exists():
            from . import build
            build.build_oracle()
        lib = ctypes.CDLL(str(path))
        sig = [_p, _i, _i, _i, _f, _i, _i, _i, _i, _i, _i, _i, _i, _i, _p]
        lib.oracle_bm3d_f32.argtypes = sig
        lib.oracle_bm3d_f32.restype = _i
        lib.oracle_bm3d_f64.argtypes = sig
        lib.oracle_bm3d_f64.restype = _i
        lib.oracle_bm3d_matches_f32.argtypes = [_p, _i, _i, _i, _f, _i, _i, _i, _i, _i, _i, _i, _p]
        lib.oracle_bm3d_matches_f32.restype = _i
        lib.oracle_bm3d_final.argtypes = [_p, _p, _i, _i, _i, _f, _i, _i, _i, _i, _i, _i, _i,
                                          _i, _i, _i, _p]
        lib.oracle_bm3d_final.restype = _i
        lib.oracle_bm3d_frozen_state.argtypes = [_p, _i, _i, _i, _f, _i, _i, _i, _i, _i, _i,
                                                 _i, _i, _p, _p]
        lib.oracle_bm3d_frozen_state.restype = _i
        lib.oracle_bm3d_stack_f32.argtypes = [_p, _i, _i, _i, _f, _i, _i, _i, _i, _i, _i, _i, _i, _p]
        lib.oracle_bm3d_stack_f32.restype = _i
        lib.oracle_block_count.argtypes = [_i, _i, _i]
        lib.oracle_block_count.restype = _i
        lib.oracle_agg_z.argtypes = [_i, _i, _i, _i]
        lib.oracle_agg_z.restype = _i
        lib.oracle_threshold.argtypes = [_f]
        lib.oracle_threshold.restype = _f
        for name in ("oracle_dct8_fwd_f32", "oracle_dct8_inv_f32"):
            getattr(lib, name).argtypes = [_p]
            getattr(lib, name).restype = None
        for name in ("oracle_dct8_fwd_f64", "oracle_dct8_inv_f64"):
            getattr(lib, name).argtypes = [_p]
            getattr(lib, name).restype = None
        self.lib = lib

    def bm3d(self, frames, params: Params, out_first=0, out_count=None, nthreads=None,
             fp64=False, ref=None) -> np.ndarray:
        """ref: the basic estimate; given, runs the final (Wiener) pass."""
        a = _frames(frames)
        n, h, w = a.shape
        out_count = n - out_first if out_count is None else out_count
        out = np.empty((out_count, h, w), dtype=np.float64 if fp64 else np.float32)
        if ref is not None:
            r = _frames(ref)
            if r.shape != a.shape:
                raise ValueError("ref must have the clip's shape")
            rc = self.lib.oracle_bm3d_final(_ptr(a), _ptr(r), n, w, h, *params.args(),
                                            params.extractor_exp, out_first, out_count,
                                            nthreads or _default_threads(), 1 if fp64 else 0,
                                            _ptr(out))
            if rc != 0:
                raise ValueError("oracle rejected the arguments")
            return out
        fn = self.lib.oracle_bm3d_f64 if fp64 else self.lib.oracle_bm3d_f32
        rc = fn(_ptr(a), n, w, h, *params.args(), params.extractor_exp, out_first, out_count,
                nthreads or _default_threads(), _ptr(out))
        if rc != 0:
            raise ValueError("oracle rejected the arguments")
        return out

    def matches(self, frames, params: Params, m: int, nthreads=None) -> np.ndarray:
        a = _frames(frames)
        n, h, w = a.shape
        nb = self.block_count(w, h, params.block_step)
        table = np.empty((nb, 8, 3), dtype=np.int32)
        rc = self.lib.oracle_bm3d_matches_f32(_ptr(a), n, w, h, *params.args(), m,
                                              nthreads or _default_threads(), _ptr(table))
        if rc != 0:
            raise ValueError("oracle rejected the arguments")
        return table

    def frozen_state(self, frames, params: Params, m: int, fp64=False, nthreads=None):
        """(match table [nblocks, 8, 3] int32, keep bits [nblocks, 8] uint64) of
        stack m, in the layout of the library's saved state."""
        a = _frames(frames)
        n, h, w = a.shape
        nb = self.block_count(w, h, params.block_step)
        table = np.empty((nb, 8, 3), dtype=np.int32)
        keep = np.empty((nb, 8), dtype=np.uint64)
        rc = self.lib.oracle_bm3d_frozen_state(_ptr(a), n, w, h, *params.args(), m,
                                               1 if fp64 else 0, nthreads or _default_threads(),
                                               _ptr(table), _ptr(keep))
        if rc != 0:
            raise ValueError("oracle rejected the arguments")
        return table, keep

    def stack(self, frames, params: Params, m: int, nthreads=None) -> np.ndarray:
        a = _frames(frames)
        n, h, w = a.shape
        tw = 2 * params.radius + 1
        out = np.empty((tw, 2, h, w), dtype=np.float32)
        rc = self.lib.oracle_bm3d_stack_f32(_ptr(a), n, w, h, *params.args(),
                                            params.extractor_exp, m,
                                            nthreads or _default_threads(), _ptr(out))
        if rc != 0:
            raise ValueError("oracle rejected the arguments")
        return out

    def block_count(self, width, height, block_step) -> int:
        return self.lib.oracle_block_count(width, height, block_step)

    def agg_z(self, i, n, nframes, radius) -> int:
        return self.lib.oracle_agg_z(i, n, nframes, radius)

    def threshold(self, sigma) -> float:
        return float(self.lib.oracle_threshold(sigma))

    def dct8(self, v, inverse=False, fp64=False) -> np.ndarray:
        a = np.array(v, dtype=np.float64 if fp64 else np.float32).copy()
        name = f"oracle_dct8_{'inv' if inverse else 'fwd'}_{'f64' if fp64 else 'f32'}"
        getattr(self.lib, name)(_ptr(a))
        return a


class ReferenceShaders:
    """The reference's bm3d.comp / bm3d_agg.comp executed on the CPU."""

    PATH = HERE / "_ref" / "libvsfeel_ref.so"

    def __init__(self, path: str | os.PathLike | None = None):
        path = Path(path) if path else self.PATH
        if not path.exists():
            from . import build
            if build.build_ref() is None:
                raise FileNotFoundError("reference shaders are not built (no reference tree)")
        lib = ctypes.CDLL(str(path))
        lib.ref_bm3d_clip.argtypes = [_p, _p, _i, _i, _i, _f, _i, _i, _i, _i, _i, _i, _i, _i, _i,
                                      _p]
        lib.ref_bm3d_clip.restype = _i
        lib.ref_bm3d_stack.argtypes = [_p, _i, _i, _i, _f, _i, _i, _i, _i, _i, _i, _i, _i, _p]
        lib.ref_bm3d_stack.restype = _i
        lib.ref_bm3d_stack_rows.argtypes = [_p, _i, _i, _i, _f, _i, _i, _i, _i, _i, _i, _i, _i, _i,
                                            _i]
        lib.ref_bm3d_stack_rows.restype = _i
        self.lib = lib

    def stack_rows(self, frames, params: Params, m: int, row_first: int, row_count: int,
                   nthreads=None) -> None:
        """Runs stack m's estimation over block rows [row_first, row_first+row_count)
        only (a timing sample; the result is discarded)."""
        a = _frames(frames)
        n, h, w = a.shape
        p = params
        rc = self.lib.ref_bm3d_stack_rows(_ptr(a), n, w, h, _f(p.sigma), p.block_step, p.bm_range,
                                          p.radius, p.ps_num, p.ps_range, p.extractor_exp, m,
                                          row_first, row_count, nthreads or _default_threads())
        if rc != 0:
            raise ValueError("reference harness rejected the arguments")

    @classmethod
    def available(cls) -> bool:
        return cls.PATH.exists()

    def bm3d(self, frames, params: Params, out_first=0, out_count=None, nthreads=1,
             ref=None) -> np.ndarray:
        """ref: the basic estimate for the final (Wiener) pass."""
        a = _frames(frames)
        n, h, w = a.shape
        out_count = n - out_first if out_count is None else out_count
        out = np.empty((out_count, h, w), dtype=np.float32)
        p = params
        r = None if ref is None else _frames(ref)
        if r is not None and r.shape != a.shape:
            raise ValueError("ref must have the clip's shape")
        rc = self.lib.ref_bm3d_clip(_ptr(a), None if r is None else _ptr(r), n, w, h, _f(p.sigma),
                                    p.block_step, p.bm_range,
                                    p.radius, p.ps_num, p.ps_range, p.extractor_exp, out_first,
                                    out_count, nthreads, _ptr(out))
        if rc != 0:
            raise ValueError("reference harness rejected the arguments")
        return out

    def stack(self, frames, params: Params, m: int, nthreads=1) -> np.ndarray:
        a = _frames(frames)
        n, h, w = a.shape
        tw = 2 * params.radius + 1
        out = np.empty((tw, 2, h, w), dtype=np.float32)
        p = params
        rc = self.lib.ref_bm3d_stack(_ptr(a), n, w, h, _f(p.sigma), p.block_step, p.bm_range,
                                     p.radius, p.ps_num, p.ps_range, p.extractor_exp, m, nthreads,
                                     _ptr(out))
        if rc != 0:
            raise ValueError("reference harness rejected the arguments")
        return out
