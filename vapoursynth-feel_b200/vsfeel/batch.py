"""Batched BM3Dv2: many clips of uneven sizes and settings in one run.

``Batch`` wraps the library's vsfeel_bm3d_batch_* entry points: the clips
are bound at construction (CUDA float32 tensors, (N, H, W) with contiguous
rows, one output tensor per clip), grouped into shape classes, each class's
work captured in a CUDA graph (one persistent match-and-filter launch over a
device work queue, one normalise launch), optionally after the autotuner has
picked each class's tile shape. ``run()`` replays the graphs on torch's
current stream; write new frames into the bound input tensors between runs.
"""

from __future__ import annotations

import ctypes

from . import Error, _lib, _make_args


class Batch:
    def __init__(self, clips, device: int = 0, autotune: bool = True,
                 tile_shape: str | None = None, lanes: int | None = None):
        """clips: sequence of (src, dst, params) with params the BM3Dv2
        keyword arguments (sigma, block_step, bm_range, radius, ps_num,
        ps_range, extractor_exp). tile_shape ("8x4", "16x2", "4x8", "8x2",
        "4x4") forces that shape on every class it fits; lanes (8 or 16)
        forces the lanes per reference block of every tiled class."""
        import torch

        self.lib = _lib.load()
        self.device = int(device)
        self._keep = []
        arr = (_lib.BatchClip * len(clips))()
        for i, (src, dst, params) in enumerate(clips):
            for name, t in (("src", src), ("dst", dst)):
                if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32
                        and t.dim() == 3 and t.stride(2) == 1):
                    raise Error(f"BM3D: clip {i}: {name} must be a CUDA float32 (N, H, W) tensor "
                                "with contiguous rows")
                if t.device.index != self.device:
                    raise Error(f"BM3D: clip {i}: {name} is not on cuda:{self.device}")
            if tuple(src.shape) != tuple(dst.shape):
                raise Error(f"BM3D: clip {i}: src and dst shapes differ")
            args, _ = _make_args(None, params.get("sigma"), params.get("block_step"),
                                 params.get("bm_range"), params.get("radius"),
                                 params.get("ps_num"), params.get("ps_range"), None,
                                 params.get("extractor_exp"))
            c = arr[i]
            c.args = args
            c.num_frames, c.height, c.width = (int(v) for v in src.shape)
            c.src, c.src_frame_stride, c.src_row_stride = src.data_ptr(), src.stride(0), src.stride(1)
            c.dst, c.dst_frame_stride, c.dst_row_stride = dst.data_ptr(), dst.stride(0), dst.stride(1)
            self._keep += [src, dst]
        handle = ctypes.c_void_p()
        flags = _lib.BATCH_AUTOTUNE if autotune else 0
        if tile_shape is not None:
            flags |= ((_lib.TILE_SHAPES.index(tile_shape) + 1) & 15) << 4
        if lanes is not None:
            if lanes not in (8, 16):
                raise Error("BM3D: lanes must be 8 or 16")
            flags |= (2 if lanes == 16 else 1) << 8
        rc = self.lib.vsfeel_bm3d_batch_create(arr, len(clips), self.device, flags,
                                               ctypes.byref(handle))
        if rc != _lib.OK:
            raise Error(_lib.last_error(self.lib))
        self.handle = handle

    def _check(self, rc: int) -> None:
        if rc != _lib.OK:
            raise Error(_lib.last_error(self.lib))

    def run(self) -> None:
        """Enqueues one denoising of every clip on torch's current stream."""
        import torch

        stream = torch.cuda.current_stream(self.device).cuda_stream
        self._check(self.lib.vsfeel_bm3d_batch_run(self.handle, stream))

    def finish(self) -> None:
        """Waits for the enqueued work; raises on a flagged internal error."""
        self._check(self.lib.vsfeel_bm3d_batch_finish(self.handle))

    @property
    def device_bytes(self) -> int:
        n, b = ctypes.c_int(), ctypes.c_int64()
        self._check(self.lib.vsfeel_bm3d_batch_classes(self.handle, ctypes.byref(n), ctypes.byref(b)))
        return b.value

    def classes(self) -> list[dict]:
        n, b = ctypes.c_int(), ctypes.c_int64()
        self._check(self.lib.vsfeel_bm3d_batch_classes(self.handle, ctypes.byref(n), ctypes.byref(b)))
        out = []
        for i in range(n.value):
            info = _lib.BatchClassInfo()
            self._check(self.lib.vsfeel_bm3d_batch_class(self.handle, i, ctypes.byref(info)))
            shape = info.tile_shape
            out.append({
                "radius": info.radius, "block_step": info.block_step, "bm_range": info.bm_range,
                "ps_num": info.ps_num, "ps_range": info.ps_range, "clips": info.clips,
                "stacks": info.stacks, "tiles": info.tiles,
                "tile_shape": _lib.TILE_SHAPES[shape] if shape >= 0 else "direct",
                "lanes": info.lanes,
                "tuned_ms": {_lib.TILE_SHAPES[s]: info.tuned_ms[s]
                             for s in range(len(_lib.TILE_SHAPES)) if info.tuned_ms[s] > 0},
                "tuned_ms_16": {_lib.TILE_SHAPES[s]: info.tuned_ms_16[s]
                                for s in range(len(_lib.TILE_SHAPES)) if info.tuned_ms_16[s] > 0},
            })
        return out

    def close(self) -> None:
        h = getattr(self, "handle", None)
        if h:
            self.lib.vsfeel_bm3d_batch_free(h)
            self.handle = None

    def __del__(self):
        self.close()
