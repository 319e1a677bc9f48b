"""ctypes binding of the C ABI in include/vsfeel_bm3d.h.

The library is vsfeel/libvsfeel_bm3d.so, built in-tree for sm_100a by
csrc/build.py. There is no fallback: if the library cannot be loaded, every
call raises.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libvsfeel_bm3d.so"

# Every symbol include/vsfeel_bm3d.h declares.
EXPORTS = (
    "vsfeel_bm3d_args_init",
    "vsfeel_bm3d_create",
    "vsfeel_bm3d_create_plane",
    "vsfeel_bm3d_plane_params",
    "vsfeel_bm3d_free",
    "vsfeel_bm3d_frame_range",
    "vsfeel_bm3d_get_frame",
    "vsfeel_bm3d_get_frame_ref",
    "vsfeel_bm3d_process_host",
    "vsfeel_bm3d_process_host_ref",
    "vsfeel_bm3d_process_device",
    "vsfeel_bm3d_process_device_ref",
    "vsfeel_bm3d_get_info",
    "vsfeel_bm3d_match_table_device",
    "vsfeel_bm3d_launch_count",
    "vsfeel_bm3d_trace",
    "vsfeel_bm3d_trace_read",
    "vsfeel_bm3d_saved_layout",
    "vsfeel_bm3d_forward_saved",
    "vsfeel_bm3d_backward",
    "vsfeel_bm3d_batch_create",
    "vsfeel_bm3d_batch_run",
    "vsfeel_bm3d_batch_finish",
    "vsfeel_bm3d_batch_classes",
    "vsfeel_bm3d_batch_class",
    "vsfeel_bm3d_batch_free",
    "vsfeel_bm3d_process_device_noalloc",
    "vsfeel_bm3d_noalloc_scratch_bytes",
    "vsfeel_bm3d_last_error",
    "vsfeel_bm3d_abi_version",
)

ABI_VERSION = 3

OK = 0
E_ARG = -1
E_FORMAT = -2
E_CUDA = -3
E_MEMORY = -4
E_TIMEOUT = -5
E_FETCH = -6
E_UNSUPPORTED = -7

KERNEL_MATCH = 0
KERNEL_FILTER = 1
KERNEL_NORMALIZE = 2
KERNEL_ADJOINT = 3
KERNEL_KINDS = 4
KERNEL_NAMES = ("bm3d_match_kernel", "bm3d_filter_kernel", "bm3d_normalize_kernel",
                "bm3d_adjoint_kernel")

CF_GRAY = 1
CF_YUV = 3
ST_INTEGER = 0
ST_FLOAT = 1


class VideoInfo(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int),
        ("height", ctypes.c_int),
        ("num_frames", ctypes.c_int),
        ("color_family", ctypes.c_int),
        ("sample_type", ctypes.c_int),
        ("bits_per_sample", ctypes.c_int),
        ("sub_sampling_w", ctypes.c_int),
        ("sub_sampling_h", ctypes.c_int),
    ]


class Args(ctypes.Structure):
    _fields_ = [
        ("sigma", ctypes.c_float * 3), ("sigma_count", ctypes.c_int),
        ("block_step", ctypes.c_int * 3), ("block_step_count", ctypes.c_int),
        ("bm_range", ctypes.c_int * 3), ("bm_range_count", ctypes.c_int),
        ("radius", ctypes.c_int), ("radius_set", ctypes.c_int),
        ("ps_num", ctypes.c_int * 3), ("ps_num_count", ctypes.c_int),
        ("ps_range", ctypes.c_int * 3), ("ps_range_count", ctypes.c_int),
        ("num_streams", ctypes.c_int), ("num_streams_set", ctypes.c_int),
        ("extractor_exp", ctypes.c_int), ("extractor_exp_set", ctypes.c_int),
        ("has_ref", ctypes.c_int),
        ("ref_info", ctypes.POINTER(VideoInfo)),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("num_frames", ctypes.c_int),
        ("radius", ctypes.c_int), ("block_step", ctypes.c_int), ("bm_range", ctypes.c_int),
        ("ps_num", ctypes.c_int), ("ps_range", ctypes.c_int), ("num_streams", ctypes.c_int),
        ("sigma", ctypes.c_float), ("threshold", ctypes.c_float), ("extractor", ctypes.c_float),
        ("blocks_x", ctypes.c_int), ("blocks_y", ctypes.c_int),
        ("device_bytes", ctypes.c_int64),
        ("match_tile_shape", ctypes.c_int), ("match_lanes", ctypes.c_int),
        ("autotuned", ctypes.c_int),
    ]


class SavedInfo(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in (
        "bytes", "stack_bytes", "match_xy_offset", "match_z_offset", "mask_offset",
        "den_offset", "den_row_stride", "den_frame_stride", "num_blocks")]


BATCH_AUTOTUNE = 1
TILE_SHAPES = ("8x4", "16x2", "4x8", "8x2", "4x4")


class BatchClip(ctypes.Structure):
    _fields_ = [
        ("args", Args),
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("num_frames", ctypes.c_int),
        ("src", ctypes.c_void_p),
        ("src_frame_stride", ctypes.c_int64), ("src_row_stride", ctypes.c_int64),
        ("dst", ctypes.c_void_p),
        ("dst_frame_stride", ctypes.c_int64), ("dst_row_stride", ctypes.c_int64),
    ]


class BatchClassInfo(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_int), ("block_step", ctypes.c_int), ("bm_range", ctypes.c_int),
        ("ps_num", ctypes.c_int), ("ps_range", ctypes.c_int),
        ("clips", ctypes.c_int), ("stacks", ctypes.c_int),
        ("tiles", ctypes.c_int64),
        ("tile_shape", ctypes.c_int),
        ("tuned_ms", ctypes.c_double * len(TILE_SHAPES)),
        ("lanes", ctypes.c_int),
        ("tuned_ms_16", ctypes.c_double * len(TILE_SHAPES)),
    ]


FETCH_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                            ctypes.POINTER(ctypes.c_ssize_t))
RELEASE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int)
FETCH2_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                             ctypes.POINTER(ctypes.c_ssize_t))
RELEASE2_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_int)

_lib = None


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Loads (once) and returns the library; raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with vapoursynth-feel_b200/csrc/build.py "
            "(the BM3D path has no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    c_int, c_p, c_i64, c_sz = ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_ssize_t
    lib.vsfeel_bm3d_args_init.argtypes = [ctypes.POINTER(Args)]
    lib.vsfeel_bm3d_args_init.restype = None
    lib.vsfeel_bm3d_create.argtypes = [ctypes.POINTER(Args), ctypes.POINTER(VideoInfo), c_int,
                                       ctypes.POINTER(c_p)]
    lib.vsfeel_bm3d_create.restype = c_int
    lib.vsfeel_bm3d_create_plane.argtypes = [ctypes.POINTER(Args), ctypes.POINTER(VideoInfo), c_int,
                                             c_int, ctypes.POINTER(c_p)]
    lib.vsfeel_bm3d_create_plane.restype = c_int
    lib.vsfeel_bm3d_plane_params.argtypes = [ctypes.POINTER(Args), ctypes.POINTER(VideoInfo), c_int,
                                             ctypes.POINTER(Info)]
    lib.vsfeel_bm3d_plane_params.restype = c_int
    lib.vsfeel_bm3d_free.argtypes = [c_p]
    lib.vsfeel_bm3d_free.restype = None
    lib.vsfeel_bm3d_frame_range.argtypes = [c_p, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]
    lib.vsfeel_bm3d_frame_range.restype = c_int
    lib.vsfeel_bm3d_get_frame.argtypes = [c_p, c_int, FETCH_FN, RELEASE_FN, c_p, c_p, c_sz]
    lib.vsfeel_bm3d_get_frame.restype = c_int
    lib.vsfeel_bm3d_process_host.argtypes = [c_p, c_p, c_sz, c_sz, c_p, c_sz, c_sz, c_int, c_int]
    lib.vsfeel_bm3d_process_host.restype = c_int
    lib.vsfeel_bm3d_process_host_ref.argtypes = [c_p, c_p, c_sz, c_sz, c_p, c_sz, c_sz, c_p, c_sz,
                                                 c_sz, c_int, c_int]
    lib.vsfeel_bm3d_process_host_ref.restype = c_int
    lib.vsfeel_bm3d_process_device_ref.argtypes = [c_p, c_p, c_i64, c_i64, c_p, c_i64, c_i64, c_p,
                                                   c_i64, c_i64, c_int, c_int, c_p]
    lib.vsfeel_bm3d_process_device_ref.restype = c_int
    lib.vsfeel_bm3d_get_frame_ref.argtypes = [c_p, c_int, FETCH2_FN, RELEASE2_FN, c_p, c_p, c_sz]
    lib.vsfeel_bm3d_get_frame_ref.restype = c_int
    lib.vsfeel_bm3d_process_device.argtypes = [c_p, c_p, c_i64, c_i64, c_p, c_i64, c_i64, c_int,
                                               c_int, c_p]
    lib.vsfeel_bm3d_process_device.restype = c_int
    lib.vsfeel_bm3d_get_info.argtypes = [c_p, ctypes.POINTER(Info)]
    lib.vsfeel_bm3d_get_info.restype = c_int
    lib.vsfeel_bm3d_match_table_device.argtypes = [c_p, c_p, c_i64, c_i64, c_int, c_p]
    lib.vsfeel_bm3d_match_table_device.restype = c_int
    lib.vsfeel_bm3d_launch_count.argtypes = [c_p]
    lib.vsfeel_bm3d_launch_count.restype = c_i64
    lib.vsfeel_bm3d_trace.argtypes = [c_p, c_int]
    lib.vsfeel_bm3d_trace.restype = c_int
    lib.vsfeel_bm3d_trace_read.argtypes = [c_p, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(c_i64)]
    lib.vsfeel_bm3d_trace_read.restype = c_int
    lib.vsfeel_bm3d_saved_layout.argtypes = [c_p, ctypes.POINTER(SavedInfo)]
    lib.vsfeel_bm3d_saved_layout.restype = c_int
    lib.vsfeel_bm3d_forward_saved.argtypes = [c_p, c_p, c_i64, c_i64, c_p, c_i64, c_i64, c_p, c_p]
    lib.vsfeel_bm3d_forward_saved.restype = c_int
    lib.vsfeel_bm3d_backward.argtypes = [c_p, c_p, c_p, c_i64, c_i64, c_p, c_i64, c_i64, c_p]
    lib.vsfeel_bm3d_backward.restype = c_int
    lib.vsfeel_bm3d_batch_create.argtypes = [ctypes.POINTER(BatchClip), c_int, c_int, c_int,
                                             ctypes.POINTER(c_p)]
    lib.vsfeel_bm3d_batch_create.restype = c_int
    lib.vsfeel_bm3d_batch_run.argtypes = [c_p, c_p]
    lib.vsfeel_bm3d_batch_run.restype = c_int
    lib.vsfeel_bm3d_batch_finish.argtypes = [c_p]
    lib.vsfeel_bm3d_batch_finish.restype = c_int
    lib.vsfeel_bm3d_batch_classes.argtypes = [c_p, ctypes.POINTER(c_int), ctypes.POINTER(c_i64)]
    lib.vsfeel_bm3d_batch_classes.restype = c_int
    lib.vsfeel_bm3d_batch_class.argtypes = [c_p, c_int, ctypes.POINTER(BatchClassInfo)]
    lib.vsfeel_bm3d_batch_class.restype = c_int
    lib.vsfeel_bm3d_batch_free.argtypes = [c_p]
    lib.vsfeel_bm3d_batch_free.restype = None
    lib.vsfeel_bm3d_process_device_noalloc.argtypes = [ctypes.POINTER(Args),
                                                       ctypes.POINTER(VideoInfo), c_p, c_i64,
                                                       c_i64, c_p, c_i64, c_i64, c_int, c_int, c_p]
    lib.vsfeel_bm3d_process_device_noalloc.restype = c_int
    lib.vsfeel_bm3d_noalloc_scratch_bytes.argtypes = []
    lib.vsfeel_bm3d_noalloc_scratch_bytes.restype = c_i64
    lib.vsfeel_bm3d_last_error.argtypes = []
    lib.vsfeel_bm3d_last_error.restype = ctypes.c_char_p
    lib.vsfeel_bm3d_abi_version.argtypes = []
    lib.vsfeel_bm3d_abi_version.restype = c_int
    if lib.vsfeel_bm3d_abi_version() != ABI_VERSION:
        raise RuntimeError("libvsfeel_bm3d.so ABI version mismatch")
    if path is None:
        _lib = lib
    return lib


def last_error(lib: ctypes.CDLL) -> str:
    msg = lib.vsfeel_bm3d_last_error()
    return msg.decode() if msg else ""
