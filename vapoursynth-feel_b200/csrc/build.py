"""Builds the product library vsfeel/libvsfeel_bm3d.so for sm_100a.

nvcc cross-compiles here without a GPU; the .so is built in-tree so that it
travels with the repository snapshot. Device code is compiled with
-fmad=false: the kernels spell every fused operation explicitly
(__fmaf_rn), so no other multiply-add may be contracted.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent
PKG = CSRC.parent / "vsfeel"
INCLUDE = CSRC.parent.parent / "include"
LIB = PKG / "libvsfeel_bm3d.so"
SOURCES = ["bm3d_kernels.cu", "bm3d_match.cu", "bm3d_match_8x4.cu", "bm3d_match_16x2.cu",
           "bm3d_match_4x8.cu", "bm3d_match_8x2.cu", "bm3d_match_4x4.cu", "bm3d_engine.cu",
           "bm3d_noalloc.cu", "bm3d_batch.cu"]
HEADERS = ["bm3d_device.cuh", "bm3d_filter.cuh", "bm3d_match.cuh"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-O2,-fvisibility=hidden", "-I", str(INCLUDE),
]


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [INCLUDE / "vsfeel_bm3d.h", Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    build_dir = CSRC / "_build"
    build_dir.mkdir(exist_ok=True)

    def compile_one(src):
        obj = build_dir / (Path(src).stem + ".o")
        cmd = [NVCC, *FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        return src, obj, subprocess.run(cmd, capture_output=True, text=True)

    from concurrent.futures import ThreadPoolExecutor

    objs = []
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        for src, obj, proc in pool.map(compile_one, SOURCES):
            if proc.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{proc.stdout}\n{proc.stderr}")
            if verbose:
                sys.stderr.write(proc.stderr)
            objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    proc = subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
                           *objs, "-o", str(tmp), "-lcudart_static", "-lrt", "-lpthread", "-ldl"],
                          capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"link failed:\n{proc.stdout}\n{proc.stderr}")
    os.replace(tmp, LIB)
    return LIB


# The VapourSynth plugin (vs_shim.cpp): built only where the SDK header
# VapourSynth4.h is installed; the SDK is not part of this repository.
SHIM_SRC = CSRC / "vs_shim.cpp"
SHIM_LIB = CSRC / "_build" / "libvsfeel.so"


def vapoursynth_include() -> Path | None:
    """The directory holding VapourSynth4.h: $VAPOURSYNTH_INCLUDE, pkg-config's
    vapoursynth flags, or the usual system locations; None when absent."""
    cands = []
    if os.environ.get("VAPOURSYNTH_INCLUDE"):
        cands.append(Path(os.environ["VAPOURSYNTH_INCLUDE"]))
    try:
        out = subprocess.run(["pkg-config", "--cflags-only-I", "vapoursynth"],
                             capture_output=True, text=True, timeout=10)
        if out.returncode == 0:
            cands += [Path(f[2:]) for f in out.stdout.split() if f.startswith("-I")]
    except (OSError, subprocess.TimeoutExpired):
        pass
    cands += [Path("/usr/include/vapoursynth"), Path("/usr/local/include/vapoursynth")]
    for c in cands:
        if (c / "VapourSynth4.h").is_file():
            return c
    return None


def build_vs_shim(force: bool = False) -> Path | None:
    """Compiles the VapourSynth plugin against libvsfeel_bm3d.so; None when
    the SDK header is not installed. Its run path finds the library in the
    installed layout (site-packages/vapoursynth/plugins/vsfeel/ ->
    site-packages/vsfeel/) and beside itself."""
    inc = vapoursynth_include()
    if inc is None:
        return None
    lib = build()
    if not force and SHIM_LIB.exists() and SHIM_LIB.stat().st_mtime > max(
            SHIM_SRC.stat().st_mtime, lib.stat().st_mtime):
        return SHIM_LIB
    SHIM_LIB.parent.mkdir(exist_ok=True)
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-fvisibility=hidden", "-I", str(inc),
           "-I", str(INCLUDE), str(SHIM_SRC), "-L", str(PKG), "-lvsfeel_bm3d",
           "-Wl,-rpath,$ORIGIN/../../../vsfeel", "-Wl,-rpath,$ORIGIN", "-o", str(SHIM_LIB)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"VapourSynth plugin build failed:\n{proc.stdout}\n{proc.stderr}")
    return SHIM_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_vs_shim(force="--force" in sys.argv) or "VapourSynth4.h not found: plugin skipped")
