"""Wheel build of the vsfeel package (metadata in pyproject.toml).

The build compiles libvsfeel_bm3d.so for sm_100a with nvcc (reusing the
in-tree library when it is newer than every source), puts it and the C
header include/vsfeel_bm3d.h inside the package, places the VapourSynth plugin
(csrc/vs_shim.cpp, built where the SDK header is installed) at
vapoursynth/plugins/vsfeel/libvsfeel.so, and tags the wheel
py3-none-<platform>: the library is native, the Python code is not tied to
an interpreter ABI (it loads the library with ctypes). This plays the part
of the reference's hatch_build.py hook (hatch_build.py:1-24), which marks
its wheel platform-specific and copies the built plugin into it.
"""

from __future__ import annotations

import importlib.util
import os
import shutil
from pathlib import Path

from setuptools import setup
from setuptools.command.bdist_wheel import bdist_wheel
from setuptools.command.build_py import build_py
from setuptools.dist import Distribution

ROOT = Path(__file__).resolve().parent
CSRC = ROOT / "vapoursynth-feel_b200" / "csrc"
HEADER = ROOT / "include" / "vsfeel_bm3d.h"


def _csrc_build():
    spec = importlib.util.spec_from_file_location("vsfeel_csrc_build", CSRC / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _vs_plugin(mod) -> Path | None:
    """The VapourSynth plugin to ship: $VSFEEL_VS_PLUGIN (a plugin built
    elsewhere against the same library), else the shim built here when the
    SDK header is installed, else none."""
    given = os.environ.get("VSFEEL_VS_PLUGIN")
    if given:
        return Path(given)
    return mod.build_vs_shim()


class BuildPy(build_py):
    def run(self):
        mod = _csrc_build()
        lib = mod.build()
        plugin = _vs_plugin(mod)
        super().run()
        dest = Path(self.build_lib) / "vsfeel"
        dest.mkdir(parents=True, exist_ok=True)
        shutil.copy2(lib, dest / lib.name)
        (dest / "include").mkdir(exist_ok=True)
        shutil.copy2(HEADER, dest / "include" / HEADER.name)
        if plugin is not None:
            # where VapourSynth autoloads plugins of a Python install, as the
            # reference's wheel does (hatch_build.py:12-24, pyproject.toml:30-37)
            pdir = Path(self.build_lib) / "vapoursynth" / "plugins" / "vsfeel"
            pdir.mkdir(parents=True, exist_ok=True)
            shutil.copy2(plugin, pdir / "libvsfeel.so")


class BinaryDistribution(Distribution):
    def has_ext_modules(self):
        return True


class BdistWheel(bdist_wheel):
    def get_tag(self):
        _, _, plat = super().get_tag()
        return "py3", "none", plat


setup(cmdclass={"build_py": BuildPy, "bdist_wheel": BdistWheel}, distclass=BinaryDistribution)
