"""The wheel: builds offline from a copy of the tree, carries the package,
the sm_100a library and the C header, is tagged py3-none-<platform>, and
imports and loads the library once installed (CPU only; no kernel runs)."""

from __future__ import annotations

import shutil
import subprocess
import sys
import zipfile

import pytest

from conftest import ROOT

PKG_FILES = ("vsfeel/__init__.py", "vsfeel/_lib.py", "vsfeel/autograd.py", "vsfeel/batch.py",
             "vsfeel/shard.py", "vsfeel/synthetic.py", "vsfeel/libvsfeel_bm3d.so",
             "vsfeel/include/vsfeel_bm3d.h")


def _build_wheel(tmp_path_factory, env=None):
    import os

    lib = ROOT / "vapoursynth-feel_b200" / "vsfeel" / "libvsfeel_bm3d.so"
    if not lib.exists():
        pytest.skip("library not built")
    src = tmp_path_factory.mktemp("src")
    for name in ("pyproject.toml", "setup.py", "README.md"):
        shutil.copy2(ROOT / name, src / name)
    shutil.copytree(ROOT / "include", src / "include")
    # copy2 keeps the times, so the build reuses the library instead of recompiling
    shutil.copytree(ROOT / "vapoursynth-feel_b200", src / "vapoursynth-feel_b200",
                    ignore=shutil.ignore_patterns("__pycache__", "*.o"))
    out = tmp_path_factory.mktemp("dist")
    subprocess.run([sys.executable, "-m", "pip", "wheel", "--no-deps", "--no-build-isolation",
                    "--no-index", "-q", "-w", str(out), str(src)], check=True, timeout=600,
                   env={**os.environ, **(env or {})})
    wheels = list(out.glob("*.whl"))
    assert len(wheels) == 1, wheels
    return wheels[0]


@pytest.fixture(scope="module")
def wheel(tmp_path_factory):
    return _build_wheel(tmp_path_factory, {"VSFEEL_VS_PLUGIN": ""})


@pytest.fixture(scope="module")
def plugin_wheel(tmp_path_factory):
    """A wheel built with a VapourSynth plugin supplied from outside (the SDK
    header is not installed here, so a stand-in shared object plays the
    plugin: only its placement is under test)."""
    d = tmp_path_factory.mktemp("plugin")
    c = d / "stand_in.c"
    c.write_text("int vsfeel_plugin_stand_in(void) { return 7; }\n")
    so = d / "stand_in.so"
    subprocess.run(["gcc", "-shared", "-fPIC", str(c), "-o", str(so)], check=True, timeout=120)
    return _build_wheel(tmp_path_factory, {"VSFEEL_VS_PLUGIN": str(so)}), so


def test_wheel_contents_and_tag(wheel):
    assert wheel.name.startswith("vapoursynth_feel_b200-1.0.0-py3-none-linux_")
    with zipfile.ZipFile(wheel) as z:
        names = set(z.namelist())
        for f in PKG_FILES:
            assert f in names, f
        assert not any(n.startswith(("oracle/", "tests/", "csrc/")) for n in names)
        info = next(n for n in names if n.endswith(".dist-info/WHEEL"))
        text = z.read(info).decode()
        assert "Root-Is-Purelib: false" in text
        header = z.read("vsfeel/include/vsfeel_bm3d.h")
    assert header == (ROOT / "include" / "vsfeel_bm3d.h").read_bytes()


def test_installed_wheel_loads_the_library(wheel, tmp_path):
    target = tmp_path / "site"
    subprocess.run([sys.executable, "-m", "pip", "install", "--no-deps", "--no-index", "-q",
                    "--target", str(target), str(wheel)], check=True, timeout=300)
    code = (
        "import sys; sys.path.insert(0, sys.argv[1]);"
        "import vsfeel, os;"
        "from vsfeel import _lib;"
        "lib = _lib.load();"
        "assert vsfeel.__file__.startswith(sys.argv[1]), vsfeel.__file__;"
        "assert vsfeel.library_path().startswith(sys.argv[1]);"
        "assert os.path.exists(os.path.join(vsfeel.get_include(), 'vsfeel_bm3d.h'));"
        "assert vsfeel.get_include().startswith(sys.argv[1]);"
        "print(lib.vsfeel_bm3d_abi_version())"
    )
    # run outside the checkout so that nothing resolves to the source tree
    res = subprocess.run([sys.executable, "-c", code, str(target)], capture_output=True,
                         text=True, cwd=tmp_path, timeout=120)
    assert res.returncode == 0, res.stderr
    from vsfeel import _lib

    assert res.stdout.strip() == str(_lib.ABI_VERSION)


def test_wheel_places_the_vapoursynth_plugin_where_vapoursynth_autoloads(plugin_wheel):
    wheel, so = plugin_wheel
    with zipfile.ZipFile(wheel) as z:
        names = set(z.namelist())
        # the reference's wheel layout (hatch_build.py:12-24): the plugin in
        # vapoursynth/plugins/vsfeel of site-packages, the library beside the
        # package (the plugin's run path: $ORIGIN/../../../vsfeel)
        assert "vapoursynth/plugins/vsfeel/libvsfeel.so" in names
        assert "vsfeel/libvsfeel_bm3d.so" in names
        assert z.read("vapoursynth/plugins/vsfeel/libvsfeel.so") == so.read_bytes()


def test_wheel_without_sdk_ships_no_plugin(wheel):
    with zipfile.ZipFile(wheel) as z:
        assert not any(n.startswith("vapoursynth/") for n in z.namelist())


def test_vapoursynth_shim_registers_the_reference_interface():
    """The shim source (compiled only where VapourSynth4.h is installed)
    registers BM3Dv2 in the reference's namespace with its argument string
    byte for byte (src/bm3d.cpp:1562-1571, src/vsfeel.cpp:350-364) and
    forwards to the C ABI."""
    import re

    src = (ROOT / "vapoursynth-feel_b200" / "csrc" / "vs_shim.cpp").read_text()
    assert "VS_EXTERNAL_API(void) VapourSynthPluginInit2(" in src
    assert '"com.thefeeltrain.vsfeel", "vsfeel"' in src
    reg = src[src.index('registerFunction("BM3Dv2"'):]
    reg = reg[:reg.index("bm3d_create")]
    joined = "".join(re.findall(r'"([^"]*)"', reg))
    assert joined == ("BM3Dv2"
                      "clip:vnode;ref:vnode:opt;sigma:float[]:opt;block_step:int[]:opt;"
                      "bm_range:int[]:opt;radius:int:opt;ps_num:int[]:opt;ps_range:int[]:opt;"
                      "num_streams:int:opt;extractor_exp:int:opt;"
                      "clip:vnode;")
    for call in ("vsfeel_bm3d_create(", "vsfeel_bm3d_frame_range(", "vsfeel_bm3d_get_frame(",
                 "vsfeel_bm3d_get_frame_ref(", "vsfeel_bm3d_free("):
        assert call in src, call
