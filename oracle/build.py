"""TEST INFRASTRUCTURE: builds the CPU checkers used by the tests and the
benchmark's CPU legs. Nothing in the product path imports this module.

* ``oracle/libbm3d_oracle.so`` -- the C++ restatement (bm3d_oracle.cpp).
* ``oracle/_ref/libvsfeel_ref.so`` -- the reference's own shaders,
  ``src/bm3d.comp`` and ``src/bm3d_agg.comp``, compiled as C++ straight from
  the reference tree, plus the SIMT executor and host driver in
  ref_harness.cpp. Built only where the reference tree is present; the
  library itself travels with the repository snapshot.

The GLSL-to-C++ step changes declarations only, never a statement of shader
code:
  - ``#version`` / ``#extension`` / ``layout(local_size...) in;`` lines become
    blank lines (line numbers are kept);
  - a specialization constant becomes a run-time ``static`` variable that the
    host sets per dispatch, and other file-scope ``const`` values become
    macros so they follow it;
  - a storage buffer ``{ T name[]; }`` becomes a ``static T*``; the push
    constant block becomes a ``static struct``; ``shared`` becomes
    ``static thread_local`` (one workgroup per thread at a time);
  - ``out``/``inout`` array parameters become plain arrays (C++ passes them by
    pointer), a scalar ``out`` parameter becomes a reference, and
    ``T[n](a, b)`` array constructors become ``{a, b}`` initialisers;
  - ``main`` is renamed ``shader_main``.
GLSL lets the driver contract ``a*b + c``; the shaders are compiled with
``-ffp-contract=fast -mfma`` so the compiler fuses those statements into
single fma instructions, as a contracting GPU compiler does.
"""

from __future__ import annotations

import hashlib
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
# The reference tree's shader directory: VSFEEL_REFERENCE_SRC, or the
# ``--reference-src DIR`` argument of ``python -m oracle.build``, else the
# path where the reference is checked out beside this repository's builds.
DEFAULT_REF_SRC = Path("/root/reference/src")
REF_SRC = Path(os.environ.get("VSFEEL_REFERENCE_SRC", str(DEFAULT_REF_SRC)))
REF_OUT = HERE / "_ref"
ORACLE_SO = HERE / "libbm3d_oracle.so"
REF_SO = REF_OUT / "libvsfeel_ref.so"

CXX = os.environ.get("CXX", "g++")
ARCH = ["-march=x86-64-v3"]


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_oracle(force: bool = False) -> Path:
    src = HERE / "bm3d_oracle.cpp"
    if force or _stale(ORACLE_SO, [src, Path(__file__)]):
        _run([CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", *ARCH,
              "-pthread", str(src), "-o", str(ORACLE_SO)])
    return ORACLE_SO


def translate_glsl(text: str, namespace: str) -> str:
    """Declaration-level GLSL -> C++ rewrite (see the module docstring)."""
    specs: list[tuple[int, str, str]] = []
    bindings: list[tuple[int, str, str]] = []
    push_members = False
    out: list[str] = []
    for line in text.splitlines():
        if line.startswith("#version") or line.startswith("#extension"):
            out.append("")
            continue
        if re.match(r"\s*layout\s*\(\s*local_size", line):
            out.append("")
            continue
        m = re.match(r"layout\s*\(\s*constant_id\s*=\s*(\d+)\s*\)\s*const\s+(int|float)\s+(\w+)\s*=\s*([^;]+);(.*)$", line)
        if m:
            specs.append((int(m[1]), m[2], m[3]))
            out.append(f"static {m[2]} {m[3]} = {m[4]};{m[5]}")
            continue
        m = re.match(r"layout\s*\(([^)]*)\)\s*(?:readonly\s+|writeonly\s+)?buffer\s+\w+\s*\{\s*(\w+)\s+(\w+)\s*\[\s*\]\s*;\s*\}\s*;(.*)$", line)
        if m:
            b = re.search(r"binding\s*=\s*(\d+)", m[1])
            bindings.append((int(b[1]), m[2], m[3]))
            out.append(f"static {m[2]}* {m[3]};{m[4]}")
            continue
        if re.match(r"layout\s*\(\s*push_constant\s*\)\s*uniform", line):
            line = re.sub(r"layout\s*\(\s*push_constant\s*\)\s*uniform\s+(\w+)", r"static struct \1", line)
            push_members = True
        m = re.match(r"const\s+(int|float)\s+(\w+)\s*=\s*([^;]+);(.*)$", line)
        if m:
            out.append(f"#define {m[2]} ({m[3]}){m[4]}")
            continue
        line = re.sub(r"^shared\s+", "static thread_local ", line)
        line = re.sub(r"\b(?:float|int)\[\d+\]\(([^()]*)\)", r"{\1}", line)
        line = re.sub(r"\bout\s+(float|int)\s+(\w+)(?=\s*[,)])", r"\1 &\2", line)
        line = re.sub(r"\b(?:out|inout)\s+", "", line)
        line = re.sub(r"\bvoid\s+main\s*\(", "void shader_main(", line)
        out.append(line)
    if not push_members:
        raise RuntimeError("no push-constant block found")
    body = "\n".join(out)
    spec_cases = "\n".join(
        f"        case {i}: {name} = ({ty})v; break;" for i, ty, name in sorted(specs))
    bind_cases = "\n".join(
        f"        case {i}: {name} = ({ty}*)p; break;" for i, ty, name in sorted(bindings))
    return f"""// generated by oracle/build.py from the reference shader; do not edit
#include <atomic>
#include <cstdint>
#include <cstring>
#include "ref_simt.h"
namespace {namespace} {{
SIMT_GLSL_BUILTINS
#line 1
{body}
void set_spec_(int id, double v) {{
    switch (id) {{
{spec_cases}
        default: break;
    }}
}}
void bind_(int binding, void* p) {{
    switch (binding) {{
{bind_cases}
        default: break;
    }}
}}
}}  // namespace {namespace}
extern "C" void {namespace}_set_spec(int id, double v) {{ {namespace}::set_spec_(id, v); }}
extern "C" void {namespace}_bind(int binding, void* p) {{ {namespace}::bind_(binding, p); }}
extern "C" void {namespace}_push(const int32_t* v, int n) {{
    std::memcpy(&{namespace}::pc, v, sizeof(int32_t) * (size_t)n);
}}
extern "C" void {namespace}_entry() {{ {namespace}::shader_main(); }}
"""


def reference_available(src: Path | None = None) -> bool:
    src = Path(src) if src else REF_SRC
    return (src / "bm3d.comp").is_file() and (src / "bm3d_agg.comp").is_file()


def build_ref(force: bool = False, src: str | os.PathLike | None = None) -> Path | None:
    """Compiles the reference shaders under ``src`` (default REF_SRC) for the
    CPU; None when the tree is absent and nothing was built before."""
    src = Path(src) if src else REF_SRC
    if not reference_available(src):
        return REF_SO if REF_SO.exists() else None
    REF_OUT.mkdir(exist_ok=True)
    shaders = {"ref_bm3d": src / "bm3d.comp", "ref_bm3d_agg": src / "bm3d_agg.comp"}
    harness = HERE / "ref_harness.cpp"
    simt_h = HERE / "ref_simt.h"
    deps = [*shaders.values(), harness, simt_h, Path(__file__)]
    if not force and not _stale(REF_SO, deps):
        return REF_SO
    objs = []
    flags = ["-O2", "-std=c++20", "-fPIC", "-ffp-contract=fast", *ARCH, "-w", f"-I{HERE}"]
    for ns, path in shaders.items():
        cpp = REF_OUT / f"{ns}.cpp"
        cpp.write_text(translate_glsl(path.read_text(), ns))
        obj = REF_OUT / f"{ns}.o"
        _run([CXX, *flags, "-c", str(cpp), "-o", str(obj)])
        objs.append(str(obj))
    obj = REF_OUT / "ref_harness.o"
    _run([CXX, *flags, "-c", str(harness), "-o", str(obj)])
    objs.append(str(obj))
    _run([CXX, "-shared", "-pthread", *objs, "-o", str(REF_SO)])
    return REF_SO


def main(argv: list[str] | None = None) -> int:
    import argparse

    ap = argparse.ArgumentParser(description="build the CPU checkers")
    ap.add_argument("--force", action="store_true", help="rebuild even when up to date")
    ap.add_argument("--reference-src", default=None,
                    help="the reference tree's src/ directory (default: VSFEEL_REFERENCE_SRC "
                         f"or {DEFAULT_REF_SRC})")
    a = ap.parse_args(argv)
    print(build_oracle(a.force))
    print(build_ref(a.force, a.reference_src))
    return 0


if __name__ == "__main__":
    sys.exit(main())
