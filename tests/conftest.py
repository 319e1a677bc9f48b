"""Shared test setup.

Markers: ``gpu`` tests need a CUDA device (B200) and run the product path
through the C ABI; everything else runs on the CPU.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "vapoursynth-feel_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden" / "bm3d_golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_golden():
    """Basic-estimate cases: [(name, params dict, input frames, reference output)]"""
    data = np.load(GOLDEN)
    meta = json.loads(bytes(data["meta"]).decode())
    return [(m["name"], m["params"], data[f"{m['name']}/input"], data[f"{m['name']}/output"])
            for m in meta if not m.get("final")]


def load_golden_final():
    """Final-pass cases: [(name, params dict, input frames, ref frames, reference output)]"""
    data = np.load(GOLDEN)
    meta = json.loads(bytes(data["meta"]).decode())
    return [(m["name"], m["params"], data[f"{m['name']}/input"], data[f"{m['name']}/ref"],
             data[f"{m['name']}/output"]) for m in meta if m.get("final")]


@pytest.fixture(scope="session")
def golden():
    return load_golden()


@pytest.fixture(scope="session")
def golden_final():
    return load_golden_final()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import Oracle
    return Oracle()
