"""Generates tests/golden/bm3d_golden.npz from the reference's own shaders.

The reference (src/bm3d.comp, src/bm3d_agg.comp) is compiled for the CPU by
oracle/build.py and executed by its SIMT executor with one thread, so atomic
adds land in a fixed order and the outputs are reproducible bit for bit.
Each case stores its seeded input frames, its arguments and the reference
output. The fixtures let machines without the reference tree (the GPU box)
check the oracle and the CUDA path against the reference itself.

Run from the repository root:  python tests/golden/make_golden.py
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "vapoursynth-feel_b200"))

from oracle import Params, ReferenceShaders  # noqa: E402
from vsfeel.synthetic import make_clip  # noqa: E402

OUT = Path(__file__).resolve().parent / "bm3d_golden.npz"

# (name, nframes, height, width, params, shift, seed): small shapes that
# cover both scan paths, every radius, odd steps, border clamping, the
# extractor, sigma 0 and a window wider than the frame.
CASES = [
    ("r0_step8", 3, 40, 48, dict(sigma=3.0, block_step=8, bm_range=9, radius=0), 3, 11),
    ("r0_step3", 2, 33, 41, dict(sigma=5.0, block_step=3, bm_range=6, radius=0), 3, 12),
    ("r1_q5", 5, 40, 48, dict(sigma=5.0, block_step=4, bm_range=12, radius=1, ps_num=2,
                               ps_range=5), 3, 13),
    ("r2_c2like", 6, 48, 64, dict(sigma=3.0, block_step=4, bm_range=16, radius=2, ps_num=2,
                                   ps_range=7), 4, 14),
    ("r2_ext", 5, 36, 44, dict(sigma=10.0, block_step=5, bm_range=7, radius=2, ps_num=3,
                                ps_range=3, extractor_exp=1), 3, 15),
    ("r3_exact", 7, 32, 40, dict(sigma=8.0, block_step=4, bm_range=6, radius=3, ps_num=3,
                                  ps_range=3, extractor_exp=2), 6, 16),
    ("r4_exact", 9, 32, 32, dict(sigma=8.0, block_step=4, bm_range=5, radius=4, ps_num=4,
                                  ps_range=2, extractor_exp=2), 6, 17),
    ("r1_sigma0", 3, 24, 24, dict(sigma=0.0, block_step=2, bm_range=3, radius=1, ps_num=1,
                                   ps_range=1), 2, 18),
    ("r2_tiny", 4, 8, 8, dict(sigma=4.0, block_step=8, bm_range=9, radius=2, ps_num=8,
                               ps_range=4), 2, 19),
    ("r1_step1", 3, 16, 20, dict(sigma=6.0, block_step=1, bm_range=4, radius=1, ps_num=2,
                                  ps_range=2), 2, 20),
]

# the final (Wiener) pass: "ref" is the reference's own basic estimate of
# the same clip
FINAL_CASES = [
    ("final_r0", 3, 40, 48, dict(sigma=4.0, block_step=8, bm_range=9, radius=0), 3, 31),
    ("final_r1", 4, 40, 48, dict(sigma=6.0, block_step=4, bm_range=8, radius=1, ps_num=2,
                                  ps_range=3), 3, 32),
    ("final_r2_ext", 5, 36, 44, dict(sigma=10.0, block_step=3, bm_range=6, radius=2, ps_num=2,
                                      ps_range=3, extractor_exp=2), 3, 33),
    ("final_r3_exact", 5, 32, 40, dict(sigma=8.0, block_step=4, bm_range=5, radius=3, ps_num=2,
                                        ps_range=2), 5, 34),
]


def main() -> int:
    ref = ReferenceShaders()
    arrays: dict[str, np.ndarray] = {}
    meta = []
    for name, n, h, w, kw, shift, seed in CASES:
        p = Params(**kw)
        frames = make_clip(n, h, w, sigma=max(p.sigma, 1.0), shift=shift, seed=seed)
        out = ref.bm3d(frames, p, nthreads=1)
        arrays[f"{name}/input"] = frames
        arrays[f"{name}/output"] = out
        meta.append(dict(name=name, params=p.as_dict()))
        print(f"{name}: {frames.shape} -> mean {float(out.mean()):.6f}")
    for name, n, h, w, kw, shift, seed in FINAL_CASES:
        p = Params(**kw)
        frames = make_clip(n, h, w, sigma=max(p.sigma, 1.0), shift=shift, seed=seed)
        basic = ref.bm3d(frames, p, nthreads=1)
        out = ref.bm3d(frames, p, nthreads=1, ref=basic)
        arrays[f"{name}/input"] = frames
        arrays[f"{name}/ref"] = basic
        arrays[f"{name}/output"] = out
        meta.append(dict(name=name, params=p.as_dict(), final=True))
        print(f"{name}: {frames.shape} -> mean {float(out.mean()):.6f}")
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
