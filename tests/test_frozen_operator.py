"""The FP64 frozen-match operator (the gradient tests' reference) on the CPU.

It is pinned to the oracle: rebuilt from the oracle's own FP64 match tables
and keep masks, it must reproduce the oracle's FP64 denoised output, so its
transform scaling, DC rule, weights and slice bookkeeping at the clip ends
are the reference algorithm's.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import Params
from oracle.frozen_operator import SavedState, agg_slice, dct_matrix, slice_reads


def test_dct_matrix_is_the_reference_transform_pair(oracle_lib):
    C = dct_matrix()
    eye = np.eye(8)
    fwd = np.stack([oracle_lib.dct8(eye[i], fp64=True) for i in range(8)], axis=1)
    inv = np.stack([oracle_lib.dct8(eye[i], inverse=True, fp64=True) for i in range(8)], axis=1)
    np.testing.assert_allclose(fwd, 4 * C, atol=1e-14)
    np.testing.assert_allclose(inv, 4 * C.T, atol=1e-14)


@pytest.mark.parametrize("nframes,radius", [(1, 0), (5, 0), (3, 1), (8, 2), (3, 2), (12, 4),
                                            (4, 4)])
def test_slice_reads_cover_each_output_tw_times(oracle_lib, nframes, radius):
    tw = 2 * radius + 1
    per_output = np.zeros(nframes, dtype=int)
    for m in range(nframes):
        for z in range(tw):
            n = min(max(m - radius + z, 0), nframes - 1)
            per_output[n] += slice_reads(m, z, nframes, radius)
    assert (per_output == tw).all()
    for n in range(nframes):
        for i in range(tw):
            assert agg_slice(i, n, nframes, radius) == (
                0 if radius == 0 else oracle_lib.agg_z(i, n, nframes, radius))


@pytest.mark.parametrize("params,n,h,w", [
    (dict(sigma=5.0, block_step=4, bm_range=6, radius=1, ps_num=2, ps_range=3), 4, 32, 40),
    (dict(sigma=8.0, block_step=3, bm_range=5, radius=0), 2, 24, 30),
    (dict(sigma=6.0, block_step=4, bm_range=5, radius=2, ps_num=2, ps_range=2), 3, 24, 32),
])
def test_frozen_operator_reproduces_the_oracle(oracle_lib, params, n, h, w):
    import torch

    from vsfeel.synthetic import make_clip as mk

    p = Params(**params)
    frames = mk(n, h, w, sigma=p.sigma, shift=2, seed=17)
    tables, words = [], []
    for m in range(n):
        t, k = oracle_lib.frozen_state(frames, p, m, fp64=True)
        tables.append(t)
        words.append(k)
    st = SavedState.from_tables(tables, words, n, h, w, p.radius)
    out = st.apply(torch.from_numpy(frames.astype(np.float64)))
    expected = oracle_lib.bm3d(frames, p, fp64=True)
    assert float(np.abs(out.numpy() - expected).max()) <= 1e-12

    # constant clips pass unchanged (only the always-kept DC survives)
    ones = st.apply(torch.ones(n, h, w, dtype=torch.float64))
    assert float((ones - 1).abs().max()) <= 1e-12

    # the operator's adjoint (autograd) satisfies <A x, y> = <x, A^T y>
    rng = np.random.default_rng(3)
    xv = torch.from_numpy(rng.standard_normal((n, h, w))).requires_grad_(True)
    yv = torch.from_numpy(rng.standard_normal((n, h, w)))
    lhs = (st.apply(xv) * yv).sum()
    lhs.backward()
    rhs = (xv.detach() * xv.grad).sum()
    lhs = float(lhs.detach())
    assert abs(lhs - float(rhs)) <= 1e-9 * max(1.0, abs(lhs))
