"""The CPU oracle: pinned to the reference's own shaders, and its building
blocks checked against first principles (CPU only)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import Params, ReferenceShaders
from vsfeel.synthetic import make_clip


def test_oracle_matches_golden_vectors_bit_exact(golden, oracle_lib):
    """Every golden case (reference shaders, executed serially) is reproduced
    bit for bit by the oracle."""
    for name, params, frames, expected in golden:
        out = oracle_lib.bm3d(frames, Params(**params), nthreads=1)
        assert out.dtype == np.float32
        assert np.array_equal(out, expected), f"{name}: oracle differs from the reference"


def test_oracle_thread_count_does_not_change_bits(golden, oracle_lib):
    name, params, frames, expected = golden[3]
    out = oracle_lib.bm3d(frames, Params(**params), nthreads=4)
    assert np.array_equal(out, expected)


@pytest.mark.skipif(not ReferenceShaders.available(), reason="reference shaders not built")
@pytest.mark.parametrize("radius,step,bm_range,ps_num,ps_range,ext", [
    (0, 4, 8, 2, 4, 0), (1, 3, 5, 1, 2, 3), (2, 6, 9, 5, 3, 0), (3, 4, 4, 2, 2, 0),
    (4, 7, 3, 8, 1, 1),
])
def test_oracle_matches_reference_shaders_random(radius, step, bm_range, ps_num, ps_range, ext,
                                                 oracle_lib):
    """Fresh seeded inputs, the reference shaders run live."""
    p = Params(sigma=4.0 + radius, block_step=step, bm_range=bm_range, radius=radius,
               ps_num=ps_num, ps_range=ps_range, extractor_exp=ext)
    frames = make_clip(2 * radius + 3, 30, 37, sigma=p.sigma, shift=4, seed=100 + radius)
    ref = ReferenceShaders().bm3d(frames, p, nthreads=1)
    out = oracle_lib.bm3d(frames, p, nthreads=2)
    assert np.array_equal(out, ref)


@pytest.mark.skipif(not ReferenceShaders.available(), reason="reference shaders not built")
def test_oracle_stack_slices_match_reference(oracle_lib):
    p = Params(sigma=5.0, block_step=4, bm_range=6, radius=2, ps_num=2, ps_range=3)
    frames = make_clip(5, 32, 40, sigma=5.0, seed=3)
    for m in (0, 2, 4):
        a = oracle_lib.stack(frames, p, m, nthreads=1)
        b = ReferenceShaders().stack(frames, p, m, nthreads=1)
        assert np.array_equal(a, b), f"stack {m}"


def test_oracle_final_pass_matches_golden_vectors_bit_exact(golden_final, oracle_lib):
    """The final (Wiener) pass: reference shaders' output with the reference's
    own basic estimate as "ref", reproduced bit for bit."""
    assert len(golden_final) >= 4
    for name, params, frames, ref, expected in golden_final:
        out = oracle_lib.bm3d(frames, Params(**params), nthreads=1, ref=ref)
        assert np.array_equal(out, expected), f"{name}: oracle differs from the reference"


@pytest.mark.skipif(not ReferenceShaders.available(), reason="reference shaders not built")
@pytest.mark.parametrize("radius,step,bm_range,ps_num,ps_range,ext", [
    (0, 5, 7, 2, 4, 0), (1, 4, 6, 2, 3, 0), (2, 3, 5, 3, 2, 1), (4, 4, 4, 4, 2, 2),
])
def test_oracle_final_pass_matches_reference_shaders(radius, step, bm_range, ps_num, ps_range,
                                                     ext, oracle_lib):
    p = Params(sigma=6.0, block_step=step, bm_range=bm_range, radius=radius, ps_num=ps_num,
               ps_range=ps_range, extractor_exp=ext)
    frames = make_clip(2 * radius + 2, 30, 37, sigma=p.sigma, shift=3, seed=200 + radius)
    basic = oracle_lib.bm3d(frames, p, nthreads=2)
    ref = ReferenceShaders().bm3d(frames, p, nthreads=1, ref=basic)
    out = oracle_lib.bm3d(frames, p, nthreads=2, ref=basic)
    assert np.array_equal(out, ref)


def test_final_pass_is_finite_and_differs_from_the_basic_estimate(oracle_lib):
    """The reference's own check of the ref pass (tests/test_bm3dv2.py:165-181):
    finite, and more than 1e-4 away from the basic estimate."""
    p = Params(sigma=8.0, block_step=4, bm_range=8, radius=1, ps_num=2, ps_range=3)
    frames = make_clip(4, 40, 48, sigma=8.0, seed=7)
    basic = oracle_lib.bm3d(frames, p)
    final = oracle_lib.bm3d(frames, p, ref=basic)
    assert np.isfinite(final).all()
    assert float(np.abs(final - basic).max()) > 1e-4
    f64 = oracle_lib.bm3d(frames, p, ref=basic, fp64=True)
    assert float(np.abs(final - f64).max()) < 1e-5


def _dct2_ortho(v):
    n = len(v)
    k = np.arange(n)[:, None]
    i = np.arange(n)[None, :]
    m = np.cos(np.pi * (2 * i + 1) * k / (2 * n)) * np.sqrt(2.0 / n)
    m[0] /= np.sqrt(2.0)
    return m @ v


def test_dct_is_four_times_orthonormal_dct2(oracle_lib):
    rng = np.random.default_rng(0)
    for _ in range(20):
        v = rng.standard_normal(8)
        got = oracle_lib.dct8(v, fp64=True)
        assert np.allclose(got, 4.0 * _dct2_ortho(v), atol=1e-12)


def test_dct_inverse_is_scaled_transpose(oracle_lib):
    rng = np.random.default_rng(1)
    for _ in range(20):
        v = rng.standard_normal(8)
        fwd = oracle_lib.dct8(v, fp64=True)
        back = oracle_lib.dct8(fwd, inverse=True, fp64=True)
        assert np.allclose(back, 16.0 * v, atol=1e-12)


def test_threshold_factor(oracle_lib):
    # src/bm3d.cpp:1103-1113: sigma * bit_cast<float>(0x3f021bb6) in float
    f = np.frombuffer(np.uint32(0x3F021BB6).tobytes(), dtype=np.float32)[0]
    for s in (0.0, 0.7, 3.0, 8.0):
        assert oracle_lib.threshold(s) == np.float32(np.float32(s) * f)


def test_agg_z_steady_state_and_boundaries(oracle_lib):
    # src/bm3d.cpp:369-371: in the steady state slice 2r-i of stack n-r+i is frame n
    n_frames, r = 20, 2
    for n in range(r, n_frames - r):
        assert [oracle_lib.agg_z(i, n, n_frames, r) for i in range(2 * r + 1)] == [4, 3, 2, 1, 0]
    # first frame: the clamped stacks all read their own frame's slice
    assert [oracle_lib.agg_z(i, 0, n_frames, r) for i in range(5)] == [2, 2, 2, 1, 0]
    assert [oracle_lib.agg_z(i, n_frames - 1, n_frames, r) for i in range(5)] == [4, 3, 2, 2, 2]


def test_block_count(oracle_lib):
    assert oracle_lib.block_count(1920, 1080, 4) == 479 * 269 == 128851
    assert oracle_lib.block_count(640, 360, 8) == 80 * 45
    assert oracle_lib.block_count(641, 360, 8) == 81 * 45  # clamped last column at x=633
    assert oracle_lib.block_count(8, 8, 8) == 1


def test_sliding_scan_differs_from_true_ssd_only_below_radius3(oracle_lib):
    """The radius<3 scan is the reference's column bookkeeping, not the full
    8x8 SSD: with radius forced to 3 (full SSD) on a single frame the
    matches change, which is why both scans are kept."""
    frames = make_clip(1, 48, 48, sigma=5.0, seed=5)
    a = oracle_lib.matches(frames, Params(block_step=4, bm_range=8, radius=0), 0)
    assert a.shape == (oracle_lib.block_count(48, 48, 4), 8, 3)
    # the forced self-match sits in every group
    nbx = (48 - 9 + 8) // 4
    for b in range(a.shape[0]):
        y, x = divmod(b, nbx)
        assert any((a[b, k, 0] == min(x * 4, 40) and a[b, k, 1] == min(y * 4, 40))
                   for k in range(8))


def test_fp64_oracle_is_close(oracle_lib):
    frames = make_clip(3, 40, 48, sigma=3.0, seed=9)
    p = Params(sigma=3.0, block_step=4, bm_range=8, radius=1, ps_num=2, ps_range=4)
    a = oracle_lib.bm3d(frames, p)
    b = oracle_lib.bm3d(frames, p, fp64=True)
    assert b.dtype == np.float64
    assert np.abs(a - b).mean() < 1e-5


def test_denoising_improves_psnr(oracle_lib):
    noisy = make_clip(3, 64, 64, sigma=8.0, seed=21)
    clean = make_clip(3, 64, 64, sigma=8.0, seed=21, noise=False)
    out = oracle_lib.bm3d(noisy, Params(sigma=8.0, block_step=4, bm_range=8, radius=1))
    mse = lambda a: float(np.mean((a - clean) ** 2))
    assert mse(out) < 0.5 * mse(noisy)


def test_oracle_rejects_bad_arguments(oracle_lib):
    frames = make_clip(2, 16, 16, seed=1)
    with pytest.raises(ValueError):
        oracle_lib.bm3d(frames, Params(radius=5))
    with pytest.raises(ValueError):
        oracle_lib.bm3d(frames[:, :7, :], Params())
