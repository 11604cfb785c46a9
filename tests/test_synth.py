"""Seeded synthetic inputs (hifde3d_b200/synth.py), CPU.

The same seeded streams feed the CUDA path, the oracle and the reference probe,
so they must be deterministic and have the stated distributions:
* splitmix64 -> uniform [0, 1) -> Box-Muller normals, reproducible from the seed;
* the Gaussian random field has standard deviation sigma and the Gaussian
  covariance exp(-r^2 / (2 ell^2)) in the generator's box units; sampled on the
  unit cube by face_coefficients_grf its correlation length is ell / 2 (the
  cube is mapped onto the generator's box of length 2);
* the high-contrast field takes values 10^U(-3, 3) on 8^3 sub-cubes.
"""
import numpy as np
import pytest

from hifde3d_b200 import synth


def test_streams_are_seeded_and_distributed():
    u = synth.uniform(7, 200000)
    assert np.array_equal(u, synth.uniform(7, 200000))
    assert not np.array_equal(u, synth.uniform(8, 200000))
    assert u.min() >= 0.0 and u.max() < 1.0
    assert u.mean() == pytest.approx(0.5, abs=0.005)
    z = synth.normal(3, 200000)
    assert z.mean() == pytest.approx(0.0, abs=0.01)
    assert z.std() == pytest.approx(1.0, abs=0.01)
    # first splitmix64 output of seed 0 (the published test value of the generator)
    assert int(synth.splitmix64(0, 1)[0]) == 0xE220A8397B1DCDAF


def test_grf_sigma_and_correlation_length():
    NC, ell = 64, 1.0 / 16
    lags = {2: [], 4: [], 8: []}
    for seed in range(4):
        g = synth.gaussian_random_field(NC, seed, ell, 1.0)
        assert g.shape == (2 * NC,) * 3
        assert g.std() == pytest.approx(1.0, rel=1e-12)
        for q in lags:
            lags[q].append(np.mean(g * np.roll(g, -q, axis=0)) / np.mean(g * g))
    for q, v in lags.items():
        # q grid steps of spacing 1 / NC in the generator's units
        r = q / NC
        assert np.mean(v) == pytest.approx(np.exp(-r * r / (2 * ell * ell)), abs=0.03)


def test_face_field_correlation_on_the_unit_cube_is_half_ell():
    N, ell = 63, 1.0 / 16
    NC = N + 1
    vals = {1: [], 2: [], 4: []}
    for seed in range(3):
        ax, _, _ = synth.face_coefficients_grf(N, seed, ell, 1.0)
        g = np.log(ax)
        for q in vals:  # q nodes apart = q / NC of the unit cube
            vals[q].append(np.mean(g * np.roll(g, -q, axis=0)) / np.mean(g * g))
    for q, v in vals.items():
        d = q / NC
        assert np.mean(v) == pytest.approx(np.exp(-d * d / (2 * (ell / 2) ** 2)), abs=0.04)


def test_high_contrast_blocks():
    N = 95
    ax, ay, az = synth.face_coefficients_blocks(N, 1)
    assert ax.shape == (N + 2,) * 3
    lo, hi = min(x.min() for x in (ax, ay, az)), max(x.max() for x in (ax, ay, az))
    assert 1e-3 <= lo and hi <= 1e3 and hi / lo > 1e4
