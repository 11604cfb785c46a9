"""Refactorization on one handle gives a fresh handle's factorization.

A handle keeps the parts of a factorization that depend on the grid alone
(level 0's cell blocks, offsets and index lists, level 0's face partition) from
its first factorization and reuses them in later ones. This checks that reuse:
a handle factors operator A, then operator B, then A again; its index data at
every level equals a fresh handle's factorization of A exactly, its inverse apply
agrees to rounding, and its factorization of B equals a fresh handle's of B.
Cases: the reference partition in FP64 (N = 31) and the clipped partition in
mixed precision (N = 47).
"""
import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth

pytestmark = pytest.mark.gpu


def setup(f, N, seed):
    n = N + 1
    ax, ay, az = synth.face_coefficients_grf(N, seed, ell=1.0 / 8, sigma=1.0)
    hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, np.zeros((n + 1,) * 3))


def handle(N, partition, precision):
    f = hb.HIFFactor(N, 4, 1e-6, partition)
    f.set_option(hb.OPT_PRECISION, precision)
    return f


def assert_same_factor(f, g, N):
    assert f.num_levels() == g.num_levels()
    for level in range(f.num_levels()):
        for kind in (0, 1):
            if level == f.num_levels() - 1 and kind == 1:
                continue
            nb = f.num_blocks(level, kind)
            assert nb == g.num_blocks(level, kind)
            for b in range(nb):
                x, y = f.block(level, kind, b), g.block(level, kind, b)
                for key in ("global", "red", "skel"):
                    np.testing.assert_array_equal(x[key], y[key], err_msg=f"{level} {kind} {b} {key}")
    u = synth.dof_vector(N, 4)
    y1, y2 = u.copy(), u.copy()
    f.Apply(y1, True)
    g.Apply(y2, True)
    assert np.linalg.norm(y1 - y2) <= 1e-12 * np.linalg.norm(y1)


@pytest.mark.parametrize("N,partition,precision", [
    (31, hb.PARTITION_REFERENCE, hb.PRECISION_FP64),
    (47, hb.PARTITION_CLIPPED, hb.PRECISION_MIXED),
])
def test_refactor_matches_fresh_handles(N, partition, precision):
    f = handle(N, partition, precision)
    ga = handle(N, partition, precision)
    gb = handle(N, partition, precision)
    try:
        setup(ga, N, 2)
        ga.Factor()
        setup(gb, N, 3)
        gb.Factor()
        setup(f, N, 2)
        f.Factor()
        setup(f, N, 3)
        f.Factor()
        assert_same_factor(f, gb, N)
        setup(f, N, 2)
        f.Factor()
        assert_same_factor(f, ga, N)
    finally:
        f.close()
        ga.close()
        gb.close()
