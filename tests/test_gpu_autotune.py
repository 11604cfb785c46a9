"""Online tile tuner of the batched FP64 products (OPT_AUTOTUNE).

The tuner only changes which of two tiles (64 x 64 FFMA, 128 x 128 DMMA) computes a
batch of products, so every factorization it makes is the same factorization up to
rounding: the apply of each must agree with the untuned factor's to 1e-10 relative,
and PCG must converge in the same iterations (within one). After two factorizations
every batch signature has tried both tiles and has a decision.
"""
import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth

pytestmark = pytest.mark.gpu


def make(n, seed, autotune):
    N = n - 1
    ax, ay, az = synth.face_coefficients_grf(N, seed, ell=1.0 / 8, sigma=1.0)
    V = np.zeros((n + 1,) * 3)
    f = hb.HIFFactor(N, 4, 1e-6)
    if autotune:
        f.set_option(hb.OPT_AUTOTUNE, 1)
    hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, V)
    return f, N


def test_autotune_decides_and_keeps_the_factor():
    ref, N = make(32, 21, False)
    tuned, _ = make(32, 21, True)
    try:
        ref.Factor()
        b = synth.dof_vector(N, 4)
        y_ref = b.copy()
        ref.Apply(y_ref, True)
        _, it_ref, _ = ref.solve_pcg(b, tol=1e-10, maxit=60)
        for rep in range(3):
            tuned.Factor()
            st = tuned.autotune_stats()
            assert st["signatures"] > 0
            if rep >= 1:
                assert st["decided"] == st["signatures"], st
            y = b.copy()
            tuned.Apply(y, True)
            assert np.linalg.norm(y - y_ref) <= 1e-10 * np.linalg.norm(y_ref), rep
            _, it, rr = tuned.solve_pcg(b, tol=1e-10, maxit=60)
            assert rr <= 1e-10 and abs(it - it_ref) <= 1
    finally:
        ref.close()
        tuned.close()


def test_autotune_off_by_default():
    f, _ = make(16, 3, False)
    try:
        f.Factor()
        st = f.autotune_stats()
        assert (st["signatures"], st["decided"], st["chose_128"]) == (0, 0, 0)
        assert st["elimination_phases"] == 0
    finally:
        f.close()


def test_autotune_picks_the_elimination_per_phase_in_mixed_precision():
    """Mixed precision on the symmetric operator: each phase signature runs once
    with Gauss-Jordan and once with Cholesky, then keeps the faster. Both are
    the same factorization up to the mixed-precision error, so every tuned
    factor's inverse apply stays within 1e-5 of the FP64 one and PCG converges
    as with the untuned mixed factor."""
    ref, N = make(32, 22, False)
    tuned, _ = make(32, 22, True)
    mixed, _ = make(32, 22, False)
    try:
        ref.Factor()
        mixed.set_option(hb.OPT_PRECISION, hb.PRECISION_MIXED)
        mixed.Factor()
        tuned.set_option(hb.OPT_PRECISION, hb.PRECISION_MIXED)
        b = synth.dof_vector(N, 6)
        y_ref = b.copy()
        ref.Apply(y_ref, True)
        _, it_mixed, _ = mixed.solve_pcg(b, tol=1e-10, maxit=60)
        for rep in range(3):
            tuned.Factor()
            st = tuned.autotune_stats()
            assert st["elimination_phases"] > 0
            if rep >= 1:
                assert st["elimination_decided"] == st["elimination_phases"], st
            y = b.copy()
            tuned.Apply(y, True)
            assert np.linalg.norm(y - y_ref) <= 1e-5 * np.linalg.norm(y_ref), rep
            _, it, rr = tuned.solve_pcg(b, tol=1e-10, maxit=60)
            assert rr <= 1e-10 and abs(it - it_mixed) <= 1
    finally:
        ref.close()
        tuned.close()
        mixed.close()
