"""Mixed-precision factorization (tensor-core Schur complements and X).

Default MIXED arithmetic: S = A11 - A12 X from 5 int8 slices per operand value
(error of order k 2^-35 max|row of A12| max|column of X|) and X = A22^{-1} A21 from
7 slices; A22^{-1}, the interpolative decompositions' pivots and rank, the factor
storage, the apply and the PCG residual stay FP64. Measured on this operator, the
mixed inverse apply differs from the FP64 factor's by 5e-8 (n = 32) and 5e-7 (n = 64)
relative, and its operator error |F^{-1} A u - u| / |u| equals the FP64 factor's
(5.0e-6 / 5.3e-6). The test bounds the difference by 1e-5 and requires PCG with the
mixed factor as preconditioner to take at most one iteration more than with the FP64
factor.

The split-TF32 Schur products (HIF_OPT_SCHUR_SLICES = 0, FP32-level products) with
FP64 X (HIF_OPT_X_SLICES = 0) remain selectable: their difference is 1.2e-5 / 1.8e-4,
bounded by 1e-3, within two PCG iterations of FP64.
"""
import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth
from oracle import hif_oracle as ho

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("n", [32, 64])
@pytest.mark.parametrize("slices,bound,extra_it", [(None, 1e-5, 1), ((0, 0), 1e-3, 2)])
def test_mixed_matches_fp64_and_converges(n, slices, bound, extra_it):
    N = n - 1
    ax, ay, az = synth.face_coefficients_grf(N, 2, ell=1.0 / 16, sigma=1.0)
    V = np.zeros((n + 1,) * 3)
    fs = {}
    for prec in (hb.PRECISION_FP64, hb.PRECISION_MIXED):
        f = hb.HIFFactor(N, 4, 1e-6)
        f.set_option(hb.OPT_PRECISION, prec)
        if slices is not None and prec == hb.PRECISION_MIXED:
            f.set_option(hb.OPT_SCHUR_SLICES, slices[0])
            f.set_option(hb.OPT_X_SLICES, slices[1])
        hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, V)
        f.Factor()
        fs[prec] = f
    u = synth.dof_vector(N, 3)
    y64 = u.copy()
    fs[hb.PRECISION_FP64].Apply(y64, True)
    ymx = u.copy()
    fs[hb.PRECISION_MIXED].Apply(ymx, True)
    assert rel(ymx, y64) < bound
    x64, it64, r64 = fs[hb.PRECISION_FP64].solve_pcg(u, 1e-10, 50)
    xmx, itmx, rmx = fs[hb.PRECISION_MIXED].solve_pcg(u, 1e-10, 50)
    assert r64 <= 1e-10 and rmx <= 1e-10
    assert itmx <= it64 + extra_it
    op = ho.setup_stencil_faces(N, 1.0 / n, ax, ay, az, V)
    assert np.linalg.norm(op @ xmx - u) / np.linalg.norm(u) < 1e-9
    for f in fs.values():
        f.close()


def test_slice_options_are_checked():
    f = hb.HIFFactor(15, 4, 1e-6)
    try:
        for opt in (hb.OPT_SCHUR_SLICES, hb.OPT_X_SLICES):
            for bad in (1, 9, -1):
                with pytest.raises(hb.HIFError):
                    f.set_option(opt, bad)
            f.set_option(opt, 0)
            f.set_option(opt, 8)
    finally:
        f.close()
