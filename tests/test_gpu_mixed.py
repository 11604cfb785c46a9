"""Mixed-precision factorization (split-TF32 Schur-complement updates).

The Schur complements S = A11 - A12 X are formed with FP32-level products, an
error of about 1e-6 |A11| per entry, which the small eigenvalues of the later
Schur complements amplify: measured on this operator, the mixed inverse apply
differs from the FP64 factor's by 1.1e-5 (n = 32) and 2.0e-4 (n = 64) relative,
and its operator error |F^{-1} A u - u| / |u| is 7.8e-6 / 3.8e-5 against the
FP64 factor's 5.0e-6 / 5.3e-6. The test bounds the difference by 1e-3 and
requires the mixed factor, as the preconditioner of the FP64-residual PCG, to
reach 1e-10 in at most two iterations more than the FP64 factor.
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
def test_mixed_matches_fp64_and_converges(n):
    N = n - 1
    ax, ay, az = synth.face_coefficients_grf(N, 2, ell=1.0 / 16, sigma=1.0)
    V = np.zeros((n + 1,) * 3)
    fs = {}
    for prec in (hb.PRECISION_FP64, hb.PRECISION_MIXED):
        f = hb.HIFFactor(N, 4, 1e-6)
        f.set_option(hb.OPT_PRECISION, prec)
        hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, V)
        f.Factor()
        fs[prec] = f
    u = synth.dof_vector(N, 3)
    y64 = u.copy()
    fs[hb.PRECISION_FP64].Apply(y64, True)
    ymx = u.copy()
    fs[hb.PRECISION_MIXED].Apply(ymx, True)
    assert rel(ymx, y64) < 1e-3
    x64, it64, r64 = fs[hb.PRECISION_FP64].solve_pcg(u, 1e-10, 50)
    xmx, itmx, rmx = fs[hb.PRECISION_MIXED].solve_pcg(u, 1e-10, 50)
    assert r64 <= 1e-10 and rmx <= 1e-10
    assert itmx <= it64 + 2
    op = ho.setup_stencil_faces(N, 1.0 / n, ax, ay, az, V)
    assert np.linalg.norm(op @ xmx - u) / np.linalg.norm(u) < 1e-9
    for f in fs.values():
        f.close()
