"""Many right-hand sides at once (one batched apply for all of them).

From 16 right-hand sides on, the apply runs every sweep stage as gather / GEMM /
emit instead of GEMVs over groups of 4 right-hand sides. Each column must match the
single-RHS apply of the same factor to rounding (the products sum in another order):
relative difference below 1e-12 per column, for the inverse and the forward apply,
and the batched PCG must reach 1e-10 on every column in the iterations the
single-column solves take.
"""
import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def factor():
    n = 32
    N = n - 1
    ax, ay, az = synth.face_coefficients_grf(N, 4, ell=1.0 / 8, sigma=1.0)
    V = np.zeros((n + 1,) * 3)
    f = hb.HIFFactor(N, 4, 1e-6)
    hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, V)
    f.Factor()
    yield f, N
    f.close()


@pytest.mark.parametrize("nrhs", [16, 64])
@pytest.mark.parametrize("inverse", [True, False])
def test_batched_apply_matches_single(factor, nrhs, inverse):
    f, N = factor
    U = np.asfortranarray(np.stack([synth.dof_vector(N, 300 + c) for c in range(nrhs)], axis=1))
    Y = U.copy(order="F")
    f.Apply(Y, inverse)
    for c in range(nrhs):
        y = U[:, c].copy()
        f.Apply(y, inverse)
        assert np.linalg.norm(Y[:, c] - y) <= 1e-12 * np.linalg.norm(y), c


def test_batched_pcg(factor):
    f, N = factor
    nrhs = 24
    B = np.asfortranarray(np.stack([synth.dof_vector(N, 500 + c) for c in range(nrhs)], axis=1))
    X, it, rr = f.solve_pcg(B, tol=1e-10, maxit=50)
    assert np.all(rr <= 1e-10)
    for c in (0, 7, 23):
        x, it1, rr1 = f.solve_pcg(B[:, c].copy(), tol=1e-10, maxit=50)
        assert abs(int(it[c]) - it1) <= 1
        assert np.linalg.norm(X[:, c] - x) <= 1e-8 * np.linalg.norm(x)
