"""The oracle's iterative solvers with the oracle's factor as preconditioner (CPU).

The reference's node operator (SetupStencil, include/setup_stencil.hpp:6-76) with a
lognormal node coefficient is about 50% asymmetric, and the reference's factor
applies X^T on the left (src/Factor.cpp:992-1081), so F^-1 A is far from the
identity. Right-preconditioned GMRES still converges in a few iterations; these
counts are what the GPU solver's tests (test_gpu_gmres.py) bound. On the
symmetric face operator GMRES and PCG agree.
"""
import numpy as np
import pytest

from hifde3d_b200 import synth
from oracle import hif_oracle as ho


@pytest.fixture(scope="module")
def node15():
    N = 15
    A, V = synth.node_lognormal(N, 1, sigma=0.5, vscale=0.1)
    fo, op = ho.factor_node(N, 4, 1e-6, A, V)
    return fo, op, N


def test_node_operator_is_nonsymmetric_and_poorly_fit_by_the_factor(node15):
    fo, op, N = node15
    assert abs(op - op.T).max() / abs(op).max() > 0.3
    u = synth.dof_vector(N, 3)
    e = np.linalg.norm(op @ fo.apply(u, True) - u) / np.linalg.norm(u)
    assert e > 1e-2  # the X^T left factor does not invert a non-symmetric operator


def test_gmres_converges_on_node_operator(node15):
    fo, op, N = node15
    b = synth.dof_vector(N, 0)
    M = lambda v: fo.apply(v, True)  # noqa: E731
    x, it, rel = ho.gmres(op, b, M, tol=1e-10)
    assert rel <= 1e-10 and it <= 15
    assert np.linalg.norm(op @ x - b) / np.linalg.norm(b) == pytest.approx(rel, abs=1e-14)
    x2, it2, rel2 = ho.gmres(op, b, M, tol=1e-10, restart=2)
    assert rel2 <= 1e-10 and it2 >= it
    # maxit reached: the residual says how far it got
    _, it1, rel1 = ho.gmres(op, b, M, tol=1e-14, maxit=1)
    assert it1 == 1 and 1e-14 < rel1 < 1.0
    assert ho.gmres(op, np.zeros_like(b), M)[1:] == (0, 0.0)


def test_gmres_and_pcg_agree_on_face_operator():
    N = 15
    n = N + 1
    ax, ay, az = synth.face_coefficients_grf(N, 2, ell=1.0 / 8, sigma=1.0)
    V = np.zeros((n + 1,) * 3)
    op = ho.setup_stencil_faces(N, 1.0 / n, ax, ay, az, V)
    fo = ho.HIFOracle(N, 4, 1e-6, "reference")
    fo.set_matrix(op)
    fo.initialize()
    fo.factor()
    b = synth.dof_vector(N, 4)
    M = lambda v: fo.apply(v, True)  # noqa: E731
    xg, itg, rg = ho.gmres(op, b, M, tol=1e-10)
    xc, itc, hist = ho.pcg(op, b, M, tol=1e-10)
    assert rg <= 1e-10 and hist[-1] <= 1e-10
    assert abs(itg - itc) <= 2
    assert np.linalg.norm(xg - xc) / np.linalg.norm(xc) < 2e-6
