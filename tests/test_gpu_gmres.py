"""Restarted GMRES with the factor's inverse apply as right preconditioner
(hif_solve_gmres).

The reference's own operator, SetupStencil's node-coefficient 7-point stencil
(include/setup_stencil.hpp:6-76), is not symmetric for variable coefficients, so
CG does not apply to it. GMRES must reach the requested relative residual
1e-10 on it, and the residual checked independently with the CPU oracle's sparse
operator must agree (1e-9). On the symmetric face operator GMRES must reach the
same residual in about as many iterations as PCG, with the same solution. Several
right-hand sides in one call must each match their single solves; a small
restart length must still converge; repeated calls are bit-identical; bad
arguments and calls out of order are refused.
"""
import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth
from oracle import hif_oracle as ho

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# Two solutions whose residuals are both below 1e-10 |b| differ by at most
# cond(A) * 2e-10 relative; cond(A) is about 4 / (pi h)^2 ~ 400 at N = 31 (with the
# coefficient contrast, a few thousand), so 2e-6 is a safe bound.
SAME_SOLUTION = 2e-6


@pytest.fixture(scope="module")
def node31():
    N = 31
    A, V = synth.node_lognormal(N, 1, sigma=0.5, vscale=0.1)
    f = hb.HIFFactor(N, 4, 1e-6)
    hb.SetupStencil(f, N, 1.0 / (N + 1), A, V)
    f.Factor()
    op = ho.setup_stencil(N, 1.0 / (N + 1), A, V)
    yield f, op, N
    f.close()


def test_node_operator_converges_to_true_residual(node31):
    f, op, N = node31
    b = synth.dof_vector(N, 0)
    asym = abs(op - op.T).max() / abs(op).max()
    assert asym > 1e-3  # the operator is far from symmetric
    x, it, rr = f.solve_gmres(b, tol=1e-10, maxit=100)
    assert rr <= 1e-10 and 1 <= it <= 30, (it, rr)  # 10 with the CPU oracle's factor
    assert np.linalg.norm(op @ x - b) / np.linalg.norm(b) < 1e-9
    # the reported residual is the true one
    assert abs(np.linalg.norm(op @ x - b) / np.linalg.norm(b) - rr) <= 1e-12


def test_small_restart_still_converges(node31):
    f, op, N = node31
    b = synth.dof_vector(N, 2)
    x30, it30, _ = f.solve_gmres(b, tol=1e-10, maxit=200, restart=30)
    x2, it2, rr2 = f.solve_gmres(b, tol=1e-10, maxit=200, restart=2)
    assert rr2 <= 1e-10 and it2 >= it30
    assert np.linalg.norm(op @ x2 - b) / np.linalg.norm(b) < 1e-9


def test_several_rhs_match_single_solves(node31):
    f, op, N = node31
    B = np.asfortranarray(synth.dof_vector(N, 11, nrhs=3))
    X, its, rrs = f.solve_gmres(B, tol=1e-10, maxit=100)
    for c in range(3):
        assert rrs[c] <= 1e-10
        assert np.linalg.norm(op @ X[:, c] - B[:, c]) / np.linalg.norm(B[:, c]) < 1e-9
        x1, it1, _ = f.solve_gmres(np.ascontiguousarray(B[:, c]), tol=1e-10, maxit=100)
        assert abs(int(its[c]) - it1) <= 1
        assert rel(X[:, c], x1) < SAME_SOLUTION


def test_bit_reproducible_and_limits(node31):
    f, op, N = node31
    b = synth.dof_vector(N, 3)
    x1, it1, r1 = f.solve_gmres(b, tol=1e-10, maxit=100)
    x2, it2, r2 = f.solve_gmres(b, tol=1e-10, maxit=100)
    assert np.array_equal(x1, x2) and it1 == it2 and r1 == r2
    # maxit reached: no error, the residual says how far it got
    x, it, rr = f.solve_gmres(b, tol=1e-14, maxit=1)
    assert it == 1 and 1e-14 < rr < 1.0
    # a zero right-hand side
    x, it, rr = f.solve_gmres(np.zeros_like(b), tol=1e-10, maxit=10)
    assert it == 0 and rr == 0.0 and not x.any()
    for bad in (0, 65):
        with pytest.raises(hb.HIFError) as e:
            f.solve_gmres(b, restart=bad)
        assert e.value.code == hb.HIF_ERR_ARG


def test_symmetric_operator_matches_pcg():
    N = 31
    n = N + 1
    ax, ay, az = synth.face_coefficients_grf(N, 2, ell=1.0 / 8, sigma=1.0)
    V = np.zeros((n + 1,) * 3)
    f = hb.HIFFactor(N, 4, 1e-6)
    try:
        hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, V)
        b = synth.dof_vector(N, 4)
        with pytest.raises(hb.HIFError) as e:
            f.solve_gmres(b)
        assert e.value.code == hb.HIF_ERR_STATE  # before Factor
        f.Factor()
        xc, itc, rc = f.solve_pcg(b, tol=1e-10, maxit=50)
        xg, itg, rg = f.solve_gmres(b, tol=1e-10, maxit=50)
        assert rg <= 1e-10 and rc <= 1e-10
        assert abs(itg - itc) <= 2
        assert rel(xg, xc) < SAME_SOLUTION
        op = ho.setup_stencil_faces(N, 1.0 / n, ax, ay, az, V)
        assert np.linalg.norm(op @ xg - b) / np.linalg.norm(b) < 1e-9
    finally:
        f.close()
