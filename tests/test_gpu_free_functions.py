"""The reference's free functions on the GPU: Schur, InterpDecomp, PivotedQR, TriangularSolve.

Checked against the CPU oracle (scipy / the reference's own OpenBLAS build) on
seeded matrices. Bars: relative 1e-10 for A22^{-1}, X, S; exact pivots and
skeleton sets (no ties in these matrices); 1e-8 for W.
"""
import numpy as np
import pytest
import scipy.linalg as sla

import hifde3d_b200 as hb
from hifde3d_b200 import synth
from oracle import hif_oracle as ho

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def dd_matrix(n, seed):
    """Diagonally dominant, non-symmetric test block."""
    A = synth.normal(seed, n * n).reshape(n, n)
    A += np.diag(np.abs(A).sum(axis=1) + 1.0)
    return A


@pytest.mark.parametrize("m,nr,ns", [(81, 27, 54), (300, 120, 150), (700, 300, 380), (40, 40, 0),
                                     (50, 0, 50)])
def test_schur_matches_oracle(m, nr, ns):
    A = dd_matrix(m, m + nr)
    perm = np.argsort(synth.uniform(7 + m, m))
    red, skel = np.sort(perm[:nr]), np.sort(perm[nr:nr + ns])
    A22, inv, X, S = hb.Schur(A, red, skel)
    blk = ho.Block(np.arange(m), red, skel)
    ho.schur(A, blk)
    if nr:
        np.testing.assert_array_equal(A22, blk.A22)
        assert rel(inv, blk.A22inv) < 1e-10
    if nr and ns:
        assert rel(X, blk.X) < 1e-10
    if ns:
        assert rel(S, blk.S) < 1e-10 or (nr == 0 and np.abs(S).max() == 0)


def lowrank(m, n, seed, decay=0.5):
    U = synth.normal(seed, m * n).reshape(m, n)
    V = synth.normal(seed + 1, n * n).reshape(n, n)
    s = decay ** np.arange(n)
    return (U * s) @ V


@pytest.mark.parametrize("m,n,eps", [(100, 9, 1e-6), (500, 49, 1e-6), (2000, 200, 1e-6),
                                     (600, 60, 1e-3)])
def test_interp_decomp_matches_oracle(m, n, eps):
    M = lowrank(m, n, m + n)
    W, sk, rd = hb.InterpDecomp(M, eps)
    Wo, sko, rdo, _, _ = ho.interp_decomp(M.copy(), eps)
    # skeleton columns: same set in the same pivot order; redundant columns: same set
    # (past the numerical rank the pivots are chosen among noise-level columns)
    np.testing.assert_array_equal(sk, sko)
    assert set(rd.tolist()) == set(rdo.tolist())
    if W.size:
        pos = {c: i for i, c in enumerate(rd.tolist())}
        assert rel(W[:, [pos[c] for c in rdo.tolist()]], Wo) < 1e-8
        # the ID reproduces the redundant columns: M[:, rd] ~= M[:, sk] W
        err = np.linalg.norm(M[:, rd] - M[:, sk] @ W) / np.linalg.norm(M)
        assert err < 10 * eps


def test_pivoted_qr_pivots():
    A = synth.normal(3, 300 * 40).reshape(300, 40)
    R, jp = hb.PivotedQR(A)
    _, jpo = ho.geqp3(A.copy())
    np.testing.assert_array_equal(jp, jpo)
    Rq = np.triu(R[:40, :])
    Ro = sla.qr(A[:, jp], mode="r")[0][:40]
    assert rel(np.abs(np.diag(Rq)), np.abs(np.diag(Ro))) < 1e-12


def test_triangular_solve():
    k, nb = 120, 37
    R = np.triu(synth.normal(5, k * k).reshape(k, k)) + 5 * np.eye(k)
    B = synth.normal(6, k * nb).reshape(k, nb)
    X = hb.TriangularSolve(R, B)
    assert rel(X, sla.solve_triangular(R, B, lower=False)) < 1e-12
