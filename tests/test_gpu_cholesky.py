"""Cholesky elimination of symmetric interiors (HIF_OPT_ELIMINATION), through the C ABI.

For the symmetric face-coefficient operator every eliminated block is
A22 = L L^T; the factor keeps L, L^{-1} and Y = L^{-1} A21, and the apply splits
A22^{-1} = L^{-T} L^{-1} around the sweeps. The reference forms the explicit
inverse instead (getrf + getri, include/Schur.hpp:72-100); in exact arithmetic
the two factorizations are the same operator, so the bars are the parity bars
of test_gpu_parity.py against the oracle on the same inputs:
* index data and skeleton sets exact;
* A22, A22^{-1}, X formed from the stored factors: relative 1e-10 (Schur
  blocks) / 1e-8 (skeletonization blocks);
* F u and F^{-1} u: relative 1e-9;
and, at n = 64, the inverse apply against the reference's own (fixture
n64_faces) at 1e-9.
"""
import os
import tempfile

import numpy as np
import pytest

import goldens
import hifde3d_b200 as hb
from hifde3d_b200 import synth
from oracle import hif_oracle as ho

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def face_inputs(N, seed=2):
    ax, ay, az = synth.face_coefficients_grf(N, seed, ell=1.0 / 8, sigma=1.0)
    return ax, ay, az, np.zeros((N + 2,) * 3)


def factor(N, elim, precision=hb.PRECISION_FP64, eps=1e-6, partition=hb.PARTITION_REFERENCE,
           seed=2):
    ax, ay, az, V = face_inputs(N, seed)
    f = hb.HIFFactor(N, 4, eps, partition)
    f.set_option(hb.OPT_PRECISION, precision)
    f.set_option(hb.OPT_ELIMINATION, elim)
    hb.SetupStencilFaces(f, N, 1.0 / (N + 1), ax, ay, az, V)
    f.Factor()
    return f


@pytest.fixture(scope="module")
def oracle31():
    N = 31
    ax, ay, az, V = face_inputs(N)
    op = ho.setup_stencil_faces(N, 1.0 / (N + 1), ax, ay, az, V)
    fo = ho.HIFOracle(N, 4, 1e-6)
    fo.set_matrix(op)
    fo.initialize()
    fo.factor()
    return fo, op


def test_cholesky_fp64_matches_oracle_blocks_and_applies(oracle31):
    fo, op = oracle31
    N = 31
    f = factor(N, hb.ELIM_CHOLESKY)
    assert f.num_levels() == fo.L
    worst = 0.0
    for lev in range(fo.L):
        for kind, blocks in ((0, fo.schur_levels[lev]), (1, fo.skel_levels[lev])):
            assert f.num_blocks(lev, kind) == len(blocks)
            tol = 1e-8 if kind else 1e-10
            for b, ob in enumerate(blocks):
                ours = f.block(lev, kind, b, matrices=True)
                np.testing.assert_array_equal(ours["global"], ob.global_inds)
                np.testing.assert_array_equal(ours["skel"], ob.skel)
                if ob.red.size == 0:
                    continue
                for name, ref in (("A22", ob.A22), ("A22inv", ob.A22inv), ("X", ob.X)):
                    if ref.size == 0:
                        continue
                    e = rel(ours[name], ref)
                    worst = max(worst, e)
                    assert e < tol, (lev, kind, b, name, e)
    u = synth.dof_vector(N, 4)
    for inv in (False, True):
        y = u.copy()
        f.Apply(y, inv)
        assert rel(y, fo.apply(u, inv)) < 1e-9, inv
    x, it, rr = f.solve_pcg(u, tol=1e-10, maxit=50)
    assert rr <= 1e-10 and it <= 5
    assert np.linalg.norm(op @ x - u) / np.linalg.norm(u) < 1e-9
    f.close()


def test_stored_factors_are_triangular_and_consistent():
    """Raw L, L^{-1}, Y (which 5-7): L lower with positive diagonal, L L^{-1} = I,
    and L^{-T} Y equal to the X formed for the readback."""
    N = 31
    f = factor(N, hb.ELIM_CHOLESKY)
    L_ = hb.lib()
    checked = 0
    for lev in range(f.num_levels()):
        for kind in (0, 1):
            for b in range(f.num_blocks(lev, kind)):
                info = f.block(lev, kind, b)
                r, s = info["red"].size, info["skel"].size
                if r < 2 or (lev < 2 and b % 37):
                    continue
                raw = {}
                for which, (h, w) in ((5, (r, r)), (6, (r, r)), (7, (r, s))):
                    if h * w == 0:
                        continue
                    buf = np.zeros(h * w)
                    assert L_.hif_block_matrix(f._h, lev, kind, b, which,
                                               hb._dptr(buf)) == hb.HIF_OK
                    raw[which] = buf.reshape(w, h).T
                L, Li = raw[5], raw[6]
                assert np.all(np.triu(L, 1) == 0) and np.all(np.triu(Li, 1) == 0)
                assert np.all(np.diag(L) > 0)
                assert np.abs(L @ Li - np.eye(r)).max() < 1e-10
                if 7 in raw:
                    X = f.block(lev, kind, b, matrices=True)["X"]
                    assert rel(Li.T @ raw[7], X) < 1e-12
                checked += 1
    assert checked > 10
    f.close()


def test_cholesky_at_n64_against_the_reference():
    """FP64 Cholesky factor of the bench operator at n = 64 against the reference's
    own factor-apply (fixture n64_faces): same skeleton sets, applies at 1e-9."""
    g = goldens.load("n64_faces")
    N = int(g["N"])
    f = factor(N, hb.ELIM_CHOLESKY)
    for lev in range(int(g["L"])):
        for b, (_, gg, rr, ss) in enumerate(goldens.blocks(g, lev, "skel")):
            ours = f.block(lev, 1, b)
            np.testing.assert_array_equal(ours["skel"], ss)
    u = synth.dof_vector(N, int(g["u_seed"]))
    for inv, key in ((False, "Fu"), (True, "Finv_u")):
        y = u.copy()
        f.Apply(y, inv)
        assert rel(y, g[key]) < 1e-9, key
    f.close()


@pytest.mark.parametrize("N,partition", [(31, hb.PARTITION_REFERENCE),
                                         (47, hb.PARTITION_CLIPPED)])
def test_mixed_cholesky_close_to_fp64(N, partition):
    """Mixed precision (the default for symmetric operators: Cholesky, int8-slice
    products for Y and S) against the FP64 Gauss-Jordan factor; PCG converges."""
    fm = factor(N, hb.ELIM_AUTO, hb.PRECISION_MIXED, partition=partition)
    fd = factor(N, hb.ELIM_GAUSS_JORDAN, hb.PRECISION_FP64, partition=partition)
    u = synth.dof_vector(N, 5)
    ym, yd = u.copy(), u.copy()
    fm.Apply(ym, True)
    fd.Apply(yd, True)
    assert rel(ym, yd) < 1e-5
    _, itm, rrm = fm.solve_pcg(u, tol=1e-10, maxit=50)
    _, itd, rrd = fd.solve_pcg(u, tol=1e-10, maxit=50)
    assert rrm <= 1e-10 and itm <= itd + 1
    fm.close()
    fd.close()


def test_mixed_cholesky_int8_factor_products():
    """HIF_OPT_CHOL_SLICES: the products forming L^{-1} from 7 int8 slices (the
    default) against FP64 products (0), at n = 64 where the top blocks span many
    128-pivot blocks: the
    stored factors stay consistent (L lower, L L^{-1} = I to 1e-10), the inverse
    applies agree to the mixed arithmetic's own level and PCG needs no more
    iterations."""
    N = 63
    ax, ay, az, V = face_inputs(N)
    fs = {}
    for slices in (0, 7):
        f = hb.HIFFactor(N, 4, 1e-6)
        f.set_option(hb.OPT_PRECISION, hb.PRECISION_MIXED)
        f.set_option(hb.OPT_ELIMINATION, hb.ELIM_CHOLESKY)
        f.set_option(hb.OPT_CHOL_SLICES, slices)
        hb.SetupStencilFaces(f, N, 1.0 / (N + 1), ax, ay, az, V)
        f.Factor()
        fs[slices] = f
    f = fs[7]
    top = f.num_levels() - 1
    info = f.block(top, 0, 0)
    r = info["red"].size
    assert r > 4 * 128
    raw = {}
    for which in (5, 6):
        buf = np.zeros(r * r)
        assert hb.lib().hif_block_matrix(f._h, top, 0, 0, which, hb._dptr(buf)) == hb.HIF_OK
        raw[which] = buf.reshape(r, r).T
    L, Li = raw[5], raw[6]
    assert np.all(np.triu(L, 1) == 0) and np.all(np.triu(Li, 1) == 0)
    assert np.abs(L @ Li - np.eye(r)).max() < 1e-10
    u = synth.dof_vector(N, 5)
    y0, y7 = u.copy(), u.copy()
    fs[0].Apply(y0, True)
    fs[7].Apply(y7, True)
    assert rel(y7, y0) < 1e-5
    _, it0, _ = fs[0].solve_pcg(u, tol=1e-10, maxit=50)
    _, it7, rr7 = fs[7].solve_pcg(u, tol=1e-10, maxit=50)
    assert rr7 <= 1e-10 and it7 <= it0
    for g in fs.values():
        g.close()
    with pytest.raises(hb.HIFError):
        h = hb.HIFFactor(N, 4, 1e-6)
        try:
            h.set_option(hb.OPT_CHOL_SLICES, 9)
        finally:
            h.close()


def test_cholesky_multi_rhs_and_save_load():
    """16+ right-hand sides (gather / GEMM / emit apply) equal the single-RHS apply;
    a saved Cholesky factor reloads bit-identically."""
    N = 31
    f = factor(N, hb.ELIM_CHOLESKY)
    U = np.asfortranarray(np.stack([synth.dof_vector(N, s) for s in range(20)], axis=1))
    for inv in (False, True):
        Y = U.copy(order="F")
        f.Apply(Y, inv)
        for c in (0, 7, 19):
            y = np.ascontiguousarray(U[:, c])
            f.Apply(y, inv)
            assert rel(Y[:, c], y) < 1e-13
    u = U[:, 3].copy()
    y0 = u.copy()
    f.Apply(y0, True)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "chol.hif")
        f.save(path)
        g = hb.HIFFactor(N, 4, 1e-6)
        g.load(path)
        y1 = u.copy()
        g.Apply(y1, True)
        assert np.array_equal(y0, y1)
        g.close()
    f.close()


def test_cholesky_refused_for_the_node_operator():
    N = 15
    A, V = synth.node_lognormal(N, 3, sigma=0.3)
    f = hb.HIFFactor(N, 4, 1e-6)
    hb.SetupStencil(f, N, 1.0 / (N + 1), A, V)
    f.set_option(hb.OPT_ELIMINATION, hb.ELIM_CHOLESKY)
    with pytest.raises(hb.HIFError) as ei:
        f.Factor()
    assert ei.value.code == hb.HIF_ERR_ARG
    f.close()
