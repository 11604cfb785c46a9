"""FP64 products from int8 slices on the tcgen05 tensor cores (Ozaki scheme)
against an FP64 product of the same operands.

Every row i of op(A) is scaled by 2^e_i (e_i the frexp exponent of its largest
magnitude) and cut into S truncated 7-bit slices, so its representation error is
below 2^(e_i - 7S); the same holds for the columns j of op(B) with exponents f_j.
The slice pairs with s + t >= S are dropped and the kept ones are summed exactly in
int32, so every entry of C must lie within
    k (S + 3) 2^(e_i + f_j - 7S) + 1e-15 (|op(A)| |op(B)| + |beta C|)_ij
of the FP64 product, for every S in 2..8, ragged shapes, both operand
orientations, alpha / beta, leading dimensions larger than the rows, k = 0, k above
the single-launch limit (16384), rows of zeros and rows spanning 30 binades. The
integer accumulation makes the result bit-identical from run to run.
"""
import numpy as np
import pytest

import hifde3d_b200 as hb

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SHAPES = [(128, 128, 64), (1, 1, 1), (200, 130, 77), (128, 256, 512), (300, 5, 1000),
          (37, 300, 129), (64, 64, 0), (513, 257, 40)]


def op_mat(rng, rows, cols, trans, pad, spread=2.0):
    """Column-major operand of op() shape rows x cols stored with ld = stored rows + pad."""
    sr, sc = (cols, rows) if trans else (rows, cols)
    ld = sr + pad
    buf = rng.standard_normal((sc, ld)) * np.exp(rng.uniform(-spread, spread, (sc, 1)))
    stored = buf[:, :sr].T  # sr x sc view, column-major in buf
    opm = stored.T if trans else stored
    return buf, ld, opm


def bound(A, B, S):
    k = A.shape[1]
    ea = np.frexp(np.max(np.abs(A), axis=1, initial=0.0))[1].astype(np.float64)
    eb = np.frexp(np.max(np.abs(B), axis=0, initial=0.0))[1].astype(np.float64)
    return k * (S + 3) * np.exp2(ea[:, None] + eb[None, :] - 7 * S)


def run(ta, tb, m, n, k, alpha, bufA, lda, bufB, ldb, beta, bufC, ldc, S):
    dev = torch.device("cuda", 0)
    dA = torch.from_numpy(np.ascontiguousarray(bufA)).to(dev)
    dB = torch.from_numpy(np.ascontiguousarray(bufB)).to(dev)
    dC = torch.from_numpy(np.ascontiguousarray(bufC)).to(dev)
    torch.cuda.synchronize()
    hb.GemmInt8Device(ta, tb, m, n, k, alpha, dA.data_ptr(), lda, dB.data_ptr(), ldb, beta,
                      dC.data_ptr(), ldc, S)
    return dC.cpu().numpy()


@pytest.mark.parametrize("S", [2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1)])
def test_int8_gemm_against_fp64(S, shape, ta, tb):
    m, n, k = shape
    rng = np.random.default_rng(m * 7919 + n * 31 + k + 2 * ta + tb + 1000 * S)
    bufA, lda, A = op_mat(rng, m, k, ta, 3)
    bufB, ldb, B = op_mat(rng, k, n, tb, 5)
    ldc = m + 2
    bufC = rng.standard_normal((n, ldc))
    C0 = bufC[:, :m].T.copy()
    alpha, beta = -1.0, (1.0 if (m + n) % 2 else 0.5)
    out = run(ta, tb, m, n, k, alpha, bufA, lda, bufB, ldb, beta, bufC, ldc, S)
    C = out[:, :m].T
    ref = alpha * (A @ B) + beta * C0
    err = np.abs(C - ref)
    bnd = bound(A, B, S) + 1e-15 * (np.abs(A) @ np.abs(B) + np.abs(beta * C0)) + 1e-300
    assert np.all(err <= bnd), float(np.max(err / bnd))
    assert np.array_equal(out[:, m:], bufC[:, m:])  # padding rows untouched


@pytest.mark.parametrize("ta,tb", [(1, 0), (0, 1)])
def test_int8_gemm_mixed_orientations(ta, tb):
    m, n, k, S = 190, 70, 300, 7
    rng = np.random.default_rng(11 + ta)
    bufA, lda, A = op_mat(rng, m, k, ta, 1)
    bufB, ldb, B = op_mat(rng, k, n, tb, 2)
    bufC = np.zeros((n, m))
    C = run(ta, tb, m, n, k, 1.0, bufA, lda, bufB, ldb, 0.0, bufC, m, S).T
    err = np.abs(C - A @ B)
    assert np.all(err <= bound(A, B, S) + 1e-15 * (np.abs(A) @ np.abs(B)))


def test_int8_gemm_long_k_zero_rows_and_wide_range():
    # k above the single-launch limit runs as consecutive k ranges; zero rows of
    # op(A) and columns of op(B) give exact zeros; rows spread over 30 binades
    m, n, k, S = 130, 66, 20000, 6
    rng = np.random.default_rng(3)
    A = rng.standard_normal((m, k)) * np.exp2(rng.integers(-15, 15, (m, 1)))
    B = rng.standard_normal((k, n)) * np.exp2(rng.integers(-15, 15, (1, n)))
    A[7, :] = 0.0
    B[:, 3] = 0.0
    C = run(0, 0, m, n, k, 1.0, np.asfortranarray(A).T.copy(), m,
            np.asfortranarray(B).T.copy(), k, 0.0, np.zeros((n, m)), m, S).T
    err = np.abs(C - A @ B)
    assert np.all(err <= bound(A, B, S) + 1e-15 * (np.abs(A) @ np.abs(B)))
    assert not C[7, :].any() and not C[:, 3].any()


def test_int8_gemm_near_fp64_at_eight_slices():
    m, n, k = 256, 256, 1024
    rng = np.random.default_rng(9)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    C = run(0, 0, m, n, k, 1.0, A.T.copy(), m, B.T.copy(), k, 0.0, np.zeros((n, m)), m, 8).T
    ref = A @ B
    assert np.linalg.norm(C - ref) <= 1e-14 * np.linalg.norm(ref)


def test_int8_gemm_is_deterministic():
    m, n, k = 256, 384, 700
    rng = np.random.default_rng(5)
    dev = torch.device("cuda", 0)
    A = torch.from_numpy(rng.standard_normal((k, m))).to(dev)  # m x k, ld m
    B = torch.from_numpy(rng.standard_normal((n, k))).to(dev)  # k x n, ld k
    for S in (4, 7):
        outs = []
        for _ in range(2):
            C = torch.zeros((n, m), dtype=torch.float64, device=dev)
            hb.GemmInt8Device(0, 0, m, n, k, 1.0, A.data_ptr(), m, B.data_ptr(), k, 0.0,
                              C.data_ptr(), m, S)
            outs.append(C.cpu().numpy())
        assert np.array_equal(outs[0], outs[1])


def test_int8_gemm_rejects_bad_slices():
    with pytest.raises(hb.HIFError):
        hb.GemmInt8Device(0, 0, 1, 1, 1, 1.0, 0, 1, 0, 1, 0.0, 0, 1, 9)
