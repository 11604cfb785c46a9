"""The tcgen05 split-TF32 GEMM (kernel of the mixed-precision Schur updates)
against an FP64 product of the same operands.

Each FP64 operand is split into a TF32 pair and hi*hi + hi*lo + lo*hi is
accumulated in FP32, so every entry of C must lie within
(2e-6 + 1.2e-7 k) (|op(A)| |op(B)|)_ij of the FP64 product (TF32 pair
representation error ~2^-21 per operand, FP32 accumulation ~2^-24 per term),
for ragged shapes, both operand orientations, alpha / beta, leading dimensions
larger than the rows, and k = 0.
"""
import numpy as np
import pytest

import hifde3d_b200 as hb

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SHAPES = [(128, 128, 32), (1, 1, 1), (200, 130, 77), (128, 256, 512), (300, 5, 1000),
          (37, 300, 129), (64, 64, 0), (513, 257, 40)]


def op_mat(rng, rows, cols, trans, pad):
    """Column-major operand of op() shape rows x cols stored with ld = stored rows + pad."""
    sr, sc = (cols, rows) if trans else (rows, cols)
    ld = sr + pad
    buf = rng.standard_normal((sc, ld)) * np.exp(rng.uniform(-2, 2, (sc, 1)))
    stored = buf[:, :sr].T  # sr x sc view, column-major in buf
    opm = stored.T if trans else stored
    return buf, ld, opm


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_tc_gemm_against_fp64(shape, ta, tb):
    m, n, k = shape
    rng = np.random.default_rng(m * 7919 + n * 31 + k + 2 * ta + tb)
    bufA, lda, A = op_mat(rng, m, k, ta, 3)
    bufB, ldb, B = op_mat(rng, k, n, tb, 5)
    ldc = m + 2
    bufC = rng.standard_normal((n, ldc))
    C0 = bufC[:, :m].T.copy()
    alpha, beta = -1.0, 1.0 if (m + n) % 2 else 0.5
    dev = torch.device("cuda", 0)
    dA = torch.from_numpy(np.ascontiguousarray(bufA)).to(dev)
    dB = torch.from_numpy(np.ascontiguousarray(bufB)).to(dev)
    dC = torch.from_numpy(np.ascontiguousarray(bufC)).to(dev)
    torch.cuda.synchronize()
    hb.GemmMixedDevice(ta, tb, m, n, k, alpha, dA.data_ptr(), lda, dB.data_ptr(), ldb, beta,
                       dC.data_ptr(), ldc)
    C = dC.cpu().numpy()[:, :m].T
    ref = alpha * (A @ B) + beta * C0
    bound = (2e-6 + 1.2e-7 * k) * (np.abs(A) @ np.abs(B)) + 1e-300
    err = np.abs(C - ref)
    assert np.all(err <= bound + 1e-15 * np.abs(beta * C0)), float(np.max(err / bound))
    # the padding rows of C are untouched
    assert np.array_equal(dC.cpu().numpy()[:, m:], bufC[:, m:])


def test_tc_gemm_is_deterministic():
    m, n, k = 256, 384, 700
    rng = np.random.default_rng(5)
    dev = torch.device("cuda", 0)
    A = torch.from_numpy(rng.standard_normal((k, m))).to(dev)  # m x k, ld m
    B = torch.from_numpy(rng.standard_normal((n, k))).to(dev)  # k x n, ld k
    outs = []
    for _ in range(2):
        C = torch.zeros((n, m), dtype=torch.float64, device=dev)
        hb.GemmMixedDevice(0, 0, m, n, k, 1.0, A.data_ptr(), m, B.data_ptr(), k, 0.0,
                           C.data_ptr(), m)
        outs.append(C.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
