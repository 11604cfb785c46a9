"""hif_schur_device_noalloc gives hif_schur_device's results without allocating.

The allocation-free entry point serves callers that cannot allocate device
memory (their framework's allocator already holds the GPU, or they must not call
the allocator inside their own loop); its scratch is a fixed array inside the
library. Two calls in a row must both match the allocating entry point within the
elimination tolerance of the other tests (relative 1e-10), which also shows the
shared scratch carries nothing over from one call to the next.
This file is collected last so a failure here does not hide the other tests.
"""
import ctypes

import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _block(n, r, seed):
    A = synth.normal(seed, n * n).reshape(n, n)
    A += np.diag(np.abs(A).sum(axis=1) + 1.0)
    return np.asfortranarray(A)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_noalloc_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    L = hb.lib()
    dev = torch.device("cuda", 0)
    for seed, (n, r) in enumerate([(300, 120), (512, 200), (97, 97)]):
        B = torch.from_numpy(_block(n, r, 11 + seed).ravel(order="F")).to(dev)
        s = n - r
        ref = [torch.zeros(max(r * r, 1), dtype=torch.float64, device=dev),
               torch.zeros(max(r * s, 1), dtype=torch.float64, device=dev),
               torch.zeros(max(s * s, 1), dtype=torch.float64, device=dev)]
        torch.cuda.synchronize()
        assert L.hif_schur_device(ctypes.c_void_p(B.data_ptr()), n, r,
                                  *[ctypes.c_void_p(t.data_ptr()) for t in ref]) == hb.HIF_OK
        for _call in range(2):
            out = [torch.full_like(t, float("nan")) for t in ref]
            torch.cuda.synchronize()
            rc = L.hif_schur_device_noalloc(ctypes.c_void_p(B.data_ptr()), n, r,
                                            *[ctypes.c_void_p(t.data_ptr()) for t in out],
                                            ctypes.c_void_p(0))
            assert rc == hb.HIF_OK, L.hif_last_error()
            torch.cuda.synchronize()
            for a, b, size in zip(out, ref, (r * r, r * s, s * s)):
                if size:
                    assert _rel(a[:size].cpu().numpy(), b[:size].cpu().numpy()) < TOL


def test_noalloc_on_a_side_stream_and_without_redundant_dofs():
    """A non-default stream (nothing else queued on it), and r = 0, where nothing
    is eliminated and S must come back all zeros as from hif_schur_device."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    L = hb.lib()
    dev = torch.device("cuda", 0)
    side = torch.cuda.Stream(device=dev)
    for seed, (n, r) in enumerate([(200, 80), (64, 0)]):
        B = torch.from_numpy(_block(n, r, 31 + seed).ravel(order="F")).to(dev)
        s = n - r
        ref = [torch.zeros(max(r * r, 1), dtype=torch.float64, device=dev),
               torch.zeros(max(r * s, 1), dtype=torch.float64, device=dev),
               torch.full((max(s * s, 1),), float("nan"), dtype=torch.float64, device=dev)]
        torch.cuda.synchronize()
        assert L.hif_schur_device(ctypes.c_void_p(B.data_ptr()), n, r,
                                  *[ctypes.c_void_p(t.data_ptr()) for t in ref]) == hb.HIF_OK
        for _call in range(2):
            out = [torch.full_like(t, float("nan")) for t in ref]
            torch.cuda.synchronize()
            rc = L.hif_schur_device_noalloc(ctypes.c_void_p(B.data_ptr()), n, r,
                                            *[ctypes.c_void_p(t.data_ptr()) for t in out],
                                            ctypes.c_void_p(side.cuda_stream))
            assert rc == hb.HIF_OK, L.hif_last_error()
            torch.cuda.synchronize()
            for a, b, size in zip(out, ref, (r * r, r * s, s * s)):
                if size:
                    assert _rel(a[:size].cpu().numpy(), b[:size].cpu().numpy()) < TOL
            if r == 0:
                assert bool((out[2][:s * s] == 0).all())


def test_noalloc_empty_block_is_a_no_op():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    L = hb.lib()
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    assert L.hif_schur_device_noalloc(p, 0, 0, p, p, p, ctypes.c_void_p(0)) == hb.HIF_OK
    assert L.hif_schur_device(p, 0, 0, p, p, p) == hb.HIF_OK


def test_noalloc_rejects_oversized_block():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    L = hb.lib()
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    assert L.hif_schur_device_noalloc(p, 513, 10, p, p, p, ctypes.c_void_p(0)) == hb.HIF_ERR_ARG
    assert b"512" in L.hif_last_error()
