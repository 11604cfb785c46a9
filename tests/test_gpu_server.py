"""Serving loop: several factored operators resident on one GPU, solves batched
across operators at every PCG iteration.

The reference runs one operator per process (tests/HIFDE3D/main.cpp: Factor, then
PCG-free Apply checks); the server must give every request exactly what
hif_solve_pcg gives for the same operator and right-hand sides when run alone:
same x bit for bit, same iteration count, same residual, whatever requests of
other operators and sizes share its iterations.
"""
import threading

import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth

pytestmark = pytest.mark.gpu

# (op id, n, seed, precision)
OPS = [(1, 16, 11, hb.PRECISION_FP64), (2, 24, 12, hb.PRECISION_FP64),
       (3, 32, 13, hb.PRECISION_FP64), (4, 32, 14, hb.PRECISION_MIXED)]


def coeffs(n, seed):
    N = n - 1
    ax, ay, az = synth.face_coefficients_grf(N, seed, ell=1.0 / 8, sigma=1.0)
    V = np.zeros((n + 1,) * 3)
    return N, ax, ay, az, V


def rhs(n, seed, nrhs):
    N = n - 1
    cols = [synth.dof_vector(N, seed * 100 + c) for c in range(nrhs)]
    return np.asfortranarray(np.stack(cols, axis=1))


@pytest.fixture(scope="module")
def alone():
    """Factors built one at a time through HIFFactor, and their solves."""
    out = {}
    for op, n, seed, prec in OPS:
        N, ax, ay, az, V = coeffs(n, seed)
        f = hb.HIFFactor(N, 4, 1e-6)
        f.set_option(hb.OPT_PRECISION, prec)
        hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, V)
        f.Factor()
        out[op] = f
    yield out
    for f in out.values():
        f.close()


def requests():
    # (op, seed, nrhs, tol, maxit): several per operator, mixed sizes
    reqs = []
    for k in range(12):
        op, n, _, _ = OPS[k % len(OPS)]
        reqs.append((op, 500 + k, 1 + (k * 5) % 7, 1e-10 if k % 3 else 1e-8, 60))
    reqs.append((1, 999, 3, 1e-10, 1))  # stops at maxit
    return reqs


def test_server_matches_alone_in_the_mix(alone):
    srv = hb.Server(budget_bytes=16 << 30, max_active_solves=64, factor_workers=2)
    try:
        fids = []
        for op, n, seed, prec in OPS:
            N, ax, ay, az, V = coeffs(n, seed)
            fids.append(srv.submit_factor(op, N, ax, ay, az, V, precision=prec))
        reqs = requests()
        ns = {op: n for op, n, _, _ in OPS}
        # submit every solve at once (before the factorizations finish), from
        # two threads, so that requests of all operators share iterations
        ids = [None] * len(reqs)

        def submit(idx):
            for i in idx:
                op, seed, nrhs, tol, maxit = reqs[i]
                ids[i] = srv.submit_solve(op, rhs(ns[op], seed, nrhs), tol=tol, maxit=maxit)

        ths = [threading.Thread(target=submit, args=(range(t, len(reqs), 2),)) for t in range(2)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        for fid in fids:
            r = srv.wait(fid)
            assert r["status"] == hb.HIF_OK, r
        results = [srv.wait(i) for i in ids]
        st = srv.stats()
        for (op, seed, nrhs, tol, maxit), r in zip(reqs, results):
            assert r["status"] == hb.HIF_OK, r
            b = rhs(ns[op], seed, nrhs)
            x, it, rr = alone[op].solve_pcg(b, tol=tol, maxit=maxit)
            assert np.array_equal(r["x"], x), (op, seed, nrhs)
            assert r["iters"] == int(np.max(it))
            assert r["relres"] == float(np.max(rr))
            assert r["latency_ms"] > 0
        # the batching happened: fewer iterations of the server loop than the
        # requests' own iteration counts added up, merged apply launches
        assert st["iterations"] < sum(r["iters"] + 1 for r in results)
        assert st["batched_launches"] > 0
        assert st["resident_ops"] == len(OPS)
    finally:
        srv.close()


def test_server_single_request_and_release(alone):
    srv = hb.Server(budget_bytes=4 << 30, max_active_solves=4, factor_workers=1)
    try:
        op, n, seed, prec = OPS[1]
        N, ax, ay, az, V = coeffs(n, seed)
        assert srv.wait(srv.submit_factor(op, N, ax, ay, az, V, precision=prec))["status"] == 0
        b = rhs(n, 77, 1)[:, 0].copy()
        r = srv.wait(srv.submit_solve(op, b, tol=1e-10, maxit=50))
        x, it, rr = alone[op].solve_pcg(b, tol=1e-10, maxit=50)
        assert np.array_equal(r["x"], x) and r["iters"] == it and r["relres"] == rr
        # zero right-hand side: done before the first iteration, x = 0
        r0 = srv.wait(srv.submit_solve(op, np.zeros_like(b)))
        assert r0["status"] == 0 and r0["iters"] == 0 and not r0["x"].any()
        srv.release(op)
        with pytest.raises(hb.HIFError):
            srv.submit_solve(op, b)
        with pytest.raises(hb.HIFError):
            srv.submit_solve(12345, b)
        assert srv.stats()["resident_ops"] == 0
    finally:
        srv.close()


def test_server_factor_failure_is_reported():
    srv = hb.Server(budget_bytes=2 << 30, max_active_solves=2, factor_workers=1)
    try:
        # clipped partition needs (N+1) divisible by P: the factorization fails on
        # the worker and the failure reaches both the factor and the solve request
        N = 16
        ax, ay, az = [np.ones((N + 2,) * 3)] * 3
        V = np.zeros((N + 2,) * 3)
        fid = srv.submit_factor(7, N, ax, ay, az, V, partition=hb.PARTITION_CLIPPED)
        sid = srv.submit_solve(7, np.ones((N + 1) ** 3))
        rf = srv.wait(fid)
        rs = srv.wait(sid)
        assert rf["status"] == hb.HIF_ERR_ARG and "clipped" in rf["error"]
        assert rs["status"] == hb.HIF_ERR_STATE
    finally:
        srv.close()
