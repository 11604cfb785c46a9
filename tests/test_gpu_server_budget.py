"""Serving loop: the device-memory budget decides when factorizations run.

* A factorization whose expected footprint does not fit beside the resident
  factors waits until an operator is released, then runs; its wait is reported
  as queue time (submit to admission), separate from its service time.
* A factorization whose expected footprint exceeds the whole budget can never
  fit and is refused with HIF_ERR_BUDGET (so are the solves submitted for it),
  whatever is resident.
The footprint of a size not factored before is estimated per DOF (12 KiB per
DOF plus 256 MiB); after a factorization the measured peak is used.
"""
import threading
import time

import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth

pytestmark = pytest.mark.gpu

GIB = 1 << 30


def coeffs(n, seed):
    N = n - 1
    ax, ay, az = synth.face_coefficients_grf(N, seed, ell=1.0 / 8, sigma=1.0)
    return N, ax, ay, az, np.zeros((n + 1,) * 3)


def test_budget_defers_a_factorization_until_a_release():
    # n = 32 fits (estimate 0.62 GiB); afterwards it holds its factor arena
    # (at least one 256 MiB chunk), and n = 64 (estimate 3.25 GiB) fits in 3.4 GiB
    # alone but not beside it
    srv = hb.Server(budget_bytes=int(3.4 * GIB), max_active_solves=8, factor_workers=2)
    N, ax, ay, az, V = coeffs(32, 3)
    r1 = srv.wait(srv.submit_factor(1, N, ax, ay, az, V, eps=1e-6))
    assert r1["status"] == hb.HIF_OK
    N2, bx, by, bz, V2 = coeffs(64, 4)
    rid = srv.submit_factor(2, N2, bx, by, bz, V2, eps=1e-6)
    res = {}
    t = threading.Thread(target=lambda: res.update(srv.wait(rid)))
    t.start()
    time.sleep(1.5)
    assert t.is_alive(), "the second factorization ran although it does not fit"
    # a solve on the resident operator still runs meanwhile
    b = synth.dof_vector(N, 7)
    sr = srv.wait(srv.submit_solve(1, b, tol=1e-10, maxit=50))
    assert sr["status"] == hb.HIF_OK and sr["relres"] <= 1e-10
    srv.release(1)
    t.join(timeout=120)
    assert not t.is_alive()
    assert res["status"] == hb.HIF_OK
    assert res["queue_ms"] >= 1000.0
    assert res["service_ms"] > 0 and res["latency_ms"] >= res["queue_ms"]
    b2 = synth.dof_vector(N2, 8)
    sr2 = srv.wait(srv.submit_solve(2, b2, tol=1e-10, maxit=50))
    assert sr2["status"] == hb.HIF_OK and sr2["relres"] <= 1e-10
    srv.release(2)
    srv.close()


def test_factorization_larger_than_the_budget_is_refused():
    srv = hb.Server(budget_bytes=1 * GIB, max_active_solves=8, factor_workers=1)
    N, ax, ay, az, V = coeffs(64, 5)  # estimate ~3.4 GiB > 1 GiB, nothing resident
    fid = srv.submit_factor(1, N, ax, ay, az, V, eps=1e-6)
    sid = srv.submit_solve(1, synth.dof_vector(N, 1), tol=1e-10, maxit=50)
    r = srv.wait(fid)
    assert r["status"] == hb.HIF_ERR_BUDGET
    assert "budget" in r["error"]
    s = srv.wait(sid)
    assert s["status"] != hb.HIF_OK
    # the server stays usable: a size that fits is factored and solved
    N2, bx, by, bz, V2 = coeffs(24, 6)
    assert srv.wait(srv.submit_factor(2, N2, bx, by, bz, V2, eps=1e-6))["status"] == hb.HIF_OK
    s2 = srv.wait(srv.submit_solve(2, synth.dof_vector(N2, 2), tol=1e-10, maxit=50))
    assert s2["status"] == hb.HIF_OK
    srv.release(2)
    srv.close()
