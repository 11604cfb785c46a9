"""Factor save / load (hif_save_factor, hif_load_factor).

A factorization written to a file and read into a new handle of the same N, P,
epsilon and partition must give the saved factorization's results bit for bit:
forward and inverse applies (one and several right-hand sides), PCG solves
(iterates, iteration counts, residuals) and the per-block index data and
matrices read back through the introspection calls. Cases: the face operator in
FP64 (reference partition), in mixed precision with the clipped partition
(n = 48), and the node operator. A load replaces whatever the handle held, and
the operator saved with the factor lets the loaded handle refactor.

Bad input never reaches the device: a handle of another N / epsilon / partition
is refused with HIF_ERR_ARG; a missing, foreign, truncated or corrupted file
(any single byte changed past the header) with HIF_ERR_IO, after which the handle
holds no factorization (Apply reports HIF_ERR_STATE) and a good file still loads.
"""
import os

import numpy as np
import pytest

import hifde3d_b200 as hb
from hifde3d_b200 import synth

pytestmark = pytest.mark.gpu

HEADER_BYTES = 64  # magic, version, byte-order marker, 8 ints, eps, NC^3


def make_face(N, eps=1e-6, partition=hb.PARTITION_REFERENCE, precision=hb.PRECISION_FP64,
              seed=2, factor=True):
    n = N + 1
    ax, ay, az = synth.face_coefficients_grf(N, seed, ell=1.0 / 8, sigma=1.0)
    V = np.zeros((n + 1,) * 3)
    f = hb.HIFFactor(N, 4, eps, partition)
    f.set_option(hb.OPT_PRECISION, precision)
    hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, V)
    if factor:
        f.Factor()
    return f


def make_node(N, eps=1e-6):
    A, V = synth.node_lognormal(N, 1, sigma=0.5, vscale=0.1)
    f = hb.HIFFactor(N, 4, eps)
    hb.SetupStencil(f, N, 1.0 / (N + 1), A, V)
    f.Factor()
    return f


def assert_same_results(f, g, N, pcg=True):
    u = synth.dof_vector(N, 5)
    for inverse in (True, False):
        y1, y2 = u.copy(), u.copy()
        f.Apply(y1, inverse)
        g.Apply(y2, inverse)
        assert np.array_equal(y1, y2), inverse
    U = np.asfortranarray(synth.dof_vector(N, 9, nrhs=3))
    Y1, Y2 = U.copy(order="F"), U.copy(order="F")
    f.Apply(Y1, True)
    g.Apply(Y2, True)
    assert np.array_equal(Y1, Y2)
    if pcg:
        x1, it1, r1 = f.solve_pcg(u, 1e-10, 40)
        x2, it2, r2 = g.solve_pcg(u, 1e-10, 40)
        assert np.array_equal(x1, x2) and it1 == it2 and r1 == r2


def assert_same_blocks(f, g):
    assert f.num_levels() == g.num_levels()
    for level in range(f.num_levels()):
        for kind in (0, 1):
            nb = f.num_blocks(level, kind)  # 0: no such phase (the top level has no skeletonization)
            assert g.num_blocks(level, kind) == nb
            if nb == 0:
                continue
            for b in sorted({0, nb // 2, nb - 1}):
                x, y = f.block(level, kind, b, matrices=True), g.block(level, kind, b, matrices=True)
                assert x.keys() == y.keys()
                for key in x:
                    assert np.array_equal(x[key], y[key]), (level, kind, b, key)


CASES = {
    "face_fp64": lambda: (make_face(31), 31, dict(eps=1e-6), True),
    "face_mixed_clipped": lambda: (make_face(47, partition=hb.PARTITION_CLIPPED,
                                             precision=hb.PRECISION_MIXED), 47,
                                   dict(eps=1e-6, partition=hb.PARTITION_CLIPPED), True),
    "node": lambda: (make_node(15), 15, dict(eps=1e-6), False),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_round_trip_is_bit_identical(case, tmp_path):
    f, N, kw, pcg = CASES[case]()
    path = str(tmp_path / "factor.hif")
    try:
        f.save(path)
        assert os.path.getsize(path) > 0 and not os.path.exists(path + ".tmp")
        g = hb.HIFFactor(N, 4, kw["eps"], kw.get("partition", hb.PARTITION_REFERENCE))
        try:
            g.load(path)
            assert_same_results(f, g, N, pcg)
            assert_same_blocks(f, g)
            # a second save of the loaded factor writes the same bytes
            path2 = str(tmp_path / "again.hif")
            g.save(path2)
            with open(path, "rb") as a, open(path2, "rb") as b:
                assert a.read() == b.read()
        finally:
            g.close()
    finally:
        f.close()


def test_load_replaces_the_factor_and_refactors(tmp_path):
    N = 31
    f = make_face(N, seed=2)
    g = make_face(N, seed=3)  # another operator, already factored
    path = str(tmp_path / "f.hif")
    try:
        f.save(path)
        g.load(path)
        assert_same_results(f, g, N)
        # the operator came with the factor: refactoring reproduces the factor
        g.Factor()
        u = synth.dof_vector(N, 6)
        y1, y2 = u.copy(), u.copy()
        f.Apply(y1, True)
        g.Apply(y2, True)
        assert np.linalg.norm(y1 - y2) <= 1e-12 * np.linalg.norm(y1)
    finally:
        f.close()
        g.close()


def expect(code, fn, *args):
    with pytest.raises(hb.HIFError) as e:
        fn(*args)
    assert e.value.code == code, str(e.value)


def test_bad_files_and_handles_are_refused(tmp_path):
    N = 15
    f = make_face(N)
    path = str(tmp_path / "f.hif")
    f.save(path)
    data = open(path, "rb").read()
    u = synth.dof_vector(N, 1)
    y_ref = u.copy()
    f.Apply(y_ref, True)

    unfactored = make_face(N, factor=False)
    expect(hb.HIF_ERR_STATE, unfactored.save, str(tmp_path / "none.hif"))
    assert not os.path.exists(str(tmp_path / "none.hif"))
    unfactored.close()

    # handles of another size, epsilon or partition
    for args in ((23, 4, 1e-6, hb.PARTITION_REFERENCE), (N, 4, 1e-3, hb.PARTITION_REFERENCE),
                 (N, 4, 1e-6, hb.PARTITION_CLIPPED)):
        h = hb.HIFFactor(*args)
        expect(hb.HIF_ERR_ARG, h.load, path)
        h.close()

    g = hb.HIFFactor(N, 4, 1e-6)
    try:
        def bad(name, content):
            p = str(tmp_path / name)
            with open(p, "wb") as fh:
                fh.write(content)
            expect(hb.HIF_ERR_IO, g.load, p)
            y = u.copy()
            expect(hb.HIF_ERR_STATE, g.Apply, y, True)

        expect(hb.HIF_ERR_IO, g.load, str(tmp_path / "missing.hif"))
        bad("foreign.hif", b"not a factor file" * 8)
        bad("empty.hif", b"")
        for frac in (0.1, 0.5, 0.999):
            bad(f"trunc{frac}.hif", data[:int(len(data) * frac)])
        bad("trailing.hif", data + b"\0")
        rng = np.random.default_rng(0)
        positions = sorted(set(rng.integers(HEADER_BYTES, len(data), 24).tolist())
                           | {HEADER_BYTES, len(data) - 1})
        for pos in positions:
            c = bytearray(data)
            c[pos] ^= 0x5A
            bad(f"flip{pos}.hif", bytes(c))
        # the good file still loads after all of that
        g.load(path)
        y = u.copy()
        g.Apply(y, True)
        assert np.array_equal(y, y_ref)
    finally:
        g.close()
        f.close()


def test_save_into_a_missing_directory_fails_cleanly(tmp_path):
    f = make_face(15)
    try:
        target = str(tmp_path / "no" / "such" / "dir" / "f.hif")
        expect(hb.HIF_ERR_IO, f.save, target)
        assert not os.path.exists(target)
        # overwriting an existing file replaces it
        path = str(tmp_path / "f.hif")
        with open(path, "wb") as fh:
            fh.write(b"old")
        f.save(path)
        assert os.path.getsize(path) > 3
    finally:
        f.close()
