"""Regenerate the golden fixtures from the reference itself.

Runs the reference's factor/apply (built from its own sources by
``make -C oracle``; driver oracle/ref_probe.cpp) on seeded inputs and writes
one ``<case>.npz`` per case next to this script.

Each fixture holds, for every level and phase (Schur, skeletonization) and
every block, the exact index data (global / redundant / skeleton lists, face)
and, for the matrices A_22, A_22^{-1}, X, S and W, either the full matrices
(small cases) or sketches: M @ zc, M.T @ zr and ||M||_F with the fixed probe
vectors of ``probe_vector``. It also holds Apply(u, false), Apply(u, true),
Apply(A u, true) for a seeded u, and the driver's e_a / e_s
(tests/HIFDE3D/main.cpp:121-134).

Cases at the bench's sizes are packed compactly ("compact"): the index data in
full, per block and matrix only ||M||_F and one bilinear sketch zr^T M zc, and
the apply outputs Apply(u, false) and Apply(u, true) in full. The face-operator
cases run the reference's own factor on the symmetric face-coefficient operator
(ref_probe dumpf). The clipped-partition case, which the reference cannot
partition (NC / P not a power of two), is produced by the CPU restatement
(oracle/hif_oracle.py) instead and says so in its "source" entry.

Usage: python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import mmap
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hifde3d_b200 import synth  # noqa: E402

PROBE = os.path.join(ROOT, "oracle", "_ref", "hif_ref_probe")

# name: (N, P, eps, operator, packing: True = full matrices, False = sketches,
#        "compact" = per-block norms and bilinear sketches)
CASES = {
    "n8_unit": (7, 4, 1e-6, "unit", True),
    "n16_unit": (15, 4, 1e-6, "unit", False),
    "n16_unit_e3": (15, 4, 1e-3, "unit", False),
    "n16_rand": (15, 4, 1e-6, "rand", False),
    "n32_unit": (31, 4, 1e-6, "unit", False),
    "n32_rand": (31, 4, 1e-6, "rand", False),
    # the bench's face operator a = exp(GRF) (correlation length 1/16 of the
    # unit cube, sigma 1, seed 2) at n = 64, factored by the reference itself
    "n64_faces": (63, 4, 1e-6, "faces", "compact"),
    # the same field family at n = 48 on the clipped partition: the restatement
    "n48_faces_clipped": (47, 4, 1e-6, "faces_clipped", "compact"),
}
RAND_SEED = 11
U_SEED = 3
FACE_SEED = 2
FACE_ELL_PARAM = 1.0 / 8  # the generator's length: correlation length 1/16 on the unit cube


def operator_inputs(N: int, kind: str):
    if kind == "unit":
        NC = N + 1
        return np.ones((NC + 1,) * 3), np.zeros((NC + 1,) * 3)
    return synth.node_lognormal(N, RAND_SEED, sigma=0.5, vscale=1.0)


def face_inputs(N: int):
    """(ax, ay, az, V) of the face-operator cases."""
    ax, ay, az = synth.face_coefficients_grf(N, FACE_SEED, FACE_ELL_PARAM, 1.0)
    return ax, ay, az, np.zeros((N + 2,) * 3)


def probe_vector(n: int, salt: float) -> np.ndarray:
    """Fixed, machine-independent sketch vector."""
    j = np.arange(n, dtype=np.float64)
    return np.cos(0.7 * j + salt) + 0.25 * np.sin(1.3 * j * j % 17.0 + salt)


def sketch(M: np.ndarray):
    r, c = M.shape
    return M @ probe_vector(c, 0.3), M.T @ probe_vector(r, 1.1), np.linalg.norm(M)


def bilinear(M: np.ndarray) -> float:
    """zr^T M zc with the fixed probe vectors (0 for an empty matrix)."""
    r, c = M.shape
    if M.size == 0:
        return 0.0
    return float(probe_vector(r, 1.1) @ (M @ probe_vector(c, 0.3)))


class Reader:
    def __init__(self, path):
        # mapped, not read: the dumps of the bench-size cases run to gigabytes
        self._f = open(path, "rb")
        self.b = mmap.mmap(self._f.fileno(), 0, access=mmap.ACCESS_READ)
        self.o = 0

    def i32(self):
        v = struct.unpack_from("<i", self.b, self.o)[0]
        self.o += 4
        return v

    def f64(self):
        v = struct.unpack_from("<d", self.b, self.o)[0]
        self.o += 8
        return v

    def ivec(self):
        n = self.i32()
        v = np.frombuffer(self.b, "<i4", n, self.o).astype(np.int64)
        self.o += 4 * n
        return v

    def dense(self):
        h, w = self.i32(), self.i32()
        v = np.frombuffer(self.b, "<f8", h * w, self.o).reshape(w, h).T.copy()
        self.o += 8 * h * w
        return v

    def vec(self):
        n = self.i32()
        v = np.frombuffer(self.b, "<f8", n, self.o).copy()
        self.o += 8 * n
        return v


def compact_mats(mats):
    """Per matrix: (shape, ||M||_F, zr^T M zc) instead of the entries."""
    return {k: (m.shape, float(np.linalg.norm(m)), bilinear(m)) for k, m in mats.items()}


def parse_dump(path, compact: bool = False):
    rd = Reader(path)
    assert rd.b[:4] == b"HIFG"
    rd.o = 4
    assert rd.i32() == 1
    N, P, L = rd.i32(), rd.i32(), rd.i32()
    eps = rd.f64()
    levels = []
    for _ in range(L):
        phases = []
        for _kind in range(2):
            nb = rd.i32()
            blocks = []
            for _ in range(nb):
                face = rd.i32()
                g, red, skl = rd.ivec(), rd.ivec(), rd.ivec()
                mats = {k: rd.dense() for k in ("A22", "A22inv", "X", "S", "W")}
                blocks.append((face, g, red, skl, compact_mats(mats) if compact else mats))
            phases.append(blocks)
        levels.append(phases)
    out = {"N": N, "P": P, "L": L, "eps": eps, "levels": levels}
    out["Au"], out["Fu"], out["Finv_u"], out["Finv_Au"] = rd.vec(), rd.vec(), rd.vec(), rd.vec()
    out["e_a"], out["e_s"] = rd.f64(), rd.f64()
    return out


def pack(d, full: bool):
    arrs = {"N": d["N"], "P": d["P"], "L": d["L"], "eps": d["eps"],
            "Au": d["Au"], "Fu": d["Fu"], "Finv_u": d["Finv_u"], "Finv_Au": d["Finv_Au"],
            "e_a": d["e_a"], "e_s": d["e_s"]}
    for lev, phases in enumerate(d["levels"]):
        for kind, blocks in zip(("schur", "skel"), phases):
            pre = f"L{lev}_{kind}_"
            arrs[pre + "nblk"] = len(blocks)
            arrs[pre + "face"] = np.array([b[0] for b in blocks], np.int32)
            for key, idx in (("g", 1), ("r", 2), ("s", 3)):
                lens = np.array([b[idx].size for b in blocks], np.int64)
                arrs[pre + key + "_off"] = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
                arrs[pre + key] = (np.concatenate([b[idx] for b in blocks]).astype(np.int32)
                                   if blocks else np.zeros(0, np.int32))
            for m in ("A22", "A22inv", "X", "S", "W"):
                mats = [b[4][m] for b in blocks]
                if full == "compact":
                    arrs[pre + m + "_shape"] = np.array([x[0] for x in mats],
                                                        np.int32).reshape(-1, 2)
                    arrs[pre + m + "_fro"] = np.array([x[1] for x in mats])
                    arrs[pre + m + "_bil"] = np.array([x[2] for x in mats])
                    continue
                arrs[pre + m + "_shape"] = np.array([x.shape for x in mats], np.int32).reshape(-1, 2)
                if full:
                    arrs[pre + m] = (np.concatenate([x.T.ravel() for x in mats])
                                     if mats else np.zeros(0))
                else:
                    sk = [sketch(x) if x.size else (np.zeros(x.shape[0]), np.zeros(x.shape[1]), 0.0)
                          for x in mats]
                    arrs[pre + m + "_sr"] = (np.concatenate([s[0] for s in sk]) if sk else np.zeros(0))
                    arrs[pre + m + "_sc"] = (np.concatenate([s[1] for s in sk]) if sk else np.zeros(0))
                    arrs[pre + m + "_fro"] = np.array([s[2] for s in sk])
    arrs["full"] = full
    return arrs


def oracle_dump(N: int, P: int, eps: float, u: np.ndarray):
    """The restatement's factor on the face operator with the clipped partition,
    in parse_dump's compact layout (no driver check: e_a / e_s are NaN)."""
    from oracle import hif_oracle as ho

    ax, ay, az, V = face_inputs(N)
    NC = N + 1
    op = ho.setup_stencil_faces(N, 1.0 / NC, ax, ay, az, V)
    fo = ho.HIFOracle(N, P, eps, partition="clipped")
    fo.set_matrix(op)
    fo.initialize()
    fo.factor()
    levels = []
    for lev in range(fo.L):
        phases = []
        for blocks, skel in ((fo.schur_levels[lev], False), (fo.skel_levels[lev], True)):
            out = []
            for b in blocks:
                mats = {"A22": b.A22, "A22inv": b.A22inv, "X": b.X, "S": b.S,
                        "W": b.W if b.W is not None else np.zeros((0, 0))}
                mats = {k: (np.zeros((0, 0)) if m is None else np.atleast_2d(m))
                        for k, m in mats.items()}
                out.append((b.face if skel else -1, b.global_inds, b.red, b.skel,
                            compact_mats(mats)))
            phases.append(out)
        levels.append(phases)
    Au = op @ u
    return {"N": N, "P": P, "L": fo.L, "eps": eps, "levels": levels, "Au": Au,
            "Fu": fo.apply(u, False), "Finv_u": fo.apply(u, True),
            "Finv_Au": fo.apply(Au, True), "e_a": float("nan"), "e_s": float("nan")}


def make_case(name):
    N, P, eps, kind, full = CASES[name]
    NC = N + 1
    u = synth.dof_vector(N, U_SEED)
    compact = full == "compact"
    if kind == "faces_clipped":
        d = oracle_dump(N, P, eps, u)
        source = "restatement (oracle/hif_oracle.py), clipped partition"
    else:
        with tempfile.TemporaryDirectory() as td:
            fu, fo = os.path.join(td, "u.bin"), os.path.join(td, "out.bin")
            u.astype("<f8").tofile(fu)
            if kind == "faces":
                names = [os.path.join(td, x + ".bin") for x in ("ax", "ay", "az", "V")]
                for path, a in zip(names, face_inputs(N)):
                    a.ravel(order="F").astype("<f8").tofile(path)
                cmd = [PROBE, "dumpf", str(N), str(P), repr(eps), *names, fu, fo]
            else:
                A, V = operator_inputs(N, kind)
                fa, fv = os.path.join(td, "A.bin"), os.path.join(td, "V.bin")
                # NumTns order is i fastest: A[i, j, k] -> i + m j + m n k (Fortran order)
                A.ravel(order="F").astype("<f8").tofile(fa)
                V.ravel(order="F").astype("<f8").tofile(fv)
                cmd = [PROBE, "dump", str(N), str(P), repr(eps), fa, fv, fu, fo]
            subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            d = parse_dump(fo, compact)
        source = "reference (oracle/_ref/hif_ref_probe)"
    assert d["Au"].size == NC ** 3
    arrs = pack(d, full)
    if compact:  # the apply outputs the tests read, not the driver's extra vectors
        del arrs["Au"], arrs["Finv_Au"]
    arrs["operator"] = kind
    arrs["source"] = source
    arrs["rand_seed"] = RAND_SEED
    arrs["face_seed"] = FACE_SEED
    arrs["u_seed"] = U_SEED
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    print(f"{name}: L={d['L']} e_a={d['e_a']:.3e} e_s={d['e_s']:.3e}")


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for n in names:
        make_case(n)
