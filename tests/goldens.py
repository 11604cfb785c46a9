"""Helpers for reading the golden fixtures written by tests/golden/make_golden.py."""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from hifde3d_b200 import synth  # noqa: E402

sys.path.insert(0, os.path.join(GOLDEN))
from make_golden import RAND_SEED, U_SEED, operator_inputs, probe_vector  # noqa: E402,F401


def load(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def blocks(g: dict, level: int, kind: str):
    """Yield (face, global, red, skel) per block of one level phase."""
    pre = f"L{level}_{kind}_"
    nb = int(g[pre + "nblk"])
    go, ro, so = g[pre + "g_off"], g[pre + "r_off"], g[pre + "s_off"]
    for b in range(nb):
        yield (int(g[pre + "face"][b]), g[pre + "g"][go[b]:go[b + 1]].astype(np.int64),
               g[pre + "r"][ro[b]:ro[b + 1]].astype(np.int64),
               g[pre + "s"][so[b]:so[b + 1]].astype(np.int64))


def is_compact(g: dict) -> bool:
    return str(g["full"]) == "compact"


def compact_matrices(g: dict, level: int, kind: str, name: str):
    """Per block of a compact fixture: (shape, ||M||_F, zr^T M zc)."""
    pre = f"L{level}_{kind}_"
    return [(tuple(int(x) for x in sh), float(fr), float(bl))
            for sh, fr, bl in zip(g[pre + name + "_shape"], g[pre + name + "_fro"],
                                  g[pre + name + "_bil"])]


def bilinear_error(M: np.ndarray, fro: float, bil: float) -> float:
    """Distance of M from a compact fixture's (||M||_F, zr^T M zc), relative to
    ||M||_F (the bilinear form scaled by the probe vectors' norms)."""
    r, c = M.shape
    zr, zc = probe_vector(r, 1.1), probe_vector(c, 0.3)
    scale = max(fro, 1e-300)
    e_fro = abs(float(np.linalg.norm(M)) - fro) / scale
    e_bil = abs(float(zr @ (M @ zc)) - bil) / (scale * np.linalg.norm(zr) * np.linalg.norm(zc))
    return max(e_fro, e_bil)


def matrices(g: dict, level: int, kind: str, name: str):
    """Per block: the full matrix (full fixtures) or (M@zc, M.T@zr, ||M||_F)."""
    pre = f"L{level}_{kind}_"
    shapes = g[pre + name + "_shape"]
    out = []
    if is_compact(g):
        raise ValueError("compact fixture: use compact_matrices")
    if bool(g["full"]):
        flat = g[pre + name]
        o = 0
        for h, w in shapes:
            out.append(flat[o:o + h * w].reshape(w, h).T)
            o += h * w
        return out
    sr, sc, fro = g[pre + name + "_sr"], g[pre + name + "_sc"], g[pre + name + "_fro"]
    orr = oc = 0
    for b, (h, w) in enumerate(shapes):
        out.append((sr[orr:orr + h], sc[oc:oc + w], float(fro[b])))
        orr += h
        oc += w
    return out


def sketch(M: np.ndarray):
    r, c = M.shape
    return M @ probe_vector(c, 0.3), M.T @ probe_vector(r, 1.1), float(np.linalg.norm(M))


def face_case_inputs(g: dict):
    """(ax, ay, az, V, u) of a face-operator fixture."""
    from make_golden import face_inputs
    N = int(g["N"])
    ax, ay, az, V = face_inputs(N)
    return ax, ay, az, V, synth.dof_vector(N, int(g["u_seed"]))


def case_inputs(g: dict):
    N = int(g["N"])
    A, V = operator_inputs(N, str(g["operator"]))
    u = synth.dof_vector(N, int(g["u_seed"]))
    return A, V, u


def pivot_orders(g: dict):
    """Per level, per skeletonized face: the reference's column order
    (skeleton columns then redundant columns, both in pivot order)."""
    out = []
    for lev in range(int(g["L"])):
        out.append([np.concatenate([s, r]) for _f, _g, r, s in blocks(g, lev, "skel")])
    return out


# Fixtures whose faces meet exact ties in the pivoted QR (a = 1 is symmetric
# under reflections of a face); their pivot choices are replayed.
TIED = {"n16_unit_e3", "n32_unit"}
