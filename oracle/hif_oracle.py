"""CPU restatement of the reference's HIF factor / apply path.

TEST INFRASTRUCTURE ONLY. This module is the checker that the CUDA path is
compared against; only tests, the smoke check and the bench's CPU-baseline leg
import it. The product (hifde3d_b200) never imports or calls it.

It restates, in numpy/scipy, what arbenson/HIFDE3D computes for
``HIFFactor<double>`` (all references are files of that project):

* operator:  ``SetupStencil``              include/setup_stencil.hpp:6-76
* partition: ``InteriorCellIndexData``     src/Factor.cpp:359-392
             ``InteriorFaceDOFs``          src/Factor.cpp:402-521
             ``InteriorEdgeDOFs``          src/Factor.cpp:523-643
             ``SkelInteractionIndexData``  src/Factor.cpp:645-755
             ``IsInterior`` & friends      src/Factor.cpp:313-357
* elimination: ``Schur``                   include/Schur.hpp:72-100
             (``hmat_tools::Invert`` = LAPACK getrf + getri,
             src/hmat_tools/Invert.cpp:37-41; scipy.linalg.inv calls the same
             two routines)
* ID:        ``InterpDecomp``              src/InterpDecomp.cpp:86-138
             (LAPACK geqp3 through scipy.linalg.qr(pivoting=True); the
             triangular solve is trsm through scipy.linalg.solve_triangular)
* ``SchurAfterID``                         src/Factor.cpp:113-153
* level loop / update: ``Factor``, ``UpdateMatrixAndDOFs``
                                           src/Factor.cpp:41-63, 262-311
* ``Apply``                                src/Factor.cpp:992-1081
* ``SpMV`` (y = A^T x: the reference walks columns), ``RelativeErrorNorm2``
                                           src/Factor.cpp:1083-1113

Beyond the reference (no reference result exists for these; the restatement
is the only oracle):

* ``partition="clipped"``: cells_per_dir = ceil(NC / width) with the last cell
  clipped at N, and L = ceil(log2(NC / P)) + 1 levels. For NC / P a power of two
  this is identical to the reference's partition; otherwise the reference's
  integer division leaves part of the domain uncovered (src/Factor.cpp:51-53).
* ``setup_stencil_faces``: the symmetric flux form -div(a grad u) + b u with a
  given at cell faces.
* ``pcg`` and ``gmres``: the iterative solves that use the factor as
  preconditioner (the reference has none; its driver only reports e_a / e_s).

Parity of this module with the reference itself is pinned by the golden files
under tests/golden (written by tests/golden/make_golden.py from the reference
built by oracle/Makefile).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

# Face enum of the reference (include/data.hpp:6).
TOP, BOTTOM, RIGHT, LEFT, FRONT, BACK = range(6)


def num_levels(N: int, P: int, partition: str = "reference") -> int:
    NC = N + 1
    if partition == "reference":
        return int(round(math.log2(NC // P))) + 1  # src/Factor.cpp:36
    return int(math.ceil(math.log2(NC / P) - 1e-12)) + 1


def cells_per_dir(N: int, P: int, level: int, partition: str = "reference") -> int:
    NC = N + 1
    width = (1 << level) * P
    if partition == "reference":
        return NC // width  # src/Factor.cpp:52-53
    return -(-NC // width)


# ----------------------------------------------------------------------------
# Operators
# ----------------------------------------------------------------------------

def setup_stencil(N: int, h: float, A: np.ndarray, V: np.ndarray) -> sp.csc_matrix:
    """Node-coefficient 7-point operator, include/setup_stencil.hpp:18-75.

    ``A`` and ``V`` are (NC+1)^3 tensors indexed [i, j, k]. Entry (row p, col q)
    for a neighbour q is -A(q)/h^2; the diagonal is the sum of the six
    neighbours' A over h^2 plus V(p). Rows and columns are DOF ids
    i + NC*j + NC^2*k.
    """
    NC = N + 1
    hh = h * h
    rng = np.arange(1, N + 1)
    I, J, K = np.meshgrid(rng, rng, rng, indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    row = I + NC * J + NC * NC * K
    diag = ((A[I - 1, J, K] + A[I + 1, J, K]) / hh + (A[I, J - 1, K] + A[I, J + 1, K]) / hh
            + (A[I, J, K - 1] + A[I, J, K + 1]) / hh + V[I, J, K])
    rows, cols, vals = [row], [row], [diag]
    for di, dj, dk in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
        ii, jj, kk = I + di, J + dj, K + dk
        ok = (ii >= 1) & (ii <= N) & (jj >= 1) & (jj <= N) & (kk >= 1) & (kk <= N)
        rows.append(row[ok])
        cols.append((ii + NC * jj + NC * NC * kk)[ok])
        vals.append(-A[ii[ok], jj[ok], kk[ok]] / hh)
    n = NC ** 3
    return sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, n))


def setup_stencil_faces(N: int, h: float, ax: np.ndarray, ay: np.ndarray, az: np.ndarray,
                        V: np.ndarray) -> sp.csc_matrix:
    """Symmetric flux form of -div(a grad u) + b u (no reference counterpart).

    ``ax[i, j, k]`` is the coefficient on the face between nodes (i, j, k) and
    (i+1, j, k) (shape (NC, NC+1, NC+1) at least covering 0..N), likewise ``ay``
    (j -> j+1) and ``az`` (k -> k+1). The diagonal is the sum of the six face
    coefficients over h^2 plus V; the off-diagonal for the face is -a/h^2.
    """
    NC = N + 1
    hh = h * h
    rng = np.arange(1, N + 1)
    I, J, K = np.meshgrid(rng, rng, rng, indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    row = I + NC * J + NC * NC * K
    faces = [(-1, 0, 0, ax[I - 1, J, K]), (1, 0, 0, ax[I, J, K]),
             (0, -1, 0, ay[I, J - 1, K]), (0, 1, 0, ay[I, J, K]),
             (0, 0, -1, az[I, J, K - 1]), (0, 0, 1, az[I, J, K])]
    diag = V[I, J, K].astype(np.float64).copy()
    for _, _, _, a in faces:
        diag = diag + a / hh
    rows, cols, vals = [row], [row], [diag]
    for di, dj, dk, a in faces:
        ii, jj, kk = I + di, J + dj, K + dk
        ok = (ii >= 1) & (ii <= N) & (jj >= 1) & (jj <= N) & (kk >= 1) & (kk <= N)
        rows.append(row[ok])
        cols.append((ii + NC * jj + NC * NC * kk)[ok])
        vals.append(-a[ok] / hh)
    n = NC ** 3
    return sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, n))


def spmv(A: sp.spmatrix, x: np.ndarray) -> np.ndarray:
    """``SpMV`` (src/Factor.cpp:1099-1113): y_i = sum over column i, i.e. A^T x."""
    return A.T @ x


def relative_error_norm2(x: np.ndarray, y: np.ndarray) -> float:
    """``RelativeErrorNorm2`` (src/Factor.cpp:1083-1097): ||x - y|| / ||x||."""
    return float(math.sqrt(np.sum(np.abs(x - y) ** 2) / np.sum(np.abs(x) ** 2)))


# ----------------------------------------------------------------------------
# Dense kernels (the reference's BLAS/LAPACK call sites)
# ----------------------------------------------------------------------------

@dataclass
class Block:
    """One ``FactorData`` (include/data.hpp:84-110) plus its ``IndexData``."""
    global_inds: np.ndarray
    red: np.ndarray          # positions into global_inds (redundant_inds)
    skel: np.ndarray         # positions into global_inds (skeleton_inds)
    face: int = -1
    A22: np.ndarray = field(default=None, repr=False)
    A22inv: np.ndarray = field(default=None, repr=False)
    X: np.ndarray = field(default=None, repr=False)
    S: np.ndarray = field(default=None, repr=False)
    W: np.ndarray = field(default=None, repr=False)


def schur(mat: np.ndarray, blk: Block) -> None:
    """``Schur`` (include/Schur.hpp:72-100)."""
    r, s = blk.red, blk.skel
    A12 = mat[np.ix_(s, r)]
    A21 = mat[np.ix_(r, s)]
    blk.A22 = mat[np.ix_(r, r)].copy()
    blk.A22inv = sla.inv(blk.A22) if len(r) else np.zeros((0, 0))  # getrf + getri
    blk.X = blk.A22inv @ A21
    blk.S = -(A12 @ blk.X)


class _ReferenceLapack:
    """dgeqp3 from the very OpenBLAS library the reference build links.

    Column-pivoted QR meets exact ties when the operator is symmetric under
    reflections of a face (a = 1); which tied column a LAPACK build picks
    depends on its rounding. Calling the same library with the same workspace
    size as ``PivotedQRWrapper`` (2n + (n+1)*32, src/InterpDecomp.cpp:161 and
    include/hifde3d/core/lapack.hpp:26,537) reproduces the reference's pivots
    bit for bit. Falls back to scipy's geqp3 when that library is absent.
    """

    _lib = None
    _tried = False

    @classmethod
    def lib(cls):
        if cls._tried:
            return cls._lib
        cls._tried = True
        import ctypes
        import glob
        import sysconfig
        d = os.path.join(sysconfig.get_paths()["purelib"], "opencv_python_headless.libs")
        try:
            for pat in ("libquadmath-*.so*", "libgfortran-*.so*"):
                for p in glob.glob(os.path.join(d, pat)):
                    ctypes.CDLL(p, mode=ctypes.RTLD_GLOBAL)
            cands = glob.glob(os.path.join(d, "libopenblasp-*.so"))
            if cands:
                lib = ctypes.CDLL(cands[0])
                lib.openblas_set_num_threads(ctypes.c_int(1))
                cls._lib = lib
        except OSError:
            cls._lib = None
        return cls._lib

    @classmethod
    def geqp3(cls, M: np.ndarray):
        """Returns (raw array as LAPACK leaves it, 0-based jpvt) or None."""
        lib = cls.lib()
        if lib is None:
            return None
        import ctypes
        m, n = M.shape
        a = np.asfortranarray(M, dtype=np.float64).copy(order="F")
        jpvt = np.zeros(n, np.int32)
        tau = np.zeros(max(n, 1))
        lwork = 2 * n + (n + 1) * 32
        work = np.zeros(lwork)
        ci = ctypes.c_int
        info = ci(0)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.dgeqp3_(ctypes.byref(ci(m)), ctypes.byref(ci(n)), a.ctypes.data_as(dp),
                    ctypes.byref(ci(max(m, 1))), jpvt.ctypes.data_as(ip), tau.ctypes.data_as(dp),
                    work.ctypes.data_as(dp), ctypes.byref(ci(lwork)), ctypes.byref(info))
        if info.value != 0:
            raise RuntimeError(f"dgeqp3 info={info.value}")
        return a, jpvt.astype(np.int64) - 1


def geqp3(M: np.ndarray):
    """Column-pivoted QR: (raw LAPACK array, 0-based pivots)."""
    r = _ReferenceLapack.geqp3(M)
    if r is not None:
        return r
    (R, _tau), _r, jpvt = sla.qr(M, mode="raw", pivoting=True)
    return R, jpvt


def interp_decomp(M: np.ndarray, eps: float, order=None):
    """``InterpDecomp`` (src/InterpDecomp.cpp:86-138).

    Returns (W, skeleton_cols, redundant_cols, R_diag, jpvt). skeleton_cols and
    redundant_cols are in pivot order: jpvt[i] for the diagonal positions i that
    pass / fail |R_ii| > eps |R_00|.

    ``order`` (test hook): a prescribed column order replaces the pivot search
    (unpivoted Householder QR of M[:, order], LAPACK geqrf). Used to replay the
    reference's pivot decisions where its pivoted QR broke an exact tie.
    """
    m, n = M.shape
    if m < n:
        raise ValueError("InterpDecomp restatement needs at least as many rows as columns")
    # mode="raw" returns geqp3's output array as LAPACK leaves it: R on and above
    # the diagonal, Householder vectors below. The reference reads rows of that
    # array (src/InterpDecomp.cpp:116-123), so the restatement does too.
    if order is None:
        R, jpvt = geqp3(M)
    else:
        jpvt = np.asarray(order, np.int64)
        (R, _tau), _r = sla.qr(M[:, jpvt], mode="raw")
    tol = abs(R[0, 0]) * eps
    diag = np.array([R[i, i] for i in range(n)])
    skel = [i for i in range(n) if abs(diag[i]) > tol]
    red = [i for i in range(n) if not abs(diag[i]) > tol]
    k = len(skel)
    W_full = np.zeros((k, n))
    for a, i in enumerate(skel):
        W_full[a, :] = np.where(np.arange(n) >= a, R[i, :], 0.0)
    if k:
        R_skel = W_full[:, :k].copy()
        W_full = sla.solve_triangular(R_skel, W_full, lower=False)  # trsm 'L','U','N','N'
    W = W_full[:, red]
    return W, jpvt[skel], jpvt[red], diag, jpvt


# ----------------------------------------------------------------------------
# Partition (exact integer data)
# ----------------------------------------------------------------------------

class Partition:
    """DOF classification of src/Factor.cpp:313-755 for one frozen DOF mask."""

    def __init__(self, N: int, P: int, remaining: np.ndarray):
        self.N, self.P, self.NC = N, P, N + 1
        self.rem = remaining  # [i, j, k] uint8, shape (NC, NC, NC)

    def lin(self, i, j, k):
        NC = self.NC
        return i + NC * j + NC * NC * k

    def _interior(self, level, a):
        w = (1 << level) * self.P
        return (a > 0) & (a <= self.N) & (a % w != 0)

    def _box(self, cell, level):
        w = (1 << level) * self.P
        lo = [max(w * c, 1) for c in cell]
        hi = [min(w * (c + 1), self.N) for c in cell]
        return lo, hi

    def _scan(self, ii, jj, kk):
        I, J, K = np.meshgrid(np.asarray(ii), np.asarray(jj), np.asarray(kk), indexing="ij")
        return I.ravel(), J.ravel(), K.ravel()

    def cell_index_data(self, cell, level):
        """``InteriorCellIndexData`` (src/Factor.cpp:359-392)."""
        lo, hi = self._box(cell, level)
        I, J, K = self._scan(range(lo[0], hi[0] + 1), range(lo[1], hi[1] + 1),
                             range(lo[2], hi[2] + 1))
        if I.size == 0:
            return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.int64)
        a, b, c = self._interior(level, I), self._interior(level, J), self._interior(level, K)
        rem = self.rem[I, J, K] != 0
        cell_int = a & b & c
        face_int = (a & b & ~c) | (a & ~b & c) | (~a & b & c)
        keep = rem & (cell_int | face_int)
        g = self.lin(I, J, K)[keep]
        is_red = cell_int[keep]
        pos = np.arange(g.size)
        return g, pos[is_red], pos[~is_red]

    def _face_plane(self, cell, face, level):
        lo, hi = self._box(cell, level)
        if face == TOP:
            if lo[0] == 1:
                return None
            return [lo[0]], range(lo[1], hi[1] + 1), range(lo[2], hi[2] + 1)
        if face == BOTTOM:
            if hi[0] == self.N:
                return None
            return [hi[0]], range(lo[1], hi[1] + 1), range(lo[2], hi[2] + 1)
        if face == LEFT:
            if lo[1] == 1:
                return None
            return range(lo[0], hi[0] + 1), [lo[1]], range(lo[2], hi[2] + 1)
        if face == RIGHT:
            if hi[1] == self.N:
                return None
            return range(lo[0], hi[0] + 1), [hi[1]], range(lo[2], hi[2] + 1)
        if face == FRONT:
            # The reference tests k == 0 here (src/Factor.cpp:486), which never
            # holds because the box starts at max(width*c, 1); so a cell on the
            # k = 1 plane scans that plane. Reproduced as is.
            if lo[2] == 0:
                return None
            return range(lo[0], hi[0] + 1), range(lo[1], hi[1] + 1), [lo[2]]
        if face == BACK:
            if hi[2] == self.N:
                return None
            return range(lo[0], hi[0] + 1), range(lo[1], hi[1] + 1), [hi[2]]
        raise ValueError(face)

    def _plane_dofs(self, cell, face, level, want_edge):
        pl = self._face_plane(cell, face, level)
        if pl is None:
            return np.zeros(0, np.int64)
        I, J, K = self._scan(*pl)
        if I.size == 0:
            return np.zeros(0, np.int64)
        a, b, c = self._interior(level, I), self._interior(level, J), self._interior(level, K)
        if want_edge:
            sel = (a & ~b & ~c) | (~a & b & ~c) | (~a & ~b & c)
        else:
            sel = (a & b & ~c) | (a & ~b & c) | (~a & b & c)
        keep = (self.rem[I, J, K] != 0) & sel
        return self.lin(I, J, K)[keep]

    def face_dofs(self, cell, face, level):
        """``InteriorFaceDOFs`` (src/Factor.cpp:402-521)."""
        return self._plane_dofs(cell, face, level, False)

    def edge_dofs(self, cell, face, level):
        """``InteriorEdgeDOFs`` (src/Factor.cpp:523-643)."""
        return self._plane_dofs(cell, face, level, True)

    def skel_interaction(self, cell, face, level):
        """``SkelInteractionIndexData`` (src/Factor.cpp:645-755): (rows, cols)."""
        lo, _ = self._box(cell, level)
        empty = (np.zeros(0, np.int64), np.zeros(0, np.int64))
        if face == TOP:
            if lo[0] == 1:
                return empty
            own = [BOTTOM, LEFT, RIGHT, FRONT, BACK]
            nb = (cell[0] - 1, cell[1], cell[2])
            nbf = [TOP, LEFT, RIGHT, FRONT, BACK]
        elif face == LEFT:
            if lo[1] == 1:
                return empty
            own = [TOP, BOTTOM, RIGHT, FRONT, BACK]
            nb = (cell[0], cell[1] - 1, cell[2])
            nbf = [TOP, BOTTOM, LEFT, FRONT, BACK]
        elif face == FRONT:
            if lo[2] == 1:
                return empty
            own = [TOP, BOTTOM, LEFT, RIGHT, BACK]
            nb = (cell[0], cell[1], cell[2] - 1)
            nbf = [TOP, BOTTOM, LEFT, RIGHT, FRONT]
        else:
            raise ValueError("only TOP, LEFT, FRONT are skeletonized")
        cols = self.face_dofs(cell, face, level)
        rows = [self.edge_dofs(cell, face, level)]
        rows += [self.face_dofs(cell, f, level) for f in own]
        rows += [self.face_dofs(nb, f, level) for f in nbf]
        return np.concatenate(rows), cols


# ----------------------------------------------------------------------------
# Factorization
# ----------------------------------------------------------------------------

class HIFOracle:
    """``HIFFactor<double>`` restated (include/Factor.hpp:8-203)."""

    def __init__(self, N: int, P: int, epsilon: float, partition: str = "reference",
                 replay_pivots=None):
        self.N, self.P, self.eps = N, P, epsilon
        # replay_pivots[level][face block] -> column order (test hook, see interp_decomp)
        self.replay_pivots = replay_pivots
        self.NC = N + 1
        self.partition = partition
        self.A = None
        self.schur_levels: list[list[Block]] = []
        self.skel_levels: list[list[Block]] = []
        self.record_M = False
        self.M_blocks: list[list[np.ndarray]] = []

    def set_matrix(self, A: sp.spmatrix) -> None:
        self.A = sp.csr_matrix(A)

    def initialize(self) -> None:
        """``Initialize`` (src/Factor.cpp:6-39)."""
        NC = self.NC
        self.rem = np.ones((NC, NC, NC), np.uint8)
        self.rem[0, :, :] = 0
        self.rem[:, 0, :] = 0
        self.rem[:, :, 0] = 0
        self.L = num_levels(self.N, self.P, self.partition)
        self.schur_levels = [[] for _ in range(self.L)]
        self.skel_levels = [[] for _ in range(self.L)]
        self.M_blocks = [[] for _ in range(self.L)]

    def _sub(self, rows, cols):
        return self.A[rows][:, cols].toarray()

    def level_factor_schur(self, cpd, level):
        """``LevelFactorSchur`` (src/Factor.cpp:184-213)."""
        part = Partition(self.N, self.P, self.rem)
        out = []
        for ci in range(cpd):
            for cj in range(cpd):
                for ck in range(cpd):
                    g, red, skl = part.cell_index_data((ci, cj, ck), level)
                    blk = Block(g, red, skl)
                    schur(self._sub(g, g), blk)
                    out.append(blk)
        self.schur_levels[level] = out

    def level_factor_skel(self, cpd, level):
        """``LevelFactorSkel`` (src/Factor.cpp:232-260) + ``Skeletonize``."""
        part = Partition(self.N, self.P, self.rem)
        out = []
        for ci in range(cpd):
            for cj in range(cpd):
                for ck in range(cpd):
                    for face in (TOP, FRONT, LEFT):
                        rows, cols = part.skel_interaction((ci, cj, ck), face, level)
                        if cols.size == 0:
                            continue
                        M = self._sub(rows, cols)
                        if self.record_M:
                            self.M_blocks[level].append(M.copy())
                        order = None
                        if self.replay_pivots is not None:
                            order = self.replay_pivots[level][len(out)]
                        W, skel_cols, red_cols, _, _ = interp_decomp(M, self.eps, order)
                        blk = Block(cols.copy(), np.asarray(red_cols, np.int64),
                                    np.asarray(skel_cols, np.int64), face=face)
                        blk.W = W
                        self._schur_after_id(blk)
                        out.append(blk)
        self.skel_levels[level] = out

    def _schur_after_id(self, blk: Block):
        """``SchurAfterID`` (src/Factor.cpp:113-153)."""
        g = blk.global_inds
        n = g.size
        Rot = np.eye(n)
        if blk.red.size and blk.skel.size:
            Rot[np.ix_(blk.skel, blk.red)] = -blk.W
        sub = self._sub(g, g)
        tmp = sub @ Rot
        result = Rot.conj().T @ tmp
        schur(result, blk)

    def update_matrix_and_dofs(self, blocks):
        """``UpdateMatrixAndDOFs`` (src/Factor.cpp:262-311)."""
        rows, cols, vals, dels = [], [], [], []
        for b in blocks:
            sg = b.global_inds[b.skel]
            if sg.size:
                rr, cc = np.meshgrid(sg, sg, indexing="ij")
                rows.append(rr.ravel())
                cols.append(cc.ravel())
                vals.append(b.S.ravel())
            dels.append(b.global_inds[b.red])
        n = self.A.shape[0]
        keep = np.ones(n)
        if dels:
            d = np.concatenate(dels)
            keep[d] = 0.0
        D = sp.diags(keep)
        A = D @ self.A @ D
        if rows:
            A = A + sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows),
                                                          np.concatenate(cols))), shape=(n, n))
        A.eliminate_zeros()
        self.A = sp.csr_matrix(A)
        if dels:
            d = np.concatenate(dels)
            NC = self.NC
            self.rem[d % NC, (d // NC) % NC, d // (NC * NC)] = 0
        for b in blocks:
            b.S_kept = b.S  # the reference clears S here; keep it for checks

    def factor(self):
        """``Factor`` (src/Factor.cpp:41-63)."""
        for level in range(self.L):
            cpd = cells_per_dir(self.N, self.P, level, self.partition)
            self.level_factor_schur(cpd, level)
            self.update_matrix_and_dofs(self.schur_levels[level])
            if level < self.L - 1:
                self.level_factor_skel(cpd, level)
                self.update_matrix_and_dofs(self.skel_levels[level])

    # ------------------------------------------------------------------ apply
    def apply(self, u: np.ndarray, apply_inverse: bool = False) -> np.ndarray:
        """``Apply`` (src/Factor.cpp:992-1081). Returns a new vector."""
        u = np.array(u, dtype=np.float64, copy=True)
        NC = self.NC
        u3 = u.reshape(NC, NC, NC)  # [k, j, i] view of i + NC j + NC^2 k
        u3[0, :, :] = 0
        u3[:, 0, :] = 0
        u3[:, :, 0] = 0
        L = len(self.schur_levels)

        def parts(b):
            return b.global_inds[b.skel], b.global_inds[b.red]

        for level in range(L - 1):
            for b in self.schur_levels[level]:
                gs, gr = parts(b)
                if gs.size and gr.size:
                    if apply_inverse:
                        u[gs] = u[gs] - b.X.T @ u[gr]
                    else:
                        u[gr] = u[gr] + b.X @ u[gs]
            for b in self.skel_levels[level]:
                gs, gr = parts(b)
                if gs.size and gr.size:
                    if apply_inverse:
                        u[gr] = u[gr] - b.W.T @ u[gs]
                        u[gs] = u[gs] - b.X.T @ u[gr]
                    else:
                        u[gs] = u[gs] + b.W @ u[gr]
                        u[gr] = u[gr] + b.X @ u[gs]
        for level in range(L):
            for b in self.schur_levels[level] + self.skel_levels[level]:
                gr = b.global_inds[b.red]
                if gr.size:
                    u[gr] = (b.A22inv if apply_inverse else b.A22) @ u[gr]
        for level in range(L - 2, -1, -1):
            for b in self.skel_levels[level]:
                gs, gr = parts(b)
                if gs.size and gr.size:
                    if apply_inverse:
                        u[gr] = u[gr] - b.X @ u[gs]
                        u[gs] = u[gs] - b.W @ u[gr]
                    else:
                        u[gs] = u[gs] + b.X.T @ u[gr]
                        u[gr] = u[gr] + b.W.T @ u[gs]
            for b in self.schur_levels[level]:
                gs, gr = parts(b)
                if gs.size and gr.size:
                    if apply_inverse:
                        u[gr] = u[gr] - b.X @ u[gs]
                    else:
                        u[gs] = u[gs] + b.X.T @ u[gr]
        return u


# ----------------------------------------------------------------------------
# Convenience drivers
# ----------------------------------------------------------------------------

def unit_tensors(N: int):
    """A = 1, V = 0 on the (NC+1)^3 grid (tests/HIFDE3D/main.cpp:59-74)."""
    NC = N + 1
    return np.ones((NC + 1,) * 3), np.zeros((NC + 1,) * 3)


def factor_node(N: int, P: int, eps: float, A: np.ndarray, V: np.ndarray,
                partition: str = "reference", replay_pivots=None
                ) -> tuple[HIFOracle, sp.spmatrix]:
    """SetupStencil + Initialize + Factor, returning the factor and the operator."""
    NC = N + 1
    op = setup_stencil(N, 1.0 / NC, A, V)
    f = HIFOracle(N, P, eps, partition, replay_pivots)
    f.set_matrix(op)
    f.initialize()
    f.factor()
    return f, op


def pcg(op: sp.spmatrix, b: np.ndarray, precond, tol: float = 1e-10, maxit: int = 200):
    """Preconditioned CG on y = A x (the reference has no iterative solver)."""
    x = np.zeros_like(b)
    r = b.copy()
    z = precond(r)
    p = z.copy()
    rz = r @ z
    bn = np.linalg.norm(b)
    hist = []
    for it in range(1, maxit + 1):
        q = op @ p
        al = rz / (p @ q)
        x += al * p
        r -= al * q
        rel = np.linalg.norm(r) / bn
        hist.append(rel)
        if rel <= tol:
            return x, it, hist
        z = precond(r)
        rz2 = r @ z
        p = z + (rz2 / rz) * p
        rz = rz2
    return x, maxit, hist


def gmres(op: sp.spmatrix, b: np.ndarray, precond, tol: float = 1e-10, restart: int = 30,
          maxit: int = 200):
    """Restarted GMRES(restart) on A x = b with ``precond`` as right preconditioner
    (the reference has no iterative solver). Same steps as the library's solver:
    Krylov space of A M^-1 from r0 = b - A x0 (x0 = 0), classical Gram-Schmidt
    applied twice, Givens rotations on the Hessenberg matrix, a cycle ends when
    the rotated residual estimate reaches tol (or maxit Arnoldi steps in all),
    x += M^-1 V y, and convergence is decided on the true residual.
    Returns (x, Arnoldi steps, true relative residual)."""
    x = np.zeros_like(b)
    bn = np.linalg.norm(b)
    if bn == 0:
        return x, 0, 0.0
    r = b.copy()
    total = 0
    rel = 1.0
    while total < maxit:
        beta = np.linalg.norm(r)
        if beta == 0:
            break
        V = [r / beta]
        R = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        k = 0
        for j in range(restart):
            w = op @ precond(V[j])
            h = np.zeros(j + 2)
            for _ in range(2):
                c = np.array([v @ w for v in V])
                w = w - np.asarray(V).T @ c
                h[:j + 1] += c
            hn = np.linalg.norm(w)
            h[j + 1] = hn
            for i in range(j):
                t = cs[i] * h[i] + sn[i] * h[i + 1]
                h[i + 1] = -sn[i] * h[i] + cs[i] * h[i + 1]
                h[i] = t
            den = np.hypot(h[j], h[j + 1])
            cs[j], sn[j] = (h[j] / den, h[j + 1] / den) if den > 0 else (1.0, 0.0)
            h[j], h[j + 1] = den, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            R[:j + 1, j] = h[:j + 1]
            total += 1
            k = j + 1
            if abs(g[j + 1]) / bn <= tol or total >= maxit or not hn > 0 or den == 0:
                break
            V.append(w / hn)
        y = np.zeros(k)
        for i in range(k - 1, -1, -1):
            y[i] = (g[i] - R[i, i + 1:k] @ y[i + 1:k]) / R[i, i] if R[i, i] != 0 else 0.0
        x = x + precond(np.asarray(V[:k]).T @ y)
        r = b - op @ x
        rel = np.linalg.norm(r) / bn
        if rel <= tol:
            break
    return x, total, rel
