"""B200 implementation of HIFDE3D's hierarchical interpolative factorization.

Python mirror of the reference's C++ API (arbenson/HIFDE3D include/Factor.hpp,
include/setup_stencil.hpp) over the C ABI of libhif_b200.so
(include/hif_b200.h). Names, argument meaning and call order follow the
reference::

    f = HIFFactor(N, P, epsilon)                 # HIFFactor<double>(N, P, eps)
    SetupStencil(f, N, 1.0 / (N + 1), A, V)      # include/setup_stencil.hpp:6
    f.Initialize(); f.Factor()                   # src/Factor.cpp:6, 41
    f.Apply(u, apply_inverse=True)               # src/Factor.cpp:992 (in place)

Vectors are float64 numpy arrays of NC^3 entries (NC = N + 1) in DOF order
i + NC*j + NC^2*k, or (NC^3, nrhs) column blocks. Errors raise HIFError with the
C status code. There is no CPU fallback: without the compiled library or a CUDA
device every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libhif_b200.so")
_lib = None

HIF_OK, HIF_ERR_ARG, HIF_ERR_CUDA, HIF_ERR_NOMEM, HIF_ERR_SINGULAR = 0, 1, 2, 3, 4
HIF_ERR_STATE, HIF_ERR_NODEVICE, HIF_ERR_BUDGET, HIF_ERR_IO = 5, 6, 7, 8
PARTITION_REFERENCE, PARTITION_CLIPPED = 0, 1
OPT_KEEP_SCHUR, OPT_VERBOSE, OPT_MEM_BUDGET_MB, OPT_PROFILE, OPT_ID_GROUP_MIN_N = 1, 2, 3, 4, 5
OPT_PRECISION, OPT_AUTOTUNE, OPT_SCHUR_SLICES, OPT_X_SLICES = 6, 7, 8, 9
OPT_ELIMINATION, OPT_Y_SLICES, OPT_GRAM_MIN_N, OPT_GRAM_SLICES, OPT_CHOL_SLICES = 10, 11, 12, 13, 14
PRECISION_FP64, PRECISION_MIXED = 0, 1
ELIM_AUTO, ELIM_GAUSS_JORDAN, ELIM_CHOLESKY = 0, 1, 2
KCLASS_NAMES = ["gather", "gemm", "sweep_small", "sweep_panel", "id", "gemv", "copy", "vector",
                "qr", "gemm_mixed", "gemm_int8"]
TOP, BOTTOM, RIGHT, LEFT, FRONT, BACK = range(6)


class HIFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hif status {code}: {msg}")
        self.code = code


_i, _d, _ll, _p = ctypes.c_int, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)
_llp = ctypes.POINTER(ctypes.c_longlong)

_SIGNATURES = {
    "hif_create": [_i, _i, _d, _i, ctypes.POINTER(_p)],
    "hif_destroy": [_p],
    "hif_set_stream": [_p, _p],
    "hif_setup_stencil": [_p, _i, _d, _dp, _dp],
    "hif_setup_stencil_device": [_p, _i, _d, _p, _p],
    "hif_setup_stencil_faces": [_p, _i, _d, _dp, _dp, _dp, _dp],
    "hif_setup_stencil_faces_device": [_p, _i, _d, _p, _p, _p, _p],
    "hif_initialize": [_p],
    "hif_factor": [_p],
    "hif_save_factor": [_p, ctypes.c_char_p],
    "hif_load_factor": [_p, ctypes.c_char_p],
    "hif_apply": [_p, _dp, _i, _ll, _i],
    "hif_apply_device": [_p, _p, _i, _ll, _i],
    "hif_spmv": [_p, _dp, _dp, _i, _ll, _i],
    "hif_spmv_device": [_p, _p, _p, _i, _ll, _i],
    "hif_solve_pcg": [_p, _dp, _dp, _i, _ll, _d, _i, _ip, _dp],
    "hif_solve_pcg_device": [_p, _p, _p, _i, _ll, _d, _i, _ip, _dp],
    "hif_solve_gmres": [_p, _dp, _dp, _i, _ll, _d, _i, _i, _ip, _dp],
    "hif_solve_gmres_device": [_p, _p, _p, _i, _ll, _d, _i, _i, _ip, _dp],
    "hif_num_levels": [_p, _ip],
    "hif_num_blocks": [_p, _i, _i, _ip],
    "hif_block_info": [_p, _i, _i, _i, _ip, _ip, _ip, _ip],
    "hif_block_indices": [_p, _i, _i, _i, _ip, _ip, _ip],
    "hif_block_matrix": [_p, _i, _i, _i, _i, _dp],
    "hif_block_pivots": [_p, _i, _i, _ip, _dp],
    "hif_dof_levels": [_p, _ip],
    "hif_set_option": [_p, _i, _ll],
    "hif_set_replay_pivots": [_p, _i, _i, _ip, _ip],
    "hif_factor_stats": [_p, _dp, _dp, _dp, _dp, _dp, _llp],
    "hif_kernel_stats": [_p, _i, _llp, _dp, _dp, _dp],
    "hif_autotune_stats": [_p, _ip, _ip, _ip],
    "hif_autotune_elimination": [_p, _ip, _ip, _ip],
    "hif_memory": [_p, _llp, _llp],
    "hif_trim": [_p],
    "hif_trim_device_pool": [],
    "hif_schur": [_dp, _i, _ll, _ip, _i, _ip, _i, _dp, _dp, _dp, _dp],
    "hif_schur_device": [_p, _i, _i, _p, _p, _p],
    "hif_schur_device_noalloc": [_p, _i, _i, _p, _p, _p, _p],
    "hif_interp_decomp": [_dp, _i, _i, _ll, _d, _dp, _ip, _ip, _ip],
    "hif_pivoted_qr": [_dp, _i, _i, _ll, _ip],
    "hif_triangular_solve": [_dp, _i, _ll, _dp, _i, _ll],
    "hif_gemm_mixed_device": [_i, _i, _i, _i, _i, _d, _p, _ll, _p, _ll, _d, _p, _ll],
    "hif_gemm_int8_device": [_i, _i, _i, _i, _i, _d, _p, _ll, _p, _ll, _d, _p, _ll, _i],
    "hif_server_create": [_ll, _i, _i, ctypes.POINTER(_p)],
    "hif_server_destroy": [_p],
    "hif_server_submit_factor": [_p, _i, _i, _i, _d, _i, _i, _d, _dp, _dp, _dp, _dp, _llp],
    "hif_server_submit_solve": [_p, _i, _dp, _i, _d, _i, _dp, _llp],
    "hif_server_wait": [_p, _ll, _ip, _ip, _dp, _dp],
    "hif_server_wait_detail": [_p, _ll, _ip, _ip, _dp, _dp, _dp],
    "hif_server_release": [_p, _i],
    "hif_server_stats": [_p, _llp, _llp, _llp, _llp, _llp],
    "hif_partition_cell": [_i, _i, _i, _i, _i, _i, _i, ctypes.POINTER(ctypes.c_ubyte),
                           _ip, _ip, _ip, _ip],
    "hif_partition_face": [_i, _i, _i, _i, _i, _i, _i, _i, ctypes.POINTER(ctypes.c_ubyte),
                           _ip, _ip],
}


def library_path() -> str:
    return _LIB_PATH


def lib():
    """Load libhif_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise HIFError(HIF_ERR_NODEVICE,
                           f"{_LIB_PATH} missing: run python -m hifde3d_b200.build")
        L = ctypes.CDLL(_LIB_PATH)
        for name, args in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.hif_last_error.restype = ctypes.c_char_p
        L.hif_last_error.argtypes = []
        _lib = L
    return _lib


def _check(code: int):
    if code != HIF_OK:
        raise HIFError(code, lib().hif_last_error().decode())


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


class Index3(tuple):
    """Vec3T<int> (include/vec3t.hpp:197)."""

    def __new__(cls, i, j, k):
        return super().__new__(cls, (int(i), int(j), int(k)))


class HIFFactor:
    """``HIFFactor<double>`` (include/Factor.hpp:8-203) on one B200."""

    def __init__(self, N: int, P: int, epsilon: float, partition: int = PARTITION_REFERENCE):
        self._N, self._P, self._eps = int(N), int(P), float(epsilon)
        self._h = _p()
        _check(lib().hif_create(self._N, self._P, self._eps, int(partition),
                                ctypes.byref(self._h)))
        self.NC = self._N + 1

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().hif_destroy(self._h)
            self._h = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- accessors (include/Factor.hpp:41-48) ----
    def N(self) -> int:
        return self._N

    def P(self) -> int:
        return self._P

    def epsilon(self) -> float:
        return self._eps

    # ---- index maps (src/Factor.cpp:65-89) ----
    def Tensor2LinearInd(self, ind) -> int:
        i, j, k = ind
        return i + self.NC * j + self.NC * self.NC * k

    def Linear2TensorInd(self, ind: int) -> Index3:
        NC = self.NC
        return Index3(ind % NC, (ind // NC) % NC, ind // (NC * NC))

    # ---- factor (src/Factor.cpp:6-63) ----
    def Initialize(self):
        _check(lib().hif_initialize(self._h))

    def Factor(self):
        _check(lib().hif_factor(self._h))

    def save(self, path: str):
        """Write the factorization (and the operator, when set) to `path`
        (hif_save_factor)."""
        _check(lib().hif_save_factor(self._h, os.fsencode(path)))

    def load(self, path: str):
        """Replace this handle's factorization by the one saved in `path`; the
        handle must have the saved N, P, epsilon and partition (hif_load_factor)."""
        _check(lib().hif_load_factor(self._h, os.fsencode(path)))

    def set_option(self, option: int, value: int):
        _check(lib().hif_set_option(self._h, int(option), int(value)))

    def set_replay_pivots(self, level: int, orders):
        """Test hook: prescribe each face's ID column order at ``level``."""
        if not orders:
            _check(lib().hif_set_replay_pivots(self._h, level, 0, None, None))
            return
        off = np.zeros(len(orders) + 1, np.int32)
        off[1:] = np.cumsum([len(o) for o in orders])
        flat = np.ascontiguousarray(np.concatenate(orders).astype(np.int32))
        _check(lib().hif_set_replay_pivots(self._h, level, len(orders), _iptr(off), _iptr(flat)))

    # ---- apply (src/Factor.cpp:992-1081) ----
    def Apply(self, u: np.ndarray, apply_inverse: bool = False) -> np.ndarray:
        """In place on ``u`` (float64, C-contiguous or (n, nrhs) Fortran order)."""
        n3 = self.NC ** 3
        if u.dtype != np.float64:
            raise HIFError(HIF_ERR_ARG, "u must be float64")
        if u.ndim == 1:
            if u.size != n3 or not u.flags.c_contiguous:
                raise HIFError(HIF_ERR_ARG, "u must have NC^3 contiguous entries")
            _check(lib().hif_apply(self._h, _dptr(u), 1, n3, int(bool(apply_inverse))))
            return u
        if u.shape[0] != n3 or not u.flags.f_contiguous:
            raise HIFError(HIF_ERR_ARG, "multi-RHS u must be (NC^3, nrhs) Fortran-ordered")
        _check(lib().hif_apply(self._h, _dptr(u), u.shape[1], n3, int(bool(apply_inverse))))
        return u

    def apply_device(self, ptr: int, nrhs: int, ldu: int, apply_inverse: bool):
        _check(lib().hif_apply_device(self._h, _p(ptr), nrhs, ldu, int(bool(apply_inverse))))

    def spmv(self, x: np.ndarray, transpose: bool = True) -> np.ndarray:
        """y = A^T x (``SpMV``, the reference walks columns) or y = A x."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        _check(lib().hif_spmv(self._h, _dptr(x), _dptr(y), 1, x.size, int(bool(transpose))))
        return y

    def solve_pcg(self, b: np.ndarray, tol: float = 1e-10, maxit: int = 200):
        """PCG on A x = b preconditioned by the inverse apply. Returns (x, iters, relres);
        for b of shape (NC^3, nrhs) iters and relres are per right-hand side."""
        b = np.asarray(b, dtype=np.float64)
        if b.ndim == 1:
            b = np.ascontiguousarray(b)
            x = np.zeros_like(b)
            it = np.zeros(1, np.int32)
            rr = np.zeros(1)
            _check(lib().hif_solve_pcg(self._h, _dptr(b), _dptr(x), 1, b.size, tol, maxit,
                                       _iptr(it), _dptr(rr)))
            return x, int(it[0]), float(rr[0])
        b = np.asfortranarray(b)
        n, nrhs = b.shape
        x = np.zeros((n, nrhs), order="F")
        it = np.zeros(nrhs, np.int32)
        rr = np.zeros(nrhs)
        _check(lib().hif_solve_pcg(self._h, _dptr(b), _dptr(x), nrhs, n, tol, maxit,
                                   _iptr(it), _dptr(rr)))
        return x, it, rr

    def solve_gmres(self, b: np.ndarray, tol: float = 1e-10, maxit: int = 200,
                    restart: int = 30):
        """Restarted GMRES on A x = b, right-preconditioned by the inverse apply (the
        solver for the non-symmetric node operator). Returns (x, iters, relres); for
        b of shape (NC^3, nrhs) iters and relres are per right-hand side."""
        b = np.asarray(b, dtype=np.float64)
        single = b.ndim == 1
        b2 = np.asfortranarray(b.reshape(-1, 1) if single else b)
        n, nrhs = b2.shape
        x = np.zeros((n, nrhs), order="F")
        it = np.zeros(nrhs, np.int32)
        rr = np.zeros(nrhs)
        _check(lib().hif_solve_gmres(self._h, _dptr(b2), _dptr(x), nrhs, n, tol, maxit,
                                     int(restart), _iptr(it), _dptr(rr)))
        if single:
            return x[:, 0].copy(), int(it[0]), float(rr[0])
        return x, it, rr

    def solve_gmres_device(self, db: int, dx: int, nrhs: int, ld: int, tol: float, maxit: int,
                           restart: int = 30):
        it = np.zeros(nrhs, np.int32)
        rr = np.zeros(nrhs)
        _check(lib().hif_solve_gmres_device(self._h, _p(db), _p(dx), nrhs, ld, tol, maxit,
                                            int(restart), _iptr(it), _dptr(rr)))
        return it, rr

    def solve_pcg_device(self, db: int, dx: int, nrhs: int, ld: int, tol: float, maxit: int):
        it = np.zeros(nrhs, np.int32)
        rr = np.zeros(nrhs)
        _check(lib().hif_solve_pcg_device(self._h, _p(db), _p(dx), nrhs, ld, tol, maxit,
                                          _iptr(it), _dptr(rr)))
        return it, rr

    # ---- introspection (schur_level_data / skel_level_data) ----
    def num_levels(self) -> int:
        v = ctypes.c_int()
        _check(lib().hif_num_levels(self._h, ctypes.byref(v)))
        return v.value

    def num_blocks(self, level: int, kind: int) -> int:
        v = ctypes.c_int()
        _check(lib().hif_num_blocks(self._h, level, kind, ctypes.byref(v)))
        return v.value

    def block(self, level: int, kind: int, b: int, matrices: bool = False):
        ng, nr, ns, face = (ctypes.c_int() for _ in range(4))
        _check(lib().hif_block_info(self._h, level, kind, b, ctypes.byref(ng), ctypes.byref(nr),
                                    ctypes.byref(ns), ctypes.byref(face)))
        g = np.zeros(max(ng.value, 1), np.int32)
        r = np.zeros(max(nr.value, 1), np.int32)
        s = np.zeros(max(ns.value, 1), np.int32)
        _check(lib().hif_block_indices(self._h, level, kind, b, _iptr(g), _iptr(r), _iptr(s)))
        out = {"face": face.value, "global": g[:ng.value].astype(np.int64),
               "red": r[:nr.value].astype(np.int64), "skel": s[:ns.value].astype(np.int64)}
        if matrices:
            R, K = nr.value, ns.value
            shapes = {"A22": (R, R), "A22inv": (R, R), "X": (R, K)}
            if kind == 1:
                shapes["W"] = (K, R)
            for which, name in enumerate(["A22", "A22inv", "X", "W"]):
                if name not in shapes:
                    continue
                h, w = shapes[name]
                buf = np.zeros(max(h * w, 1))
                _check(lib().hif_block_matrix(self._h, level, kind, b, which, _dptr(buf)))
                out[name] = buf[:h * w].reshape(w, h).T.copy()
        return out

    def schur_complement(self, level: int, kind: int, b: int) -> np.ndarray:
        info = self.block(level, kind, b)
        k = info["skel"].size
        buf = np.zeros(max(k * k, 1))
        _check(lib().hif_block_matrix(self._h, level, kind, b, 4, _dptr(buf)))
        return buf[:k * k].reshape(k, k).T.copy()

    def pivots(self, level: int, b: int):
        info = self.block(level, 1, b)
        n = info["global"].size
        jp = np.zeros(max(n, 1), np.int32)
        rd = np.zeros(max(n, 1))
        _check(lib().hif_block_pivots(self._h, level, b, _iptr(jp), _dptr(rd)))
        return jp[:n].astype(np.int64), rd[:n]

    def dof_levels(self) -> np.ndarray:
        """Per DOF id: the phase that eliminated it (2 * level + kind), -1 on the
        index-0 planes."""
        out = np.zeros(self.NC ** 3, np.int32)
        _check(lib().hif_dof_levels(self._h, _iptr(out)))
        return out

    def kernel_stats(self) -> dict:
        """Per kernel class: launches, ms, algorithmic flops and bytes (needs OPT_PROFILE)."""
        out = {}
        for c, name in enumerate(KCLASS_NAMES):
            n = ctypes.c_longlong()
            ms, fl, by = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
            _check(lib().hif_kernel_stats(self._h, c, ctypes.byref(n), ctypes.byref(ms),
                                          ctypes.byref(fl), ctypes.byref(by)))
            out[name] = {"launches": n.value, "ms": ms.value, "flops": fl.value, "bytes": by.value}
        return out

    def autotune_stats(self) -> dict:
        """OPT_AUTOTUNE tuner: batch signatures seen, decided, and how many chose 128 x 128."""
        n, d, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().hif_autotune_stats(self._h, ctypes.byref(n), ctypes.byref(d),
                                        ctypes.byref(c)))
        e_n, e_d, e_c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().hif_autotune_elimination(self._h, ctypes.byref(e_n), ctypes.byref(e_d),
                                              ctypes.byref(e_c)))
        return {"signatures": n.value, "decided": d.value, "chose_128": c.value,
                "elimination_phases": e_n.value, "elimination_decided": e_d.value,
                "elimination_chose_cholesky": e_c.value}

    def memory(self) -> dict:
        fb, wb = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().hif_memory(self._h, ctypes.byref(fb), ctypes.byref(wb)))
        return {"factor_bytes": fb.value, "workspace_bytes": wb.value}

    def trim(self):
        """Return the factorization workspace to the device (the factor stays)."""
        _check(lib().hif_trim(self._h))

    def factor_stats(self) -> dict:
        vals = [ctypes.c_double() for _ in range(5)]
        nb = ctypes.c_longlong()
        _check(lib().hif_factor_stats(self._h, *[ctypes.byref(v) for v in vals], ctypes.byref(nb)))
        keys = ["total_s", "gather_s", "elim_s", "id_s", "host_s"]
        d = {k: v.value for k, v in zip(keys, vals)}
        d["device_bytes"] = nb.value
        return d


def trim_device_pool() -> None:
    """Return the unused reserved memory of the current device's default pool."""
    _check(lib().hif_trim_device_pool())


def GemmMixedDevice(transA: int, transB: int, m: int, n: int, k: int, alpha: float, dA: int,
                    lda: int, dB: int, ldb: int, beta: float, dC: int, ldc: int) -> None:
    """C = alpha op(A) op(B) + beta C on device pointers (column-major), split-TF32
    products on the tcgen05 tensor cores with FP32 accumulation."""
    _check(lib().hif_gemm_mixed_device(int(transA), int(transB), m, n, k, float(alpha), _p(dA),
                                       lda, _p(dB), ldb, float(beta), _p(dC), ldc))


def GemmInt8Device(transA: int, transB: int, m: int, n: int, k: int, alpha: float, dA: int,
                   lda: int, dB: int, ldb: int, beta: float, dC: int, ldc: int,
                   slices: int = 7) -> None:
    """C = alpha op(A) op(B) + beta C on device pointers (column-major), FP64 from
    exact int8 slice products on the tcgen05 tensor cores (Ozaki scheme)."""
    _check(lib().hif_gemm_int8_device(int(transA), int(transB), m, n, k, float(alpha), _p(dA),
                                      lda, _p(dB), ldb, float(beta), _p(dC), ldc, int(slices)))


class Server:
    """Many factored operators resident on one GPU, with iteration-level batched
    PCG solves across them (``hif_server_*`` in include/hif_b200.h).

    ``submit_factor`` / ``submit_solve`` return a request id at once; ``wait``
    blocks until the request ends and returns a dict with ``status``, ``iters``,
    ``relres``, ``latency_ms`` and, for solves, ``x`` (NC^3 x nrhs, float64,
    column-major like the right-hand sides)."""

    def __init__(self, budget_bytes: int, max_active_solves: int = 64, factor_workers: int = 2):
        h = _p()
        _check(lib().hif_server_create(int(budget_bytes), int(max_active_solves),
                                       int(factor_workers), ctypes.byref(h)))
        self._h = h
        self._out = {}
        self._n3 = {}

    def close(self):
        if self._h:
            _check(lib().hif_server_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit_factor(self, op_id: int, N: int, ax, ay, az, V, P: int = 4, eps: float = 1e-6,
                      precision: int = 0, partition: int = 0, h: float | None = None) -> int:
        arrs = [np.ascontiguousarray(np.asarray(x, np.float64).ravel(order="F"))
                for x in (ax, ay, az, V)]
        for x in arrs:
            if x.size != (N + 2) ** 3:
                raise HIFError(HIF_ERR_ARG, "face arrays must be (N+2)^3")
        rid = _ll()
        hstep = 1.0 / (N + 1) if h is None else float(h)
        _check(lib().hif_server_submit_factor(self._h, int(op_id), N, P, float(eps),
                                              int(partition), int(precision), hstep,
                                              *[_dptr(x) for x in arrs], ctypes.byref(rid)))
        self._n3[int(op_id)] = (N + 1) ** 3
        self._out[rid.value] = (None, arrs)  # inputs stay alive until the copy
        return rid.value

    def submit_solve(self, op_id: int, b, tol: float = 1e-10, maxit: int = 100) -> int:
        n3 = self._n3.get(int(op_id))
        if n3 is None:
            raise HIFError(HIF_ERR_ARG, f"unknown operator {op_id}")
        bb = np.asarray(b, np.float64)
        nrhs = 1 if bb.ndim == 1 else bb.shape[1]
        bf = np.ascontiguousarray(bb.reshape(n3, nrhs, order="F").T).ravel()
        x = np.zeros(n3 * nrhs)
        rid = _ll()
        _check(lib().hif_server_submit_solve(self._h, int(op_id), _dptr(bf), nrhs, float(tol),
                                             int(maxit), _dptr(x), ctypes.byref(rid)))
        self._out[rid.value] = (x, (nrhs, bb.ndim))
        return rid.value

    def wait(self, request_id: int) -> dict:
        """Blocks until the request ends. latency_ms = submit to completion,
        queue_ms = submit to admission, service_ms = the rest."""
        st, it = _i(), _i()
        rr, lat, qu = _d(), _d(), _d()
        code = lib().hif_server_wait_detail(self._h, int(request_id), ctypes.byref(st),
                                            ctypes.byref(it), ctypes.byref(rr),
                                            ctypes.byref(lat), ctypes.byref(qu))
        _check(code)
        x, meta = self._out.pop(int(request_id), (None, None))
        res = {"status": st.value, "iters": it.value, "relres": rr.value,
               "latency_ms": lat.value, "queue_ms": qu.value,
               "service_ms": lat.value - qu.value}
        if st.value != HIF_OK:
            res["error"] = lib().hif_last_error().decode()
        if x is not None:
            nrhs, ndim = meta
            xm = x.reshape(nrhs, -1).T
            res["x"] = xm[:, 0].copy() if ndim == 1 else np.asfortranarray(xm)
        return res

    def release(self, op_id: int) -> None:
        _check(lib().hif_server_release(self._h, int(op_id)))
        self._n3.pop(int(op_id), None)

    def stats(self) -> dict:
        vals = [_ll() for _ in range(5)]
        _check(lib().hif_server_stats(self._h, *[ctypes.byref(v) for v in vals]))
        keys = ("device_bytes", "resident_ops", "completed", "iterations", "batched_launches")
        return {k: v.value for k, v in zip(keys, vals)}


def SetupStencil(factor: HIFFactor, N: int, h: float, A: np.ndarray, V: np.ndarray) -> None:
    """``SetupStencil`` (include/setup_stencil.hpp:6-76). A, V: (N+2)^3 arrays indexed
    [i, j, k] (NumTns order i fastest is handled here)."""
    NC = N + 1
    if A.shape != (NC + 1,) * 3 or V.shape != (NC + 1,) * 3:
        raise HIFError(HIF_ERR_ARG, "A and V must be (N+2)^3")
    a = np.ascontiguousarray(A.astype(np.float64).ravel(order="F"))
    v = np.ascontiguousarray(V.astype(np.float64).ravel(order="F"))
    _check(lib().hif_setup_stencil(factor._h, N, h, _dptr(a), _dptr(v)))


def SetupStencilFaces(factor: HIFFactor, N: int, h: float, ax, ay, az, V) -> None:
    """Symmetric flux-form operator; face arrays (N+2)^3 indexed [i, j, k]."""
    arrs = [np.ascontiguousarray(np.asarray(x, np.float64).ravel(order="F")) for x in (ax, ay, az, V)]
    NC = N + 1
    for x in arrs:
        if x.size != (NC + 1) ** 3:
            raise HIFError(HIF_ERR_ARG, "face arrays must be (N+2)^3")
    _check(lib().hif_setup_stencil_faces(factor._h, N, h, *[_dptr(x) for x in arrs]))


def SetupStencilFacesDevice(factor: HIFFactor, N: int, h: float, dax: int, day: int, daz: int,
                            dV: int) -> None:
    """Face-coefficient operator from device pointers ((N+2)^3 float64 each, i fastest)."""
    _check(lib().hif_setup_stencil_faces_device(factor._h, N, h, _p(dax), _p(day), _p(daz),
                                                _p(dV)))


def set_stream(factor: HIFFactor, stream_ptr: int) -> None:
    _check(lib().hif_set_stream(factor._h, _p(stream_ptr)))


def SpMV(factor: HIFFactor, x: np.ndarray, y: np.ndarray) -> None:
    """``SpMV(sp_matrix, x, y)`` (src/Factor.cpp:1099-1113): y = A^T x."""
    y[...] = factor.spmv(x, transpose=True)


def RelativeErrorNorm2(x: np.ndarray, y: np.ndarray) -> float:
    """``RelativeErrorNorm2`` (src/Factor.cpp:1083-1097): ||x - y|| / ||x||."""
    return float(np.sqrt(np.sum(np.abs(x - y) ** 2) / np.sum(np.abs(x) ** 2)))


def Schur(matrix: np.ndarray, red, skel):
    """``Schur`` (include/Schur.hpp:72-100) on the GPU: returns (A22, A22inv, X, S)."""
    M = np.asfortranarray(matrix, dtype=np.float64)
    r = np.ascontiguousarray(red, np.int32)
    s = np.ascontiguousarray(skel, np.int32)
    nr, ns = r.size, s.size
    out = [np.zeros((max(nr, 1), max(nr, 1)), order="F"), np.zeros((max(nr, 1), max(nr, 1)), order="F"),
           np.zeros((max(nr, 1), max(ns, 1)), order="F"), np.zeros((max(ns, 1), max(ns, 1)), order="F")]
    _check(lib().hif_schur(_dptr(M), M.shape[0], M.shape[0], _iptr(r), nr, _iptr(s), ns,
                           *[_dptr(o) for o in out]))
    A22, inv, X, S = out
    return A22[:nr, :nr], inv[:nr, :nr], X[:nr, :ns], S[:ns, :ns]


def InterpDecomp(M: np.ndarray, eps: float):
    """``InterpDecomp`` (src/InterpDecomp.cpp:86-138) on the GPU.

    Returns (W, skeleton_cols, redundant_cols); M is not modified (the C entry point
    overwrites its argument as the reference does; this wrapper passes a copy)."""
    A = np.array(M, dtype=np.float64, order="F", copy=True)
    m, n = A.shape
    W = np.zeros(n * n // 4 + n + 1)
    sk = np.zeros(n, np.int32)
    rd = np.zeros(n, np.int32)
    k = ctypes.c_int()
    _check(lib().hif_interp_decomp(_dptr(A), m, n, m, float(eps), _dptr(W), _iptr(sk), _iptr(rd),
                                   ctypes.byref(k)))
    k = k.value
    return (W[:k * (n - k)].reshape(n - k, k).T.copy(), sk[:k].astype(np.int64),
            rd[:n - k].astype(np.int64))


def PivotedQR(A: np.ndarray):
    """``PivotedQRWrapper`` (src/InterpDecomp.cpp:198-211): returns (R-array, jpvt)."""
    X = np.array(A, dtype=np.float64, order="F", copy=True)
    jp = np.zeros(X.shape[1], np.int32)
    _check(lib().hif_pivoted_qr(_dptr(X), X.shape[0], X.shape[1], X.shape[0], _iptr(jp)))
    return X, jp.astype(np.int64)


def TriangularSolve(R: np.ndarray, B: np.ndarray) -> np.ndarray:
    """``TriangularSolveWrapper`` (src/InterpDecomp.cpp:213-231): returns R^{-1} B."""
    Rf = np.asfortranarray(R, dtype=np.float64)
    Bf = np.array(B, dtype=np.float64, order="F", copy=True)
    k, nb = Bf.shape
    _check(lib().hif_triangular_solve(_dptr(Rf), k, Rf.shape[0], _dptr(Bf), nb, k))
    return Bf


def partition_cell(N: int, P: int, level: int, cell, mask: np.ndarray):
    """Host partitioner (test hook): InteriorCellIndexData of one cell over a mask
    (uint8, NC^3, DOF order). Returns (global, red, skel)."""
    n3 = (N + 1) ** 3
    m = np.ascontiguousarray(mask, np.uint8)
    g = np.zeros(n3, np.int32)
    r = np.zeros(n3, np.int32)
    s = np.zeros(n3, np.int32)
    cnt = np.zeros(3, np.int32)
    _check(lib().hif_partition_cell(N, P, level, cell[0], cell[1], cell[2], 0,
                                    m.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                    _iptr(g), _iptr(r), _iptr(s), _iptr(cnt)))
    return g[:cnt[0]].astype(np.int64), r[:cnt[1]].astype(np.int64), s[:cnt[2]].astype(np.int64)


def partition_face(N: int, P: int, level: int, cell, face: int, mask: np.ndarray):
    """Host partitioner (test hook): SkelInteractionIndexData -> (rows, cols)."""
    n3 = (N + 1) ** 3
    m = np.ascontiguousarray(mask, np.uint8)
    rows = np.zeros(n3 + 1, np.int32)
    cols = np.zeros(n3 + 1, np.int32)
    _check(lib().hif_partition_face(N, P, level, cell[0], cell[1], cell[2], face, 0,
                                    m.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                    _iptr(rows), _iptr(cols)))
    return rows[1:1 + rows[0]].astype(np.int64), cols[1:1 + cols[0]].astype(np.int64)
