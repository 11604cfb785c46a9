"""Seeded synthetic inputs (host side, numpy).

One generator for every workload so that the CUDA path, the CPU oracle and the
reference probe see bit-identical inputs on any machine: splitmix64 ->
uniform doubles in [0, 1) -> Box-Muller normals. ``numpy.random`` and
``std::normal_distribution`` are avoided because their streams are
implementation-defined.

Operators described here follow the workloads of the hot path:

* unit Poisson (a = 1, V = 0): tests/HIFDE3D/main.cpp:59-74 of the reference;
* node-coefficient fields for the reference's ``SetupStencil``;
* face coefficients a = exp(g) with g a Gaussian random field (Gaussian
  covariance, correlation length ell, standard deviation sigma) synthesised by
  FFT on a (2n)^3 periodic grid and sampled at face midpoints;
* piecewise-constant high-contrast a on 8^3 sub-cubes with values 10^U(-3, 3).
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n outputs of splitmix64 started at ``seed`` (uint64 array)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int) -> np.ndarray:
    """Uniform doubles in [0, 1) from the top 53 bits of splitmix64."""
    return (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, n: int) -> np.ndarray:
    """Standard normals by Box-Muller on consecutive uniform pairs."""
    m = (n + 1) // 2
    u = uniform(seed, 2 * m)
    u1, u2 = 1.0 - u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.empty(2 * m)
    z[0::2] = r * np.cos(2 * np.pi * u2)
    z[1::2] = r * np.sin(2 * np.pi * u2)
    return z[:n]


def dof_vector(N: int, seed: int, nrhs: int = 1) -> np.ndarray:
    """RHS with N(0,1) entries on the DOFs and zeros on the index-0 planes.

    Layout: NC^3 x nrhs, column-major, DOF id i + NC*j + NC^2*k.
    """
    NC = N + 1
    out = np.zeros((nrhs, NC, NC, NC))
    for r in range(nrhs):
        z = normal(seed + 7919 * r, NC ** 3).reshape(NC, NC, NC)  # [k, j, i]
        z[0, :, :] = 0
        z[:, 0, :] = 0
        z[:, :, 0] = 0
        out[r] = z
    return out.reshape(nrhs, NC ** 3).T.copy() if nrhs > 1 else out.reshape(NC ** 3).copy()


def node_lognormal(N: int, seed: int, sigma: float = 0.5, vscale: float = 0.0):
    """(A, V) node tensors of shape (NC+1)^3, indexed [i, j, k]:
    A = exp(sigma * z) with z i.i.d. N(0,1); V = vscale * U[0,1)."""
    NC = N + 1
    n = (NC + 1) ** 3
    A = np.exp(sigma * normal(seed, n)).reshape(NC + 1, NC + 1, NC + 1)
    V = vscale * uniform(seed ^ 0x5DEECE66D, n).reshape(NC + 1, NC + 1, NC + 1)
    return A, V


def gaussian_random_field(n: int, seed: int, ell: float, sigma: float) -> np.ndarray:
    """Periodic GRF on an m^3 grid (m = 2n, spacing 1/n) over the box [0, 2)^3 with
    Gaussian covariance exp(-r^2 / (2 ell^2)), standard deviation sigma; ell is in
    the box's units. Spectral synthesis: white noise filtered by sqrt of the
    covariance's FFT."""
    m = 2 * n
    h = 1.0 / n
    x = np.fft.fftfreq(m, d=1.0 / m) * h  # signed periodic distance
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    cov = np.exp(-(X * X + Y * Y + Z * Z) / (2.0 * ell * ell))
    spec = np.sqrt(np.maximum(np.fft.fftn(cov).real, 0.0))
    noise = normal(seed, m ** 3).reshape(m, m, m)
    g = np.fft.ifftn(np.fft.fftn(noise) * spec).real
    g *= sigma / max(g.std(), 1e-300)
    return g


def face_coefficients_grf(N: int, seed: int, ell: float = 1.0 / 16, sigma: float = 1.0):
    """Face coefficients (ax, ay, az) of a = exp(g), g a GRF sampled at face
    midpoints of the (N+1)-cell grid. Each array has shape (NC+1)^3 and
    ax[i, j, k] couples nodes (i, j, k) and (i+1, j, k).

    The unit cube is mapped onto the generator's whole box [0, 2)^3 (node i at
    grid point 2i, spacing 1/NC per grid step), so distances on the cube are half
    the box's: the field's correlation length on the unit cube is ell / 2."""
    NC = N + 1
    g = gaussian_random_field(NC, seed, ell, sigma)
    # node (i, j, k) sits at g[2i, 2j, 2k]; the x-face midpoint at g[2i+1, 2j, 2k].
    m = g.shape[0]
    idx = np.arange(NC + 1)
    ev = (2 * idx) % m
    od = (2 * idx + 1) % m
    ax = np.exp(g[np.ix_(od, ev, ev)])
    ay = np.exp(g[np.ix_(ev, od, ev)])
    az = np.exp(g[np.ix_(ev, ev, od)])
    return ax, ay, az


def face_coefficients_blocks(N: int, seed: int, nblk: int = 8, lo: float = -3.0, hi: float = 3.0):
    """Piecewise-constant a on nblk^3 sub-cubes with values 10^U(lo, hi); a face
    takes the harmonic mean of its two nodes' sub-cube values."""
    NC = N + 1
    vals = 10.0 ** (lo + (hi - lo) * uniform(seed, nblk ** 3)).reshape(nblk, nblk, nblk)
    idx = np.minimum((np.arange(NC + 2) * nblk) // (NC + 1), nblk - 1)
    node = vals[np.ix_(idx, idx, idx)]

    def hm(a, b):
        return 2.0 * a * b / (a + b)

    ax = hm(node[:-1, :-1, :-1], node[1:, :-1, :-1])
    ay = hm(node[:-1, :-1, :-1], node[:-1, 1:, :-1])
    az = hm(node[:-1, :-1, :-1], node[:-1, :-1, 1:])
    return ax, ay, az


def face_coefficients_lognormal(N: int, seed: int, sigma: float = 1.0):
    """Face coefficients a = exp(sigma z), z i.i.d. N(0,1) per face: a lognormal
    field with no spatial correlation. Arrays of shape (NC+1)^3 as
    face_coefficients_grf."""
    T = N + 2
    z = normal(seed, 3 * T ** 3).reshape(3, T, T, T)
    ax, ay, az = (np.exp(sigma * z[q]) for q in range(3))
    return ax, ay, az
