"""ORACLE -- test infrastructure only: seeded synthetic workloads without the
product library.

Only tests/ and bench.py's reference arm may import this module. It restates,
in numpy, the generators the product uses for its benchmark inputs
(gpu-conjugate-gradient-solver_b200/csrc/setup.cc: SplitMix64, uniform_rhs,
grf_coefficients, loguniform_coefficients, poisson7, varcoef7), so that the
reference arm can build the same system without loading the product.
Elementary functions go through Python's math module (the C library's exp,
log and cos, as the product's host code calls them) and every sum keeps the
product's order, so the arrays are bit-identical to the product's
(tests/test_oracle_sa.py checks this).
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, start: int = 0) -> np.ndarray:
    """Outputs start .. start+count-1 of SplitMix64(seed) (Steele, Lea & Flood
    2014): state_i = seed + (i + 1) * golden, then the two xor-shift-multiply
    rounds and a final xor-shift."""
    i = np.arange(start + 1, start + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def uniform01(seed: int, count: int, start: int = 0) -> np.ndarray:
    return (splitmix64(seed, count, start) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform_rhs(n: int, seed: int) -> np.ndarray:
    """U[-1, 1): a + (b - a) * u with a = -1, b = 1."""
    return -1.0 + 2.0 * uniform01(seed, n)


def normals(seed: int, n: int) -> np.ndarray:
    """Box-Muller on consecutive pairs (u1, u2), cosine branch, u1 >= 1e-300."""
    u = uniform01(seed, 2 * n)
    u1 = np.maximum(u[0::2], 1e-300)
    u2 = u[1::2]
    log, cos = math.log, math.cos
    return np.array([math.sqrt(-2.0 * log(a)) * cos(6.283185307179586 * b) for a, b in zip(u1.tolist(), u2.tolist())])


def grf_coefficients(nx: int, ny: int, nz: int, corr: float, sigma: float, seed: int) -> np.ndarray:
    """exp(sigma * standardised Gaussian random field): white noise smoothed by
    a periodic separable Gaussian kernel of standard deviation corr / sqrt(2)
    cells (radius ceil(4 s)), x then y then z."""
    n = nx * ny * nz
    f = normals(seed, n).reshape(nz, ny, nx)
    s = corr / math.sqrt(2.0)
    rad = int(math.ceil(4.0 * s))
    w = [math.exp(-0.5 * d * d / (s * s)) for d in range(-rad, rad + 1)]
    for axis in (2, 1, 0):  # x, y, z in the C-order array
        acc = np.zeros_like(f)
        for d in range(-rad, rad + 1):
            acc += w[d + rad] * np.roll(f, -d, axis=axis)  # f[(c + d) mod len]
        f = acc
    f = f.reshape(-1)
    mean = float(np.cumsum(f)[-1]) / n
    var = float(np.cumsum((f - mean) * (f - mean))[-1])
    sd = math.sqrt(var / n)
    z = (sigma * (f - mean) / sd).tolist()
    return np.array([math.exp(v) for v in z])


def loguniform_coefficients(n: int, lo: float, hi: float, seed: int) -> np.ndarray:
    a, b = math.log(lo), math.log(hi)
    u = (a + (b - a) * uniform01(seed, n)).tolist()
    return np.array([math.exp(v) for v in u])


class Csr:
    def __init__(self, rows, cols, row_ptr, col_idx, val):
        self.rows, self.cols = int(rows), int(cols)
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        self.col_idx = np.ascontiguousarray(col_idx, np.int32)
        self.val = np.ascontiguousarray(val, np.float64)

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col_idx, self.row_ptr), shape=(self.rows, self.cols))


def _stencil7(nx: int, ny: int, nz: int, offdiag, diag) -> Csr:
    """CSR of a 7-point stencil: per row the inside neighbours in ascending
    column order with the diagonal in place; offdiag[f] and diag are arrays
    over the grid, faces f = (z-, y-, x-, x+, y+, z+)."""
    n = nx * ny * nz
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    z, y, x = z.reshape(-1), y.reshape(-1), x.reshape(-1)
    i = np.arange(n)
    inside = [z > 0, y > 0, x > 0, x + 1 < nx, y + 1 < ny, z + 1 < nz]
    step = [-nx * ny, -nx, -1, 1, nx, nx * ny]
    cols = np.empty((n, 7), np.int64)
    vals = np.empty((n, 7))
    used = np.zeros((n, 7), bool)
    for f in range(3):
        cols[:, f], vals[:, f], used[:, f] = i + step[f], offdiag[f], inside[f]
    cols[:, 3], vals[:, 3], used[:, 3] = i, diag, True
    for f in range(3, 6):
        cols[:, f + 1], vals[:, f + 1], used[:, f + 1] = i + step[f], offdiag[f], inside[f]
    counts = used.sum(axis=1)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=rp[1:])
    return Csr(n, n, rp, cols[used], vals[used])


def poisson7(nx: int, ny: int = None, nz: int = None) -> Csr:
    ny, nz = ny or nx, nz or nx
    n = nx * ny * nz
    return _stencil7(nx, ny, nz, [np.full(n, -1.0)] * 6, np.full(n, 6.0))


def varcoef7(nx: int, ny: int, nz: int, k: np.ndarray) -> Csr:
    """Cell coefficients k, face coefficient 2 p q / (p + q), a boundary face
    adds 2 k_i to the diagonal; the diagonal sums the faces in the order
    z-, y-, x-, x+, y+, z+."""
    n = nx * ny * nz
    k = np.asarray(k, np.float64)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    z, y, x = z.reshape(-1), y.reshape(-1), x.reshape(-1)
    i = np.arange(n)
    inside = [z > 0, y > 0, x > 0, x + 1 < nx, y + 1 < ny, z + 1 < nz]
    step = [-nx * ny, -nx, -1, 1, nx, nx * ny]
    diag = np.zeros(n)
    off = []
    for f in range(6):
        j = np.where(inside[f], i + step[f], i)
        q = k[j]
        t = 2.0 * (k * q) / (k + q)
        diag = diag + np.where(inside[f], t, 2.0 * k)
        off.append(-t)
    return _stencil7(nx, ny, nz, off, diag)


def p128(side: int = 128, seed: int = 4):
    """The 128^3 variable-coefficient Poisson of the benchmark and its RHS."""
    a = varcoef7(side, side, side, grf_coefficients(side, side, side, 8.0, 2.3, seed))
    return a, uniform_rhs(a.rows, seed)
