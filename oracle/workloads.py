"""ORACLE -- test infrastructure only: seeded synthetic workloads without the
product library.

Only tests/ and bench.py's reference arm may import this module. It restates,
in numpy, the generators the product uses for its benchmark inputs
(gpu-conjugate-gradient-solver_b200/csrc/setup.cc: SplitMix64, uniform_rhs,
grf_coefficients, loguniform_coefficients, poisson7, varcoef7, kuhn_laplacian,
elasticity_p1), so that the
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


# Kuhn tetrahedra of a unit cube ({0, e_a, e_a + e_b, e_a + e_b + e_c} for each
# ordering (a, b, c) of the axes) as corner bit masks, bit 0 = x, 1 = y, 2 = z
_KUHN_AXES = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
_KUHN_CORNERS = tuple((0, 1 << p[0], (1 << p[0]) | (1 << p[1]), 7) for p in _KUHN_AXES)
# the 15 vertex offsets of a Kuhn mesh (every nonzero component of one sign),
# in ascending linear order dz, dy, dx
_KUHN_OFFSETS = tuple((dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
                      if not ((dx < 0 or dy < 0 or dz < 0) and (dx > 0 or dy > 0 or dz > 0)))
_KUHN_SLOT = {o: s for s, o in enumerate(_KUHN_OFFSETS)}


def kuhn_laplacian(m: int, jitter: float, seed: int) -> Csr:
    """P1 Laplacian on m^3 cubes of six Kuhn tetrahedra each, interior vertices
    jittered by U[-jitter h, jitter h) per axis, Dirichlet boundary vertices
    dropped. Each tetrahedron's gradients come from the inverse of the matrix
    of edge vectors (columns p_i - p_0, cofactors over the determinant), its
    element entries vol (g_a . g_b) are added per (row, offset slot) in cell,
    tetrahedron, a, b order, and each row lists its used slots in slot order."""
    if m < 2:
        raise ValueError("kuhn_laplacian: need at least 2 cells per side")
    nv, ni = m + 1, m - 1
    h = 1.0 / m
    z, y, x = np.meshgrid(np.arange(nv), np.arange(nv), np.arange(nv), indexing="ij")
    x, y, z = x.reshape(-1), y.reshape(-1), z.reshape(-1)
    xyz = np.stack([x * h, y * h, z * h], axis=1)
    interior = (x > 0) & (x < m) & (y > 0) & (y < m) & (z > 0) & (z < m)
    lo, hi = -jitter * h, jitter * h
    u = lo + (hi - lo) * uniform01(seed, 3 * int(interior.sum()))
    xyz[interior] += u.reshape(-1, 3)

    def unknown(vx, vy, vz):
        ok = (vx > 0) & (vx < m) & (vy > 0) & (vy < m) & (vz > 0) & (vz < m)
        return np.where(ok, ((vz - 1) * ni + (vy - 1)) * ni + (vx - 1), -1)

    n = ni ** 3
    acc = np.zeros(n * 15)
    used = np.zeros(n * 15, bool)
    cz, cy, cx = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    cz, cy, cx = cz.reshape(-1), cy.reshape(-1), cx.reshape(-1)
    for z0 in range(0, m):  # one layer of cells at a time, in loop order
        sel = cz == z0
        bx, by, bz = cx[sel], cy[sel], cz[sel]
        idx, val = [], []
        # (cell, t) in loop order: cells outer, tetrahedra inner
        vx = np.empty((len(bx), 6, 4), np.int64)
        vy, vz = np.empty_like(vx), np.empty_like(vx)
        for t, corner in enumerate(_KUHN_CORNERS):
            for a, cm in enumerate(corner):
                vx[:, t, a] = bx + (cm & 1)
                vy[:, t, a] = by + ((cm >> 1) & 1)
                vz[:, t, a] = bz + ((cm >> 2) & 1)
        vx, vy, vz = vx.reshape(-1, 4), vy.reshape(-1, 4), vz.reshape(-1, 4)
        p = xyz[(vz * nv + vy) * nv + vx]  # (T, 4, 3)
        j = [[p[:, c + 1, r] - p[:, 0, r] for c in range(3)] for r in range(3)]
        det = (j[0][0] * (j[1][1] * j[2][2] - j[1][2] * j[2][1]) -
               j[0][1] * (j[1][0] * j[2][2] - j[1][2] * j[2][0]) +
               j[0][2] * (j[1][0] * j[2][1] - j[1][1] * j[2][0]))
        inv = [[(j[1][1] * j[2][2] - j[1][2] * j[2][1]) / det, (j[0][2] * j[2][1] - j[0][1] * j[2][2]) / det,
                (j[0][1] * j[1][2] - j[0][2] * j[1][1]) / det],
               [(j[1][2] * j[2][0] - j[1][0] * j[2][2]) / det, (j[0][0] * j[2][2] - j[0][2] * j[2][0]) / det,
                (j[0][2] * j[1][0] - j[0][0] * j[1][2]) / det],
               [(j[1][0] * j[2][1] - j[1][1] * j[2][0]) / det, (j[0][1] * j[2][0] - j[0][0] * j[2][1]) / det,
                (j[0][0] * j[1][1] - j[0][1] * j[1][0]) / det]]
        g = [None, inv[0], inv[1], inv[2]]
        g[0] = [-((g[1][d] + g[2][d]) + g[3][d]) for d in range(3)]
        vol = np.abs(det) / 6.0
        ua = unknown(vx, vy, vz)  # (T, 4)
        T = len(vol)
        rows = np.empty((T, 4, 4), np.int64)
        slots = np.empty((T, 4, 4), np.int64)
        kab = np.empty((T, 4, 4))
        ok = np.empty((T, 4, 4), bool)
        for a in range(4):
            for b in range(4):
                ok[:, a, b] = (ua[:, a] >= 0) & (ua[:, b] >= 0)
                rows[:, a, b] = ua[:, a]
                key = (vx[:, b] - vx[:, a]) + 3 * (vy[:, b] - vy[:, a]) + 9 * (vz[:, b] - vz[:, a])
                slots[:, a, b] = key
                kab[:, a, b] = vol * ((g[a][0] * g[b][0] + g[a][1] * g[b][1]) + g[a][2] * g[b][2])
        keymap = np.full(27, -1, np.int64)
        for (dx, dy, dz), s in _KUHN_SLOT.items():
            keymap[dx + 3 * dy + 9 * dz + 13] = s
        flat = ok.reshape(-1)
        where = rows.reshape(-1)[flat] * 15 + keymap[slots.reshape(-1)[flat] + 13]
        np.add.at(acc, where, kab.reshape(-1)[flat])
        used[where] = True
    used = used.reshape(n, 15)
    r, s = np.nonzero(used)  # row-major: rows in order, slots ascending
    iz, rem = np.divmod(r, ni * ni)
    iy, ix = np.divmod(rem, ni)
    off = np.array(_KUHN_OFFSETS, np.int64)
    cols = unknown(ix + 1 + off[s, 0], iy + 1 + off[s, 1], iz + 1 + off[s, 2])
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(used.sum(axis=1), out=rp[1:])
    return Csr(n, n, rp, cols, acc.reshape(n, 15)[r, s])


def k80(side: int = 80, jitter: float = 0.2, seed: int = 1):
    """The Kuhn-tetrahedra P1 Laplacian of the benchmark (80^3 cubes) and its RHS."""
    a = kuhn_laplacian(side, jitter, seed)
    return a, uniform_rhs(a.rows, seed)


def _p1_gradients(p):
    """Gradients (4 lists of 3 arrays) and volumes of the tetrahedra p[:, 4, 3]:
    the inverse of the edge-vector matrix by cofactors over the determinant,
    gradient 0 the negated sum of the other three."""
    j = [[p[:, c + 1, r] - p[:, 0, r] for c in range(3)] for r in range(3)]
    det = (j[0][0] * (j[1][1] * j[2][2] - j[1][2] * j[2][1]) -
           j[0][1] * (j[1][0] * j[2][2] - j[1][2] * j[2][0]) +
           j[0][2] * (j[1][0] * j[2][1] - j[1][1] * j[2][0]))
    inv = [[(j[1][1] * j[2][2] - j[1][2] * j[2][1]) / det, (j[0][2] * j[2][1] - j[0][1] * j[2][2]) / det,
            (j[0][1] * j[1][2] - j[0][2] * j[1][1]) / det],
           [(j[1][2] * j[2][0] - j[1][0] * j[2][2]) / det, (j[0][0] * j[2][2] - j[0][2] * j[2][0]) / det,
            (j[0][2] * j[1][0] - j[0][0] * j[1][2]) / det],
           [(j[1][0] * j[2][1] - j[1][1] * j[2][0]) / det, (j[0][1] * j[2][0] - j[0][0] * j[2][1]) / det,
            (j[0][0] * j[1][1] - j[0][1] * j[1][0]) / det]]
    g = [None, inv[0], inv[1], inv[2]]
    g[0] = [-((g[1][d] + g[2][d]) + g[3][d]) for d in range(3)]
    return g, np.abs(det) / 6.0


def elasticity_p1(v: int, nu: float, seed: int):
    """P1 linear elasticity on a v^3-vertex grid of Kuhn tetrahedra (no jitter),
    Young's modulus exp(N(0, 1)) per tetrahedron (one Box-Muller normal each, in
    cell and tetrahedron order), Poisson ratio nu, the x = 0 face clamped, a
    unit body force in -z (vol / 4 to each vertex's z row). Element block (a, b)
    adds vol (lam g_a g_b^T + mu g_b g_a^T + mu (g_a . g_b) I) per (node, slot);
    each node row lists its used slots in slot order, 3 columns each.
    Returns (Csr, rhs)."""
    if v < 2:
        raise ValueError("elasticity_p1: need at least 2 vertices per side")
    m = v - 1
    h = 1.0 / m

    def unknown(x, y, z):
        ok = (x > 0) & (x <= m) & (y >= 0) & (y <= m) & (z >= 0) & (z <= m)
        return np.where(ok, (z * v + y) * m + (x - 1), -1)

    nvu = m * v * v
    acc = np.zeros(nvu * 15 * 9)
    used = np.zeros(nvu * 15, bool)
    rhs = np.zeros(3 * nvu)
    young = np.array([math.exp(z) for z in normals(seed, m * m * m * 6).tolist()])
    keymap = np.full(27, -1, np.int64)
    for (dx, dy, dz), s in _KUHN_SLOT.items():
        keymap[dx + 3 * dy + 9 * dz + 13] = s
    cz, cy, cx = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    cz, cy, cx = cz.reshape(-1), cy.reshape(-1), cx.reshape(-1)
    for z0 in range(m):
        sel = cz == z0
        bx, by, bz = cx[sel], cy[sel], cz[sel]
        vx = np.empty((len(bx), 6, 4), np.int64)
        vy, vz = np.empty_like(vx), np.empty_like(vx)
        for t, corner in enumerate(_KUHN_CORNERS):
            for a, cm in enumerate(corner):
                vx[:, t, a] = bx + (cm & 1)
                vy[:, t, a] = by + ((cm >> 1) & 1)
                vz[:, t, a] = bz + ((cm >> 2) & 1)
        vx, vy, vz = vx.reshape(-1, 4), vy.reshape(-1, 4), vz.reshape(-1, 4)
        E = young[z0 * m * m * 6:(z0 + 1) * m * m * 6]
        lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        mu = E / (2.0 * (1.0 + nu))
        p = np.stack([vx * h, vy * h, vz * h], axis=2).astype(np.float64)
        g, vol = _p1_gradients(p)
        ua = unknown(vx, vy, vz)
        T = len(vol)
        # the body force, in (tetrahedron, a) order
        okr = ua >= 0
        np.add.at(rhs, (3 * ua + 2)[okr], np.broadcast_to((-vol / 4.0)[:, None], (T, 4))[okr])
        idx = np.empty((T, 4, 4, 3, 3), np.int64)
        val = np.empty((T, 4, 4, 3, 3))
        ok = np.empty((T, 4, 4), bool)
        for a in range(4):
            for b in range(4):
                ok[:, a, b] = (ua[:, a] >= 0) & (ua[:, b] >= 0)
                key = (vx[:, b] - vx[:, a]) + 3 * (vy[:, b] - vy[:, a]) + 9 * (vz[:, b] - vz[:, a])
                slot = keymap[key + 13]
                gg = (g[a][0] * g[b][0] + g[a][1] * g[b][1]) + g[a][2] * g[b][2]
                base = (ua[:, a] * 15 + slot) * 9
                for i in range(3):
                    for jj in range(3):
                        idx[:, a, b, i, jj] = base + 3 * i + jj
                        val[:, a, b, i, jj] = vol * ((lam * g[a][i] * g[b][jj] + mu * g[b][i] * g[a][jj]) +
                                                     (mu * gg if i == jj else 0.0))
                used_rows = ok[:, a, b]
                used[(ua[:, a] * 15 + slot)[used_rows]] = True
        flat = np.broadcast_to(ok[:, :, :, None, None], (T, 4, 4, 3, 3)).reshape(-1)
        np.add.at(acc, idx.reshape(-1)[flat], val.reshape(-1)[flat])
    used = used.reshape(nvu, 15)
    acc = acc.reshape(nvu, 15, 9)
    node, s = np.nonzero(used)  # nodes in (z, y, x) order, slots ascending
    z, rem = np.divmod(node, v * m)
    y, xm = np.divmod(rem, m)
    x = xm + 1
    off = np.array(_KUHN_OFFSETS, np.int64)
    jv = unknown(x + off[s, 0], y + off[s, 1], z + off[s, 2])
    counts = used.sum(axis=1)
    # rows 3 iv + i: for each node, component i lists (slot, j) in order
    nslot = counts.repeat(3)
    rp = np.zeros(3 * nvu + 1, np.int64)
    np.cumsum(3 * nslot, out=rp[1:])
    start = np.zeros(nvu + 1, np.int64)
    np.cumsum(counts, out=start[1:])
    cols = np.empty(rp[-1], np.int64)
    vals = np.empty(rp[-1])
    for iv_comp in range(3):
        # entries of component iv_comp of every node: its used slots, 3 columns each
        k = np.arange(len(node))
        row = 3 * node + iv_comp
        pos = rp[row] + 3 * (k - start[node])
        for jj in range(3):
            cols[pos + jj] = 3 * jv + jj
            vals[pos + jj] = acc[node, s, 3 * iv_comp + jj]
    return Csr(3 * nvu, 3 * nvu, rp, cols, vals), rhs


def e64(v: int = 64, nu: float = 0.3, seed: int = 2):
    """The P1 elasticity system of the benchmark (64^3 vertices) and its RHS."""
    return elasticity_p1(v, nu, seed)
