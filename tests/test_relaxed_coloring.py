"""The colouring of the strong couplings (gs_relaxed_coloring, the coarse levels
under coloring 2) on the CPU: no strong coupling joins two rows of one colour,
every row keeps its same-colour off-diagonal mass below rho |a_ii| (so D - W
stays strictly diagonally dominant and the forward / backward sweeps a
convergent symmetric pair), the colour lists partition the rows, the result
is deterministic; and the oracle's relaxed Gauss-Seidel over it converges."""
import numpy as np
import pytest


def levels(H):
    return ([H.A(k) for k in range(H.levels)], [H.P(k) for k in range(H.levels - 1)],
            [H.R(k) for k in range(H.levels - 1)])


def check(m, theta, rho, out):
    nc, col, verts, offs = out
    n = m.rows
    rp, ci, v = m.row_ptr, m.col_idx, m.val
    rows = np.repeat(np.arange(n), np.diff(rp))
    diag = np.zeros(n)
    own = rows == ci
    np.add.at(diag, rows[own], np.abs(v[own]))
    strong = ~own & (np.abs(v) >= theta * np.sqrt(diag[rows] * diag[ci]))
    assert not np.any(strong & (col[rows] == col[ci])), "a strong coupling inside a colour"
    same = ~own & (col[rows] == col[ci])
    mass = np.zeros(n)
    np.add.at(mass, rows[same], np.abs(v[same]))
    assert np.all(mass < rho * diag), "same-colour mass reaches rho |a_ii|"
    assert offs[0] == 0 and offs[-1] == n and np.all(np.diff(offs) > 0)
    assert sorted(verts.tolist()) == list(range(n))
    for c in range(nc):
        block = verts[offs[c]:offs[c + 1]]
        assert np.all(col[block] == c) and np.all(np.diff(block) > 0)


@pytest.fixture(scope="module")
def grf(gs):
    a = gs.varcoef_grf(24, 8.0, 2.3, 4)
    return a, gs.Hierarchy.build(a, 1, 0.1, 10, 100)


@pytest.mark.parametrize("theta,rho", [(0.05, 0.5), (0.02, 0.5), (0.1, 0.3), (0.0, 0.5)])
def test_relaxed_colouring_invariants(gs, grf, theta, rho):
    a, H = grf
    for k in range(1, H.levels):
        m = H.A(k)
        out = gs.relaxed_coloring(m, theta, rho)
        check(m, theta, rho, out)
        again = gs.relaxed_coloring(m, theta, rho)
        assert out[0] == again[0] and np.array_equal(out[1], again[1])


def test_relaxed_colouring_needs_fewer_colours(gs, grf):
    """theta 0 keeps every coupling strong: a proper colouring of the whole
    graph; theta 0.05 colours a Galerkin level with far fewer colours."""
    a, H = grf
    m = H.A(1)
    exact = gs.greedy_coloring(m)[0]
    full = gs.relaxed_coloring(m, 0.0, 0.5)
    assert full[0] <= exact
    assert gs.relaxed_coloring(m, 0.05, 0.5)[0] < exact


def test_relaxed_colouring_rejects_bad_arguments(gs, grf):
    a, H = grf
    m = H.A(1)
    for theta, rho in ((-1.0, 0.5), (float("nan"), 0.5), (0.05, 0.0), (0.05, 1.0), (0.05, float("inf"))):
        with pytest.raises(gs.SolverError):
            gs.relaxed_coloring(m, theta, rho)


@pytest.mark.parametrize("half", [0, 1])
def test_oracle_relaxed_gauss_seidel_converges(gs, orc, grf, half):
    """The oracle's V-cycle with the relaxed colourings on the coarse levels
    (Jacobi within a colour) still converges, within a few iterations of the
    exact colouring, and its true residual meets the tolerance."""
    a, H = grf
    A, P, R = levels(H)
    b = gs.uniform_rhs(a.rows, 4)
    x0, it0, st0, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, half_sweeps=half)
    cols = [None] + [gs.relaxed_coloring(A[k], 0.05, 0.5) for k in range(1, len(A))]
    x1, it1, st1, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, half_sweeps=half,
                                  colourings=[None] + [(c[2], c[3]) for c in cols[1:]], relaxed=1)
    assert st0 == 1 and st1 == 1
    assert it1 <= it0 + 3
    rp, ci, v = a.row_ptr, a.col_idx, a.val
    r = b - np.array([np.dot(v[rp[i]:rp[i + 1]], x1[ci[rp[i]:rp[i + 1]]]) for i in range(a.rows)])
    assert np.linalg.norm(r) <= 1.5e-8 * np.linalg.norm(b)


@pytest.fixture(scope="module")
def e8(gs):
    e = gs.elasticity(8, 0.3, 2)
    return e, gs.Hierarchy.build(e, 3, 0.1, 10, 100)


def block_norms(m):
    """Frobenius norms of the 3x3 blocks (dict (I, J) -> norm) and the node
    budgets 1 / ||A_II^-1||_F."""
    rp, ci, v = m.row_ptr, m.col_idx, m.val
    nn = m.rows // 3
    sq, diag = {}, np.zeros((nn, 3, 3))
    for r in range(m.rows):
        for e in range(rp[r], rp[r + 1]):
            I, J = r // 3, ci[e] // 3
            if I == J:
                diag[I, r % 3, ci[e] % 3] += v[e]
            else:
                sq[(I, J)] = sq.get((I, J), 0.0) + v[e] * v[e]
    norms = {k: np.sqrt(x) for k, x in sq.items()}
    sd = np.sqrt((diag ** 2).sum(axis=(1, 2)))
    mu = 1.0 / np.sqrt((np.linalg.inv(diag) ** 2).sum(axis=(1, 2)))
    return norms, sd, mu


@pytest.mark.parametrize("theta,rho", [(0.05, 0.5), (0.1, 0.3)])
def test_relaxed_block_colouring_invariants(gs, e8, theta, rho):
    e, H = e8
    for k in range(1, H.levels):
        m = H.A(k)
        nc, col, verts, offs = gs.relaxed_coloring(m, theta, rho, block=3)
        norms, sd, mu = block_norms(m)
        mass = np.zeros(m.rows // 3)
        for (I, J), w in norms.items():
            if col[I] == col[J]:
                assert w < theta * np.sqrt(sd[I] * sd[J]), "a strong block coupling inside a colour"
                mass[I] += w
        assert np.all(mass < rho * mu)
        assert offs[-1] == m.rows // 3 and sorted(verts.tolist()) == list(range(m.rows // 3))


def test_oracle_relaxed_block_gauss_seidel_converges(gs, orc, e8):
    e, H = e8
    A, P, R = levels(H)
    x0, it0, st0, _ = orc.amg_pcg(A, P, R, e.rhs, smoother=1, tol=1e-8)
    cols = [None] + [gs.relaxed_coloring(A[k], 0.05, 0.5, block=3) for k in range(1, len(A))]
    x1, it1, st1, _ = orc.amg_pcg(A, P, R, e.rhs, smoother=1, tol=1e-8,
                                  colourings=[None] + [(c[2], c[3]) for c in cols[1:]], relaxed=1)
    assert st0 == 1 and st1 == 1 and it1 <= it0 + 3
