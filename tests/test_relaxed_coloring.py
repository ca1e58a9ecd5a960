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
