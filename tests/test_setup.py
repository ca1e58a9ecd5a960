"""Host setup of the product against the reference (bit-exact integer work)
and against the numpy restatement of smoothed aggregation."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.csgraph  # noqa: F401

from conftest import golden


@pytest.mark.parametrize("name", ["poisson16", "kuhn12"])
def test_setup_matches_reference_golden(gs, name):
    g = golden(f"setup_{name}.npz")
    n = len(g["row_ptr"]) - 1
    m = gs.Csr(n, n, g["row_ptr"], g["col_idx"], g["val"].astype(np.float64))
    nc, colors, verts, offs = gs.greedy_coloring(m)
    assert nc == int(g["ncolors"])
    assert np.array_equal(colors, g["colors"]) and np.array_equal(verts, g["verts"])
    assert np.array_equal(offs, g["offs"])
    o2n, n2o = gs.rcm(m)
    assert np.array_equal(o2n, g["o2n"]) and np.array_equal(n2o, g["n2o"])
    ap = gs.apply_permutation(m, o2n, n2o)
    assert np.array_equal(ap.row_ptr, g["ap_row_ptr"]) and np.array_equal(ap.col_idx, g["ap_col"])
    assert np.array_equal(ap.val.astype(np.float32), g["ap_val"])
    pm = gs.permute_matrix(m, o2n, o2n)
    assert np.array_equal(pm.row_ptr, g["pm_row_ptr"]) and np.array_equal(pm.col_idx, g["pm_col"])
    assert np.array_equal(pm.val.astype(np.float32), g["pm_val"])
    ec, ev, orp, oc, ov = gs.ell_build(m, 7)
    assert np.array_equal(ec, g["ell_col"]) and np.array_equal(ev.astype(np.float32), g["ell_val"])
    assert np.array_equal(orp, g["ovf_row_ptr"]) and np.array_equal(oc, g["ovf_col"])
    assert np.array_equal(ov.astype(np.float32), g["ovf_val"])


def test_setup_matches_reference_live(gs, ref):
    for m in (gs.poisson7(7, 5, 6), gs.varcoef_loguniform(9, 4, 3), gs.kuhn_laplacian(7, seed=9),
              gs.elasticity(4)):
        assert gs.greedy_coloring(m)[2].tolist() == ref.ref_coloring(m)[2].tolist()
        o2n, n2o = gs.rcm(m)
        r_o2n, r_n2o = ref.ref_rcm(m)
        assert np.array_equal(o2n, r_o2n) and np.array_equal(n2o, r_n2o)
    e = gs.elasticity(4)
    grp, gci = gs.block_graph(e)
    rrp, rci = ref.ref_block_graph(e)
    assert np.array_equal(grp, rrp) and np.array_equal(gci, rci)
    d = gs.block_inverses3x3(e)
    dr = ref.ref_block_inverses(e)
    assert np.allclose(d, dr, rtol=1e-5, atol=1e-6 * np.abs(d).max())


def test_block_permutation_expansion(gs):
    e = gs.elasticity(4)
    grp, gci = gs.block_graph(e)
    g = gs.Csr(len(grp) - 1, len(grp) - 1, grp, gci, np.ones(len(gci)))
    no2n, nn2o = gs.rcm(g)
    o2n, n2o = gs.expand_block_permutation(no2n, nn2o)
    assert np.array_equal(o2n[n2o], np.arange(e.rows))
    assert np.array_equal(o2n[3 * 5 + 2], 3 * no2n[5] + 2)


def _compare_hierarchy(gs, orc, a, block, min_dofs, aggregation=0):
    if aggregation == 0:
        H = gs.Hierarchy.build(a, block, 0.1, 10, min_dofs)
    else:
        H = gs.Hierarchy.build_ex(a, block, 0.1, 10, min_dofs, aggregation=aggregation, device=-1)
    A, P, R, aggs = orc.build_hierarchy(orc.CsrView.of(a), block, 0.1, 10, min_dofs, aggregation)
    assert H.levels == len(A)
    for k in range(H.levels - 1):
        assert np.array_equal(H.aggregates(k, block), aggs[k])
        for mine, theirs in ((H.P(k), P[k]), (H.R(k), R[k]), (H.A(k + 1), A[k + 1])):
            ms = mine.to_scipy()
            ms.eliminate_zeros()
            ts = theirs.tocsr()
            ts.eliminate_zeros()
            assert ms.shape == ts.shape
            assert np.array_equal(ms.indptr, ts.indptr) and np.array_equal(ms.indices, ts.indices)
            scale = np.abs(ts.data).max()
            assert np.abs(ms.data - ts.data).max() <= 1e-13 * scale
    return H


def test_smoothed_aggregation_matches_restatement_scalar(gs, orc):
    _compare_hierarchy(gs, orc, gs.poisson7(14, 12, 10), 1, 100)
    _compare_hierarchy(gs, orc, gs.varcoef_loguniform(11, 9, 8, seed=2), 1, 80)
    _compare_hierarchy(gs, orc, gs.kuhn_laplacian(10, seed=4), 1, 60)


def test_smoothed_aggregation_matches_restatement_block(gs, orc):
    _compare_hierarchy(gs, orc, gs.elasticity(6), 3, 90)


def test_independent_set_aggregation_matches_restatement(gs, orc):
    """The parallel (distance-2 independent set) aggregation, host build of
    the product against the numpy restatement: aggregates bit-exact, P, R and
    the Galerkin levels to 1e-13."""
    _compare_hierarchy(gs, orc, gs.poisson7(14, 12, 10), 1, 100, aggregation=1)
    _compare_hierarchy(gs, orc, gs.varcoef_loguniform(11, 9, 8, seed=2), 1, 80, aggregation=1)
    _compare_hierarchy(gs, orc, gs.kuhn_laplacian(10, seed=4), 1, 60, aggregation=1)
    _compare_hierarchy(gs, orc, gs.elasticity(6), 3, 90, aggregation=1)


def test_independent_set_aggregation_isolated_and_disconnected(gs, orc):
    """Rows with only a diagonal stay out of every aggregate (-1, empty P row)
    and a disconnected block aggregates on its own, host build of the product
    against the numpy restatement."""
    p = gs.poisson7(6).to_scipy()
    q = gs.poisson7(3).to_scipy()
    iso = sp.identity(7, format="csr") * 4.0
    m = sp.block_diag([p, iso, q]).tocsr()
    m.sort_indices()
    a = gs.Csr.from_scipy(m)
    H = gs.Hierarchy.build_ex(a, 1, 0.1, 2, 10, aggregation=1, device=-1)
    A, P, R, aggs = orc.build_hierarchy(orc.CsrView.of(a), 1, 0.1, 2, 10, aggregation=1)
    agg = H.aggregates(0)
    assert np.array_equal(agg, aggs[0])
    n0 = p.shape[0]
    assert np.all(agg[n0:n0 + 7] == -1)
    assert set(agg[:n0]).isdisjoint(set(agg[n0 + 7:]))
    Ph = H.P(0).to_scipy()
    assert np.all(np.diff(Ph.indptr)[n0:n0 + 7] == 0)
    assert abs(Ph - P[0]).max() <= 1e-13 * abs(P[0]).max()


def test_independent_set_aggregation_properties(gs, orc):
    """Every non-isolated node is aggregated and each aggregate is connected
    in the strength graph."""
    for a, block in ((gs.poisson7(10, 9, 8), 1), (gs.kuhn_laplacian(8, seed=3), 1), (gs.elasticity(5), 3)):
        H = gs.Hierarchy.build_ex(a, block, 0.1, 1, 10, aggregation=1, device=-1)
        agg = H.aggregates(0, block)
        # strength graph of the restatement (node couplings, eps 0.1)
        v = orc.CsrView.of(a)
        nn = v.rows // block
        m = sp.csr_matrix((v.val ** 2, v.col_idx // block, v.row_ptr), shape=(v.rows, nn))
        Rb = sp.csr_matrix((np.ones(v.rows), (np.arange(v.rows) // block, np.arange(v.rows))), shape=(nn, v.rows))
        W = (Rb @ m).tocsr()
        W.data = np.sqrt(W.data)
        d = W.diagonal()
        W = W.tocoo()
        off = W.row != W.col
        s = off & (W.data ** 2 >= 0.01 * d[W.row] * d[W.col])
        S = sp.csr_matrix((np.ones(int(s.sum())), (W.row[s], W.col[s])), shape=(nn, nn))
        isolated = np.asarray(S.sum(axis=1)).ravel() == 0
        assert np.all((agg >= 0) | isolated)
        nagg = agg.max() + 1
        sizes = np.bincount(agg[agg >= 0], minlength=nagg)
        assert sizes.min() >= 1
        for g in range(nagg):
            members = np.flatnonzero(agg == g)
            if len(members) == 1:
                continue
            ncomp, _ = sp.csgraph.connected_components(S[members][:, members], directed=False)
            assert ncomp == 1


def test_smallest_last_coloring(gs):
    """Proper colourings with the known counts on a path, an even cycle, a
    complete graph and a 2-D grid (2, 2, n, 2), vertices grouped by colour in
    increasing order, and never more colours than the greedy order on the
    AMG levels of a Kuhn mesh."""
    def graph(n, edges):
        rows = [i for i, j in edges] + [j for i, j in edges] + list(range(n))
        cols = [j for i, j in edges] + [i for i, j in edges] + list(range(n))
        m = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
        m.sum_duplicates()
        m.sort_indices()
        return gs.Csr.from_scipy(m)
    g10 = [(x + 10 * y, x + 1 + 10 * y) for y in range(10) for x in range(9)] + \
          [(x + 10 * y, x + 10 * (y + 1)) for y in range(9) for x in range(10)]
    for m, want in ((graph(9, [(i, i + 1) for i in range(8)]), 2),
                    (graph(8, [(i, (i + 1) % 8) for i in range(8)]), 2),
                    (graph(7, [(i, j) for i in range(7) for j in range(i + 1, 7)]), 7),
                    (graph(100, g10), 2)):
        nc, colors, verts, offs = gs.smallest_last_coloring(m)
        assert nc == want
        s = m.to_scipy().tocoo()
        assert np.all((colors[s.row] != colors[s.col]) | (s.row == s.col))
        for c in range(nc):
            block = verts[offs[c]:offs[c + 1]]
            assert np.all(colors[block] == c) and np.all(np.diff(block) > 0)
    H = gs.Hierarchy.build(gs.kuhn_laplacian(10, seed=4), 1, 0.1, 10, 60)
    for k in range(H.levels):
        assert gs.smallest_last_coloring(H.A(k))[0] <= gs.greedy_coloring(H.A(k))[0]


def vector_laplacian(nx, ny, nz):
    """examples/amgSolver/tests/MultigridUnitTests.cc:90-147: 3 dofs per
    vertex graph Laplacian plus a 0.1 diagonal shift."""
    idx = lambda x, y, z: (z * ny + y) * nx + x
    rows, cols, vals = [], [], []
    def edge(a, b):
        for c in range(3):
            i, j = 3 * a + c, 3 * b + c
            rows.extend([i, j, i, j]); cols.extend([i, j, j, i]); vals.extend([1.0, 1.0, -1.0, -1.0])
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                v = idx(x, y, z)
                if x + 1 < nx: edge(v, idx(x + 1, y, z))
                if y + 1 < ny: edge(v, idx(x, y + 1, z))
                if z + 1 < nz: edge(v, idx(x, y, z + 1))
    n = 3 * nx * ny * nz
    rows += list(range(n)); cols += list(range(n)); vals += [0.1] * n
    m = sp.csr_matrix((np.array(vals, np.float32).astype(np.float64), (rows, cols)), shape=(n, n))
    m.sum_duplicates()
    m.sort_indices()
    return m


def test_galerkin_operators_are_consistent(gs):
    """MultigridUnitTests.cc:239-266: ||A_{k+1} - R A_k P|| / ||A_{k+1}|| < 1e-4
    with SmoothedAggregationCoarsener(1, 0.1) and AMGHierarchyBuilder(10, 1000)."""
    a = gs.Csr.from_scipy(vector_laplacian(8, 8, 8))
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 1000)
    assert H.levels >= 2
    for k in range(H.levels - 1):
        Ak, Ac = H.A(k).to_scipy(), H.A(k + 1).to_scipy()
        proj = H.R(k).to_scipy() @ Ak @ H.P(k).to_scipy()
        assert sp.linalg.norm(Ac - proj) / sp.linalg.norm(Ac) < 1e-4
        assert abs(H.R(k).to_scipy() - H.P(k).to_scipy().T).max() == 0.0


def test_hierarchical_permutations_are_valid(gs):
    """MultigridUnitTests.cc:268-299, with RCM per level."""
    a = gs.Csr.from_scipy(vector_laplacian(8, 8, 8))
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 1000)
    for k in range(H.levels):
        o2n, n2o = gs.rcm(H.A(k))
        assert np.array_equal(np.sort(o2n), np.arange(H.A(k).rows))
        assert np.array_equal(o2n[n2o], np.arange(H.A(k).rows))


def test_problem_generators(gs):
    p = gs.poisson7(32)
    assert (p.rows, p.nnz) == (32768, 223232)
    s = p.to_scipy()
    assert abs(s - s.T).max() == 0 and np.allclose(s.diagonal(), 6.0)
    k = gs.kuhn_laplacian(20)
    assert k.rows == 19 ** 3
    ks = k.to_scipy()
    assert abs(ks - ks.T).max() < 1e-12 and np.all(ks.diagonal() > 0)
    e = gs.elasticity(8)
    assert e.rows == 3 * 7 * 8 * 8 and e.rhs is not None and e.rhs[2::3].sum() < 0
    es = e.to_scipy()
    assert abs(es - es.T).max() < 1e-12
    v = gs.varcoef_grf(16)
    vs = v.to_scipy()
    assert (v.rows, v.nnz) == (4096, 7 * 4096 - 6 * 16 * 16)
    rowsum = np.asarray(vs.sum(axis=1)).ravel()
    assert abs(vs - vs.T).max() == 0 and np.all(rowsum > -1e-10 * vs.diagonal())
    b = gs.uniform_rhs(1000, 0)
    assert b.min() >= -1 and b.max() < 1 and np.array_equal(b, gs.uniform_rhs(1000, 0))


@pytest.mark.parametrize("make", ["poisson", "kuhn", "varcoef"])
def test_hierarchical_reordering_matches_reference(gs, orc, ref, make):
    """HierarchicalReordering::compute: bit-identical orderings to the reference's own code
    (oracle/_ref) and to the numpy restatement, on every level."""
    if make == "poisson":
        a = gs.poisson7(14)
    elif make == "kuhn":
        a = gs.kuhn_laplacian(9)
    else:
        a = gs.varcoef_loguniform(12, 10, 9, 0.1, 10.0, seed=4)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 30)
    assert H.levels >= 3
    A = [H.A(k) for k in range(H.levels)]
    P = [H.P(k) for k in range(H.levels - 1)]
    R = [H.R(k) for k in range(H.levels - 1)]
    mine = gs.hierarchical_reordering(H)
    theirs = orc.ref_hierarchical_reordering(A, P, R)
    restated = orc.hierarchical_reordering(A, R)
    for (o1, n1), (o2, n2), (o3, n3) in zip(mine, theirs, restated):
        assert np.array_equal(o1, o2) and np.array_equal(n1, n2)
        assert np.array_equal(o1, o3) and np.array_equal(n1, n3)
        assert np.array_equal(np.sort(n1), np.arange(len(n1)))
