"""Smoothed-aggregation setup on the GPU (gs_hierarchy_build_ex with a device),
against the host build of the same algorithm -- bit for bit: every level,
transfer operator and aggregate -- and against the numpy restatement of the
independent-set aggregation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bitwise_same(hd, hh, block):
    assert hd.levels == hh.levels
    for k in range(hh.levels):
        for which in ((0,) if k == hh.levels - 1 else (0, 1, 2)):
            x, y = hd.matrix(k, which), hh.matrix(k, which)
            assert (x.rows, x.cols) == (y.rows, y.cols)
            assert np.array_equal(x.row_ptr, y.row_ptr)
            assert np.array_equal(x.col_idx, y.col_idx)
            assert np.array_equal(x.val.view(np.uint64), y.val.view(np.uint64))
        if k < hh.levels - 1:
            assert np.array_equal(hd.aggregates(k, block), hh.aggregates(k, block))


CASES = {
    "poisson32": (lambda gs: gs.poisson7(32), 1, 100),
    "varcoef": (lambda gs: gs.varcoef_loguniform(24, 20, 16, seed=2), 1, 100),
    "kuhn16": (lambda gs: gs.kuhn_laplacian(16, seed=4), 1, 100),
    "grf48": (lambda gs: gs.varcoef_grf(48, 8.0, 2.3, 4), 1, 1000),
    "elasticity12": (lambda gs: gs.elasticity(12), 3, 150),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_device_setup_matches_host_build(gs, device, case):
    make, block, min_dofs = CASES[case]
    a = make(gs)
    hd = gs.Hierarchy.build_ex(a, block, 0.1, 10, min_dofs, aggregation=1, device=device)
    hh = gs.Hierarchy.build_ex(a, block, 0.1, 10, min_dofs, aggregation=1, device=-1)
    assert hd.levels >= 2
    assert hd.setup_stats["mis_rounds"] >= hd.levels - 1
    _bitwise_same(hd, hh, block)


def test_device_setup_matches_restatement(gs, orc, device):
    for a, block, min_dofs in ((gs.poisson7(12), 1, 100), (gs.elasticity(5), 3, 60)):
        hd = gs.Hierarchy.build_ex(a, block, 0.1, 10, min_dofs, aggregation=1, device=device)
        A, P, R, aggs = orc.build_hierarchy(orc.CsrView.of(a), block, 0.1, 10, min_dofs, aggregation=1)
        assert hd.levels == len(A)
        for k in range(len(A) - 1):
            assert np.array_equal(hd.aggregates(k, block), aggs[k])
            for mine, theirs in ((hd.P(k), P[k]), (hd.R(k), R[k]), (hd.A(k + 1), A[k + 1])):
                ms, ts = mine.to_scipy(), theirs.tocsr()
                ms.eliminate_zeros()
                ts.eliminate_zeros()
                assert np.array_equal(ms.indptr, ts.indptr) and np.array_equal(ms.indices, ts.indices)
                assert np.abs(ms.data - ts.data).max() <= 1e-13 * np.abs(ts.data).max()


def test_device_setup_full_size_solve(gs, device):
    """P128 (2.1 M rows): the device build equals the host build of the same
    algorithm and its hierarchy solves to 1e-8 (FP64-verified residual)."""
    a = gs.varcoef_grf(128, 8.0, 2.3, 4)
    b = gs.uniform_rhs(a.rows, 4)
    hd = gs.Hierarchy.build_ex(a, 1, 0.1, 10, 1000, aggregation=1, device=device)
    hh = gs.Hierarchy.build_ex(a, 1, 0.1, 10, 1000, aggregation=1, device=-1)
    _bitwise_same(hd, hh, 1)
    s = gs.Solver(hd, gs.SolverOptions(tol=1e-8, precision=1, flexible=1, use_graph=1,
                                       coarse_rows=24576), device=device)
    # the dense FP32 inverse sits on the second coarse level (19670 rows)
    assert [lv["rows"] for lv in s.level_info()] == [hd.A(k).rows for k in range(3)]
    x, st = s.solve(b)
    assert st.status == 1
    r = np.linalg.norm(b - a.to_scipy() @ x) / np.linalg.norm(b)
    assert r <= 1.5e-8


def test_device_setup_rejects_bad_input(gs, device):
    a = gs.poisson7(6)
    rp, ci, v = a.row_ptr.copy(), a.col_idx.copy(), a.val.copy()
    ci[rp[3]], ci[rp[3] + 1] = ci[rp[3] + 1], ci[rp[3]]  # row 3 out of order
    v[rp[3]], v[rp[3] + 1] = v[rp[3] + 1], v[rp[3]]
    bad = gs.Csr(a.rows, a.cols, rp, ci, v)
    with pytest.raises(gs.SolverError, match="sorted"):
        gs.Hierarchy.build_ex(bad, 1, 0.1, 10, 10, aggregation=1, device=device)
    with pytest.raises(gs.SolverError, match="aggregation 1"):
        gs.Hierarchy.build_ex(a, 1, 0.1, 10, 10, aggregation=0, device=device)
    # the host build accepts the unsorted matrix
    gs.Hierarchy.build_ex(bad, 1, 0.1, 10, 10, aggregation=1, device=-1)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["poisson32", "grf24", "kuhn12", "elasticity8", "p128"])
def test_value_refresh_on_device_equals_host(gs, device, case):
    """The Galerkin refresh of a hierarchy for new finest values (the solver's
    update_matrix, and Hierarchy.refresh): the products on the GPU equal the
    host's bit for bit on every level."""
    if case == "poisson32":
        a, block = gs.poisson7(32), 1
    elif case == "grf24":
        a, block = gs.varcoef_grf(24, 8.0, 2.3, 4), 1
    elif case == "kuhn12":
        a, block = gs.kuhn_laplacian(12, 0.2, 1), 1
    elif case == "elasticity8":
        a, block = gs.elasticity(8, 0.3, 2), 3
    else:
        a, block = gs.varcoef_grf(128, 8.0, 2.3, 4), 1
    H = gs.Hierarchy.build_ex(a, block, 0.1, 10, 200 if case != "p128" else 1000, aggregation=1, device=device)
    rows = np.repeat(np.arange(a.rows), np.diff(a.row_ptr))
    d = 1.0 + 0.25 * np.cos(np.arange(a.rows))
    values = a.val * d[rows] * d[a.col_idx]  # D A D: same sparsity, still SPD
    hd = H.refresh(values, device)
    hh = H.refresh(values, -1)
    assert hd.levels == hh.levels == H.levels >= 2
    for k in range(H.levels):
        x, y = hd.A(k), hh.A(k)
        assert np.array_equal(x.row_ptr, y.row_ptr) and np.array_equal(x.col_idx, y.col_idx)
        assert np.array_equal(x.val, y.val), k
