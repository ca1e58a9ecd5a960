"""Property-based checks of the host smoothed-aggregation setup
(gs_hierarchy_build_ex on the host, both aggregations) on small random
symmetric matrices, degenerate ones included (zero or negative diagonal
entries, isolated rows, empty rows, dense rows, 3x3 blocks): the build
returns an error or a hierarchy whose levels fit together -- square A_k,
P_k of shape (n_k, n_{k+1}) with every fine row in at most one aggregate,
R_k = P_k^T, A_{k+1} = R_k A_k P_k -- and it never crashes. On the
diagonally dominant ones the build equals the oracle's numpy restatement
(aggregates exactly, values within 1e-13 of their scale)."""
import numpy as np
import pytest
import scipy.sparse as sp
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

SETTINGS = settings(max_examples=150, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])


@st.composite
def matrices(draw, degenerate=True):
    block = draw(st.sampled_from([1, 1, 3]))
    rng = np.random.default_rng(draw(st.integers(0, 2 ** 31)))
    if draw(st.booleans()):
        # a 2-D grid graph (coarsens over several levels) with random positive
        # couplings, optionally with random long-range couplings added
        r, c = draw(st.integers(2, 14)), draw(st.integers(2, 14))
        nodes = r * c
        i = np.arange(nodes).reshape(r, c)
        pairs = np.concatenate([np.stack([i[:, :-1].ravel(), i[:, 1:].ravel()], 1),
                                np.stack([i[:-1, :].ravel(), i[1:, :].ravel()], 1)])
        if draw(st.booleans()):
            pairs = np.concatenate([pairs, rng.integers(0, nodes, size=(nodes // 4 + 1, 2))])
        w = rng.uniform(0.01, 1.0, len(pairs)) * draw(st.sampled_from([1.0, 1e-3, 1e3]))
        g = sp.coo_matrix((-w, (pairs[:, 0], pairs[:, 1])), shape=(nodes, nodes)).tocsr()
        g.setdiag(0)
        g.eliminate_zeros()
        off = sp.kron(g, sp.identity(block) if block > 1 else 1.0, format="csr")
        n = nodes * block
    else:
        nodes = draw(st.integers(1, 80 if block == 1 else 20))
        n = nodes * block
        density = draw(st.sampled_from([0.0, 0.05, 0.2, 0.6]))
        off = sp.random(n, n, density=density, random_state=rng, format="csr")
        off.data = -off.data * draw(st.sampled_from([1.0, 1e-3, 1e3]))
    off = off + off.T
    kinds = ["dominant", "zero_some", "negative_some", "tiny"] if degenerate else ["dominant"]
    diag_kind = draw(st.sampled_from(kinds))
    d = np.asarray(abs(off).sum(axis=1)).ravel() + 1.0
    if diag_kind == "zero_some":
        d[rng.random(n) < 0.3] = 0.0
    elif diag_kind == "negative_some":
        d[rng.random(n) < 0.3] *= -1.0
    elif diag_kind == "tiny":
        d *= 1e-12
    a = (off + sp.diags(d)).tocsr()
    a.sort_indices()
    eps = draw(st.sampled_from([0.0, 0.08, 0.1, 0.5]))
    return a, block, eps


@SETTINGS
@given(m=matrices(), aggregation=st.integers(0, 1), min_dofs=st.sampled_from([1, 2, 6]))
def test_host_setup_is_consistent_or_refuses(gs, m, aggregation, min_dofs):
    a, block, eps = m
    csr = gs.Csr.from_scipy(a)
    try:
        H = gs.Hierarchy.build_ex(csr, block, eps, 6, min_dofs, aggregation=aggregation, device=-1)
    except gs.SolverError:
        return
    assert H.levels >= 1
    assert H.A(0).rows == a.shape[0]
    for k in range(H.levels - 1):
        A, P, R, Ac = (H.A(k).to_scipy(), H.P(k).to_scipy(), H.R(k).to_scipy(), H.A(k + 1).to_scipy())
        n, nc = A.shape[0], Ac.shape[0]
        assert A.shape == (n, n) and Ac.shape == (nc, nc)
        assert P.shape == (n, nc) and R.shape == (nc, n)
        assert 0 < nc < n
        assert abs(R - P.T).max() == 0 if R.nnz else P.nnz == 0
        agg = H.aggregates(k, block)
        assert len(agg) == n // block and np.all((agg >= -1) & (agg < nc // block))
        galerkin = (R @ A @ P).toarray()
        assert np.allclose(Ac.toarray(), galerkin, rtol=1e-10, atol=1e-10 * max(1.0, abs(galerkin).max()))
        assert np.all(np.isfinite(Ac.data))


@SETTINGS
@given(m=matrices(degenerate=False), aggregation=st.integers(0, 1), min_dofs=st.sampled_from([1, 2, 6]))
def test_host_setup_matches_restatement(gs, orc, m, aggregation, min_dofs):
    a, block, eps = m
    csr = gs.Csr.from_scipy(a)
    H = gs.Hierarchy.build_ex(csr, block, eps, 6, min_dofs, aggregation=aggregation, device=-1)
    A, P, R, aggs = orc.build_hierarchy(orc.CsrView.of(csr), block, eps, 6, min_dofs, aggregation)
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
            if ts.nnz:
                assert np.abs(ms.data - ts.data).max() <= 1e-13 * np.abs(ts.data).max()
