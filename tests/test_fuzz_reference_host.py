"""The host setup routines of the product against the reference's own code
(oracle/_ref, compiled from the reference's sources) on random symmetric
patterns -- several components, isolated rows, rows listed out of order,
many equal degrees (ties in RCM's degree sort) -- with FP32 values:
GraphColoring, RCMReordering, HostCSRMatrix::applyPermutation,
permuteMatrix, HostELLMatrix and buildBlockGraph bit for bit, and
extractInverseDiagonalBlocks3x3 to FP32 accuracy (the reference factors in
FP32, the product in FP64)."""
import numpy as np
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

SETTINGS = settings(max_examples=120, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])


@st.composite
def symmetric(draw, block=1):
    nodes = draw(st.integers(1, 40))
    rng = np.random.default_rng(draw(st.integers(0, 2 ** 31)))
    kind = draw(st.sampled_from(["random", "ring", "grid", "components"]))
    edges = set()
    if kind == "random":
        for _ in range(int(rng.integers(0, 3 * nodes + 1))):
            i, j = rng.integers(0, nodes, 2)
            edges.add((int(i), int(j)))
    elif kind == "ring":  # every degree equal: RCM's ties everywhere
        edges = {(i, (i + 1) % nodes) for i in range(nodes)}
    elif kind == "grid":
        w = max(1, int(np.sqrt(nodes)))
        edges = {(i, i + 1) for i in range(nodes - 1) if (i + 1) % w} | {(i, i + w) for i in range(nodes - w)}
    else:  # several components, some isolated nodes
        for _ in range(int(rng.integers(1, 5))):
            a, b = sorted(rng.integers(0, nodes, 2))
            edges |= {(i, i + 1) for i in range(int(a), int(b))}
    adj = [{v} for v in range(nodes)]
    for i, j in edges:
        adj[i].add(j)
        adj[j].add(i)
    n = nodes * block
    rows = [[] for _ in range(n)]
    for v in range(nodes):
        for u in adj[v]:
            for r in range(block):
                for c in range(block):
                    rows[block * v + r].append(block * u + c)
    rp, ci, val = [0], [], []
    for r in range(n):
        cols = rows[r] if rng.random() < 0.7 else list(rng.permutation(rows[r]))
        for c in cols:
            ci.append(int(c))
            d = abs(r - int(c))
            val.append(np.float32(4.0 * block + 1.0 if r == c else (0.5 if r // block == int(c) // block else -1.0 / (1 + d))))
        rp.append(len(ci))
    return n, np.array(rp, np.int32), np.array(ci, np.int32), np.array(val, np.float32).astype(np.float64)


def _csr(gs, g):
    n, rp, ci, v = g
    return gs.Csr(n, n, rp, ci, v)


@SETTINGS
@given(g=symmetric())
def test_coloring_and_rcm_equal_reference(gs, ref, g):
    m = _csr(gs, g)
    mine, theirs = gs.greedy_coloring(m), ref.ref_coloring(m)
    assert mine[0] == theirs[0]
    for a, b in zip(mine[1:], theirs[1:]):
        assert np.array_equal(a, b)
    o2n, n2o = gs.rcm(m)
    r_o2n, r_n2o = ref.ref_rcm(m)
    assert np.array_equal(o2n, r_o2n) and np.array_equal(n2o, r_n2o)


@SETTINGS
@given(g=symmetric(), data=st.data())
def test_permutations_and_ell_equal_reference(gs, ref, g, data):
    m = _csr(gs, g)
    n = m.rows
    o2n, n2o = gs.rcm(m)
    ap = gs.apply_permutation(m, o2n, n2o)
    rrp, rci, rv = ref.ref_apply_permutation(m, o2n, n2o)
    assert np.array_equal(ap.row_ptr, rrp) and np.array_equal(ap.col_idx, rci)
    assert np.array_equal(ap.val.astype(np.float32), rv)
    ro2n = np.array(data.draw(st.permutations(list(range(n)))), np.int32)
    pm = gs.permute_matrix(m, ro2n, o2n)
    prp, pci, pv = ref.ref_permute_matrix(m, ro2n, o2n)
    assert np.array_equal(pm.row_ptr, prp) and np.array_equal(pm.col_idx, pci)
    assert np.array_equal(pm.val.astype(np.float32), pv)
    width = data.draw(st.integers(1, 6))
    ec, ev, orp, oc, ov = gs.ell_build(m, width)
    rec, rev, rorp, roc, rov = ref.ref_ell(m, width)
    assert np.array_equal(ec, rec) and np.array_equal(ev.astype(np.float32), rev)
    assert np.array_equal(orp, rorp) and np.array_equal(oc, roc) and np.array_equal(ov.astype(np.float32), rov)


@SETTINGS
@given(g=symmetric(block=3))
def test_block_helpers_equal_reference(gs, ref, g):
    m = _csr(gs, g)
    grp, gci = gs.block_graph(m, 3)
    rrp, rci = ref.ref_block_graph(m)
    assert np.array_equal(grp, rrp) and np.array_equal(gci, rci)
    d = gs.block_inverses3x3(m)
    rd = ref.ref_block_inverses(m)
    assert np.abs(d - rd).max() <= 1e-6 * max(1.0, np.abs(d).max())
