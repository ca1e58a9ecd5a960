"""Known answers from the reference's own unit tests, checked on the oracle
restatement, on the reference compiled from its sources (oracle/_ref) and,
for the host-side setup, on the product's C ABI."""
import numpy as np
import pytest
import scipy.sparse as sp


def csr_from_triplets(n, trip):
    r, c, v = zip(*trip)
    m = sp.csr_matrix((np.array(v, float), (np.array(r), np.array(c))), shape=(n, n))
    m.sort_indices()
    return m


TRIDIAG4 = [(0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0), (1, 1, 4.0), (1, 2, -1.0),
            (2, 1, -1.0), (2, 2, 4.0), (2, 3, -1.0), (3, 2, -1.0), (3, 3, 4.0)]


def test_gs_one_color(orc):
    # tests/cuda/testCudaGaussSeidel.cc:15-111
    m = orc.CsrView.from_scipy(csr_from_triplets(4, TRIDIAG4))
    order = np.array([0, 2, 1, 3], np.int32)
    rhs = np.array([4.0, 8.0, 12.0, 16.0])
    for f32 in (False, True):
        x = orc.gs_color(m, order, 0, 2, rhs, np.zeros(4), 1.0, f32=f32)
        assert np.allclose(x, [1.0, 0.0, 3.0, 0.0], atol=1e-5)


def test_gs_full_two_color_sweep(orc):
    # tests/cuda/testCudaGaussSeidel.cc:114-222
    m = orc.CsrView.from_scipy(csr_from_triplets(4, TRIDIAG4))
    order = np.array([0, 2, 1, 3], np.int32)
    rhs = np.array([4.0, 8.0, 12.0, 16.0])
    x = orc.gs_color(m, order, 0, 2, rhs, np.zeros(4), 1.0)
    x = orc.gs_color(m, order, 2, 2, rhs, x, 1.0)
    assert np.allclose(x, [1.0, 3.0, 3.0, 4.75], atol=1e-5)


def test_gs_known_answers_reference(ref):
    m = ref.CsrView.from_scipy(csr_from_triplets(4, TRIDIAG4))
    order = np.array([0, 2, 1, 3], np.int32)
    rhs = np.array([4.0, 8.0, 12.0, 16.0], np.float32)
    x = ref.ref_gs_color(m, order, 0, 2, rhs, np.zeros(4, np.float32), 1.0)
    assert np.array_equal(x, np.array([1, 0, 3, 0], np.float32))
    x = ref.ref_gs_color(m, order, 2, 2, rhs, x, 1.0)
    assert np.array_equal(x, np.array([1, 3, 3, 4.75], np.float32))


def test_apply_two_inverse_blocks(ref):
    # tests/cuda/testCudaBlockOps.cc:15-...
    dinv = np.array([2, 0, 0, 0, 3, 0, 0, 0, 4, 1, 1, 0, 0, 2, 0, 0, 0, 3], np.float32)
    r = np.array([1, 2, 3, 4, 5, 6], np.float32)
    assert np.array_equal(ref.ref_apply_block_inverses(dinv, r), [2, 6, 12, 9, 10, 18])


def test_spmv_three_by_three(orc, ref):
    # tests/cuda/testCudaSpmv.cc:123-195
    m = orc.CsrView.from_scipy(csr_from_triplets(3, [(0, 0, 4), (0, 1, 1), (1, 0, 1), (1, 1, 3),
                                                      (1, 2, 2), (2, 1, 2), (2, 2, 5)]))
    x = np.array([1.0, 2.0, 3.0])
    assert np.array_equal(orc.spmv(m, x), [6, 13, 19])
    assert np.array_equal(orc.spmv(m, x, f32=True), [6, 13, 19])
    assert np.array_equal(ref.ref_spmv(m, x), [6, 13, 19])


def test_dot_products(orc, ref):
    # tests/cuda/testCudaSpmv.cc:17-56 and tests/metal/DotProductTests.cc:65-140
    assert orc.dot([1, 2, 3], [4, 5, 6]) == 32.0
    assert ref.ref_dot(np.array([1, 2, 3], np.float32), np.array([4, 5, 6], np.float32)) == 32.0
    for n in (1, 17, 255, 256, 257, 1000, 100000):
        ones = np.ones(n)
        assert orc.dot(ones, ones) == n
        assert ref.ref_dot(ones, ones) == n
        assert orc.dot(ones, np.zeros(n)) == 0.0
    i = np.arange(10000, dtype=np.float32)
    x, y = np.sin(0.001 * i), np.cos(0.002 * i)
    exact = float(np.dot(x.astype(np.float64), y.astype(np.float64)))
    assert abs(ref.ref_dot(x, y) - exact) <= 1e-3 * max(1.0, abs(exact))
    assert abs(orc.dot(x, y, f32=True) - exact) <= 1e-3 * max(1.0, abs(exact))


def _graph(n, edges):
    trip = [(i, i, 1.0) for i in range(n)]
    for a, b in edges:
        trip += [(a, b, -1.0), (b, a, -1.0)]
    return csr_from_triplets(n, trip)


GRAPHS = {
    # tests/metal/graphColoringTest.cc:222-410
    "path": (_graph(6, [(i, i + 1) for i in range(5)]), 2),
    "triangle": (_graph(3, [(0, 1), (1, 2), (2, 0)]), 3),
    "even_cycle": (_graph(4, [(0, 1), (1, 2), (2, 3), (3, 0)]), 2),
    "complete5": (_graph(5, [(i, j) for i in range(5) for j in range(i + 1, 5)]), 5),
    # tests/metal/graphColoringTest.cc:412-507
    "grid10x10": (_graph(100, [(y * 10 + x, y * 10 + x + 1) for y in range(10) for x in range(9)]
                         + [(y * 10 + x, (y + 1) * 10 + x) for y in range(9) for x in range(10)]), 2),
}


def validate_coloring(m, nc, colors, verts, offs):
    """tests/metal/graphColoringTest.cc:40-200: proper, complete, contiguous."""
    n = m.shape[0]
    assert len(offs) == nc + 1 and offs[0] == 0 and offs[-1] == n
    assert sorted(verts.tolist()) == list(range(n))
    for c in range(nc):
        block = verts[offs[c]:offs[c + 1]]
        assert np.all(colors[block] == c)
    coo = m.tocoo()
    off = coo.row != coo.col
    assert np.all(colors[coo.row[off]] != colors[coo.col[off]])


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_coloring_counts(name, gs, orc, ref):
    m, expected = GRAPHS[name]
    c = gs.Csr.from_scipy(m)
    nc, colors, verts, offs = gs.greedy_coloring(c)
    assert nc == expected
    validate_coloring(m, nc, colors, verts, offs)
    rnc, rcolors, rverts, roffs = ref.ref_coloring(c)
    assert nc == rnc and np.array_equal(colors, rcolors) and np.array_equal(verts, rverts)
    assert np.array_equal(offs, roffs)
    onc, overts, ooffs = orc.coloring(c)
    assert onc == nc and np.array_equal(overts, verts) and np.array_equal(ooffs, offs)


def test_sgs_poisson8x8_golden(orc):
    """tests/metal/gaussSeidelSymmUnittest.cc:163-302: one symmetric GS
    application from zero; the golden vector comes from the reference's
    SymmetricGaussSeidelPreconditioner on its CPU backend."""
    from conftest import golden
    g = golden("sgs_poisson8x8.npz")
    m = orc.CsrView(64, 64, g["row_ptr"], g["col_idx"], g["val"])
    # a one-level hierarchy whose coarsest smoother runs one symmetric step
    z = orc.precondition([m], [], [], g["rhs"].astype(np.float64), precision=orc.PREC_F32,
                         coarse_solver=0, coarse_steps=1)
    assert np.array_equal(z.astype(np.float32), g["z"])
    z64 = orc.precondition([m], [], [], g["rhs"].astype(np.float64), coarse_solver=0, coarse_steps=1)
    assert np.linalg.norm(z64 - g["z"]) / np.linalg.norm(z64) < 1e-5
    rhs = g["rhs"].astype(np.float64)
    A = m.to_scipy()
    assert np.linalg.norm(rhs - A @ z64) < np.linalg.norm(rhs)
    assert rhs @ z64 > 0
