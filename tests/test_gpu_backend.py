"""Kernel-level Backend operations through the C ABI, against the known
answers of the reference's own CUDA tests (tests/cuda/*.cc) and the oracle."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

TRIDIAG4 = [(0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0), (1, 1, 4.0), (1, 2, -1.0),
            (2, 1, -1.0), (2, 2, 4.0), (2, 3, -1.0), (3, 2, -1.0), (3, 3, 4.0)]


def csr(gs, n, trip):
    r, c, v = zip(*trip)
    m = sp.csr_matrix((np.array(v, float), (np.array(r), np.array(c))), shape=(n, n))
    m.sort_indices()
    return gs.Csr.from_scipy(m)


def dev(a, dtype="float32"):
    import torch
    return torch.tensor(np.asarray(a), dtype=getattr(torch, dtype), device="cuda")


@pytest.fixture
def torch_mod(device):
    import torch
    return torch


@pytest.mark.parametrize("dt", ["float32", "float64"])
def test_gauss_seidel_one_color_and_sweep(gs, torch_mod, dt):
    # tests/cuda/testCudaGaussSeidel.cc:15-222
    torch = torch_mod
    kind = gs.F32 if dt == "float32" else gs.F64
    A = gs.DeviceCsr(csr(gs, 4, TRIDIAG4), kind)
    order = dev([0, 2, 1, 3], "int32")
    rhs = dev([4, 8, 12, 16], dt)
    x = dev([0, 0, 0, 0], dt)
    gs.gauss_seidel_color(A, order.data_ptr(), 0, 2, rhs.data_ptr(), x.data_ptr(), 1.0)
    torch.cuda.synchronize()
    assert x.cpu().tolist() == [1.0, 0.0, 3.0, 0.0]
    gs.gauss_seidel_color(A, order.data_ptr(), 2, 2, rhs.data_ptr(), x.data_ptr(), 1.0)
    torch.cuda.synchronize()
    assert x.cpu().tolist() == [1.0, 3.0, 3.0, 4.75]


def test_spmv_known_and_updated_values(gs, torch_mod):
    # tests/cuda/testCudaSpmv.cc:123-272
    torch = torch_mod
    A = gs.DeviceCsr(csr(gs, 3, [(0, 0, 4), (0, 1, 1), (1, 0, 1), (1, 1, 3), (1, 2, 2), (2, 1, 2), (2, 2, 5)]), gs.F32)
    x, y = dev([1, 2, 3]), dev([0, 0, 0])
    gs.spmv(A, x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    assert y.cpu().tolist() == [6.0, 13.0, 19.0]
    B = gs.DeviceCsr(csr(gs, 2, [(0, 0, 2), (0, 1, 1), (1, 0, 1), (1, 1, 3)]), gs.F32)
    B.update_values(np.array([4.0, 2.0, 2.0, 6.0]))
    x, y = dev([1, 2]), dev([0, 0])
    gs.spmv(B, x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    assert y.cpu().tolist() == [8.0, 14.0]


def test_spmv_random_sparse_against_oracle(gs, orc, torch_mod):
    # tests/cuda/testCudaSpmv.cc:275-...: n = 300 banded matrix
    torch = torch_mod
    n = 300
    trip = []
    for r in range(n):
        trip.append((r, r, 4.0))
        if r > 0: trip.append((r, r - 1, -1.0))
        if r + 1 < n: trip.append((r, r + 1, -1.0))
        if r + 7 < n: trip.append((r, r + 7, 0.25))
    m = csr(gs, n, trip)
    xv = np.sin(0.1 * np.arange(n)) + 0.3
    for dt, kind, tol in (("float32", gs.F32, 1e-5), ("float64", gs.F64, 1e-14)):
        A = gs.DeviceCsr(m, kind)
        x, y = dev(xv, dt), dev(np.zeros(n), dt)
        gs.spmv(A, x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        ref = orc.spmv(m, xv)
        assert np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref) < tol


def test_dot_products(gs, orc, torch_mod):
    # tests/cuda/testCudaSpmv.cc:17-120, tests/metal/DotProductTests.cc:65-140
    torch = torch_mod
    out = dev([0.0])
    # keep every operand referenced: a tensor freed before the kernel runs
    # hands its block to the next allocation
    xa3, ya3 = dev([1, 2, 3]), dev([4, 5, 6])
    gs.dot(3, xa3.data_ptr(), ya3.data_ptr(), out.data_ptr(), gs.F32)
    torch.cuda.synchronize()
    assert out.item() == 32.0
    for n in (1, 17, 255, 256, 257, 1000, 100000):
        ones = dev(np.ones(n), "float64")
        o = dev([0.0], "float64")
        gs.dot(n, ones.data_ptr(), ones.data_ptr(), o.data_ptr(), gs.F64)
        torch.cuda.synchronize()
        assert o.item() == n
    i = np.arange(10000)
    xa, ya = np.sin(0.001 * i), np.cos(0.002 * i)
    o = dev([0.0], "float64")
    xd, yd = dev(xa, "float64"), dev(ya, "float64")
    gs.dot(10000, xd.data_ptr(), yd.data_ptr(), o.data_ptr(), gs.F64)
    torch.cuda.synchronize()
    assert abs(o.item() - float(xa @ ya)) <= 1e-12 * abs(float(xa @ ya))


def test_block_ops(gs, orc, torch_mod):
    # tests/cuda/testCudaBlockOps.cc:15-...
    torch = torch_mod
    dinv = dev([2, 0, 0, 0, 3, 0, 0, 0, 4, 1, 1, 0, 0, 2, 0, 0, 0, 3])
    r = dev([1, 2, 3, 4, 5, 6])
    c = dev([0] * 6)
    gs.apply_block_inverses3x3(6, dinv.data_ptr(), r.data_ptr(), c.data_ptr(), gs.F32)
    torch.cuda.synchronize()
    assert c.cpu().tolist() == [2, 6, 12, 9, 10, 18]
    # one block GS colour pass on a small elasticity matrix against the oracle
    e = gs.elasticity(4)
    d64 = gs.block_inverses3x3(e)
    nc, colors, verts, offs = gs.greedy_coloring(gs.Csr(e.rows // 3, e.rows // 3, *gs.block_graph(e), np.ones(len(gs.block_graph(e)[1]))))
    A = gs.DeviceCsr(e, gs.F64)
    x0 = np.linspace(-1, 1, e.rows)
    xd = dev(x0, "float64")
    rhs = dev(e.rhs, "float64")
    dinv_d = dev(d64, "float64")
    order = dev(verts, "int32")
    for c_ in range(nc):
        gs.block_gauss_seidel_color3x3(A, order.data_ptr(), int(offs[c_]), int(offs[c_ + 1] - offs[c_]),
                                       dinv_d.data_ptr(), rhs.data_ptr(), xd.data_ptr(), 0.9)
    torch.cuda.synchronize()
    xo = x0.copy()
    for c_ in range(nc):
        xo = orc.block_gs_color(e, verts, int(offs[c_]), int(offs[c_ + 1] - offs[c_]), d64, e.rhs, xo, 0.9)
    assert np.linalg.norm(xd.cpu().numpy() - xo) / np.linalg.norm(xo) < 1e-13


def test_vector_and_scalar_ops(gs, torch_mod):
    # tests/cuda/testCudaVectorOps.cc, tests/cuda/testCudaScalarOps.cc
    torch = torch_mod
    x, y = dev([1, 2, 3]), dev([10, 20, 30])
    gs.vector_op(gs.VEC_AXPY, 3, x.data_ptr(), y.data_ptr(), 2.0, dtype=gs.F32)
    gs.vector_op(gs.VEC_SCALE, 3, 0, y.data_ptr(), 0.5, dtype=gs.F32)
    torch.cuda.synchronize()
    assert y.cpu().tolist() == [6.0, 12.0, 18.0]
    a = dev([3.0])
    gs.vector_op(gs.VEC_AXPY, 3, x.data_ptr(), y.data_ptr(), alpha_ptr=a.data_ptr(), dtype=gs.F32)
    gs.vector_op(gs.VEC_SCALE_BY_VECTOR, 3, x.data_ptr(), y.data_ptr(), dtype=gs.F32)
    torch.cuda.synchronize()
    assert y.cpu().tolist() == [9.0, 36.0, 81.0]
    gs.vector_op(gs.VEC_COPY, 3, x.data_ptr(), y.data_ptr(), dtype=gs.F32)
    torch.cuda.synchronize()
    assert y.cpu().tolist() == [1.0, 2.0, 3.0]
    gs.vector_op(gs.VEC_SET_ZERO, 3, 0, y.data_ptr(), dtype=gs.F32)
    torch.cuda.synchronize()
    assert y.cpu().tolist() == [0.0, 0.0, 0.0]
    s1, s2, o = dev([6.0]), dev([4.0]), dev([0.0])
    gs.scalar_op(gs.SCALAR_DIVIDE, s1.data_ptr(), s2.data_ptr(), o.data_ptr(), dtype=gs.F32)
    gs.scalar_op(gs.SCALAR_MULTIPLY, o.data_ptr(), s2.data_ptr(), o.data_ptr(), dtype=gs.F32)
    gs.scalar_op(gs.SCALAR_NEGATE, o.data_ptr(), None, o.data_ptr(), dtype=gs.F32)
    torch.cuda.synchronize()
    assert o.item() == -6.0
    gs.scalar_op(gs.SCALAR_SET, None, None, o.data_ptr(), 16.0, dtype=gs.F32)
    gs.scalar_op(gs.SCALAR_SQRT, o.data_ptr(), None, o.data_ptr(), dtype=gs.F32)
    gs.scalar_op(gs.SCALAR_COPY, o.data_ptr(), None, s1.data_ptr(), dtype=gs.F32)
    torch.cuda.synchronize()
    assert s1.item() == 4.0


def test_zero_diagonal_is_rejected(gs, torch_mod):
    m = csr(gs, 2, [(0, 0, 1.0), (0, 1, 1.0), (1, 0, 1.0)])
    A = gs.DeviceCsr(m, gs.F64)
    order = dev([0, 1], "int32")
    v = dev([1.0, 1.0], "float64")
    with pytest.raises(gs.SolverError, match="zero diagonal"):
        gs.gauss_seidel_color(A, order.data_ptr(), 0, 2, v.data_ptr(), v.data_ptr(), 1.0)
