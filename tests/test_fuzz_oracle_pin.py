"""The FP32 restatement in the oracle against the reference's own code
(oracle/_ref, built from the reference's sources; one thread, so its FP32
reductions run in order) on random problems: SPD graph Laplacians of random
2-D and 3-D grids with random coefficients, the host SA hierarchy, no or
per-level RCM permutations, and random V-cycle options (SGS or damped
Jacobi, 1-2 pre/post steps, 1-2 V-cycles, weights), and their 3x3-block
forms under the multigrid block-Jacobi preconditioner. Iteration counts must
be equal and the FP32 iterates bit-identical -- the pin the GPU path's
parity stands on, checked beyond the fixed problems. HierarchicalReordering
is compared with the reference's class on the same hierarchies."""
import numpy as np
import scipy.sparse as sp
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

SETTINGS = settings(max_examples=40, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])


@st.composite
def problems(draw):
    dims = draw(st.sampled_from([(draw(st.integers(4, 16)), draw(st.integers(4, 16))),
                                 (draw(st.integers(3, 7)), draw(st.integers(3, 7)), draw(st.integers(3, 7)))]))
    rng = np.random.default_rng(draw(st.integers(0, 2 ** 31)))
    n = int(np.prod(dims))
    idx = np.arange(n).reshape(dims)
    pairs = []
    for ax in range(len(dims)):
        lo = [slice(None)] * len(dims)
        hi = [slice(None)] * len(dims)
        lo[ax], hi[ax] = slice(None, -1), slice(1, None)
        pairs.append(np.stack([idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()], 1))
    pairs = np.concatenate(pairs)
    w = np.exp(rng.uniform(-draw(st.sampled_from([0.0, 1.0, 3.0])), 0.0, len(pairs)))
    g = sp.coo_matrix((w, (pairs[:, 0], pairs[:, 1])), shape=(n, n))
    g = (g + g.T).tocsr()
    lap = sp.diags(np.asarray(g.sum(axis=1)).ravel()) - g
    a = (lap + sp.diags(rng.uniform(1e-3, 0.1, n))).tocsr()
    a.sort_indices()
    opts = dict(
        smoother=draw(st.sampled_from([0, 2])),
        pre=draw(st.integers(1, 2)),
        post=draw(st.integers(1, 2)),
        vcycles=draw(st.integers(1, 2)),
        omega=draw(st.sampled_from([0.7, 0.9, 1.0])),
    )
    return a, draw(st.booleans()), draw(st.sampled_from([8, 20, 60])), opts, int(rng.integers(0, 1000))


def _f32_levels(ref, H):
    f32 = lambda m: ref.CsrView(m.rows, m.cols, m.row_ptr, m.col_idx, m.val.astype(np.float32).astype(np.float64))
    return ([f32(H.A(k)) for k in range(H.levels)], [f32(H.P(k)) for k in range(H.levels - 1)],
            [f32(H.R(k)) for k in range(H.levels - 1)])


@SETTINGS
@given(p=problems())
def test_fp32_restatement_equals_reference_on_random_problems(gs, ref, p):
    a, rcm, min_dofs, opts, seed = p
    csr = gs.Csr.from_scipy(a)
    H = gs.Hierarchy.build(csr, 1, 0.1, 10, min_dofs)
    f32 = lambda m: ref.CsrView(m.rows, m.cols, m.row_ptr, m.col_idx, m.val.astype(np.float32).astype(np.float64))
    A = [f32(H.A(k)) for k in range(H.levels)]
    P = [f32(H.P(k)) for k in range(H.levels - 1)]
    R = [f32(H.R(k)) for k in range(H.levels - 1)]
    perms = [gs.rcm(H.A(k)) for k in range(H.levels)] if rcm else None
    b = gs.uniform_rhs(a.shape[0], seed).astype(np.float32)
    code = 0 if opts["smoother"] == 0 else 2  # MultigridGaussSeidel / MultigridDampedJacobi preconditioner
    xr, itr, _, _ = ref.ref_amg_pcg(A, P, R, b, perms=perms, smoother=code, pre=opts["pre"], post=opts["post"],
                                    vcycles=opts["vcycles"], omega=opts["omega"], tol=1e-5, max_iter=300)
    xo, ito, _, _ = ref.amg_pcg(A, P, R, b.astype(np.float64), perms=perms, precision=ref.PREC_F32,
                                smoother=opts["smoother"], pre=opts["pre"], post=opts["post"],
                                vcycles=opts["vcycles"], omega=opts["omega"], coarse_solver=0, tol=1e-5,
                                max_iter=300, alias=1)
    assert itr == ito
    assert np.array_equal(xr, xo.astype(np.float32))


@SETTINGS
@given(p=problems(), data=st.data())
def test_block_jacobi_multigrid_equals_reference_on_random_problems(gs, ref, p, data):
    """MultigridBlockJacobiPreconditioner (3x3 block Jacobi on every level) on
    (graph Laplacian) x (random SPD 3x3 block), the block form of the problems
    above: the reference's code and the FP32 restatement agree bit for bit."""
    a, rcm, min_dofs, opts, seed = p
    rng = np.random.default_rng(seed)
    m = rng.uniform(-1, 1, (3, 3))
    blk = m @ m.T + 3 * np.eye(3)
    ab = sp.kron(a, blk, format="csr")
    ab.sort_indices()
    H = gs.Hierarchy.build(gs.Csr.from_scipy(ab), 3, 0.1, 10, 3 * min_dofs)
    A, P, R = _f32_levels(ref, H)
    perms = [gs.rcm(H.A(k)) for k in range(H.levels)] if rcm else None
    b = gs.uniform_rhs(ab.shape[0], seed).astype(np.float32)
    coarse = data.draw(st.integers(1, 4))
    omega = data.draw(st.sampled_from([0.5, 0.6, 0.8]))
    xr, itr, _, _ = ref.ref_amg_pcg(A, P, R, b, perms=perms, smoother=3, pre=opts["pre"], post=opts["post"],
                                    coarse=coarse, vcycles=opts["vcycles"], omega=omega, tol=1e-5, max_iter=300)
    xo, ito, _, _ = ref.amg_pcg(A, P, R, b.astype(np.float64), perms=perms, precision=ref.PREC_F32, smoother=3,
                                pre=opts["pre"], post=opts["post"], coarse_steps=coarse, vcycles=opts["vcycles"],
                                omega=omega, coarse_solver=0, tol=1e-5, max_iter=300, alias=1)
    assert itr == ito
    assert np.array_equal(xr, xo.astype(np.float32))


@SETTINGS
@given(p=problems())
def test_hierarchical_reordering_equals_reference_on_random_problems(gs, ref, p):
    """HierarchicalReordering::compute: the product, the reference's own class
    and the numpy restatement give the same permutation on every level."""
    a, _, min_dofs, _, _ = p
    H = gs.Hierarchy.build(gs.Csr.from_scipy(a), 1, 0.1, 10, min_dofs)
    A = [H.A(k) for k in range(H.levels)]
    P = [H.P(k) for k in range(H.levels - 1)]
    R = [H.R(k) for k in range(H.levels - 1)]
    mine = gs.hierarchical_reordering(H)
    theirs = ref.ref_hierarchical_reordering(A, P, R)
    restated = ref.hierarchical_reordering(A, R)
    for (o1, n1), (o2, n2), (o3, n3) in zip(mine, theirs, restated):
        assert np.array_equal(o1, o2) and np.array_equal(n1, n2)
        assert np.array_equal(o1, o3) and np.array_equal(n1, n3)
        assert np.array_equal(o1[n1], np.arange(len(n1)))
