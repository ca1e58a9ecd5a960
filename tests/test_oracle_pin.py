"""Pins the oracle restatement (oracle/oracle.cc) to the reference's own
FP32 CPU path, bit for bit, on the golden fixture and on live runs of the
reference compiled from its sources."""
import numpy as np
import pytest

from conftest import golden


def _fixture_levels(orc, g):
    L = int(g["levels"])
    mk = lambda tag: orc.CsrView(g[f"{tag}_shape"][0], g[f"{tag}_shape"][1], g[f"{tag}_rp"],
                                 g[f"{tag}_ci"], g[f"{tag}_v"].astype(np.float64))
    A = [mk(f"A{k}") for k in range(L)]
    P = [mk(f"P{k}") for k in range(L - 1)]
    R = [mk(f"R{k}") for k in range(L - 1)]
    perms = [(g[f"o2n{k}"], g[f"n2o{k}"]) for k in range(L)]
    return A, P, R, perms


def test_fp32_amg_pcg_matches_reference_golden(orc):
    g = golden("amg_pcg_poisson16_f32.npz")
    A, P, R, perms = _fixture_levels(orc, g)
    x, it, status, _ = orc.amg_pcg(A, P, R, g["b"].astype(np.float64), perms=perms,
                                   precision=orc.PREC_F32, coarse_solver=0, tol=1e-6, max_iter=100,
                                   alias=1)
    assert it == int(g["iterations"])
    assert np.array_equal(x.astype(np.float32), g["x"])


def test_fp32_amg_pcg_matches_reference_live(gs, ref):
    """Same pin on a second problem (variable coefficients, identity
    permutations, two V-cycles, omega 0.9), run live against oracle/_ref."""
    a0 = gs.varcoef_loguniform(12, 10, 9, seed=7)
    H = gs.Hierarchy.build(a0, 1, 0.1, 10, 100)
    f32 = lambda m: ref.CsrView(m.rows, m.cols, m.row_ptr, m.col_idx,
                                m.val.astype(np.float32).astype(np.float64))
    A = [f32(H.A(k)) for k in range(H.levels)]
    P = [f32(H.P(k)) for k in range(H.levels - 1)]
    R = [f32(H.R(k)) for k in range(H.levels - 1)]
    b = gs.uniform_rhs(a0.rows, 11).astype(np.float32)
    xr, itr, _, _ = ref.ref_amg_pcg(A, P, R, b, pre=1, post=2, vcycles=2, omega=0.9, tol=1e-5)
    xo, ito, _, _ = ref.amg_pcg(A, P, R, b.astype(np.float64), precision=ref.PREC_F32, pre=1,
                                post=2, vcycles=2, omega=0.9, coarse_solver=0, tol=1e-5,
                                alias=1)
    assert itr == ito
    assert np.array_equal(xr, xo.astype(np.float32))


def test_fp32_pin_with_rcm_permutations_live(gs, ref):
    a0 = gs.kuhn_laplacian(9, seed=5)
    H = gs.Hierarchy.build(a0, 1, 0.1, 10, 60)
    f32 = lambda m: ref.CsrView(m.rows, m.cols, m.row_ptr, m.col_idx,
                                m.val.astype(np.float32).astype(np.float64))
    A = [f32(H.A(k)) for k in range(H.levels)]
    P = [f32(H.P(k)) for k in range(H.levels - 1)]
    R = [f32(H.R(k)) for k in range(H.levels - 1)]
    perms = [ref.ref_rcm(m) for m in A]
    b = gs.uniform_rhs(a0.rows, 3).astype(np.float32)
    xr, itr, _, _ = ref.ref_amg_pcg(A, P, R, b, perms=perms, tol=1e-6)
    xo, ito, _, _ = ref.amg_pcg(A, P, R, b.astype(np.float64), perms=perms,
                                precision=ref.PREC_F32, coarse_solver=0, tol=1e-6, alias=1)
    assert itr == ito and np.array_equal(xr, xo.astype(np.float32))


def test_fp64_oracle_tracks_fp32_reference(gs, orc):
    """The FP64 restatement and the FP32 reference agree to FP32 accuracy."""
    g = golden("amg_pcg_poisson16_f32.npz")
    A, P, R, perms = _fixture_levels(orc, g)
    x64, it64, _, _ = orc.amg_pcg(A, P, R, g["b"].astype(np.float64), perms=perms,
                                  coarse_solver=0, tol=1e-6, max_iter=100, alias=1)
    assert abs(it64 - int(g["iterations"])) <= 1
    assert np.linalg.norm(x64 - g["x"]) / np.linalg.norm(x64) < 1e-5


def test_reference_vcycle_aliasing_is_what_the_reference_computes(gs, ref):
    """With three or more levels the reference's V-cycle overwrites the
    pre-smoothed iterate of every intermediate level with P x_c and adds it
    to itself (src/Smoothers/MultigridSmoother.cc:394-404). The oracle
    reproduces the reference only with that aliasing; the textbook V-cycle
    (x_k += P x_{k+1}) gives a different iterate."""
    a0 = gs.poisson7(14)
    H = gs.Hierarchy.build(a0, 1, 0.1, 10, 60)
    assert H.levels >= 3
    f32 = lambda m: ref.CsrView(m.rows, m.cols, m.row_ptr, m.col_idx,
                                m.val.astype(np.float32).astype(np.float64))
    A = [f32(H.A(k)) for k in range(H.levels)]
    P = [f32(H.P(k)) for k in range(H.levels - 1)]
    R = [f32(H.R(k)) for k in range(H.levels - 1)]
    b = gs.uniform_rhs(a0.rows, 1).astype(np.float32)
    xr, _, _, _ = ref.ref_amg_pcg(A, P, R, b, tol=1e-30, max_iter=1)
    xa, _, _, _ = ref.amg_pcg(A, P, R, b.astype(np.float64), precision=ref.PREC_F32,
                              coarse_solver=0, tol=1e-30, max_iter=1, alias=1)
    xs, _, _, _ = ref.amg_pcg(A, P, R, b.astype(np.float64), precision=ref.PREC_F32,
                              coarse_solver=0, tol=1e-30, max_iter=1, alias=0)
    assert np.array_equal(xr, xa.astype(np.float32))
    assert np.abs(xr - xs).max() > 1e-3


def _f32_levels(ref, H):
    f32 = lambda m: ref.CsrView(m.rows, m.cols, m.row_ptr, m.col_idx,
                                m.val.astype(np.float32).astype(np.float64))
    return ([f32(H.A(k)) for k in range(H.levels)], [f32(H.P(k)) for k in range(H.levels - 1)],
            [f32(H.R(k)) for k in range(H.levels - 1)])


# reference preconditioner code -> oracle options
#   2 MultigridDampedJacobiPreconditioner: damped Jacobi everywhere, coarse steps = pre + post
#   3 MultigridBlockJacobiPreconditioner: block Jacobi everywhere, coarse steps given
#   4 MultigridHybridBlockPreconditioner: block GS on the finest level, block Jacobi below
@pytest.mark.parametrize("code", [2, 3, 4])
def test_fp32_jacobi_family_multigrid_matches_reference(gs, ref, code):
    if code == 2:
        a0 = gs.varcoef_loguniform(11, 9, 10, seed=8)
        H = gs.Hierarchy.build(a0, 1, 0.1, 10, 80)
        b = gs.uniform_rhs(a0.rows, 4)
    else:
        a0 = gs.elasticity(5)
        H = gs.Hierarchy.build(a0, 3, 0.1, 10, 60)
        b = a0.rhs
    assert H.levels >= 2
    A, P, R = _f32_levels(ref, H)
    b32 = b.astype(np.float32)
    omega, coarse = (0.7, None) if code == 2 else (0.6, 3)
    xr, itr, _, _ = ref.ref_amg_pcg(A, P, R, b32, smoother=code, pre=2, post=1, coarse=coarse,
                                    omega=omega, tol=1e-5, max_iter=300)
    kw = dict(smoother=2) if code == 2 else dict(smoother=3) if code == 3 else dict(smoother=1, coarse_smoother=3)
    xo, ito, _, _ = ref.amg_pcg(A, P, R, b32.astype(np.float64), precision=ref.PREC_F32, pre=2, post=1,
                                coarse_steps=coarse, omega=omega, coarse_solver=0, tol=1e-5, max_iter=300,
                                alias=1, **kw)
    if code == 4:
        # block Gauss-Seidel on the finest level: the reference's CPU backend reads the
        # smoother's (colour start, colour count) as (start, end) (src/CPU/CPUBackend.cc:350-364),
        # so its hybrid preconditioner sweeps wrong ranges and stalls; the oracle (and the
        # product) use the intended (start, count) reading and converge
        assert itr == 300 and ito < 300
        return
    assert itr == ito
    assert np.array_equal(xr, xo.astype(np.float32))


# single-level preconditioners: a one-level hierarchy whose only level is smoothed
#   0 Identity, 1 Jacobi, 2 SymmetricGaussSeidel(w, n), 3 DampedJacobi(n, w),
#   4 BlockJacobi(n, w), 5 BlockGaussSeidel(w, n)
@pytest.mark.parametrize("code", [0, 1, 2, 3, 4, 5])
def test_fp32_single_level_preconditioners_match_reference(gs, ref, code):
    block = code in (4, 5)
    a = gs.elasticity(4) if block else gs.varcoef_loguniform(9, 8, 7, seed=9)
    b = (a.rhs if block else gs.uniform_rhs(a.rows, 6)).astype(np.float32)
    m = ref.CsrView(a.rows, a.cols, a.row_ptr, a.col_idx, a.val.astype(np.float32).astype(np.float64))
    omega, sweeps = (1.0, 1) if code in (0, 1) else (0.8, 3)
    kind = {0: 4, 1: 2, 2: 0, 3: 2, 4: 3, 5: 1}[code]
    xo, ito, _, _ = ref.amg_pcg([m], [], [], b.astype(np.float64), precision=ref.PREC_F32, smoother=kind,
                                coarse_steps=sweeps, omega=omega, coarse_solver=0, tol=1e-5, max_iter=2000)
    if code == 5:
        # the same (start, count) vs (start, end) reading in the reference's block GS
        # makes its BlockGaussSeidelPreconditioner diverge; the intended reading converges
        with pytest.raises(RuntimeError, match="NaN"):
            ref.ref_pcg(m, b, preconditioner=code, omega=omega, sweeps=sweeps, tol=1e-5, max_iter=2000)
        assert ito < 2000
        return
    xr, itr = ref.ref_pcg(m, b, preconditioner=code, omega=omega, sweeps=sweeps, tol=1e-5, max_iter=2000)
    assert itr == ito
    assert np.array_equal(xr, xo.astype(np.float32))
