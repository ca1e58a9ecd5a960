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
