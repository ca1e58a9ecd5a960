"""Parity of the CUDA AMG-PCG path with the oracle, called through the C ABI.

Tolerances: the plain FP64 solve must give iterates within 1e-10 relative
of the FP64 oracle and iteration counts within +-1; the FP32 V-cycle path
must reach the same FP64-verified residual and stay within the error bound
the residual implies (stated per test).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def levels(H):
    return ([H.A(k) for k in range(H.levels)], [H.P(k) for k in range(H.levels - 1)],
            [H.R(k) for k in range(H.levels - 1)])


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def true_residual(a, x, b):
    return float(np.linalg.norm(b - a.to_scipy() @ x) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def p32(gs):
    # min_dofs 100 gives 4 levels, so the coarse tail spans three of them
    a = gs.poisson7(32)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 100)
    assert H.levels >= 4
    return a, H, gs.uniform_rhs(a.rows, 0)


CASES = {
    # name: (solver options, oracle options)
    "cholesky": (dict(), dict()),
    "reference_coarse": (dict(coarse_solver=0, coarse_steps=2), dict(coarse_solver=0, coarse_steps=2)),
    "two_vcycles_omega": (dict(vcycles=2, omega=0.8, pre_steps=2, post_steps=1),
                          dict(vcycles=2, omega=0.8, pre=2, post=1)),
    "flexible": (dict(flexible=1), dict(flexible=1)),
    "graph": (dict(use_graph=1), dict()),
    "reference_vcycle": (dict(reference_vcycle=1, coarse_solver=0, coarse_steps=2),
                         dict(alias=1, coarse_solver=0, coarse_steps=2)),
    "no_tail_no_autotune": (dict(coarse_tail=0, autotune=0), dict()),
    "tail": (dict(coarse_tail=2), dict()),
    "tail_reference_vcycle": (dict(coarse_tail=2, reference_vcycle=1, coarse_solver=0, coarse_steps=2),
                              dict(alias=1, coarse_solver=0, coarse_steps=2)),
    "tail_graph_flexible": (dict(coarse_tail=2, use_graph=1, flexible=1), dict(flexible=1)),
    "lanes_1": (dict(lanes=1, coarse_tail=0), dict()),
    "lanes_8": (dict(lanes=8, coarse_tail=0), dict()),
    "lanes_32": (dict(lanes=32, coarse_tail=0), dict()),
    "sliced_2": (dict(sliced_lanes=2, coarse_tail=0), dict()),
    "sliced_4": (dict(sliced_lanes=4, coarse_tail=0), dict()),
    "sliced_8_graph_flexible": (dict(sliced_lanes=8, coarse_tail=0, use_graph=1, flexible=1), dict(flexible=1)),
    "plain_stream_order": (dict(overlap_launch=0), dict()),
    "coop_sweeps": (dict(sweep_launch=2, coarse_tail=0), dict()),
    "coop_graph_flexible": (dict(sweep_launch=2, coarse_tail=0, use_graph=1, flexible=1), dict(flexible=1)),
    "coop_omega_two_steps": (dict(sweep_launch=2, coarse_tail=0, vcycles=2, omega=0.8, pre_steps=2, post_steps=1),
                             dict(vcycles=2, omega=0.8, pre=2, post=1)),
    "coop_reference_coarse": (dict(sweep_launch=2, coarse_tail=0, coarse_solver=0, coarse_steps=2),
                              dict(coarse_solver=0, coarse_steps=2)),
    "coop_lanes_8": (dict(sweep_launch=2, coarse_tail=0, lanes=8), dict()),
    "coop_sliced_4": (dict(sweep_launch=2, coarse_tail=0, sliced_lanes=4), dict()),
    "per_colour_launches": (dict(sweep_launch=0, coarse_tail=0), dict()),
    "half_sweeps": (dict(half_sweeps=1), dict(half_sweeps=1)),
    "half_sweeps_two_steps_omega": (dict(half_sweeps=1, pre_steps=2, post_steps=2, omega=0.9, vcycles=2),
                                    dict(half_sweeps=1, pre=2, post=2, omega=0.9, vcycles=2)),
    "half_sweeps_graph_flexible": (dict(half_sweeps=1, use_graph=1, flexible=1), dict(half_sweeps=1, flexible=1)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_p32_fp64_matches_oracle(gs, orc, device, p32, case):
    a, H, b = p32
    so, oo = CASES[case]
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, **so), device=device)
    x, st = s.solve(b)
    A, P, R = levels(H)
    xo, it, status, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, **oo)
    assert st.status == gs.STATUS_CONVERGED and status == 1
    assert abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10
    assert true_residual(a, x, b) <= 1.5e-8


def test_p32_rcm_permutations_match_oracle(gs, orc, device, p32):
    a, H, b = p32
    A, P, R = levels(H)
    perms = [gs.rcm(m) for m in A]
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8), permutations=perms, device=device)
    x, st = s.solve(b)
    xo, it, _, _ = orc.amg_pcg(A, P, R, b, perms=perms, tol=1e-8)
    assert abs(st.iterations - it) <= 1 and rel(x, xo) <= 1e-10


def test_p32_hierarchical_permutations_match_oracle(gs, orc, device, p32):
    """HierarchicalReordering permutations passed to the solver (and to the oracle)."""
    a, H, b = p32
    A, P, R = levels(H)
    perms = gs.hierarchical_reordering(H)
    for opts in (dict(), dict(precision=1, flexible=1, use_graph=1)):
        s = gs.Solver(H, gs.SolverOptions(tol=1e-8, **opts), permutations=perms, device=device)
        x, st = s.solve(b)
        assert true_residual(a, x, b) <= 1.5e-8
        if not opts:
            xo, it, _, _ = orc.amg_pcg(A, P, R, b, perms=perms, tol=1e-8)
            assert abs(st.iterations - it) <= 1 and rel(x, xo) <= 1e-10


def test_preconditioner_matches_oracle(gs, orc, device, p32):
    import torch
    a, H, b = p32
    A, P, R = levels(H)
    for opts, oo in ((dict(), dict()), (dict(coarse_solver=0), dict(coarse_solver=0)),
                     (dict(reference_vcycle=1), dict(alias=1))):
        s = gs.Solver(H, gs.SolverOptions(**opts), device=device)
        r = torch.tensor(b, dtype=torch.float64, device="cuda")
        z = torch.empty_like(r)
        s.apply_preconditioner_device(r.data_ptr(), z.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        zo = orc.precondition(A, P, R, b, **oo)
        assert rel(z.cpu().numpy(), zo) <= 1e-12


def test_max_iterations_and_counts(gs, orc, device, p32):
    a, H, b = p32
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-14, max_iter=3), device=device)
    x, st = s.solve(b)
    xo, it, status, _ = orc.amg_pcg(A, P, R, b, tol=1e-14, max_iter=3)
    assert st.status == gs.STATUS_MAX_ITER and st.iterations == 3 == it and status == 2
    assert rel(x, xo) <= 1e-12


def test_edge_cases(gs, device, p32):
    a, H, b = p32
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8), device=device)
    x, st = s.solve(np.zeros(a.rows), np.ones(a.rows))
    assert st.status == gs.STATUS_ZERO_RHS and not x.any()
    x1, _ = s.solve(b)
    x2, st2 = s.solve(b, x1)  # already converged: returns without an iteration, x unchanged
    assert st2.status == gs.STATUS_INITIAL_CONVERGED and np.array_equal(x1, x2)
    bad = b.copy()
    bad[5] = np.nan
    with pytest.raises(gs.NotFiniteError):
        s.solve(bad)
    x3, st3 = s.solve(b)  # the solver stays usable after an error
    assert st3.status == gs.STATUS_CONVERGED and rel(x3, x1) == 0.0


def test_float_entry_point_and_device_solve(gs, device, p32):
    import torch
    a, H, b = p32
    s = gs.Solver(H, gs.SolverOptions(tol=1e-6), device=device)
    xf, stf = s.solve_f32(b.astype(np.float32))
    assert xf.dtype == np.float32 and true_residual(a, xf.astype(np.float64), b) < 2e-6
    xh, sth = s.solve(b)
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros_like(bd)
    std = s.solve_device(bd.data_ptr(), xd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert std.iterations == sth.iterations
    assert np.array_equal(xd.cpu().numpy(), xh)  # deterministic reductions: bit-identical


def test_mixed_precision_vcycle(gs, orc, device, p32):
    """FP32 V-cycle inside the FP64 flexible CG: the FP64-verified residual
    reaches 1e-8 and the iterate agrees with the FP64 oracle within the
    bound that residual implies (||dx||/||x|| <= cond * 2e-8, cond(P32) < 500)."""
    a, H, b = p32
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, precision=1, flexible=1, use_graph=1), device=device)
    x, st = s.solve(b)
    xo, it, _, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, precision=orc.PREC_MIXED, flexible=1)
    x64, it64, _, _ = orc.amg_pcg(A, P, R, b, tol=1e-12)
    assert true_residual(a, x, b) <= 1.5e-8
    assert abs(st.iterations - it) <= 1
    assert rel(x, x64) <= 1e-5


@pytest.fixture(scope="module")
def e8(gs):
    e = gs.elasticity(8)
    H = gs.Hierarchy.build(e, 3, 0.1, 10, 150)
    assert H.levels >= 2
    return e, H


@pytest.mark.parametrize("lanes,sliced", [(0, 0), (1, 0), (4, 0), (32, 0), (0, 2), (0, 4), (0, 8)])
def test_block_smoother_elasticity_matches_oracle(gs, orc, device, e8, lanes, sliced):
    e, H = e8
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(smoother=1, tol=1e-8, lanes=lanes, sliced_lanes=sliced), device=device)
    if sliced:
        assert all(l["sliced"] == 1 and l["lanes"] == sliced for l in s.level_info()[:-1])
    x, st = s.solve(e.rhs)
    xo, it, status, _ = orc.amg_pcg(A, P, R, e.rhs, smoother=1, tol=1e-8)
    assert status == 1 and abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10
    assert true_residual(e, x, e.rhs) <= 1.5e-8


def test_smallest_last_colouring_solves(gs, device, p32, e8):
    """coloring 1 (first-fit in smallest-last order): no more colours per level
    than the reference's greedy colouring, and the solve reaches the FP64-
    verified residual in FP64 and in the FP32 graph path (scalar and 3x3 block)."""
    for a, H, b, smoother in ((p32[0], p32[1], p32[2], 0), (e8[0], e8[1], e8[0].rhs, 1)):
        base = gs.Solver(H, gs.SolverOptions(smoother=smoother, tol=1e-8), device=device)
        for extra in (dict(), dict(precision=1, flexible=1, use_graph=1)):
            s = gs.Solver(H, gs.SolverOptions(smoother=smoother, tol=1e-8, coloring=1, **extra), device=device)
            assert all(c["colors"] <= g["colors"] for c, g in zip(s.level_info(), base.level_info()))
            x, st = s.solve(b)
            assert st.status == gs.STATUS_CONVERGED and true_residual(a, x, b) <= 1.5e-8


@pytest.mark.parametrize("graph", [0, 1])
@pytest.mark.parametrize("precision", [0, 1])
def test_overlapped_launch_is_bit_identical(gs, device, p32, e8, precision, graph):
    # Programmatic dependent launch (eager, or as programmatic edges of the
    # captured graph) changes when CTAs become resident, never the order of
    # the writes: the iterates must be the same bits.
    for a, H, b, smoother in ((p32[0], p32[1], p32[2], 0), (e8[0], e8[1], e8[0].rhs, 1)):
        out = []
        for ov in ((0, 1) if graph == 0 else (0, 1, 2)):
            o = gs.SolverOptions(smoother=smoother, tol=1e-8, precision=precision, flexible=precision,
                                 autotune=0, coarse_tail=0, overlap_launch=ov, use_graph=graph)
            s = gs.Solver(H, o, device=device)
            x, st = s.solve(b)
            out.append((x, st.iterations))
        for other in out[1:]:
            assert other[1] == out[0][1]
            assert np.array_equal(other[0], out[0][0])


def test_kuhn_and_weights(gs, orc, device):
    k = gs.kuhn_laplacian(16)
    H = gs.Hierarchy.build(k, 1, 0.1, 10, 300)
    A, P, R = levels(H)
    b = gs.uniform_rhs(k.rows, 1)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8), device=device)
    info = s.level_info()
    w = [np.linspace(0.9, 1.1, lv["colors"]) for lv in info]
    s.set_colour_weights(w)
    x, st = s.solve(b)
    xo, it, _, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, weights=w)
    assert abs(st.iterations - it) <= 1 and rel(x, xo) <= 1e-10


@pytest.mark.parametrize("variant", ["plain", "fast"])
def test_full_size_p128_converges(gs, device, variant):
    """128^3 heterogeneous Poisson at full size: FP64-verified residual."""
    a = gs.varcoef_grf(128)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 1000)
    b = gs.uniform_rhs(a.rows, 4)
    opts = gs.SolverOptions(tol=1e-8) if variant == "plain" else gs.SolverOptions(
        tol=1e-8, precision=1, flexible=1, use_graph=1)
    s = gs.Solver(H, opts, device=device)
    x, st = s.solve(b)
    assert st.status == gs.STATUS_CONVERGED
    assert true_residual(a, x, b) <= 2e-8


def test_kernel_timer(gs, device, p32):
    a, H, b = p32
    s = gs.Solver(H, gs.SolverOptions(), device=device)
    for kind in (0, 1, 2):
        assert s.time_kernel(kind, 3) > 0.0


def test_tail_runs_levels(gs, device, p32):
    a, H, b = p32
    s = gs.Solver(H, gs.SolverOptions(coarse_tail=2), device=device)
    info = s.level_info()
    assert info[0]["in_tail"] == 0 and all(lv["in_tail"] > 0 for lv in info[1:])
    s0 = gs.Solver(H, gs.SolverOptions(coarse_tail=0), device=device)
    assert not any(lv["in_tail"] for lv in s0.level_info())


def test_tail_mixed_precision_and_weights(gs, orc, device, p32):
    a, H, b = p32
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, coarse_tail=2), device=device)
    w = [np.linspace(0.85, 1.15, lv["colors"]) for lv in s.level_info()]
    s.set_colour_weights(w)
    x, st = s.solve(b)
    xo, it, _, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, weights=w)
    assert abs(st.iterations - it) <= 1 and rel(x, xo) <= 1e-10
    sm = gs.Solver(H, gs.SolverOptions(tol=1e-8, coarse_tail=2, precision=1, flexible=1), device=device)
    xm, stm = sm.solve(b)
    assert true_residual(a, xm, b) <= 1.5e-8


@pytest.mark.parametrize("dims", [(13, 11, 9), (8, 8, 16), (5, 13, 1), (17, 17, 17)])
def test_dense_spd_inverse(gs, device, dims):
    """The library's tiled Cholesky and inverse on the GPU (coarsest levels above
    1000 rows), against numpy's inverse; sizes below, at and off the 64-row
    tile (1287, 1024, 65, 4913 rows)."""
    a = gs.varcoef_loguniform(*dims, 0.1, 10.0, seed=5)
    inv = gs.dense_spd_inverse(a, device)
    ref = np.linalg.inv(a.to_scipy().toarray())
    assert np.linalg.norm(inv - ref) / np.linalg.norm(ref) <= 1e-11
    assert np.array_equal(inv, inv.T)  # the upper triangle mirrors the lower one


def test_dense_spd_inverse_rejects_indefinite(gs, device):
    """A pivot that is not positive -- at the first tile or only at the last one --
    is reported as "not SPD"."""
    a = gs.varcoef_loguniform(13, 11, 9, 0.1, 10.0, seed=5)
    bad = gs.Csr.from_scipy(-a.to_scipy())
    with pytest.raises(gs.SolverError, match="not SPD"):
        gs.dense_spd_inverse(bad, device)
    m = a.to_scipy().tolil()
    m[a.rows - 1, a.rows - 1] = -1.0
    with pytest.raises(gs.SolverError, match="not SPD"):
        gs.dense_spd_inverse(gs.Csr.from_scipy(m.tocsr()), device)


@pytest.mark.parametrize("coarse_rows", [700, 5000])
def test_dense_coarse_level_moves_up(gs, orc, device, p32, coarse_rows):
    """coarse_rows: the V-cycle ends with a dense solve on the first level with at most
    coarse_rows rows; same iterates as the oracle run on the truncated hierarchy."""
    a, H, b = p32
    A, P, R = levels(H)
    d = next(k + 1 for k in range(1, len(A)) if A[k].rows <= coarse_rows)
    assert d < len(A)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, coarse_rows=coarse_rows), device=device)
    assert len(s.level_info()) == d
    x, st = s.solve(b)
    xo, it, status, _ = orc.amg_pcg(A[:d], P[:d - 1], R[:d - 1], b, tol=1e-8)
    assert st.status == gs.STATUS_CONVERGED and abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10
    # mixed precision + graph with the moved coarse level
    sf = gs.Solver(H, gs.SolverOptions(tol=1e-8, coarse_rows=coarse_rows, precision=1, flexible=1,
                                       use_graph=1), device=device)
    xf, stf = sf.solve(b)
    assert true_residual(a, xf, b) <= 1.5e-8


@pytest.mark.parametrize("coarse_rows", [700, 5000])
def test_packed_dense_coarse_level(gs, orc, device, p32, coarse_rows):
    """packed_rows 0: the dense coarsest inverse kept as tiles of its lower
    triangle (the layout of levels above 8192 rows by default): FP64 iterates
    within 1e-10 of the oracle on the truncated hierarchy, the same bits on a
    second solve, and the FP32 graph path to the FP64-verified residual."""
    a, H, b = p32
    A, P, R = levels(H)
    d = next(k + 1 for k in range(1, len(A)) if A[k].rows <= coarse_rows)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, coarse_rows=coarse_rows, packed_rows=0), device=device)
    assert len(s.level_info()) == d and A[d - 1].rows > 64
    x, st = s.solve(b)
    xo, it, status, _ = orc.amg_pcg(A[:d], P[:d - 1], R[:d - 1], b, tol=1e-8)
    assert st.status == gs.STATUS_CONVERGED and abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10
    x2, _ = s.solve(b)
    assert np.array_equal(x, x2)
    sf = gs.Solver(H, gs.SolverOptions(tol=1e-8, coarse_rows=coarse_rows, packed_rows=0, precision=1, flexible=1,
                                       use_graph=1), device=device)
    xf, stf = sf.solve(b)
    assert stf.status == gs.STATUS_CONVERGED and true_residual(a, xf, b) <= 1.5e-8


@pytest.mark.parametrize("coarse_rows", [700, 5000])
def test_packed_dense_coarse_level_in_fp16_tiles(gs, orc, device, p32, coarse_rows):
    """coarse_half: the packed inverse stored as FP16 tiles with one FP32 scale
    each (FP32 V-cycle). The coarse correction is then exact to about 5e-4; the
    FP64 outer CG still reaches the FP64-verified residual, within 2
    iterations of FP32 tiles, and its answer is within 1e-7 of the FP64 oracle's
    solution to 1e-12 (the error the residual allows)."""
    a, H, b = p32
    A, P, R = levels(H)
    out = []
    for half in (0, 1):
        s = gs.Solver(H, gs.SolverOptions(tol=1e-8, coarse_rows=coarse_rows, packed_rows=0, precision=1,
                                          flexible=1, use_graph=1, coarse_half=half), device=device)
        x, st = s.solve(b)
        assert st.status == gs.STATUS_CONVERGED and true_residual(a, x, b) <= 1.5e-8
        out.append((x, st.iterations))
    assert out[1][1] <= out[0][1] + 2
    xo, _, _, _ = orc.amg_pcg(A, P, R, b, tol=1e-12)
    assert rel(out[1][0], xo) <= 1e-7


@pytest.mark.parametrize("coarse_rows", [700, 5000])
def test_fp16_tile_apply_on_tensor_cores(gs, device, p32, coarse_rows):
    """The FP16 tiles are applied with mma.sync (the vector as a scaled FP16
    part plus its FP16 remainder): one preconditioner application agrees with
    the FP32-tile apply to the tiles' storage precision, and repeats bit for
    bit."""
    torch = pytest.importorskip("torch")
    a, H, b = p32
    z = []
    for half in (0, 1):
        s = gs.Solver(H, gs.SolverOptions(tol=1e-8, coarse_rows=coarse_rows, packed_rows=0, precision=1,
                                          flexible=1, coarse_half=half), device=device)
        r = torch.tensor(b, dtype=torch.float64, device=f"cuda:{device}")
        out = []
        for _ in range(2):
            zz = torch.zeros_like(r)
            s.apply_preconditioner_device(r.data_ptr(), zz.data_ptr(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            out.append(zz.cpu().numpy())
        assert np.array_equal(out[0], out[1])
        z.append(out[0])
    assert np.all(np.isfinite(z[1]))
    assert rel(z[1], z[0]) <= 3e-3


JACOBI_FAMILY = {
    # name: (elasticity?, solver options, oracle options) -- the reference's preconditioner
    "multigrid_damped_jacobi": (False, dict(smoother=2, coarse_solver=0, coarse_steps=2, omega=0.8),
                                dict(smoother=2, coarse_solver=0, coarse_steps=2, omega=0.8)),
    "multigrid_damped_jacobi_fp32_graph": (False, dict(smoother=2, coarse_solver=0, coarse_steps=2, omega=0.8,
                                                       precision=1, flexible=1, use_graph=1),
                                           None),
    "multigrid_block_jacobi": (True, dict(smoother=3, coarse_solver=0, coarse_steps=3, omega=0.6),
                               dict(smoother=3, coarse_solver=0, coarse_steps=3, omega=0.6)),
    "multigrid_hybrid_block": (True, dict(smoother=1, coarse_smoother=3, coarse_solver=0, coarse_steps=3,
                                          omega=0.9),
                               dict(smoother=1, coarse_smoother=3, coarse_solver=0, coarse_steps=3, omega=0.9)),
    "hybrid_block_dense_coarse": (True, dict(smoother=1, coarse_smoother=3), dict(smoother=1, coarse_smoother=3)),
}


@pytest.mark.parametrize("case", sorted(JACOBI_FAMILY))
def test_jacobi_family_multigrid_matches_oracle(gs, orc, device, p32, e8, case):
    block, so, oo = JACOBI_FAMILY[case]
    if block:
        a, H = e8
        b = a.rhs
    else:
        a, H, b = p32
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, **so), device=device)
    x, st = s.solve(b)
    assert st.status == gs.STATUS_CONVERGED and true_residual(a, x, b) <= 1.5e-8
    if oo is not None:
        xo, it, status, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, **oo)
        assert status == 1 and abs(st.iterations - it) <= 1
        assert rel(x, xo) <= 1e-10


SINGLE_LEVEL = {
    # reference class: (block?, kind, steps, omega)
    "JacobiPreconditioner": (False, 2, 1, 1.0),
    "DampedJacobiPreconditioner": (False, 2, 3, 0.8),
    "SymmetricGaussSeidelPreconditioner": (False, 0, 2, 1.0),
    "IdentityPreconditioner": (False, 4, 1, 1.0),
    "BlockJacobiPreconditioner": (True, 3, 2, 0.7),
    "BlockGaussSeidelPreconditioner": (True, 1, 1, 1.0),
}


@pytest.mark.parametrize("name", sorted(SINGLE_LEVEL))
def test_single_level_preconditioners_match_oracle(gs, orc, device, name):
    """Single-level preconditioners: a one-level hierarchy of the CG's matrix, smoothed from z = 0."""
    block, kind, steps, omega = SINGLE_LEVEL[name]
    a = gs.elasticity(4) if block else gs.varcoef_loguniform(14, 12, 10, 0.5, 2.0, seed=12)
    b = a.rhs if block else gs.uniform_rhs(a.rows, 13)
    H = gs.Hierarchy.from_levels([a], [], [], 3 if block else 1)
    opts = dict(smoother=kind, coarse_solver=0, coarse_steps=steps, omega=omega)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, max_iter=3000, **opts), device=device)
    x, st = s.solve(b)
    xo, it, status, _ = orc.amg_pcg([a], [], [], b, tol=1e-8, max_iter=3000, **opts)
    assert st.status == gs.STATUS_CONVERGED and status == 1
    assert abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-9


def _galerkin(gs, A0, H, depth):
    """A'_0 = A0, A'_{k+1} = R_k A'_k P_k with the hierarchy's transfers (scipy)."""
    A = [A0]
    for k in range(depth - 1):
        A.append(gs.Csr.from_scipy((H.R(k).to_scipy() @ A[-1].to_scipy() @ H.P(k).to_scipy()).tocsr()))
    return A


REFRESH = {
    "fp64_dense_coarse": (False, dict(), dict()),
    "fp64_damped_jacobi": (False, dict(smoother=2, coarse_solver=0, coarse_steps=2, omega=0.8),
                           dict(smoother=2, coarse_solver=0, coarse_steps=2, omega=0.8)),
    "fast_graph_moved_coarse": (False, dict(precision=1, flexible=1, use_graph=1, coarse_rows=300), None),
    "block_sliced": (True, dict(smoother=1, sliced_lanes=4), dict(smoother=1)),
}


@pytest.mark.parametrize("case", sorted(REFRESH))
def test_update_matrix_values_matches_oracle(gs, orc, device, case):
    """Matrix-value refresh: the solver built on A, refreshed with A' (same sparsity), solves
    like the oracle on the hierarchy A'_{k+1} = R_k A'_k P_k with the same transfers."""
    block, so, oo = REFRESH[case]
    if block:
        a = gs.elasticity(7)
        H = gs.Hierarchy.build(a, 3, 0.1, 10, 120)
        # D A D on the stored pattern (explicit zeros kept): still SPD, new values
        d = 1.0 + 0.2 * np.sin(np.arange(a.rows))
        rows = np.repeat(np.arange(a.rows), np.diff(a.row_ptr))
        a2 = gs.Csr(a.rows, a.cols, a.row_ptr.copy(), a.col_idx.copy(), a.val * d[rows] * d[a.col_idx])
        b = a.rhs
    else:
        a = gs.varcoef_loguniform(16, 15, 14, 0.1, 10.0, seed=21)
        H = gs.Hierarchy.build(a, 1, 0.1, 10, 60)
        a2 = gs.varcoef_loguniform(16, 15, 14, 0.1, 10.0, seed=22)
        b = gs.uniform_rhs(a.rows, 23)
    assert np.array_equal(a2.row_ptr, a.row_ptr) and np.array_equal(a2.col_idx, a.col_idx)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, **so), device=device)
    s.solve(b)  # graphs captured on the old values
    s.update_matrix(a2.val)
    x, st = s.solve(b)
    assert st.status == gs.STATUS_CONVERGED and true_residual(a2, x, b) <= 1.5e-8
    if oo is not None:
        depth = len(s.level_info())
        A = _galerkin(gs, a2, H, depth)
        P = [H.P(k) for k in range(depth - 1)]
        R = [H.R(k) for k in range(depth - 1)]
        xo, it, status, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, **oo)
        assert status == 1 and abs(st.iterations - it) <= 1
        assert rel(x, xo) <= 1e-10



@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("layout", [dict(), dict(lanes=1), dict(lanes=8), dict(lanes=32), dict(sliced_lanes=2),
                                    dict(sliced_lanes=8)])
def test_cooperative_sweeps_are_bit_identical(gs, device, precision, layout):
    """One cooperative launch per smoothing step (grid barriers between the
    colours) against one launch per colour pass: the same bits, on a level
    structure with many colours (GRF 24^3, 4 levels), eager and graph-replayed."""
    a = gs.varcoef_grf(24, 8.0, 2.3, 4)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 100)
    b = gs.uniform_rhs(a.rows, 4)
    for graph in (0, 1):
        out = []
        for sweep in (0, 2):
            o = gs.SolverOptions(tol=1e-8, precision=precision, flexible=precision, use_graph=graph,
                                 autotune=0, coarse_tail=0, sweep_launch=sweep, **layout)
            s = gs.Solver(H, o, device=device)
            x, st = s.solve(b)
            out.append((x, st.iterations, st.status))
        assert out[0][2] == out[1][2] == gs.STATUS_CONVERGED
        assert out[0][1] == out[1][1]
        assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("sweep", [0, 2])
def test_skipped_repeat_pass_is_exact(gs, device, sweep):
    """With omega 1 the colour pass repeated where a sweep turns is skipped;
    colour weights of exactly 1 keep every pass (a weight disables the skip):
    the iterates must be the same bits."""
    a = gs.varcoef_grf(20, 8.0, 2.3, 4)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 100)
    b = gs.uniform_rhs(a.rows, 4)
    out = []
    for ones in (False, True):
        o = gs.SolverOptions(tol=1e-8, autotune=0, coarse_tail=0, sweep_launch=sweep, pre_steps=2, post_steps=2)
        s = gs.Solver(H, o, device=device)
        if ones:
            s.set_colour_weights([np.ones(lv["colors"]) for lv in s.level_info()])
        x, st = s.solve(b)
        out.append((x, st.iterations))
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


def test_cooperative_sweep_with_weights_matches_oracle(gs, orc, device):
    k = gs.kuhn_laplacian(16)
    H = gs.Hierarchy.build(k, 1, 0.1, 10, 300)
    A, P, R = levels(H)
    b = gs.uniform_rhs(k.rows, 1)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, sweep_launch=2, coarse_tail=0), device=device)
    w = [np.linspace(0.9, 1.1, lv["colors"]) for lv in s.level_info()]
    s.set_colour_weights(w)
    x, st = s.solve(b)
    xo, it, _, _ = orc.amg_pcg(A, P, R, b, tol=1e-8, weights=w)
    assert abs(st.iterations - it) <= 1 and rel(x, xo) <= 1e-10


def test_half_sweeps_block_smoother_matches_oracle(gs, orc, device, e8):
    """Forward block sweeps before and backward after the coarse correction,
    3x3 block smoother, against the oracle."""
    e, H = e8
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(smoother=1, tol=1e-8, half_sweeps=1), device=device)
    x, st = s.solve(e.rhs)
    xo, it, status, _ = orc.amg_pcg(A, P, R, e.rhs, smoother=1, tol=1e-8, half_sweeps=1)
    assert status == 1 and abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10
