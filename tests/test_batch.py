"""Batched solves of many systems (gs_batch_*): every (system, right-hand side)
pair must give what the single-system path gives for that pair.

Tolerances: with the FP64 V-cycle each pair's iterate is within 1e-10
relative of the FP64 oracle (the restated CGSolver + V-cycle) with iteration
counts within +-1; with the FP32 V-cycle each pair reaches an FP64-verified
true residual of 1.5e-8 and agrees with the oracle within the error bound that
residual implies (relative error <= cond(A) * relative residual, cond from
scipy's Lanczos).
"""
import numpy as np
import pytest

from conftest import cuda_available

# uneven systems of 2, 3 and 4 levels (min_dofs 40)
SIDES = [(6, 7, 5), (11, 9, 10), (16, 16, 16), (9, 14, 12), (20, 18, 17)]


def systems(gs, sides=SIDES, min_dofs=40):
    out = []
    for i, (nx, ny, nz) in enumerate(sides):
        a = gs.varcoef_loguniform(nx, ny, nz, 0.1, 10.0, seed=30 + i)
        out.append((a, gs.Hierarchy.build(a, 1, 0.1, 10, min_dofs)))
    return out


def rhs(gs, sys, nrhs, seed=7):
    return [np.stack([gs.uniform_rhs(a.rows, seed + 10 * i + j) for j in range(nrhs)])
            for i, (a, _) in enumerate(sys)]


def levels(H):
    return ([H.A(k) for k in range(H.levels)], [H.P(k) for k in range(H.levels - 1)],
            [H.R(k) for k in range(H.levels - 1)])


def condition_number(a):
    """lambda_max / lambda_min of an SPD matrix (scipy's Lanczos; shift-invert for the smallest)."""
    from scipy.sparse.linalg import eigsh
    m = a.to_scipy().tocsc()
    hi = eigsh(m, k=1, which="LA", return_eigenvectors=False)[0]
    lo = eigsh(m, k=1, sigma=0.0, which="LM", return_eigenvectors=False)[0]
    return float(hi / lo)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_batch_plan_covers_every_colour_once(gs):
    sys = systems(gs)
    Hs = [H for _, H in sys]
    depth = [H.levels for H in Hs]
    assert len(set(depth)) >= 2  # uneven depths
    st = gs.batch_plan_check(Hs)
    assert st["levels"] == max(depth)
    # passes: per level, twice the largest colour count among the systems smoothed there
    want = 0
    for k in range(max(depth) - 1):
        cols = [gs.greedy_coloring(H.A(k))[0] for H in Hs if H.levels - 1 > k]
        want += 2 * max(cols)
    assert st["passes"] == want
    assert st["items"] > 0


def test_batch_rejects_single_level_systems(gs):
    a = gs.poisson7(4)
    H1 = gs.Hierarchy.build(a, 1, 0.1, 10, 1000)  # 64 rows: one level
    assert H1.levels == 1
    with pytest.raises(gs.SolverError, match="two levels"):
        gs.batch_plan_check([H1])


@pytest.mark.skipif(cuda_available(), reason="checks the no-device error")
def test_batch_without_device_fails_loudly(gs):
    sys = systems(gs, SIDES[:2])
    with pytest.raises(gs.NoDeviceError):
        gs.Batch([H for _, H in sys], 2)


@pytest.mark.gpu
@pytest.mark.parametrize("nrhs", [1, 3, 4])
def test_batch_fp64_matches_oracle(gs, orc, device, nrhs):
    sys = systems(gs)
    B = gs.Batch([H for _, H in sys], nrhs, gs.SolverOptions(tol=1e-8), device=device)
    bs = rhs(gs, sys, nrhs)
    x, st = B.solve(B.pack(bs))
    xs = B.unpack(x)
    for i, (a, H) in enumerate(sys):
        A, P, R = levels(H)
        for j in range(nrhs):
            xo, it, status, _ = orc.amg_pcg(A, P, R, bs[i][j], tol=1e-8)
            s = st[i * nrhs + j]
            assert s.status == gs.STATUS_CONVERGED and status == 1
            assert abs(s.iterations - it) <= 1
            assert rel(xs[i][j], xo) <= 1e-10


@pytest.mark.gpu
def test_batch_matches_single_system_solver(gs, device):
    sys = systems(gs)
    opts = gs.SolverOptions(tol=1e-8, use_graph=1, flexible=1)
    B = gs.Batch([H for _, H in sys], 2, opts, device=device)
    bs = rhs(gs, sys, 2, seed=90)
    x, st = B.solve(B.pack(bs))
    xs = B.unpack(x)
    for i, (a, H) in enumerate(sys):
        s1 = gs.Solver(H, gs.SolverOptions(tol=1e-8, flexible=1), device=device)
        for j in range(2):
            x1, t1 = s1.solve(bs[i][j])
            assert abs(st[i * 2 + j].iterations - t1.iterations) <= 1
            assert rel(xs[i][j], x1) <= 1e-10


@pytest.mark.gpu
def test_batch_graph_replay_is_bit_identical(gs, device):
    sys = systems(gs)
    bs = rhs(gs, sys, 4, seed=50)
    out = []
    for graph in (0, 1):
        B = gs.Batch([H for _, H in sys], 4, gs.SolverOptions(tol=1e-8, use_graph=graph, lanes=4),
                     device=device)
        out.append(B.solve(B.pack(bs)))
    assert np.array_equal(out[0][0], out[1][0])
    assert [s.iterations for s in out[0][1]] == [s.iterations for s in out[1][1]]


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 32])
def test_batch_formats_match_oracle(gs, orc, device, lanes):
    sys = systems(gs, SIDES[1:4])
    B = gs.Batch([H for _, H in sys], 2, gs.SolverOptions(tol=1e-8, lanes=lanes), device=device)
    assert all(l["lanes"] == lanes for l in B.level_info())
    bs = rhs(gs, sys, 2, seed=11)
    x, st = B.solve(B.pack(bs))
    xs = B.unpack(x)
    for i, (a, H) in enumerate(sys):
        A, P, R = levels(H)
        for j in range(2):
            xo, it, _, _ = orc.amg_pcg(A, P, R, bs[i][j], tol=1e-8)
            assert abs(st[i * 2 + j].iterations - it) <= 1 and rel(xs[i][j], xo) <= 1e-10


@pytest.mark.gpu
def test_batch_mixed_precision(gs, orc, device):
    sys = systems(gs)
    opts = gs.SolverOptions(tol=1e-8, precision=1, flexible=1, use_graph=1)
    B = gs.Batch([H for _, H in sys], 4, opts, device=device)
    bs = rhs(gs, sys, 4, seed=21)
    x, st = B.solve(B.pack(bs))
    xs = B.unpack(x)
    cond = [condition_number(a) for a, _ in sys]
    for i, (a, H) in enumerate(sys):
        A, P, R = levels(H)
        for j in range(4):
            assert st[i * 4 + j].status == gs.STATUS_CONVERGED
            r = np.linalg.norm(bs[i][j] - a.to_scipy() @ xs[i][j]) / np.linalg.norm(bs[i][j])
            assert r <= 1.5e-8
            xo, _, _, _ = orc.amg_pcg(A, P, R, bs[i][j], tol=1e-10)
            assert rel(xs[i][j], xo) <= cond[i] * (r + 1e-10)


@pytest.mark.gpu
def test_batch_edge_cases(gs, device):
    """Zero right-hand side (x = 0), an exact initial guess (already converged,
    x untouched), the iteration limit, a NaN right-hand side (per-pair status,
    the other pairs unaffected) -- each as the single-system solver reports it."""
    sys = systems(gs, SIDES[:3])
    B = gs.Batch([H for _, H in sys], 4, gs.SolverOptions(tol=1e-8, use_graph=1), device=device)
    bs = rhs(gs, sys, 4, seed=5)
    x0 = [np.zeros_like(v) for v in bs]
    a1 = sys[1][0]
    exact = np.linspace(-1.0, 1.0, a1.rows)
    bs[0][1][:] = 0.0                     # zero rhs
    bs[1][2] = a1.to_scipy() @ exact      # exact initial guess below
    x0[1][2] = exact
    bs[2][3][5] = np.nan                  # non-finite
    x, st = B.solve(B.pack(bs), B.pack(x0))
    xs = B.unpack(x)
    assert st[0 * 4 + 1].status == gs.STATUS_ZERO_RHS and not xs[0][1].any()
    assert st[1 * 4 + 2].status == gs.STATUS_INITIAL_CONVERGED
    assert np.array_equal(xs[1][2], exact)
    assert st[2 * 4 + 3].status == gs.STATUS_NOT_FINITE
    for i in range(3):
        for j in range(4):
            if (i, j) in ((0, 1), (1, 2), (2, 3)):
                continue
            assert st[i * 4 + j].status == gs.STATUS_CONVERGED
    B.set_tolerance(1e-14, 3)
    x, st = B.solve(B.pack(rhs(gs, sys, 4, seed=6)))
    assert all(s.status == gs.STATUS_MAX_ITER and s.iterations == 3 for s in st)


@pytest.mark.gpu
def test_batch_device_entry_point(gs, device):
    import torch
    sys = systems(gs, SIDES[:3])
    B = gs.Batch([H for _, H in sys], 3, gs.SolverOptions(tol=1e-8), device=device)
    b = B.pack(rhs(gs, sys, 3, seed=8))
    xh, sth = B.solve(b)
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros_like(bd)
    std = B.solve_device(bd.data_ptr(), xd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert [s.iterations for s in std] == [s.iterations for s in sth]
    assert np.array_equal(xd.cpu().numpy(), xh)
    assert B.launch_count() > 0


@pytest.mark.gpu
def test_batch_dense_coarse_level_moves_up(gs, orc, device):
    """coarse_rows in a batch: every system stops at min(own depth, D), D the deepest first
    level with at most coarse_rows rows over the systems; each pair matches the oracle on
    its truncated hierarchy."""
    sys = systems(gs)
    T = 300
    depth = []
    for _, H in sys:
        rows = [H.A(k).rows for k in range(H.levels)]
        depth.append(next((k + 1 for k in range(1, len(rows)) if rows[k] <= T), len(rows)))
    D = max(depth)
    B = gs.Batch([H for _, H in sys], 2, gs.SolverOptions(tol=1e-8, coarse_rows=T), device=device)
    assert B.levels == D
    bs = rhs(gs, sys, 2, seed=77)
    x, st = B.solve(B.pack(bs))
    xs = B.unpack(x)
    for i, (a, H) in enumerate(sys):
        A, P, R = levels(H)
        d = min(H.levels, D)
        for j in range(2):
            xo, it, _, _ = orc.amg_pcg(A[:d], P[:d - 1], R[:d - 1], bs[i][j], tol=1e-8)
            assert abs(st[i * 2 + j].iterations - it) <= 1 and rel(xs[i][j], xo) <= 1e-10
