"""coloring 2 on the GPU: the coarse scalar Gauss-Seidel levels coloured by
their strong couplings (gs_relaxed_coloring), each pass reading its own
colour's rows from the iterate its sweep started with. FP64 iterates within
1e-10 of the oracle run with the same colourings and the same relaxed passes;
the FP32 graph path the same bits as eager launches; the preconditioner
stays symmetric."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THETA, RHO = 0.05, 0.5


def levels(H):
    return ([H.A(k) for k in range(H.levels)], [H.P(k) for k in range(H.levels - 1)],
            [H.R(k) for k in range(H.levels - 1)])


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def grf(gs):
    a = gs.varcoef_grf(24, 8.0, 2.3, 4)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 100)
    assert H.levels >= 3
    return a, H, gs.uniform_rhs(a.rows, 4)


def finest_colouring(gs, m, block):
    """The finest level's colouring under coloring 2 (as under 1): the greedy
    colouring, or the smallest-last one where it has fewer colours. It is a
    proper colouring, so the relaxed reads of the oracle never apply there."""
    if block == 3:
        grp, gci = gs.block_graph(m, 3)
        m = gs.Csr(len(grp) - 1, len(grp) - 1, grp, gci, np.ones(len(gci)))
    g = gs.greedy_coloring(m)
    if g[0] > 2:
        s = gs.smallest_last_coloring(m)
        if s[0] < g[0]:
            g = s
    return g[2], g[3]


def colourings(gs, A, block=1):
    out = [finest_colouring(gs, A[0], block)]
    for k in range(1, len(A)):
        nc, col, verts, offs = gs.relaxed_coloring(A[k], THETA, RHO, block=block)
        out.append((verts, offs))
    return out


@pytest.mark.parametrize("extra", [dict(), dict(pre_steps=2, post_steps=2), dict(half_sweeps=1),
                                   dict(omega=0.8)])
def test_relaxed_passes_match_oracle(gs, orc, device, grf, extra):
    a, H, b = grf
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, coloring=2, **extra), device=device)
    info = s.level_info()
    cols = colourings(gs, A)
    for k in range(1, len(info) - 1):
        assert info[k]["colors"] == len(cols[k][1]) - 1
    assert info[1]["colors"] < gs.greedy_coloring(A[1])[0]
    x, st = s.solve(b)
    okw = dict(tol=1e-8, colourings=cols, relaxed=1)
    if "pre_steps" in extra:
        okw.update(pre=extra["pre_steps"], post=extra["post_steps"])
    if "half_sweeps" in extra:
        okw.update(half_sweeps=1)
    if "omega" in extra:
        okw.update(omega=extra["omega"])
    xo, it, status, _ = orc.amg_pcg(A, P, R, b, **okw)
    assert status == 1 and st.status == gs.STATUS_CONVERGED
    assert abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10


@pytest.mark.parametrize("half", [0, 1])
def test_relaxed_graph_replay_is_bit_identical(gs, device, grf, half):
    a, H, b = grf
    out = []
    for graph, ov in ((0, 0), (0, 1), (1, 1), (1, 2)):
        o = gs.SolverOptions(tol=1e-8, coloring=2, precision=1, flexible=1, use_graph=graph, overlap_launch=ov,
                             autotune=0, half_sweeps=half)
        s = gs.Solver(H, o, device=device)
        x, st = s.solve(b)
        assert st.status == gs.STATUS_CONVERGED
        out.append((x, st.iterations))
    for x, it in out[1:]:
        assert it == out[0][1] and np.array_equal(x, out[0][0])


def test_relaxed_preconditioner_is_symmetric(gs, device, grf):
    """u^T M v = v^T M u for the FP64 preconditioner with relaxed coarse
    levels (forward and backward sweeps with the copies taken at each sweep's
    start form the pair S, S^T)."""
    torch = pytest.importorskip("torch")
    a, H, b = grf
    s = gs.Solver(H, gs.SolverOptions(tol=1e-8, coloring=2), device=device)
    rng = np.random.default_rng(7)
    u, v = rng.standard_normal(a.rows), rng.standard_normal(a.rows)
    res = []
    for vec in (u, v):
        r = torch.tensor(vec, dtype=torch.float64, device=f"cuda:{device}")
        z = torch.zeros_like(r)
        s.apply_preconditioner_device(r.data_ptr(), z.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        res.append(z.cpu().numpy())
    lhs, rhs = float(u @ res[1]), float(v @ res[0])
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs))


@pytest.fixture(scope="module")
def e12(gs):
    e = gs.elasticity(12, 0.3, 2)
    return e, gs.Hierarchy.build(e, 3, 0.1, 10, 100)


@pytest.mark.parametrize("extra", [dict(), dict(half_sweeps=1), dict(pre_steps=2, post_steps=2)])
def test_relaxed_block_passes_match_oracle(gs, orc, device, e12, extra):
    e, H = e12
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(smoother=1, tol=1e-8, coloring=2, **extra), device=device)
    info = s.level_info()
    cols = colourings(gs, A, 3)
    for k in range(len(info) - 1):
        assert info[k]["colors"] == len(cols[k][1]) - 1
    x, st = s.solve(e.rhs)
    okw = dict(smoother=1, tol=1e-8, colourings=cols, relaxed=1)
    if "pre_steps" in extra:
        okw.update(pre=2, post=2)
    if "half_sweeps" in extra:
        okw.update(half_sweeps=1)
    xo, it, status, _ = orc.amg_pcg(A, P, R, e.rhs, **okw)
    assert status == 1 and st.status == gs.STATUS_CONVERGED
    assert abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10


def _apply(gs, s, vec, device):
    import torch
    r = torch.tensor(vec, dtype=torch.float64, device=f"cuda:{device}")
    z = torch.zeros_like(r)
    s.apply_preconditioner_device(r.data_ptr(), z.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return z.cpu().numpy()


@pytest.mark.parametrize("half", [0, 1])
def test_relaxed_preconditioner_matches_oracle(gs, orc, device, grf, e12, half):
    """One application z = M r (FP64) with relaxed coarse levels, scalar and
    3x3 block, against the oracle given the same colourings: 1e-12."""
    pytest.importorskip("torch")
    cases = ((grf[1], grf[2], 0, 1), (e12[1], e12[0].rhs, 1, 3))
    for H, b, smoother, block in cases:
        A, P, R = levels(H)
        s = gs.Solver(H, gs.SolverOptions(smoother=smoother, tol=1e-8, coloring=2, half_sweeps=half), device=device)
        cols = colourings(gs, A, block)
        z = _apply(gs, s, b, device)
        zo = orc.precondition(A, P, R, b, smoother=smoother, half_sweeps=half, colourings=cols, relaxed=1)
        assert rel(z, zo) <= 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_relaxed_block_layouts_are_bit_identical(gs, device, e12, precision):
    """BELL-1 register passes, bulk-copy staged passes (sweep_launch 2) and graph
    replay: the same bits under the relaxed block colouring."""
    e, H = e12
    out = []
    for graph, sweep in ((0, 0), (0, 2), (1, 0), (1, 2)):
        o = gs.SolverOptions(smoother=1, tol=1e-8, coloring=2, precision=precision, flexible=precision,
                             use_graph=graph, sweep_launch=sweep, autotune=0)
        s = gs.Solver(H, o, device=device)
        x, st = s.solve(e.rhs)
        out.append((x, st.iterations))
    for x, it in out[1:]:
        assert it == out[0][1] and np.array_equal(x, out[0][0])
