"""3x3 block Gauss-Seidel colour passes that bulk-copy each BELL-1 slice's
blocks to shared memory (sweep_launch 2 forces them on every level whose widest
slice fits, 0 keeps the register kernel): the same iterates bit for bit as the
register kernel, in FP64 and FP32 V-cycles, eager and graph-replayed, with
omega, node weights and half sweeps, and parity with the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def levels(H):
    return ([H.A(k) for k in range(H.levels)], [H.P(k) for k in range(H.levels - 1)],
            [H.R(k) for k in range(H.levels - 1)])


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def e12(gs):
    # 12^3 nodes: a fine level of 26 off-diagonal blocks per node row and
    # Galerkin levels of wider slices (the FP64 ones too wide to stage)
    e = gs.elasticity(12, 0.3, 2)
    return e, gs.Hierarchy.build(e, 3, 0.1, 10, 100)


def _solve(gs, device, H, b, sweep, **extra):
    o = gs.SolverOptions(smoother=1, tol=1e-8, autotune=0, sweep_launch=sweep, **extra)
    s = gs.Solver(H, o, device=device)
    return s, s.solve(b)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("extra", [dict(), dict(use_graph=1), dict(omega=0.8, pre_steps=2, post_steps=1),
                                   dict(half_sweeps=1), dict(overlap_launch=0)])
def test_staged_passes_are_bit_identical(gs, device, e12, precision, extra):
    e, H = e12
    out = []
    for sweep in (0, 2):
        s, (x, st) = _solve(gs, device, H, e.rhs, sweep, precision=precision, flexible=precision, **extra)
        info = s.level_info()
        if sweep == 2:
            assert info[0]["launch"] == 2  # the fine level runs the staged passes
        else:
            assert all(lv["launch"] == 0 for lv in info)
        out.append((x, st.iterations, st.status))
    assert out[0][2] == out[1][2] == gs.STATUS_CONVERGED
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("precision", [0, 1])
def test_staged_passes_with_node_weights_are_bit_identical(gs, device, e12, precision):
    e, H = e12
    rng = np.random.default_rng(5)
    out = []
    for sweep in (0, 2):
        o = gs.SolverOptions(smoother=1, tol=1e-8, autotune=0, sweep_launch=sweep, precision=precision,
                             flexible=precision)
        s = gs.Solver(H, o, device=device)
        nw = rng.uniform(0.8, 1.2, len(s.node_features())) if not out else nw
        s.set_node_weights(nw)
        out.append(s.solve(e.rhs))
    assert out[0][1].iterations == out[1][1].iterations
    assert np.array_equal(out[0][0], out[1][0])


def test_staged_passes_match_oracle(gs, orc, device, e12):
    e, H = e12
    A, P, R = levels(H)
    s, (x, st) = _solve(gs, device, H, e.rhs, 2)
    assert s.level_info()[0]["launch"] == 2
    xo, it, status, _ = orc.amg_pcg(A, P, R, e.rhs, smoother=1, tol=1e-8)
    assert status == 1 and st.status == gs.STATUS_CONVERGED
    assert abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10


def test_autotuned_staged_choice_is_recorded(gs, device, e12, tmp_path):
    """The autotuner times the staged passes against the register kernel on
    BELL-1 block levels; its choice is written to the tune cache and read back
    (the same per-level launch kinds and the same iterates)."""
    e, H = e12
    cache = str(tmp_path / "tune.txt")
    gs.set_tune_cache(cache)
    try:
        runs = []
        for _ in range(2):
            s = gs.Solver(H, gs.SolverOptions(smoother=1, tol=1e-8, precision=1, flexible=1), device=device)
            runs.append(([lv["launch"] for lv in s.level_info()], s.solve(e.rhs)))
    finally:
        gs.set_tune_cache(None)
    assert runs[0][0] == runs[1][0]
    assert all(k in (0, 2) for k in runs[0][0])
    assert np.array_equal(runs[0][1][0], runs[1][1][0])
