"""Per-block scalings of the 3x3 block Gauss-Seidel smoother (learned
relaxation weights per node), through the C ABI: parity with the FP64 oracle
given the same weights, equivalence with omega for uniform weights, graph
replay after the weights change, and what the trained network gains on an
unseen instance of the elasticity distribution."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def levels(H):
    return ([H.A(k) for k in range(H.levels)], [H.P(k) for k in range(H.levels - 1)],
            [H.R(k) for k in range(H.levels - 1)])


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def e8(gs):
    e = gs.elasticity(8, 0.3, 2)
    return e, gs.Hierarchy.build(e, 3, 0.1, 10, 100)


@pytest.mark.parametrize("lanes", [0, 8])
def test_node_weights_match_oracle(gs, orc, device, e8, lanes):
    e, H = e8
    A, P, R = levels(H)
    s = gs.Solver(H, gs.SolverOptions(smoother=1, tol=1e-8, lanes=lanes), device=device)
    feats = s.node_features()
    assert feats.shape == (sum(m.rows // 3 for m in A), 8)
    assert np.all(np.isfinite(feats)) and np.abs(feats).max() <= 2
    rng = np.random.default_rng(3)
    nw = [rng.uniform(0.8, 1.2, m.rows // 3) for m in A]
    s.set_node_weights(nw)
    x, st = s.solve(e.rhs)
    xo, it, status, _ = orc.amg_pcg(A, P, R, e.rhs, smoother=1, tol=1e-8, node_weights=nw)
    assert status == 1 and st.status == gs.STATUS_CONVERGED
    assert abs(st.iterations - it) <= 1
    assert rel(x, xo) <= 1e-10


@pytest.mark.parametrize("precision", [0, 1])
def test_uniform_node_weights_equal_omega(gs, device, e8, precision):
    """Every node weighted 0.9 is the smoother with omega = 0.9, bit for bit."""
    e, H = e8
    out = []
    for mode in ("omega", "nodes"):
        o = gs.SolverOptions(smoother=1, tol=1e-8, precision=precision, flexible=precision, autotune=0,
                             omega=0.9 if mode == "omega" else 1.0)
        s = gs.Solver(H, o, device=device)
        if mode == "nodes":
            s.set_node_weights(np.full(len(s.node_features()), 0.9))
        out.append(s.solve(e.rhs))
    assert out[0][1].iterations == out[1][1].iterations
    assert np.array_equal(out[0][0], out[1][0])


def test_weights_changed_between_graph_replays(gs, device, e8):
    """The captured CUDA graph carries the weight pointers: setting and clearing
    colour and node weights rebuilds it, so a cleared solver equals a fresh one."""
    e, H = e8
    o = gs.SolverOptions(smoother=1, tol=1e-8, precision=1, flexible=1, use_graph=1, autotune=0)
    fresh = gs.Solver(H, o, device=device).solve(e.rhs)
    s = gs.Solver(H, o, device=device)
    s.set_colour_weights([np.full(lv["colors"], 0.7) for lv in s.level_info()])
    weighted = s.solve(e.rhs)
    s.set_colour_weights(None)
    cleared = s.solve(e.rhs)
    s.set_node_weights(np.full(len(s.node_features()), 0.7))
    nodes = s.solve(e.rhs)
    s.set_node_weights(None)
    cleared2 = s.solve(e.rhs)
    assert weighted[1].iterations != fresh[1].iterations or not np.array_equal(weighted[0], fresh[0])
    assert np.array_equal(nodes[0], weighted[0])  # 0.7 per node = 0.7 per colour
    for c in (cleared, cleared2):
        assert c[1].iterations == fresh[1].iterations and np.array_equal(c[0], fresh[0])


def test_learned_node_weights_on_unseen_instance(gs, device):
    """What the trained per-block scalings do on an unseen instance of the
    elasticity distribution (56^3 vertices, seed 400; training seeds 100-123),
    fast configuration. They gain on their training objective -- one V-cycle
    contracts a random error strictly more in the A-norm than with omega = 1 --
    but not in iterations: omega = 1 is already at the optimum of this smoother
    (uniform weights 0.8-1.2 all take 74-75 iterations) and the iterations are
    set by modes the smoother cannot reach. So the selector must keep omega = 1
    whenever the learned weights are not faster, and never install a slower
    configuration."""
    import torch
    from gpusolver_b200 import learned
    params = learned.load_params(learned.DEFAULT_NODE_PARAMS)
    if params is None:
        pytest.skip("no trained per-block scalings committed")
    a = gs.elasticity(56, 0.3, 400)
    H = gs.Hierarchy.build_ex(a, 3, 0.1, 10, 1000, aggregation=1, device=device)
    s = gs.Solver(H, learned.fast_block_options(), device=device)
    w = learned.node_weights_for(learned.Model(params), s)
    assert np.all((w > 0) & (w < 2)) and w.std() > 0  # weights do vary per node
    e0 = torch.tensor(np.random.default_rng(5).uniform(-1, 1, a.rows), device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    s.set_node_weights(None)
    rho_plain = s.error_reduction(e0.data_ptr(), st)
    s.set_node_weights(w)
    rho_learned = s.error_reduction(e0.data_ptr(), st)
    assert rho_learned < rho_plain  # the training objective improves (about 10 %)
    b = torch.tensor(a.rhs, device="cuda")
    j = learned.select_node_weights(s, w, b, repeats=3)
    print(f"error reduction plain {rho_plain:.4f} learned {rho_learned:.4f}; iterations plain "
          f"{j.iterations_plain} learned {j.iterations_learned}; ms plain {j.ms_plain:.2f} learned "
          f"{j.ms_learned:.2f}; use learned {j.use_learned}")
    assert abs(j.iterations_learned - j.iterations_plain) <= 1
    assert j.use_learned == (j.ms_learned < j.ms_plain)
