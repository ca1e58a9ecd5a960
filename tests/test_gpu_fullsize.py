"""Oracle parity at the benchmarked sizes, through the C ABI.

The plain FP64 drop-in on the full-size configs of the benchmark -- P128
(128^3 variable-coefficient Poisson, 2.1 M unknowns), K80 (Kuhn P1 Laplacian,
493 k unknowns), E64 (P1 elasticity with 3x3 block Gauss-Seidel, 786 k
unknowns) and the four largest B64 systems with all four right-hand sides
(batched) -- against the FP64 oracle (oracle/oracle.cc) run on the host cores
on the same hierarchy: iterates within 1e-10 relative, iteration counts
within +-1 (the tolerance the plain drop-in is held to).
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def levels(H):
    return ([H.A(k) for k in range(H.levels)], [H.P(k) for k in range(H.levels - 1)],
            [H.R(k) for k in range(H.levels - 1)])


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def plain_options(gs, smoother=0):
    # the benchmark's plain FP64 drop-in
    return gs.SolverOptions(smoother=smoother, tol=1e-8, max_iter=1000, coarse_solver=1)


@pytest.fixture(scope="module")
def fullsize(gs, orc):
    """The three single-system configs with their host-built hierarchies; the
    oracle solves start at once on host threads (the oracle releases the
    GIL) and each test waits for its own."""
    cases = {}
    for name in ("p128", "k80", "e64"):
        if name == "p128":
            a, block = gs.varcoef_grf(128, 8.0, 2.3, 4), 1
            b = gs.uniform_rhs(a.rows, 4)
        elif name == "k80":
            a, block = gs.kuhn_laplacian(80, 0.2, 1), 1
            b = gs.uniform_rhs(a.rows, 1)
        else:
            a, block = gs.elasticity(64, 0.3, 2), 3
            b = a.rhs
        cases[name] = (a, block, b, gs.Hierarchy.build(a, block, 0.1, 10, 1000))
    ex = ThreadPoolExecutor(max_workers=3)

    def oracle(name):
        a, block, b, H = cases[name]
        A, P, R = levels(H)
        return orc.amg_pcg(A, P, R, b, smoother=1 if block == 3 else 0, tol=1e-8)

    futures = {name: ex.submit(oracle, name) for name in ("e64", "p128", "k80")}
    yield cases, futures
    ex.shutdown(wait=True)


@pytest.mark.parametrize("name", ["p128", "k80", "e64"])
def test_full_size_plain_fp64_matches_oracle(gs, device, fullsize, name):
    cases, futures = fullsize
    a, block, b, H = cases[name]
    s = gs.Solver(H, plain_options(gs, 1 if block == 3 else 0), device=device)
    x, st = s.solve(b)
    xo, it, status, _ = futures[name].result()
    assert st.status == gs.STATUS_CONVERGED and status == 1
    assert abs(st.iterations - it) <= 1, (st.iterations, it)
    assert rel(x, xo) <= 1e-10, rel(x, xo)


def test_full_size_b64_largest_systems_match_oracle(gs, orc, device):
    """The four largest of the 64 seeded B64 systems, all four right-hand
    sides, solved in one batch; every (system, RHS) pair against the oracle."""
    u = gs.uniform_rhs(64, 3)
    sides = [16 + min(80, int((v + 1.0) / 2.0 * 81)) for v in u]
    big = sorted(range(64), key=lambda i: (-sides[i], i))[:4]
    mats = [gs.varcoef_loguniform(sides[i], sides[i], sides[i], 0.1, 10.0, seed=1000 * 3 + i) for i in big]
    bs = [np.stack([gs.uniform_rhs(a.rows, 100000 * 3 + 4 * i + j) for j in range(4)]) for i, a in zip(big, mats)]
    Hs = [gs.Hierarchy.build(a, 1, 0.1, 10, 1000) for a in mats]
    B = gs.Batch(Hs, 4, plain_options(gs), device=device)
    x, st = B.solve(B.pack(bs))
    xs = B.unpack(x)

    def oracle(pair):
        i, j = pair
        A, P, R = levels(Hs[i])
        return orc.amg_pcg(A, P, R, bs[i][j], tol=1e-8)

    pairs = [(i, j) for i in range(4) for j in range(4)]
    with ThreadPoolExecutor(max_workers=8) as ex:  # the oracle releases the GIL
        results = list(ex.map(oracle, pairs))
    for (i, j), (xo, it, status, _) in zip(pairs, results):
        s = st[i * 4 + j]
        assert s.status == gs.STATUS_CONVERGED and status == 1
        assert abs(s.iterations - it) <= 1, (i, j, s.iterations, it)
        assert rel(xs[i][j], xo) <= 1e-10, (i, j, rel(xs[i][j], xo))
