"""The oracle's product-free workload path: numpy restatements of the
benchmark generators (oracle/workloads.py: the Poissons, the GRF and
log-uniform coefficients, the Kuhn-tetrahedra Laplacian, P1 elasticity, the
right-hand sides) and the C++ smoothed-aggregation
restatement (oracle/sa.cc) against the product's generators and host build,
and the benchmark's reference arm loading no product code."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _same(x, y):
    return (x.rows == y.rows and np.array_equal(x.row_ptr, y.row_ptr) and np.array_equal(x.col_idx, y.col_idx)
            and np.array_equal(x.val, y.val))


def test_generators_bit_identical(gs):
    from oracle import workloads as W
    for side in (7, 16, 33):
        assert _same(gs.varcoef_grf(side, 8.0, 2.3, 4), W.varcoef7(side, side, side,
                                                                   W.grf_coefficients(side, side, side, 8.0, 2.3, 4)))
    assert _same(gs.poisson7(11), W.poisson7(11))
    assert _same(gs.poisson7(5, 7, 3), W.poisson7(5, 7, 3))
    assert _same(gs.varcoef_loguniform(9, 9, 9, 0.1, 10.0, seed=3007),
                 W.varcoef7(9, 9, 9, W.loguniform_coefficients(729, 0.1, 10.0, 3007)))
    for n, seed in ((1, 0), (1000, 4), (4097, 300012)):
        assert np.array_equal(gs.uniform_rhs(n, seed), W.uniform_rhs(n, seed))
    # the Kuhn-tetrahedra P1 Laplacian (K80's generator), jittered and not
    for m, jitter, seed in ((2, 0.2, 1), (5, 0.0, 3), (9, 0.2, 1), (14, 0.3, 7)):
        assert _same(gs.kuhn_laplacian(m, jitter, seed), W.kuhn_laplacian(m, jitter, seed))
    # the P1 elasticity system (E64's generator) and its body-force RHS
    for v, nu, seed in ((2, 0.3, 2), (6, 0.25, 9), (11, 0.3, 2)):
        e = gs.elasticity(v, nu, seed)
        a, rhs = W.elasticity_p1(v, nu, seed)
        assert _same(e, a) and np.array_equal(e.rhs, rhs)


@pytest.mark.parametrize("case", ["poisson16", "grf24", "kuhn12", "elasticity8"])
def test_sa_restatement_equals_host_build(gs, orc, case):
    """Bit for bit: every level, P and R of the oracle's C++ smoothed
    aggregation equal the product's host build (sequential aggregation)."""
    a, block = {"poisson16": (lambda: gs.poisson7(16), 1), "grf24": (lambda: gs.varcoef_grf(24, 8.0, 2.3, 4), 1),
                "kuhn12": (lambda: gs.kuhn_laplacian(12, 0.2, 1), 1),
                "elasticity8": (lambda: gs.elasticity(8, 0.3, 2), 3)}[case]
    a = a()
    H = gs.Hierarchy.build(a, block, 0.1, 10, 200)
    A, P, R = orc.sa_hierarchy(a, block, 0.1, 10, 200)
    assert len(A) == H.levels >= 2
    for k in range(H.levels):
        assert _same(H.A(k), A[k])
        if k + 1 < H.levels:
            assert _same(H.P(k), P[k]) and _same(H.R(k), R[k])


def test_sa_restatement_equals_numpy_restatement(gs, orc):
    a = gs.varcoef_grf(12, 8.0, 2.3, 4)
    An, Pn, Rn, _ = orc.build_hierarchy(a, 1, 0.1, 10, 100)
    A, P, R = orc.sa_hierarchy(a, 1, 0.1, 10, 100)
    assert len(A) == len(An)
    for k in range(len(A)):
        d = np.abs(An[k].toarray() - A[k].to_scipy().toarray()).max()
        assert d <= 1e-13 * np.abs(An[k].toarray()).max()


def test_reference_arm_loads_no_product_code(tmp_path):
    """bench.py --impl reference, run in a fresh process: the product's
    package is never imported and its shared library never mapped."""
    probe = (
        "import runpy, sys, json\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'p32', '--steps', '1', '--warmup', '0']\n"
        f"runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'module': 'gpusolver_b200' in sys.modules, 'so': 'libgpusolver_b200' in maps}))\n")
    out = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    line, flags = lines[0], lines[-1]
    assert line["impl"] == "reference" and "unavailable" not in line and line["value"] > 0
    assert line["iterations"] > 0 and "note" in line
    assert flags == {"module": False, "so": False}
