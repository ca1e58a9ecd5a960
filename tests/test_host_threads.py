"""The host setup's parallel loops give the same bits on one thread as on all
of them: hierarchies (both aggregations, scalar and 3x3 block), the
permutation, the node graph and the colourings, built in fresh processes with
GS_HOST_THREADS=1 and without it."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import hashlib, sys
sys.path.insert(0, "gpu-conjugate-gradient-solver_b200")
import numpy as np
import gpusolver_b200 as gs
h = hashlib.sha256()
def add(*arrays):
    for x in arrays:
        h.update(np.ascontiguousarray(x).tobytes())
for a, block in ((gs.varcoef_grf(40, 8.0, 2.3, 4), 1), (gs.kuhn_laplacian(24, seed=3), 1), (gs.elasticity(16), 3)):
    for aggregation in (0, 1):
        H = gs.Hierarchy.build_ex(a, block, 0.1, 10, 200, aggregation=aggregation, device=-1)
        for k in range(H.levels):
            m = H.A(k)
            add(m.row_ptr, m.col_idx, m.val)
            if k + 1 < H.levels:
                for m in (H.P(k), H.R(k)):
                    add(m.row_ptr, m.col_idx, m.val)
                add(H.aggregates(k, block))
    o2n, n2o = gs.rcm(a)
    pm = gs.permute_matrix(a, o2n, o2n)
    add(pm.row_ptr, pm.col_idx, pm.val)
    add(*gs.greedy_coloring(a)[1:], *gs.smallest_last_coloring(a)[1:])
    if block == 3:
        add(*gs.block_graph(a))
print(h.hexdigest())
"""


def _digest(threads):
    env = dict(os.environ)
    env.pop("GS_HOST_THREADS", None)
    if threads is not None:
        env["GS_HOST_THREADS"] = str(threads)
    out = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env, check=True, capture_output=True,
                         text=True, timeout=600)
    return out.stdout.strip()


def test_host_setup_is_independent_of_the_thread_count(gs):
    one = _digest(1)
    assert len(one) == 64
    assert _digest(None) == one
    assert _digest(3) == one
