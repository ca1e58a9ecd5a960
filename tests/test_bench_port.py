"""bench.py without oracle/_ref: the cpu_baseline leg and the reference arm
time the oracle's FP32 restatement of the reference's CPU path (kind "port",
one thread) instead, and the restatement gives the reference's own answer
(same iterations, bit-identical iterate on one thread)."""
import argparse
import json

import numpy as np


def _levels(H):
    return ([H.A(k) for k in range(H.levels)], [H.P(k) for k in range(H.levels - 1)],
            [H.R(k) for k in range(H.levels - 1)])


def test_port_solve_equals_the_reference(gs, orc, monkeypatch):
    import bench
    a = gs.poisson7(16)
    b = gs.uniform_rhs(a.rows, 0)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 200)
    A, P, R = _levels(H)
    reference = None
    if orc.ref_available():
        orc.ref_set_threads(1)
        f32 = lambda m: orc.CsrView(m.rows, m.cols, m.row_ptr, m.col_idx, m.val.astype(np.float32).astype(np.float64))
        reference = orc.ref_amg_pcg([f32(m) for m in A], [f32(m) for m in P], [f32(m) for m in R],
                                    b.astype(np.float32), tol=bench.TOL, max_iter=200)
    monkeypatch.setattr(orc, "ref_available", lambda: False)
    x, it, ms, kind, cores, setup = bench.reference_cpu_solve(orc, A, P, R, b, 0, 200)
    assert kind == "port" and cores == 1 and setup is None and ms > 0
    assert np.linalg.norm(b - a.to_scipy() @ np.asarray(x)) / np.linalg.norm(b) < 1e-5
    if reference is not None:
        # the port rounds the levels to FP32 itself, exactly as the reference stores them
        xr, itr, _, _ = reference
        assert it == itr and np.array_equal(np.asarray(x).astype(np.float32), xr)


def test_reference_arm_line_with_the_port(gs, orc, monkeypatch, capsys):
    import bench
    monkeypatch.setattr(orc, "ref_available", lambda: False)
    args = argparse.Namespace(workload="p32", steps=3, warmup=3, gpus=1, ref_max_iter=200)
    bench.run_reference(args, 1, 0)
    lines = [json.loads(l) for l in capsys.readouterr().out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and "unavailable" not in line
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 1
    assert "restatement" in line["cpu_baseline"]["sample"]
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"] and line["true_residual"] < 1e-5


def test_cpu_baseline_leg_and_b64_sample(gs, orc, monkeypatch):
    """The CPU legs of the GPU arm (single system and the B64 sample), with
    the reference's code where it is built and with the port, on small cases."""
    import bench
    a = gs.poisson7(12)
    b = gs.uniform_rhs(a.rows, 0)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 200)
    mats = [gs.varcoef_loguniform(m, m, m, 0.1, 10.0, seed=i) for i, m in enumerate((6, 9, 7, 8))]
    rhs = [np.stack([gs.uniform_rhs(m.rows, 10 * i + j) for j in range(bench.B64_RHS)]) for i, m in enumerate(mats)]
    kinds = (["reference"] if orc.ref_available() else []) + ["port"]
    for kind in kinds:
        if kind == "port":
            monkeypatch.setattr(orc, "ref_available", lambda: False)
        cb = bench.cpu_baseline(argparse.Namespace(ref_max_iter=200), a, b, H, 1)
        assert cb["kind"] == kind and cb["unit"] == "ms" and cb["value"] > 0 and cb["cores"] >= 1 and cb["sample"]
        v, threads, sample, k = bench.b64_cpu_sample(gs, orc, mats, rhs, stride=2)
        assert k == kind and v > 0 and threads >= 1 and "systems [0, 2]" in sample
