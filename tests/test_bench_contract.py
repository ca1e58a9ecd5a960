"""bench.py's reference arm on the host: the reference's CPU path on the
32^3 Poisson workload prints one JSON line with every key of the contract,
and under torchrun (two gloo ranks, 127.0.0.1) rank 0 alone prints it."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _ref_built():
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    return O.ref_available()


pytestmark = pytest.mark.skipif(not _ref_built(), reason="the reference's CPU library is not built")

ARGS = ["bench.py", "--impl", "reference", "--workload", "p32", "--steps", "3", "--warmup", "3"]


def _json_lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check_line(line, n_gpus):
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["n_gpus"] == n_gpus and line["steps"] == 3 and line["warmup"] == 3
    assert line["higher_is_better"] is False and line["unit"] == "ms" and line["value"] > 0
    assert line["config"]["workload"] == "p32" and line["config"]["n"] == 32 ** 3
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"] and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # 32^3 Poisson reaches 1e-8 in a handful of iterations; the FP64 true
    # residual of the FP32 reference path stays near FP32 rounding
    assert 1 <= line["iterations"] <= 20 and line["true_residual"] < 1e-5


def test_reference_arm_prints_the_contract_line():
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    out = subprocess.run([sys.executable] + ARGS, cwd=ROOT, env=env, check=True, capture_output=True, text=True,
                         timeout=600)
    lines = _json_lines(out.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 1)


def test_reference_arm_under_torchrun_prints_once():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port)] + ARGS + ["--gpus", "2"]
    out = subprocess.run(cmd, cwd=ROOT, check=True, capture_output=True, text=True, timeout=600)
    lines = _json_lines(out.stdout)
    assert len(lines) == 1
    _check_line(lines[0], 2)
