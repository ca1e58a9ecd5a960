#!/usr/bin/env python
"""AMG-preconditioned CG, time to relative residual 1e-8 on one B200.

One step = one complete solve of the workload's linear system to a relative
recurrence residual of 1e-8 (the result is re-checked with an FP64 true
residual on the host after the timed region). Inputs are resident in HBM when
the timed region starts; between timed solves the L2 is flushed, and the
default workload is larger than L2 anyway.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload p128]
                    [--impl ours|reference]

With --gpus N > 1 (launched by torchrun) every rank solves its own replica
of the system: the path has no data-parallel exchange step, so there is no
collective in the solve (weak scaling, replicas only). Rank 0 prints one
JSON line.

`--impl reference` times the reference's own CPU implementation (compiled
from its sources into oracle/_ref) on the host cores with every host thread,
same workload, metric and unit; under torchrun only rank 0 runs it. Where
oracle/_ref was not built, it and the cpu_baseline leg time the oracle's FP32
restatement of the same path on one thread instead (kind "port").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-conjugate-gradient-solver_b200"))
sys.path.insert(0, ROOT)

TOL = 1e-8
# Fast variants: the V-cycle's dense coarsest solve moves up to the first level
# with at most this many rows (one bandwidth-bound matvec instead of ~150
# latency-bound colour passes); batched: the deepest such level over the systems.
FAST_COARSE_ROWS = 24576
FAST_BATCH_COARSE_ROWS = 4096
METRIC = "AMG-PCG time-to-1e-8 residual (FP64-verified), 1 B200"

WORKLOADS = {
    "p128": dict(desc="128^3 variable-coefficient 7-point Poisson, k = exp(2.3 GRF, corr. length 8 cells), "
                      "harmonic face averaging, seed 4; RHS U[-1,1] seed 4",
                 block=1, rhs_seed=4),
    "p32": dict(desc="32^3 7-point Poisson, Dirichlet 0; RHS U[-1,1] seed 0", block=1, rhs_seed=0),
    "k80": dict(desc="Kuhn-tetrahedra P1 Laplacian, 80^3 cubes, jitter 0.2h seed 1; RHS U[-1,1] seed 1",
                block=1, rhs_seed=1),
    "e64": dict(desc="P1 linear elasticity, 64^3 vertices, E = exp(N(0,1)) seed 2, nu 0.3, x=0 clamped, "
                     "unit body force -z; 3x3 block GS, node aggregation", block=3, rhs_seed=None),
    "b64": dict(desc="64 independent 7-point variable-coefficient Poissons, sides U{16..96} (seed 3), "
                     "cell coefficients log-uniform [0.1, 10] (seed 3000 + s), 4 RHS U[-1,1] each "
                     "(seed 300000 + 4 s + j): 256 solves, one batched solve per step",
                block=1, rhs_seed=None),
}

B64_SYSTEMS, B64_RHS, B64_SEED = 64, 4, 3


def b64_problems(gs, count=B64_SYSTEMS, seed=B64_SEED):
    """Sides U{16..96} from SplitMix64(seed) (the library's uniform_rhs stream
    mapped from [-1, 1]); per system the log-uniform coefficient field and
    B64_RHS right-hand sides."""
    u = gs.uniform_rhs(count, seed)
    sides = [16 + min(80, int((v + 1.0) / 2.0 * 81)) for v in u]
    mats = [gs.varcoef_loguniform(m, m, m, 0.1, 10.0, seed=1000 * seed + i) for i, m in enumerate(sides)]
    rhs = [np.stack([gs.uniform_rhs(a.rows, 100000 * seed + B64_RHS * i + j) for j in range(B64_RHS)])
           for i, a in enumerate(mats)]
    return sides, mats, rhs


def build_hierarchies(gs, mats):
    """SA hierarchies of all systems, several at a time (ctypes releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda a: gs.Hierarchy.build(a, 1, 0.1, 10, 1000), mats))


def make_problem(gs, name):
    if name == "p128":
        a = gs.varcoef_grf(128, 8.0, 2.3, 4)
    elif name == "p32":
        a = gs.poisson7(32)
    elif name == "k80":
        a = gs.kuhn_laplacian(80, 0.2, 1)
    elif name == "e64":
        a = gs.elasticity(64, 0.3, 2)
    else:
        raise SystemExit(f"unknown workload {name}")
    w = WORKLOADS[name]
    b = a.rhs if w["rhs_seed"] is None else gs.uniform_rhs(a.rows, w["rhs_seed"])
    return a, b


def solver_options(gs, variant, block):
    smoother = 1 if block == 3 else 0
    if variant == "plain":
        # The plain FP64 drop-in: FP64 V-cycle, the reference's CG update,
        # host-checked iteration like CGSolver::solve.
        return gs.SolverOptions(smoother=smoother, tol=TOL, max_iter=1000, coarse_solver=1)
    # FP32 V-cycle inside an FP64 flexible (Polak-Ribiere) CG, graph-replayed,
    # dense coarsest solve on the first level of at most FAST_COARSE_ROWS rows,
    # first-fit colouring in smallest-last order on the finest level and of the
    # strong couplings on the coarse scalar levels (coloring 2), a forward sweep before and a
    # backward sweep after the coarse correction (half_sweeps), and a packed
    # dense inverse in FP16 tiles applied on the tensor cores (coarse_half).
    return gs.SolverOptions(smoother=smoother, tol=TOL, max_iter=1000, coarse_solver=1,
                            precision=1, flexible=1, use_graph=1, coarse_rows=FAST_COARSE_ROWS, coloring=2,
                            half_sweeps=1, coarse_half=1)


FALLBACK_HBM_GBS = 6650.0


def _peak_number(v):
    """A peak given as a number, a numeric string, or an object holding one
    under a value-like key."""
    if isinstance(v, bool):
        return None
    if isinstance(v, (int, float)):
        return float(v) if v > 0 else None
    if isinstance(v, str):
        try:
            return _peak_number(float(v))
        except ValueError:
            return None
    if isinstance(v, dict):
        for key in ("value", "gbs", "GBps", "gb_s", "median", "burst", "mean"):
            if key in v:
                x = _peak_number(v[key])
                if x is not None:
                    return x
    return None


def load_peaks(path=None):
    """HBM copy bandwidth in GB/s for the roofline denominator: the measured
    figure from MEASURED_PEAKS.json when it is there and readable, else the
    earlier measurement on this hardware (6.65 TB/s), labelled "fallback"."""
    path = path or os.path.join(ROOT, "MEASURED_PEAKS.json")
    if not os.path.exists(path):
        return FALLBACK_HBM_GBS, "fallback"
    try:
        with open(path) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return FALLBACK_HBM_GBS, "fallback (MEASURED_PEAKS.json unreadable)"
    if isinstance(d, dict):
        for key in ("hbm_gbs", "hbm_GBps", "hbm_gb_s", "hbm"):
            if key in d:
                x = _peak_number(d[key])
                if x is not None:
                    return x, "measured"
    return FALLBACK_HBM_GBS, "fallback (no HBM figure in MEASURED_PEAKS.json)"


def load_traffic(workload):
    """Per-launch DRAM bytes of the roofline kernel from the committed ncu
    summary (profiles/roofline_traffic.txt: `<workload> <kernel> <bytes>`)."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    if not os.path.exists(path):
        return {}
    out = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#") and parts[0] == workload:
                out[parts[1]] = float(parts[2])
    return out


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region.

    nvidia-smi samples every INTERVAL_MS with its own timestamp; start()
    returns once the first sample has arrived (at most 3 s), so the loop runs
    before the timed region begins, and stop() keeps the samples whose
    timestamps fall between start() returning and stop() being called (an
    idle GPU before or after the region reports its idle clock)."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 50

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.INTERVAL_MS), "-i", str(self.dev)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.time() + 3.0
            while not self.lines and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.005)
        except Exception:
            self.proc = None
        self.t0 = time.time()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    @staticmethod
    def _stamp(text):
        import datetime
        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(text, fmt).timestamp()
            except ValueError:
                continue
        return None

    def stop(self):
        self.t1 = time.time()
        if self.proc is None:
            return None
        time.sleep(self.INTERVAL_MS / 1000.0)  # the sample that covers the region's end
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        rows = []
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 10:
                continue
            try:
                rows.append((self._stamp(p[0]), float(p[2]), float(p[3]), p[6:10]))
            except ValueError:
                continue
        if not rows:
            return None
        slack = self.INTERVAL_MS / 1000.0
        inside = [r for r in rows if r[0] is not None and self.t0 <= r[0] <= self.t1 + slack]
        in_window = bool(inside)
        if not inside:  # region shorter than one interval: the sample nearest to it
            stamped = [r for r in rows if r[0] is not None]
            mid = 0.5 * (self.t0 + self.t1)
            inside = [min(stamped, key=lambda r: abs(r[0] - mid))] if stamped else rows[-1:]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, clk, cmax, flags in inside:
            sm.append(clk)
            mx = cmax
            for name, val in zip(names, flags):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "in_window": in_window}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if args.impl == "ours" else "gloo"
        import datetime
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def algorithmic_bytes(nnz, n, s, kind):
    """Byte model: SpMV nnz (s + 4) + 2 n s; one GS sweep nnz (s + 4) + 4 n s;
    3x3 blocks: nb (9 s + 4) + 2 N s (+ 9 s per node for D^-1 in GS)."""
    if kind == "spmv":
        return nnz * (s + 4) + 2 * n * s
    return nnz * (s + 4) + 4 * n * s


def block_algorithmic_bytes(nblocks, n, s, kind):
    if kind == "spmv":
        return nblocks * (9 * s + 4) + 2 * n * s
    return nblocks * (9 * s + 4) + 4 * n * s + (n // 3) * 9 * s


def reference_inputs(name):
    """The workload built without the product library: the oracle's numpy
    restatement of the product's generators (bit-identical arrays) and the
    oracle's C++ smoothed-aggregation hierarchy (bit-identical to the
    product's host build), so that the reference arm maps no product code."""
    from oracle import oracle as O, workloads as W
    if name == "p128":
        a, b = W.p128()
    elif name == "p32":
        a = W.poisson7(32)
        b = W.uniform_rhs(a.rows, WORKLOADS["p32"]["rhs_seed"])
    elif name == "k80":
        a, b = W.k80()
    elif name == "e64":
        a, b = W.e64()
    else:
        raise ValueError(name)
    A, P, R = O.sa_hierarchy(a, WORKLOADS[name]["block"], 0.1, 10, 1000)
    return a, b, A, P, R


def reference_b64_inputs(count=B64_SYSTEMS, seed=B64_SEED):
    """b64_problems without the product library (same seeds, same arrays)."""
    from oracle import workloads as W
    u = W.uniform_rhs(count, seed)
    sides = [16 + min(80, int((v + 1.0) / 2.0 * 81)) for v in u]
    mats = [W.varcoef7(m, m, m, W.loguniform_coefficients(m ** 3, 0.1, 10.0, 1000 * seed + i))
            for i, m in enumerate(sides)]
    rhs = [np.stack([W.uniform_rhs(a.rows, 100000 * seed + B64_RHS * i + j) for j in range(B64_RHS)])
           for i, a in enumerate(mats)]
    return sides, mats, rhs


REFERENCE_NOTE = ("the reference's FP32 CG stops when its recurrence residual reaches 1e-8; its FP64 true "
                  "residual stays near 1e-5 (reported as true_residual), while the GPU arm's 1e-8 is "
                  "verified by an FP64 true residual")


def run_reference(args, world, rank):
    """Reference arm: the reference's FP32 CPU path on the host cores. Inputs
    and hierarchy come from the oracle (oracle/workloads.py, oracle/sa.cc);
    this arm never loads the product library."""
    if rank != 0:
        return
    from oracle import oracle as O
    if args.workload == "b64":
        sides, mats, rhs = reference_b64_inputs()
        times = []
        for step in range(args.warmup + args.steps):
            v, threads, sample, kind = b64_cpu_sample(None, O, mats, rhs, stride=16)
            if step >= args.warmup:
                times.append(v)
        ms = float(np.mean(times))
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "b64", "desc": WORKLOADS["b64"]["desc"], "systems": len(mats),
                       "rhs_per_system": B64_RHS, "unknowns": sum(a.rows for a in mats)},
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": REFERENCE_NOTE,
        }), flush=True)
        return
    a, b, A, P, R = reference_inputs(args.workload)
    # The reference's block Gauss-Seidel reads the colour range as (start, end)
    # and does not converge past colour 0, so on the 3x3 block hierarchy its
    # scalar multicolour SGS preconditioner is timed (as the E64 leg does).
    smoother = 0
    times, iters, res = [], [], []
    for step in range(args.warmup + args.steps):
        x, it, solve_ms, kind, threads, _ = reference_cpu_solve(O, A, P, R, b, smoother, args.ref_max_iter)
        if step >= args.warmup:
            times.append(solve_ms)
            iters.append(it)
            res.append(float(np.linalg.norm(b - a.to_scipy() @ np.asarray(x, np.float64)) / np.linalg.norm(b)))
    ms = float(np.mean(times))
    sample = (f"full solve of {args.workload} per step by {_path_name(kind)}: CGSolver + "
              f"MultigridGaussSeidelPreconditioner"
              f"{' (its block variant does not converge: colour range read as (start, end))' if WORKLOADS[args.workload]['block'] == 3 else ''}"
              f" (1 pre, 1 post, 1 V-cycle, omega 1), FP32, tol 1e-8 on the "
              f"recurrence residual, {iters[-1]} iterations, FP64 true residual {res[-1]:.2e}; "
              f"setup excluded")
    line = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"],
                   "n": a.rows, "nnz": a.nnz, "levels": len(A),
                   "inputs": "oracle restatement of the generators and the host SA build (no product code)"},
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iterations": iters[-1], "true_residual": res[-1], "note": REFERENCE_NOTE,
    }
    print(json.dumps(line), flush=True)


def reference_cpu_solve(O, A, P, R, b, smoother, max_iter):
    """One solve of the reference's FP32 CPU path (CGSolver + Multigrid{GaussSeidel,
    BlockGaussSeidel}Preconditioner, 1 pre / 1 post step, 1 V-cycle) to TOL: the
    reference's own code (oracle/_ref, every host thread) when it was built,
    else the oracle's FP32 restatement of it (one thread; bit-identical to the
    reference's scalar path on one thread), timed around the call.
    Returns (x, iterations, solve ms, kind, cores, setup ms or None)."""
    if O.ref_available():
        threads = os.cpu_count() or 1
        O.ref_set_threads(threads)
        x, it, setup_ms, solve_ms = O.ref_amg_pcg(A, P, R, b, smoother=smoother, tol=TOL, max_iter=max_iter)
        return x, it, solve_ms, "reference", threads, setup_ms
    t0 = time.perf_counter()
    x, it, _, _ = O.amg_pcg(A, P, R, np.asarray(b, np.float64), precision=O.PREC_F32, smoother=smoother,
                            coarse_solver=0, alias=1, tol=TOL, max_iter=max_iter)
    return x, it, (time.perf_counter() - t0) * 1e3, "port", 1, None


def _path_name(kind):
    return ("the reference's FP32 CPUBackend path" if kind == "reference"
            else "the oracle's FP32 restatement of the reference's CPU path (oracle/_ref not built)")


def cpu_baseline(args, a, b, H, block):
    """The reference's CPU path on a bounded sample of the same workload."""
    from oracle import oracle as O
    A = [H.A(k) for k in range(H.levels)]
    P = [H.P(k) for k in range(H.levels - 1)]
    R = [H.R(k) for k in range(H.levels - 1)]
    smoother = 1 if block == 3 else 0
    x, it, solve_ms, kind, cores, setup_ms = reference_cpu_solve(O, A, P, R, b, smoother, args.ref_max_iter)
    res = float(np.linalg.norm(b - a.to_scipy() @ np.asarray(x, np.float64)) / np.linalg.norm(b))
    setup = f"setup {setup_ms:.0f} ms excluded" if setup_ms is not None else "level conversion included"
    return {"value": solve_ms, "unit": "ms", "cores": cores, "kind": kind,
            "sample": f"one full solve of the same system by {_path_name(kind)} "
                      f"({it} iterations to recurrence residual 1e-8, FP64 true residual {res:.2e}, {setup})"}


def shard_systems(rows, world, rank):
    """Systems (by size) of `rank` out of `world`: largest first to the least-loaded rank,
    ties to the lowest rank; every system goes to exactly one rank."""
    order = sorted(range(len(rows)), key=lambda i: (-rows[i], i))
    load, mine = [0] * world, []
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += rows[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def b64_cpu_sample(gs, O, mats, rhs, stride=8):
    """The reference's FP32 CPU path on every `stride`-th system (first
    right-hand side), extrapolated to all systems and right-hand sides by
    unknowns: returns (ms for the whole batch, sample description)."""
    idx = list(range(0, len(mats), stride))
    if gs is None:  # the reference arm: the oracle's hierarchy, no product code
        Hs = [O.sa_hierarchy(mats[i], 1, 0.1, 10, 1000) for i in idx]
    else:
        Hs = [(tuple(H.A(k) for k in range(H.levels)), tuple(H.P(k) for k in range(H.levels - 1)),
               tuple(H.R(k) for k in range(H.levels - 1))) for H in build_hierarchies(gs, [mats[i] for i in idx])]
    ms, rows, its, res = 0.0, 0, [], []
    kind, threads = "reference", 1
    for (A, P, R), i in zip(Hs, idx):
        a, b = mats[i], rhs[i][0]
        x, it, solve_ms, kind, threads, _ = reference_cpu_solve(O, A, P, R, b, 0, 200)
        ms += solve_ms
        rows += a.rows
        its.append(it)
        res.append(float(np.linalg.norm(b - a.to_scipy() @ np.asarray(x, np.float64)) / np.linalg.norm(b)))
    total = sum(a.rows for a in mats) * B64_RHS
    value = ms / rows * total
    sample = (f"{_path_name(kind)} (CGSolver + MultigridGaussSeidelPreconditioner, "
              f"tol 1e-8) on systems {idx} (first RHS each, {rows} unknowns, {ms:.0f} ms, "
              f"{min(its)}-{max(its)} iterations, FP64 true residual up to {max(res):.1e}), "
              f"extrapolated by unknowns to all {len(mats)} systems x {B64_RHS} RHS; setup excluded")
    return value, threads, sample, kind


def run_b64(args, world, rank, local, dist):
    """B64: one step = one batched solve of every (system, RHS) pair of this
    rank to 1e-8. With N ranks the 64 systems are split over the GPUs
    (largest first to the least-loaded rank): strong scaling, no collective."""
    import torch
    import gpusolver_b200 as gs

    torch.cuda.set_device(local)
    dev = local
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    t0 = time.time()
    sides, mats, rhs = b64_problems(gs, count=args.systems)
    if args.kernel_only == "level1":
        Hs = build_hierarchies(gs, mats)
        B = gs.Batch(Hs, B64_RHS, gs.SolverOptions(tol=TOL, precision=1, flexible=1, lanes=4), device=dev)
        print(json.dumps({"kernel_only": "level1", "systems": len(mats), "level1": B.level_info()[1],
                          "resid_ms": B.time_level(1, 1, 4, 1, sptr), "sweep_ms": B.time_level(1, 0, 4, 1, sptr)}))
        return
    mine = shard_systems([a.rows for a in mats], world, rank)
    mats_r, rhs_r = [mats[i] for i in mine], [rhs[i] for i in mine]
    Hs = build_hierarchies(gs, mats_r)
    setup_s = time.time() - t0
    if args.variant == "plain":
        opts = gs.SolverOptions(tol=TOL, max_iter=1000, coarse_solver=1)
    else:
        opts = gs.SolverOptions(tol=TOL, max_iter=1000, coarse_solver=1, precision=1, flexible=1,
                                use_graph=1, coarse_rows=FAST_BATCH_COARSE_ROWS, coloring=min(args.coloring, 1))
    t0 = time.time()
    B = gs.Batch(Hs, B64_RHS, opts, device=dev)
    upload_s = time.time() - t0
    b = B.pack(rhs_r)
    b_d = torch.tensor(b, dtype=torch.float64, device="cuda")
    x_d = torch.zeros_like(b_d)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2

    def solve_once():
        x_d.zero_()
        return B.solve_device(b_d.data_ptr(), x_d.data_ptr(), sptr)

    for _ in range(args.warmup):
        solve_once()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    torch.cuda.synchronize()
    launches0 = B.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.nvtx.range_push("timed_solve")
        ev[i][0].record(stream)
        stats = solve_once()
        ev[i][1].record(stream)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    launches = B.launch_count() - launches0
    ms = float(np.mean([e0.elapsed_time(e1) for e0, e1 in ev]))
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    clk = clocks.stop()
    xs = B.unpack(x_d.cpu().numpy())
    res = [float(np.linalg.norm(rhs_r[i][j] - a.to_scipy() @ xs[i][j]) / np.linalg.norm(rhs_r[i][j]))
           for i, a in enumerate(mats_r) for j in range(B64_RHS)]
    iters = [st.iterations for st in stats]
    statuses = sorted(set(st.status for st in stats))

    # end to end through the public host entry point (pinned host buffers)
    b_h = torch.tensor(b, dtype=torch.float64).pin_memory()
    x_h = torch.zeros_like(b_h).pin_memory()
    e2e = []
    for i in range(0 if args.no_e2e else args.warmup + args.steps):
        x_h.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        B.solve_host_ptr(b_h.data_ptr(), x_h.data_ptr())
        t1 = time.perf_counter()
        if i >= args.warmup:
            e2e.append((t1 - t0) * 1e3)
    e2e_ms = float(np.mean(e2e)) if e2e else None
    if dist is not None and e2e_ms is not None:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    # roofline: level-0 forward Gauss-Seidel sweep over all systems (4 RHS per
    # matrix read) and the outer FP64 SpMV, CUDA events on the launching stream
    info = B.level_info()
    n0, nnz0 = info[0]["rows"], info[0]["nnz"]
    vs = 4 if args.variant == "fast" else 8
    gs_ms = B.time_kernel(1, 10, sptr)
    spmv_ms = B.time_kernel(0, 10, sptr)
    vc_ms = B.time_kernel(2, 5, sptr)
    gs_bytes = (nnz0 - n0) * (vs + 4) + n0 * vs + 4 * n0 * B64_RHS * vs
    spmv_bytes = (nnz0 - n0) * 12 + n0 * 8 + 2 * n0 * B64_RHS * 8
    peak, peak_kind = load_peaks()
    gs_gbs = gs_bytes / (gs_ms * 1e-3) / 1e9
    spmv_gbs = spmv_bytes / (spmv_ms * 1e-3) / 1e9
    traffic = load_traffic("b64")
    roofline = {"bound": "hbm", "kernel": f"level-0 batched Gauss-Seidel sweep ({info[0]['max_colors']} colour "
                                          f"passes, {B64_RHS} RHS per matrix read, {'FP32' if vs == 4 else 'FP64'})",
                "achieved": gs_gbs, "peak": peak, "unit": "GB/s", "frac": gs_gbs / peak,
                "peak_kind": peak_kind, "traffic": traffic.get(f"gs_sweep_{args.variant}"),
                "algorithmic_bytes": gs_bytes, "ms_per_sweep": gs_ms, "ms_per_vcycle": vc_ms,
                "spmv_fp64": {"achieved": spmv_gbs, "frac": spmv_gbs / peak, "ms": spmv_ms,
                              "algorithmic_bytes": spmv_bytes, "traffic": traffic.get("spmv_fp64")}}

    # the single-system path, one pair after another: the plain FP64 drop-in
    # and the fast variant (each solver warmed on its system first)
    seq = {}
    for name in ([] if args.no_plain else ["plain", "fast"]):
        total, its = 0.0, []
        for H, rb in zip(Hs, rhs_r):
            sv = gs.Solver(H, solver_options(gs, name, 1), device=dev)
            bd = torch.tensor(rb, dtype=torch.float64, device="cuda")
            xd = torch.zeros(rb.shape[1], dtype=torch.float64, device="cuda")
            sv.solve_device(bd[0].data_ptr(), xd.data_ptr(), sptr)
            for j in range(B64_RHS):
                xd.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st = sv.solve_device(bd[j].data_ptr(), xd.data_ptr(), sptr)
                e1.record(stream)
                torch.cuda.synchronize()
                total += e0.elapsed_time(e1)
                its.append(st.iterations)
            del sv
        seq[name] = {"ms": total, "iterations_max": max(its), "speedup_of_batched": total / ms}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        v, threads, sample, kind = b64_cpu_sample(gs, O, mats, rhs)
        cpu = {"value": v, "unit": "ms", "cores": threads, "kind": kind, "sample": sample}

    if rank == 0:
        unknowns = sum(a.rows for a in mats)
        line = {
            "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 V-cycle + f64 CG" if args.variant == "fast" else "f64", "data": "synthetic",
            "config": {"workload": "b64", "desc": WORKLOADS["b64"]["desc"], "systems": len(mats),
                       "rhs_per_system": B64_RHS, "solves": len(mats) * B64_RHS, "unknowns": unknowns,
                       "sides_min_max": [min(sides), max(sides)], "variant": args.variant,
                       "systems_this_rank": len(mats_r), "levels": B.levels,
                       "level_rows": [lv["rows"] for lv in info],
                       "level_max_colors": [lv["max_colors"] for lv in info],
                       "level_lanes": [[lv["lanes"], lv["r_lanes"], lv["p_lanes"]] for lv in info],
                       "l2": "level-0 matrices larger than L2; 256 MB L2 flush between timed solves",
                       "parallelism": f"systems split over {world} GPU(s), no collective in the solve",
                       "host_setup_s": round(setup_s, 2), "upload_s": round(upload_s, 2)},
            "iterations_max": max(iters), "iterations_mean": float(np.mean(iters)),
            "statuses": statuses, "true_residual_max": max(res),
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 16 * b.size,
                    "d2h_bytes_per_step": 8 * b.size},
            "roofline": roofline,
            "gpu_launches": int(launches),
            "clocks": clk,
            "plain_fp64": seq.get("plain"),
            "sequential_fast": seq.get("fast"),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    del B
    if dist is not None:
        dist.destroy_process_group()


def timed_solves(torch, s, b_d, x_d, stream, flush, steps, warmup=2):
    """Mean CUDA-event ms of `steps` solves from x = 0 (L2 flushed before
    each, not timed) after `warmup` untimed ones; returns (ms, stats, x)."""
    sptr = stream.cuda_stream
    per = []
    st = None
    for i in range(warmup + steps):
        x_d.zero_()
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = s.solve_device(b_d.data_ptr(), x_d.data_ptr(), sptr)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= warmup:
            per.append(e0.elapsed_time(e1))
    return float(np.mean(per)), st, x_d.cpu().numpy()


def fp64_reference_solution(torch, s_plain, b_d, stream, n, tol=1e-12):
    """x* for the error of a result: the plain FP64 drop-in (held to the FP64
    oracle at full size by tests/test_gpu_fullsize.py) run to relative
    residual `tol`."""
    s_plain.set_tolerance(tol, 5000)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    s_plain.solve_device(b_d.data_ptr(), x.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    s_plain.set_tolerance(TOL, 1000)
    return x.cpu().numpy()


def rel_err(x, ref):
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))


def level_roofline(s, info, level, vs, peak, sptr, reps=20):
    """One forward Gauss-Seidel sweep of `level` as the solve launches it
    (layout and launch mode of the autotuner): algorithmic bytes
    nnz (s + 4) + 4 n s over the CUDA-event time of a sweep."""
    lv = info[level]
    ms = s.time_level(level, 0, 0, reps, sptr)
    nbytes = algorithmic_bytes(lv["nnz"], lv["rows"], vs, "gs")
    gbs = nbytes / (ms * 1e-3) / 1e9
    return {"level": level, "rows": lv["rows"], "nnz": lv["nnz"], "colors": lv["colors"],
            "layout": ("sliced" if lv["sliced"] else "csr-vector") + f" x{lv['lanes']}",
            "achieved": gbs, "frac": gbs / peak, "ms_per_sweep": ms, "algorithmic_bytes": nbytes}


def e64_leg(args, gs, torch, dev, stream, flush, peak, peak_kind):
    """The ~786k-dof elasticity config beside the headline: fast (FP32 V-cycle,
    graph, GPU hierarchy) against the plain FP64 drop-in, same timing rules,
    with the error of each against an FP64 solution, the 3x3 block
    Gauss-Seidel rooflines and the reference's CPU path on the host cores."""
    sptr = stream.cuda_stream
    a, b = make_problem(gs, "e64")
    n = a.rows
    H = gs.Hierarchy.build(a, 3, 0.1, 10, 1000)
    Hs = gs.Hierarchy.build_ex(a, 3, 0.1, 10, 1000, aggregation=1, device=dev)
    sf = gs.Solver(Hs, solver_options(gs, "fast", 3), device=dev)
    b_d = torch.tensor(b, dtype=torch.float64, device="cuda")
    x_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    learned_info = None
    if not args.no_learned:
        from gpusolver_b200 import learned
        params = learned.load_params(args.weights) if args.weights else learned.load_params()
        if params is not None:
            wts = learned.Model(params).weights_for(sf)
            j = learned.select_weights(sf, wts, b_d, repeats=2)
            learned_info = {"used": j.use_learned, "ms_learned": j.ms_learned, "ms_plain_omega": j.ms_plain,
                            "iterations_learned": j.iterations_learned,
                            "iterations_plain_omega": j.iterations_plain}
            # per-block scalings of the 3x3 smoother (the network trained on the
            # elasticity distribution), against the configuration chosen so far
            pn = learned.load_params(learned.DEFAULT_NODE_PARAMS)
            if pn is not None:
                kept = wts if j.use_learned else None
                nw = learned.node_weights_for(learned.Model(pn), sf)
                jn = learned.select_node_weights(sf, nw, b_d, repeats=2)
                if not jn.use_learned:
                    sf.set_colour_weights(kept)
                learned_info["per_block"] = {"used": jn.use_learned, "ms_learned": jn.ms_learned,
                                             "ms_plain_omega": jn.ms_plain,
                                             "iterations_learned": jn.iterations_learned,
                                             "iterations_plain_omega": jn.iterations_plain,
                                             "weights_range": [float(nw.min()), float(nw.max())]}
    ms_f, st_f, x_f = timed_solves(torch, sf, b_d, x_d, stream, flush, args.steps, args.warmup)
    sp = gs.Solver(H, solver_options(gs, "plain", 3), device=dev)
    ms_p, st_p, x_p = timed_solves(torch, sp, b_d, x_d, stream, flush, args.steps, 2)
    xref = fp64_reference_solution(torch, sp, b_d, stream, n)
    A = a.to_scipy()

    def res(x):
        return float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))

    info = sf.level_info()
    nblocks = (a.nnz - 9 * (n // 3)) // 9 + n // 3
    fine = level_roofline(sf, info, 0, 4, peak, sptr)
    fine["algorithmic_bytes"] = block_algorithmic_bytes(nblocks, n, 4, "gs")
    fine["achieved"] = fine["algorithmic_bytes"] / (fine["ms_per_sweep"] * 1e-3) / 1e9
    fine["frac"] = fine["achieved"] / peak
    out = {"workload": "e64", "desc": WORKLOADS["e64"]["desc"], "n": n, "nnz": a.nnz,
           "fast": {"ms": ms_f, "iterations": st_f.iterations, "true_residual": res(x_f),
                    "error_vs_fp64": rel_err(x_f, xref), "levels": [lv["rows"] for lv in info],
                    "colors": [lv["colors"] for lv in info]},
           "plain_fp64": {"ms": ms_p, "iterations": st_p.iterations, "true_residual": res(x_p),
                          "error_vs_fp64": rel_err(x_p, xref)},
           "speedup_of_fast": ms_p / ms_f,
           "fp64_reference": "plain FP64 drop-in run to relative residual 1e-12",
           "roofline": {"fine_block_gs": fine, "peak": peak, "peak_kind": peak_kind},
           "learned_weights": learned_info}
    if len(info) > 2:
        lv1 = info[1]
        l1 = level_roofline(sf, info, 1, 4, peak, sptr)
        nb1 = (lv1["nnz"] - 3 * lv1["rows"]) // 9 + lv1["rows"] // 3  # stored scalar entries / 9 per block
        l1["algorithmic_bytes"] = block_algorithmic_bytes(nb1, lv1["rows"], 4, "gs")
        l1["achieved"] = l1["algorithmic_bytes"] / (l1["ms_per_sweep"] * 1e-3) / 1e9
        l1["frac"] = l1["achieved"] / peak
        out["roofline"]["level1_block_gs"] = l1
    if not args.no_cpu:
        # The reference's CPU path on this system. Its block Gauss-Seidel
        # reads the colour range as (start, end) and does not converge past
        # colour 0, so its scalar multicolour SGS preconditioner is timed.
        from oracle import oracle as O
        Al = [H.A(k) for k in range(H.levels)]
        Pl = [H.P(k) for k in range(H.levels - 1)]
        Rl = [H.R(k) for k in range(H.levels - 1)]
        xc, it, solve_ms, kind, cores, _ = reference_cpu_solve(O, Al, Pl, Rl, b, 0, args.ref_max_iter)
        out["cpu_baseline"] = {"value": solve_ms, "unit": "ms", "cores": cores, "kind": kind,
                               "sample": f"one full solve by {_path_name(kind)} with its scalar "
                                         f"MultigridGaussSeidelPreconditioner (its block variant does not "
                                         f"converge: colour range read as (start, end)), {it} iterations, "
                                         f"FP64 true residual {res(np.asarray(xc, np.float64)):.2e}"}
    del sf, sp
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="p128")
    ap.add_argument("--variant", choices=["fast", "plain"], default="fast")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison solve")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end host-buffer leg")
    ap.add_argument("--weights", default=None,
                    help="learned relaxation weights (.npy); default: the committed network")
    ap.add_argument("--no-learned", action="store_true", help="fast variant without learned weights")
    ap.add_argument("--coloring", type=int, choices=[0, 1, 2], default=2,
                    help="fast variant's colouring: 0 the reference's greedy order, 1 smallest-last order, "
                         "2 and the strong couplings only on coarse scalar levels (batches: 1)")
    ap.add_argument("--host-setup", action="store_true",
                    help="fast variant on the host-built hierarchy (sequential aggregation) instead of the GPU build")
    ap.add_argument("--tune-cache", default=None,
                    help="autotuner decision file (profiling runs reuse the decisions of a plain run)")
    ap.add_argument("--ref-max-iter", type=int, default=200)
    ap.add_argument("--kernel-only", choices=["gs", "spmv", "level1"], default=None,
                    help="profiling aid: build the solver with one lane per row everywhere and "
                         "run only the fine-level kernel timing loop; level1: one forward sweep of "
                         "level 1 of the fast variant with the cached layouts (b64: level1 runs the "
                         "level-1 residual and one forward sweep of the batch with 4 lanes per row)")
    ap.add_argument("--systems", type=int, default=B64_SYSTEMS,
                    help="b64: number of systems (the first ones of the seeded set)")
    ap.add_argument("--no-e64", action="store_true", help="skip the elasticity leg of the default run")
    ap.add_argument("--ordering", choices=["none", "rcm", "hierarchical"], default="none",
                    help="per-level permutation given to the solver (the reference's MultigridSmoother "
                         "takes one per level): none, RCM of every level, or HierarchicalReordering")
    ap.add_argument("--no-ablation", action="store_true", help="skip the hierarchy/option ablation solves")
    args = ap.parse_args()

    world, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.workload == "b64":
        run_b64(args, world, rank, local, dist)
        return

    import torch
    import gpusolver_b200 as gs

    torch.cuda.set_device(local)
    dev = local
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    w = WORKLOADS[args.workload]
    a, b = make_problem(gs, args.workload)
    t0 = time.time()
    H = gs.Hierarchy.build(a, w["block"], 0.1, 10, 1000)
    setup_s = time.time() - t0
    opts = solver_options(gs, args.variant, w["block"])
    if args.variant == "fast":
        opts.coloring = args.coloring
    if args.tune_cache:
        gs.set_tune_cache(args.tune_cache)
    if args.kernel_only == "level1":
        # one forward sweep of level 1 of the fast variant's GPU-built hierarchy,
        # layouts from the tune cache (--tune-cache) of a plain run, so the
        # profiled sweep is the one the solve launches
        Hk = gs.Hierarchy.build_ex(a, w["block"], 0.1, 10, 1000, aggregation=1, device=dev)
        opts.coarse_tail = 0
        s = gs.Solver(Hk, opts, device=dev)
        ms = s.time_level(1, 0, 0, 5, sptr)
        print(json.dumps({"kernel_only": args.kernel_only, "ms": ms, "level1": s.level_info()[1]}))
        return
    if args.kernel_only:
        opts.autotune = 0
        opts.coarse_tail = 0  # no coarse V-cycle timing at setup: the fine-level sweep is the first GS launch
        s = gs.Solver(H, opts, device=dev)
        ms = s.time_kernel(1 if args.kernel_only == "gs" else 0, 5, sptr)
        print(json.dumps({"kernel_only": args.kernel_only, "ms": ms}))
        return
    setup_info = {"hierarchy_host_s": round(setup_s, 3)}
    Hs = H
    if args.variant == "fast" and not args.host_setup:
        # the fast variant's hierarchy: smoothed aggregation with the
        # independent-set aggregation, built on the GPU (the plain FP64 drop-in
        # and the CPU baseline keep the host build of the reference's algorithm)
        t0 = time.time()
        Hs = gs.Hierarchy.build_ex(a, w["block"], 0.1, 10, 1000, aggregation=1, device=dev)
        setup_info["hierarchy_gpu_s"] = round(time.time() - t0, 3)
        setup_info["hierarchy_gpu_phases_ms"] = {k: round(v, 1) for k, v in Hs.setup_stats.items()}
    setup_info["solve_hierarchy"] = ("gpu, independent-set aggregation" if Hs is not H
                                     else "host, sequential aggregation")
    t0 = time.time()
    perms = None
    if args.ordering == "rcm":
        perms = [gs.rcm(Hs.A(k)) for k in range(Hs.levels)]
    elif args.ordering == "hierarchical":
        perms = gs.hierarchical_reordering(Hs)
    s = gs.Solver(Hs, opts, permutations=perms, device=dev)
    upload_s = time.time() - t0
    setup_info["solver_create_s"] = round(upload_s, 3)
    setup_info["solver_create_phases_ms"] = {k: round(v) for k, v in s.setup_phases().items()}
    n = a.rows
    b_d = torch.tensor(b, dtype=torch.float64, device="cuda")
    x_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2

    def solve_once():
        x_d.zero_()
        return s.solve_device(b_d.data_ptr(), x_d.data_ptr(), sptr)

    learned_info = None
    if args.variant == "fast" and not args.no_learned:
        # learned per-colour weights, kept only if they cut the time to
        # solution (plain omega = 1 is the fallback and the yardstick)
        from gpusolver_b200 import learned
        params = learned.load_params(args.weights) if args.weights else learned.load_params()
        if params is not None:
            wts = learned.Model(params).weights_for(s)
            j = learned.select_weights(s, wts, b_d, repeats=2)
            learned_info = {"used": j.use_learned, "ms_learned": j.ms_learned, "ms_plain_omega": j.ms_plain,
                            "iterations_learned": j.iterations_learned,
                            "iterations_plain_omega": j.iterations_plain,
                            "weights_range": [float(min(x.min() for x in wts)), float(max(x.max() for x in wts))]}

    for _ in range(args.warmup):
        solve_once()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    torch.cuda.synchronize()
    launches0 = s.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    stats = []
    for i in range(args.steps):
        flush.zero_()  # L2 flush between timed solves (not timed)
        torch.cuda.nvtx.range_push("timed_solve")  # lets ncu restrict a capture to this region
        ev[i][0].record(stream)
        stats.append(solve_once())
        ev[i][1].record(stream)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    launches = s.launch_count() - launches0
    per = [e0.elapsed_time(e1) for e0, e1 in ev]
    ms = float(np.mean(per))
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    clk = clocks.stop()
    x = x_d.cpu().numpy()
    true_res = float(np.linalg.norm(b - a.to_scipy() @ x) / np.linalg.norm(b))
    iters = stats[-1].iterations

    # end to end through the public host entry point: pinned host buffers,
    # H2D of b and x0, solve, D2H of x inside the timed region
    b_h = torch.tensor(b, dtype=torch.float64).pin_memory()
    x_h = torch.zeros(n, dtype=torch.float64).pin_memory()
    e2e = []
    for i in range(0 if args.no_e2e else args.warmup + args.steps):
        x_h.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.solve_host_ptr(b_h.data_ptr(), x_h.data_ptr())
        t1 = time.perf_counter()
        if i >= args.warmup:
            e2e.append((t1 - t0) * 1e3)
    e2e_ms = float(np.mean(e2e)) if e2e else None
    if dist is not None and e2e_ms is not None:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    # roofline: the fine-level Gauss-Seidel sweep (the dominant kernel) and the
    # outer SpMV, CUDA events on the launching stream
    info = s.level_info()
    fine = info[0]
    vs = 4 if args.variant == "fast" else 8
    gs_ms = s.time_kernel(1, 20, sptr)
    spmv_ms = s.time_kernel(0, 20, sptr)
    if w["block"] == 3:
        nb = fine["stored"] // 9  # padded block slots (upper bound on blocks)
        nblocks = (a.nnz - 9 * (n // 3)) // 9 + n // 3
        gs_bytes = block_algorithmic_bytes(nblocks, n, vs, "gs")
        spmv_bytes = block_algorithmic_bytes(nblocks, n, 8, "spmv")
    else:
        gs_bytes = algorithmic_bytes(a.nnz, n, vs, "gs")
        spmv_bytes = algorithmic_bytes(a.nnz, n, 8, "spmv")
    peak, peak_kind = load_peaks()
    gs_gbs = gs_bytes / (gs_ms * 1e-3) / 1e9
    spmv_gbs = spmv_bytes / (spmv_ms * 1e-3) / 1e9
    traffic = load_traffic(args.workload)
    roofline = {"bound": "hbm", "kernel": f"fine-level Gauss-Seidel sweep ({fine['colors']} colour passes, "
                                          f"{'FP32' if vs == 4 else 'FP64'})",
                "achieved": gs_gbs, "peak": peak, "unit": "GB/s", "frac": gs_gbs / peak,
                "peak_kind": peak_kind, "traffic": traffic.get(f"gs_sweep_{args.variant}"),
                "algorithmic_bytes": gs_bytes, "ms_per_sweep": gs_ms,
                "spmv_fp64": {"achieved": spmv_gbs, "frac": spmv_gbs / peak, "ms": spmv_ms,
                              "algorithmic_bytes": spmv_bytes,
                              "traffic": traffic.get("spmv_fp64")}}
    # the dense coarsest solve: the inverse's bytes (full, or the packed lower
    # triangle -- FP16 tiles with an FP32 scale each under coarse_half -- plus
    # its partial sums, FP64 or FP32, written and read) per application
    nc = info[-1]["rows"]
    dense_ms = s.time_kernel(3, 20, sptr)
    packed = nc > opts.packed_rows
    half = packed and opts.coarse_half == 1 and vs == 4
    if packed:
        tiles = (nc + 63) // 64
        ntile = tiles * (tiles + 1) // 2
        if half:
            dense_bytes = 2 * ntile * 64 * 64 + 4 * ntile + 2 * 4 * tiles * tiles * 64 + 2 * vs * nc
        else:
            dense_bytes = vs * ntile * 64 * 64 + 2 * 8 * tiles * tiles * 64 + 2 * vs * nc
    else:
        dense_bytes = vs * nc * nc + 2 * vs * nc
    dense_gbs = dense_bytes / (dense_ms * 1e-3) / 1e9
    layout = "full"
    if packed:
        layout = ("packed lower-triangle FP16 tiles, tensor-core apply" if half
                  else "packed lower-triangle tiles")
    roofline["dense_coarse"] = {"rows": nc, "layout": layout,
                                "achieved": dense_gbs, "frac": dense_gbs / peak, "ms": dense_ms,
                                "algorithmic_bytes": dense_bytes, "traffic": traffic.get(f"dense_{args.variant}")}

    plain = None
    errors = None
    ablation = None
    if len(info) > 2:
        roofline["level1_gs"] = level_roofline(s, info, 1, vs, peak, sptr)
        roofline["level1_gs"]["traffic"] = traffic.get(f"level1_gs_{args.variant}")
    if not args.no_plain and args.variant == "fast":
        sp = gs.Solver(H, solver_options(gs, "plain", w["block"]), device=dev)
        ms_p, st, xp = timed_solves(torch, sp, b_d, x_d, stream, flush, args.steps, 2)
        plain = {"ms": ms_p, "iterations": st.iterations,
                 "true_residual": float(np.linalg.norm(b - a.to_scipy() @ xp) / np.linalg.norm(b)),
                 "speedup_of_fast": ms_p / ms}
        xref = fp64_reference_solution(torch, sp, b_d, stream, n)
        errors = {"fast": rel_err(x, xref), "plain_fp64": rel_err(xp, xref),
                  "reference": "plain FP64 drop-in (pinned to the FP64 oracle at this size) run to 1e-12"}
        plain["error_vs_fp64"] = errors["plain_fp64"]
        del sp
        if not args.no_ablation and Hs is not H:
            # where the speed-up comes from: the fast options on the plain
            # arm's host hierarchy, and the plain options on the GPU hierarchy
            ablation = {}
            for key, hier, variant in (("fast_on_host_hierarchy", H, "fast"),
                                       ("plain_on_gpu_hierarchy", Hs, "plain")):
                o = solver_options(gs, variant, w["block"])
                if variant == "fast":
                    o.coloring = args.coloring
                sa = gs.Solver(hier, o, device=dev)
                ms_a, st_a, _ = timed_solves(torch, sa, b_d, x_d, stream, flush, max(3, args.steps // 2), 2)
                ablation[key] = {"ms": ms_a, "iterations": st_a.iterations,
                                 "levels": [lv["rows"] for lv in sa.level_info()]}
                del sa
            ablation["fast"] = {"ms": ms, "iterations": iters, "levels": [lv["rows"] for lv in info]}
            ablation["plain_fp64"] = {"ms": plain["ms"], "iterations": plain["iterations"],
                                      "levels": [H.A(k).rows for k in range(H.levels)]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, a, b, H, w["block"])

    e64 = None
    if args.workload == "p128" and args.variant == "fast" and not args.no_e64 and world == 1:
        e64 = e64_leg(args, gs, torch, dev, stream, flush, peak, peak_kind)

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 V-cycle + f64 CG" if args.variant == "fast" else "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "desc": w["desc"], "n": n, "nnz": a.nnz,
                       "levels": Hs.levels, "variant": args.variant,
                       "level_rows": [lv["rows"] for lv in info],
                       "level_colors": [lv["colors"] for lv in info],
                       "level_lanes": [[lv["lanes"], lv["r_lanes"], lv["p_lanes"]] for lv in info],
                       "level_sliced": [lv["sliced"] for lv in info],
                       "level_in_tail": [lv["in_tail"] for lv in info],
                       "l2": "matrix larger than L2; 256 MB L2 flush between timed solves",
                       "ordering": args.ordering,
                       "parallelism": f"replicas x{world} (no collective in the solve)",
                       "host_setup_s": round(setup_s, 2), "upload_s": round(upload_s, 2)},
            "iterations": iters, "true_residual": true_res,
            "error_vs_fp64": None if errors is None else errors["fast"],
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 16 * n,
                    "d2h_bytes_per_step": 8 * n},
            "roofline": roofline,
            "gpu_launches": int(launches),
            "clocks": clk,
            "plain_fp64": plain,
            "errors_vs_fp64": errors,
            "ablation": ablation,
            "e64": e64,
            "learned_weights": learned_info,
            "setup": setup_info,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    del s
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
