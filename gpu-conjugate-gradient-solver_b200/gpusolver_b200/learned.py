"""Learned per-(level, colour) relaxation weights for the multigrid smoother.

An MLP (8 features -> 32 -> 32 -> 1, FP32) predicts a Gauss-Seidel weight
omega = 2 sigmoid(z), kept inside [0.02, 1.98], for every colour of every level from features
the solver computes from its own level matrices (level depth, colour
position and size, diagonal dominance, diagonal contrast, row length). The
same weight serves a colour in the forward and the backward sweep of every
smoothing step, so the V-cycle stays symmetric positive definite and the
outer CG stays valid.

Training uses data the solver generates itself: the A-norm error reduction
of one V-cycle, ||e1||_A / ||e0||_A, measured on the GPU
(``Solver.error_reduction``). Its gradient with respect to the weights is
estimated by simultaneous perturbation (two measurements per step, a random
+-1 direction), pushed through the network by the hand-written backward
kernel, and applied by the hand-written Adam kernel. PyTorch only provides
device buffers here; every computation is a kernel of this library.

``select_weights`` keeps the plain method (omega = 1 everywhere) whenever
the learned weights do not cut the time to solution: plain AMG-PCG is both
the fallback and the yardstick.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import (Hierarchy, Solver, SolverOptions, elasticity, mlp_adam, mlp_backward, mlp_forward,
               mlp_param_count, uniform_rhs, varcoef_grf)

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PARAMS = os.path.join(HERE, "weights", "mlp_p128_grf.npy")
# the per-block scalings of the 3x3 block smoother, trained on the elasticity distribution
DEFAULT_NODE_PARAMS = os.path.join(HERE, "weights", "mlp_elasticity_nodes.npy")
N_IN, N_H = 8, 32


def init_params(seed: int = 0) -> np.ndarray:
    """Xavier-uniform hidden layers, a small output layer and zero biases, so
    the untrained network predicts omega close to 1 (the plain method)."""
    rng = np.random.default_rng(seed)
    w1 = rng.uniform(-1, 1, (N_H, N_IN)) * np.sqrt(6.0 / (N_IN + N_H))
    w2 = rng.uniform(-1, 1, (N_H, N_H)) * np.sqrt(6.0 / (2 * N_H))
    w3 = rng.uniform(-1, 1, N_H) * 0.05
    p = np.concatenate([w1.ravel(), np.zeros(N_H), w2.ravel(), np.zeros(N_H), w3, [0.0]])
    assert len(p) == mlp_param_count()
    return p.astype(np.float32)


def load_params(path: str = DEFAULT_PARAMS) -> Optional[np.ndarray]:
    return np.load(path).astype(np.float32) if os.path.exists(path) else None


def split_by_level(values: np.ndarray, solver: Solver) -> List[np.ndarray]:
    out, k = [], 0
    for lv in solver.level_info():
        out.append(np.asarray(values[k:k + lv["colors"]], np.float64))
        k += lv["colors"]
    return out


class Model:
    """Parameters and Adam state on the device, evaluated by the library's kernels."""

    def __init__(self, params: np.ndarray, lr: float = 3e-3):
        import torch
        self.torch = torch
        self.p = torch.tensor(params, dtype=torch.float32, device="cuda")
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.g = torch.zeros_like(self.p)
        self.lr = lr
        self.step = 0

    def params(self) -> np.ndarray:
        return self.p.cpu().numpy()

    def forward(self, feats: np.ndarray):
        torch = self.torch
        f = torch.tensor(np.ascontiguousarray(feats, np.float32), device="cuda")
        n = f.shape[0]
        om = torch.empty(n, dtype=torch.float32, device="cuda")
        cache = torch.empty(n * (2 * N_H + 1), dtype=torch.float32, device="cuda")
        mlp_forward(self.p.data_ptr(), f.data_ptr(), n, om.data_ptr(), cache.data_ptr(),
                    torch.cuda.current_stream().cuda_stream)
        return f, om, cache

    def weights_for(self, solver: Solver) -> List[np.ndarray]:
        _, om, _ = self.forward(solver.colour_features())
        return split_by_level(om.cpu().numpy(), solver)

    def apply_gradient(self, f, cache, upstream: np.ndarray) -> None:
        torch = self.torch
        n = f.shape[0]
        up = torch.tensor(np.asarray(upstream, np.float32), device="cuda")
        delta = torch.empty(n * (2 * N_H + 1), dtype=torch.float32, device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        mlp_backward(self.p.data_ptr(), f.data_ptr(), n, cache.data_ptr(), up.data_ptr(),
                     delta.data_ptr(), self.g.data_ptr(), st)
        self.step += 1
        mlp_adam(self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                 self.p.numel(), self.lr, self.step, stream=st)


def spsa_step(model: Model, solver: Solver, e0, rng: np.random.Generator, c: float = 0.05) -> float:
    """One training step on one solver: returns the error reduction at the
    current prediction (mean of the two perturbed measurements)."""
    f, om, cache = model.forward(solver.colour_features())
    w = om.cpu().numpy().astype(np.float64)
    delta = rng.choice([-1.0, 1.0], size=len(w))
    st = model.torch.cuda.current_stream().cuda_stream
    solver.set_colour_weights(split_by_level(np.clip(w + c * delta, 0.02, 1.98), solver))
    rp = solver.error_reduction(e0.data_ptr(), st)
    solver.set_colour_weights(split_by_level(np.clip(w - c * delta, 0.02, 1.98), solver))
    rm = solver.error_reduction(e0.data_ptr(), st)
    grad_w = (rp - rm) / (2 * c) * delta
    model.apply_gradient(f, cache, grad_w)
    return 0.5 * (rp + rm)


def training_instances(count: int = 200, size: int = 48, first_seed: int = 100):
    """Instances of the P128 distribution (exp(2.3 GRF), correlation length 8
    cells, harmonic faces) at a trainable size, seeds first_seed...; yields
    (seed, matrix, hierarchy)."""
    for seed in range(first_seed, first_seed + count):
        a = varcoef_grf(size, 8.0, 2.3, seed)
        yield seed, a, Hierarchy.build(a, 1, 0.1, 10, 1000)


def train(instances, params: Optional[np.ndarray] = None, steps_per_instance: int = 4,
          lr: float = 3e-3, seed: int = 0, log=None) -> np.ndarray:
    """Trains on (seed, matrix, hierarchy) instances; FP32 V-cycle solvers,
    the configuration the weights are used in."""
    import torch
    model = Model(init_params(seed) if params is None else params, lr)
    rng = np.random.default_rng(seed)
    for i, (inst_seed, a, H) in enumerate(instances):
        s = Solver(H, SolverOptions(precision=1, flexible=1, tol=1e-8))
        e0 = torch.tensor(np.random.default_rng(inst_seed).uniform(-1, 1, a.rows),
                          dtype=torch.float64, device="cuda")
        for _ in range(steps_per_instance):
            rho = spsa_step(model, s, e0, rng)
        if log is not None:
            log(i, inst_seed, rho)
        del s
    return model.params()


def error_reduction_with(solver: Solver, weights: Optional[List[np.ndarray]], e0) -> float:
    import torch
    solver.set_colour_weights(weights)
    return solver.error_reduction(e0.data_ptr(), torch.cuda.current_stream().cuda_stream)


@dataclass
class WeightChoice:
    use_learned: bool
    ms_learned: float
    ms_plain: float
    iterations_learned: int
    iterations_plain: int


def select_weights(solver: Solver, weights: List[np.ndarray], b, repeats: int = 2) -> WeightChoice:
    """Times the solve of b (a device FP64 tensor) with the learned weights
    and with the plain method; leaves the faster configuration installed."""
    import torch
    x = torch.zeros_like(b)
    st = torch.cuda.current_stream().cuda_stream

    def timed():
        best, it = 1e30, 0
        for _ in range(repeats):
            x.zero_()
            stats = solver.solve_device(b.data_ptr(), x.data_ptr(), st)
            best, it = min(best, stats.solve_ms), stats.iterations
        return best, it

    solver.set_colour_weights(weights)
    ms_l, it_l = timed()
    solver.set_colour_weights(None)
    ms_p, it_p = timed()
    use = ms_l < ms_p
    solver.set_colour_weights(weights if use else None)
    return WeightChoice(use, ms_l, ms_p, it_l, it_p)


# ---- per-block scalings of the 3x3 block Gauss-Seidel smoother -------------------
# The same network, evaluated once per node (3x3 block row) of every level on
# the node's own features (Solver.node_features: level depth, colour
# position, block diagonal dominance, off-diagonal block contrast, blocks per
# row, diagonal norm against the level's mean, diagonal anisotropy, colour
# share). Its weight scales that node's block update in every forward and
# backward pass, so the V-cycle stays symmetric positive definite.

def node_weights_for(model: Model, solver: Solver) -> np.ndarray:
    _, om, _ = model.forward(solver.node_features())
    return om.cpu().numpy().astype(np.float64)


def spsa_node_step(model: Model, solver: Solver, e0, rng: np.random.Generator, c: float = 0.05) -> float:
    """One training step on per-node weights: a random +-1 perturbation of every
    node's weight, two measured error reductions, the estimate (r+ - r-) / 2c
    times the perturbation as each node's upstream gradient, pushed through the
    network by the backward kernel and applied by the Adam kernel."""
    f, om, cache = model.forward(solver.node_features())
    w = om.cpu().numpy().astype(np.float64)
    delta = rng.choice([-1.0, 1.0], size=len(w))
    st = model.torch.cuda.current_stream().cuda_stream
    solver.set_node_weights(np.clip(w + c * delta, 0.02, 1.98))
    rp = solver.error_reduction(e0.data_ptr(), st)
    solver.set_node_weights(np.clip(w - c * delta, 0.02, 1.98))
    rm = solver.error_reduction(e0.data_ptr(), st)
    model.apply_gradient(f, cache, (rp - rm) / (2 * c) * delta)
    return 0.5 * (rp + rm)


def fast_block_options() -> SolverOptions:
    """The fast configuration of the block path (FP32 V-cycle, flexible CG,
    dense coarsest solve moved up, smallest-last colouring)."""
    return SolverOptions(smoother=1, tol=1e-8, max_iter=1000, coarse_solver=1, precision=1, flexible=1,
                         use_graph=1, coarse_rows=24576, coloring=1, half_sweeps=1)


def elasticity_instances(count: int = 32, size: int = 56, first_seed: int = 100, device: int = 0):
    """Instances of the E64 distribution (P1 elasticity on Kuhn tetrahedra,
    Young's modulus exp(N(0, 1)) per element, nu 0.3, x = 0 clamped, unit body
    force) at a trainable size, seeds first_seed...; the hierarchy is built on
    the GPU as in the fast variant. Yields (seed, matrix, hierarchy)."""
    for seed in range(first_seed, first_seed + count):
        a = elasticity(size, 0.3, seed)
        yield seed, a, Hierarchy.build_ex(a, 3, 0.1, 10, 1000, aggregation=1, device=device)


def train_nodes(instances, params: Optional[np.ndarray] = None, steps_per_instance: int = 24,
                lr: float = 3e-3, seed: int = 0, log=None) -> np.ndarray:
    """Trains the per-block scalings on (seed, matrix, hierarchy) instances
    with fast_block_options solvers."""
    import torch
    model = Model(init_params(seed) if params is None else params, lr)
    rng = np.random.default_rng(seed)
    for i, (inst_seed, a, H) in enumerate(instances):
        s = Solver(H, fast_block_options())
        e0 = torch.tensor(np.random.default_rng(inst_seed).uniform(-1, 1, a.rows),
                          dtype=torch.float64, device="cuda")
        for _ in range(steps_per_instance):
            rho = spsa_node_step(model, s, e0, rng)
        if log is not None:
            log(i, inst_seed, rho)
        del s
    return model.params()


@dataclass
class NodeWeightChoice:
    use_learned: bool
    ms_learned: float
    ms_plain: float
    iterations_learned: int
    iterations_plain: int


def select_node_weights(solver: Solver, weights: np.ndarray, b, repeats: int = 2) -> NodeWeightChoice:
    """Times the solve of b with the learned per-block scalings and with the
    plain method (omega = 1, no colour weight); leaves the faster installed."""
    import torch
    x = torch.zeros_like(b)
    st = torch.cuda.current_stream().cuda_stream

    def timed():
        best, it = 1e30, 0
        for _ in range(repeats):
            x.zero_()
            stats = solver.solve_device(b.data_ptr(), x.data_ptr(), st)
            best, it = min(best, stats.solve_ms), stats.iterations
        return best, it

    solver.set_colour_weights(None)
    solver.set_node_weights(weights)
    ms_l, it_l = timed()
    solver.set_node_weights(None)
    ms_p, it_p = timed()
    use = ms_l < ms_p
    solver.set_node_weights(weights if use else None)
    return NodeWeightChoice(use, ms_l, ms_p, it_l, it_p)
