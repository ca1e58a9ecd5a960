"""Trains the learned relaxation weights on the GPU and writes them under
gpusolver_b200/weights/.

    python gpu-conjugate-gradient-solver_b200/train_weights.py [--count 200] [--size 48]
    python gpu-conjugate-gradient-solver_b200/train_weights.py --distribution elasticity \
        [--count 32] [--size 56] [--steps 24]

Default: per-(level, colour) weights on the 128^3 heterogeneous-Poisson
distribution (exp(2.3 GRF), correlation length 8 cells, harmonic faces) at a
trainable size, seeds 100..100+count-1. --distribution elasticity: per-block
scalings of the 3x3 block smoother on the E64 distribution (P1 elasticity,
Young's modulus exp(N(0, 1)) per element, nu 0.3), seeds 100...; hierarchies
built on the GPU as in the fast variant. Every step measures the A-norm error
reduction of one V-cycle with the library's own kernels.
"""
import argparse
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from gpusolver_b200 import learned  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--distribution", choices=["p128", "elasticity"], default="p128")
    ap.add_argument("--count", type=int, default=None)
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    t0 = time.time()

    def log(i, seed, rho):
        if i % 4 == 0 or i == count - 1:
            print(f"instance {i} seed {seed} error reduction {rho:.4f} ({time.time() - t0:.0f} s)", flush=True)

    if args.distribution == "p128":
        count, size, steps = args.count or 200, args.size or 48, args.steps or 4
        out = args.out or learned.DEFAULT_PARAMS
        params = learned.train(learned.training_instances(count, size), steps_per_instance=steps,
                               lr=args.lr, log=log)
    else:
        count, size, steps = args.count or 32, args.size or 56, args.steps or 24
        out = args.out or learned.DEFAULT_NODE_PARAMS
        params = learned.train_nodes(learned.elasticity_instances(count, size), steps_per_instance=steps,
                                     lr=args.lr, log=log)
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    np.save(out, params)
    print("wrote", out, params.shape)


if __name__ == "__main__":
    main()
