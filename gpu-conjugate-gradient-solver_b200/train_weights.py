"""Trains the learned relaxation weights on the GPU and writes them to
gpusolver_b200/weights/mlp_p128_grf.npy.

    python gpu-conjugate-gradient-solver_b200/train_weights.py [--count 200] [--size 48]

Instances: the 128^3 heterogeneous-Poisson distribution (exp(2.3 GRF),
correlation length 8 cells, harmonic faces) at a trainable size, seeds
100..100+count-1; every step measures the A-norm error reduction of one
V-cycle with the library's own kernels.
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
    ap.add_argument("--count", type=int, default=200)
    ap.add_argument("--size", type=int, default=48)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out", default=learned.DEFAULT_PARAMS)
    args = ap.parse_args()
    t0 = time.time()

    def log(i, seed, rho):
        if i % 20 == 0 or i == args.count - 1:
            print(f"instance {i} seed {seed} error reduction {rho:.4f} ({time.time() - t0:.0f} s)", flush=True)

    params = learned.train(learned.training_instances(args.count, args.size), steps_per_instance=args.steps,
                           lr=args.lr, log=log)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.save(args.out, params)
    print("wrote", args.out, params.shape)


if __name__ == "__main__":
    main()
