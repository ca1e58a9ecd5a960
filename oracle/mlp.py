"""ORACLE -- test infrastructure only: a numpy restatement of the learned-
weight network (gpu-conjugate-gradient-solver_b200/csrc/mlp.cu) used to
check the GPU forward pass, the GPU gradients and the Adam step.

Layout: W1[32][8], b1[32], W2[32][32], b2[32], W3[32], b3; omega = 2 sigmoid(z)
clamped to [0.02, 1.98], zero gradient where clamped.
"""
import numpy as np

N_IN, N_H = 8, 32
P = N_H * N_IN + N_H + N_H * N_H + N_H + N_H + 1
W_MIN, W_MAX = 0.02, 1.98


def unpack(p):
    p = np.asarray(p, np.float64)
    i = 0
    w1 = p[i:i + N_H * N_IN].reshape(N_H, N_IN); i += N_H * N_IN
    b1 = p[i:i + N_H]; i += N_H
    w2 = p[i:i + N_H * N_H].reshape(N_H, N_H); i += N_H * N_H
    b2 = p[i:i + N_H]; i += N_H
    w3 = p[i:i + N_H]; i += N_H
    b3 = p[i]
    return w1, b1, w2, b2, w3, b3


def forward(p, f):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    f = np.asarray(f, np.float64)
    h1 = np.tanh(f @ w1.T + b1)
    h2 = np.tanh(h1 @ w2.T + b2)
    z = h2 @ w3 + b3
    return np.clip(2.0 / (1.0 + np.exp(-z)), W_MIN, W_MAX), (h1, h2, z)


def grad(p, f, upstream):
    """d/dp of sum_s upstream[s] * omega[s]."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    f = np.asarray(f, np.float64)
    om, (h1, h2, z) = forward(p, f)
    sg = 1.0 / (1.0 + np.exp(-z))
    inside = (2.0 * sg >= W_MIN) & (2.0 * sg <= W_MAX)
    dz = np.where(inside, np.asarray(upstream, np.float64) * 2.0 * sg * (1.0 - sg), 0.0)
    d2 = dz[:, None] * w3[None, :] * (1.0 - h2 ** 2)
    d1 = (d2 @ w2) * (1.0 - h1 ** 2)
    g = np.concatenate([(d1.T @ f).ravel(), d1.sum(0), (d2.T @ h1).ravel(), d2.sum(0),
                        dz @ h2, [dz.sum()]])
    return g


def adam(p, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return p - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
