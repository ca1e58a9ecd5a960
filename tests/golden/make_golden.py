"""Regenerates the golden fixtures in tests/golden/ from the reference's own
CPU code (oracle/_ref/libgsref.so, compiled unmodified from the reference
sources by oracle/ref/Makefile). Run from the repository root:

    make -C oracle/ref && python tests/golden/make_golden.py

Inputs are built here from closed-form formulas (the matrices of the
reference's own unit tests: tests/cuda/testCudaGaussSeidel.cc:15-222,
tests/metal/graphColoringTest.cc:222-507,
tests/metal/gaussSeidelSymmUnittest.cc:32-75) and from the product's
problem generators (their arrays are stored in the fixture, so the fixture
is self-contained). The reference runs single-threaded so its FP32
reductions are sequential.
"""
import os
import sys

import numpy as np
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "gpu-conjugate-gradient-solver_b200"))
from oracle import oracle as O  # noqa: E402
import gpusolver_b200 as gs  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def grid2d(nx, ny, diag=4.0):
    """5-point Laplacian in the order of gaussSeidelSymmUnittest.cc:32-75."""
    rows, cols, vals = [], [], []
    for y in range(ny):
        for x in range(nx):
            i = y * nx + x
            rows.append(i); cols.append(i); vals.append(diag)
            for (cond, j) in ((x > 0, i - 1), (x + 1 < nx, i + 1), (y > 0, i - nx), (y + 1 < ny, i + nx)):
                if cond:
                    rows.append(i); cols.append(j); vals.append(-1.0)
    m = sp.csr_matrix((vals, (rows, cols)), shape=(nx * ny, nx * ny))
    m.sort_indices()
    return O.CsrView.from_scipy(m)


def save(name, **arrays):
    np.savez_compressed(os.path.join(OUT, name), **arrays)
    print("wrote", name, {k: getattr(v, "shape", None) for k, v in arrays.items()})


def main():
    O.ref_set_threads(1)
    # 1. multicolour SGS on the 8x8 Poisson of gaussSeidelSymmUnittest.cc (rhs sin(0.17 i) + 0.5)
    a = grid2d(8, 8)
    rhs = (np.sin(0.17 * np.arange(64, dtype=np.float32)) + 0.5).astype(np.float32)
    z = O.ref_sgs_apply(a, rhs, 1.0, 1)
    nc, colors, verts, offs = O.ref_coloring(a)
    save("sgs_poisson8x8.npz", row_ptr=a.row_ptr, col_idx=a.col_idx, val=a.val.astype(np.float32),
         rhs=rhs, z=z, colors=colors, verts=verts, offs=offs)

    # 2. colouring and RCM of the 7-point Poisson 16^3 and of a Kuhn P1 Laplacian 12^3
    for name, m in (("poisson16", gs.poisson7(16)), ("kuhn12", gs.kuhn_laplacian(12))):
        c = O.CsrView.of(m)
        nc, colors, verts, offs = O.ref_coloring(c)
        o2n, n2o = O.ref_rcm(c)
        prp, pci, pv = O.ref_apply_permutation(c, o2n, n2o)
        qrp, qci, qv = O.ref_permute_matrix(c, o2n, o2n)
        ec, ev, orp, oc, ov = O.ref_ell(c, 7)
        save(f"setup_{name}.npz", row_ptr=c.row_ptr, col_idx=c.col_idx, val=c.val.astype(np.float32),
             ncolors=np.int32(nc), colors=colors, verts=verts, offs=offs, o2n=o2n, n2o=n2o,
             ap_row_ptr=prp, ap_col=pci, ap_val=pv, pm_row_ptr=qrp, pm_col=qci, pm_val=qv,
             ell_col=ec, ell_val=ev, ovf_row_ptr=orp, ovf_col=oc, ovf_val=ov)

    # 3. the reference's FP32 AMG-PCG (CGSolver + MultigridGaussSeidelPreconditioner,
    #    coarse = pre + post SGS steps) on Poisson 16^3 with the product's SA hierarchy
    #    and RCM permutations per level, as examples/multigridPoisson/mainTetmeshPoisson.cc:63-98,571-579 builds it.
    A0 = gs.poisson7(16)
    H = gs.Hierarchy.build(A0, 1, 0.1, 10, 200)
    A = [H.A(k) for k in range(H.levels)]
    P = [H.P(k) for k in range(H.levels - 1)]
    R = [H.R(k) for k in range(H.levels - 1)]
    # Values rounded to FP32: this fixture is an FP32 reference run.
    f32 = lambda m: O.CsrView(m.rows, m.cols, m.row_ptr, m.col_idx, m.val.astype(np.float32).astype(np.float64))
    A, P, R = [f32(m) for m in A], [f32(m) for m in P], [f32(m) for m in R]
    perms = [O.ref_rcm(m) for m in A]
    b = gs.uniform_rhs(A0.rows, 0).astype(np.float32)
    x, it, _, _ = O.ref_amg_pcg(A, P, R, b, perms=perms, tol=1e-6, max_iter=100)
    arrays = dict(b=b, x=x, iterations=np.int32(it), levels=np.int32(len(A)))
    for k, m in enumerate(A):
        arrays.update({f"A{k}_rp": m.row_ptr, f"A{k}_ci": m.col_idx, f"A{k}_v": m.val.astype(np.float32),
                       f"A{k}_shape": np.array([m.rows, m.cols], np.int32),
                       f"o2n{k}": perms[k][0], f"n2o{k}": perms[k][1]})
    for k, (p, r) in enumerate(zip(P, R)):
        for tag, m in (("P", p), ("R", r)):
            arrays.update({f"{tag}{k}_rp": m.row_ptr, f"{tag}{k}_ci": m.col_idx,
                           f"{tag}{k}_v": m.val.astype(np.float32),
                           f"{tag}{k}_shape": np.array([m.rows, m.cols], np.int32)})
    save("amg_pcg_poisson16_f32.npz", **arrays)


if __name__ == "__main__":
    main()
