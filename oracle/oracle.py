"""ORACLE -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg and reference arm may import this module, and only as the checker or as
the timed CPU baseline; the product (``gpu-conjugate-gradient-solver_b200``)
never does.

It wraps two CPU libraries:
  * ``oracle/liboracle.so`` -- the project's restatement of the reference's
    AMG-PCG path (``oracle/oracle.cc``), FP64 / FP32 / mixed;
  * ``oracle/_ref/libgsref.so`` -- the reference's own CPU sources compiled
    unmodified (``oracle/ref/Makefile``), the pin for the restatement and
    the ``reference`` CPU baseline.
and restates, in numpy with explicit loops, the smoothed-aggregation
coarsening that the reference delegates to amgcl (absent and unpinned:
``cmake/recipes/amgcl.cmake:11-12`` fetches ``ddemidov/amgcl`` at ``master``).
The restatement follows the published method (Vanek, Mandel & Brezina,
Computing 56, 1996) with the parameter choices the product documents, and
is the bit-exact check of the product's integer coarsening output.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libgsref.so")

_orc = None
_ref = None


class _OrcCsr(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("rowptr", C.c_void_p),
                ("col", C.c_void_p), ("val", C.c_void_p)]


class _OrcOptions(C.Structure):
    _fields_ = [("smoother", C.c_int), ("pre", C.c_int), ("post", C.c_int),
                ("coarse_steps", C.c_int), ("vcycles", C.c_int), ("omega", C.c_double),
                ("coarse_solver", C.c_int), ("flexible", C.c_int), ("tol", C.c_double),
                ("max_iter", C.c_int), ("colour_weights", C.c_void_p),
                ("weight_offsets", C.c_void_p), ("alias_correction", C.c_int),
                ("coarse_smoother", C.c_int), ("node_weights", C.c_void_p), ("node_offsets", C.c_void_p),
                ("half_sweeps", C.c_int), ("colour_counts", C.c_void_p), ("colour_verts", C.c_void_p),
                ("colour_offs", C.c_void_p), ("relaxed", C.c_int)]


class _RefCsr(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("rowptr", C.c_void_p),
                ("col", C.c_void_p), ("val", C.c_void_p)]


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError(f"{ORACLE_LIB} missing: run `make -C {HERE}`")
        _orc = C.CDLL(ORACLE_LIB)
        _orc.orc_last_error.restype = C.c_char_p
        _orc.orc_sa_last_error.restype = C.c_char_p
        _orc.orc_sa_levels.argtypes = [C.c_void_p]
        _orc.orc_sa_free.argtypes = [C.c_void_p]
        _orc.orc_sa_matrix.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]
        _orc.orc_dot_f64.restype = C.c_double
        _orc.orc_dot_f32.restype = C.c_float
        _orc.orc_gs_color_f64.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double]
        _orc.orc_gs_color_f32.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_float]
        _orc.orc_block_gs_color_f64.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                                C.c_void_p, C.c_void_p, C.c_double]
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref() -> C.CDLL:
    """The reference's own CPU path (compiled from its sources)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise ImportError(f"{REF_LIB} missing: run `make -C {HERE}/ref` where the reference tree exists")
        _ref = C.CDLL(REF_LIB)
        _ref.gsref_last_error.restype = C.c_char_p
        _ref.gsref_gs_color.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_float]
        _ref.gsref_block_gs_color3x3.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_int, C.c_int, C.c_int,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_float]
        _ref.gsref_sgs_apply.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_float, C.c_int]
        _ref.gsref_pcg.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_int, C.c_float, C.c_int, C.c_float, C.c_int,
                                   C.c_void_p, C.c_void_p, C.c_void_p]
    return _ref


def _p(a: np.ndarray):
    # data_as keeps a reference to the array, so temporaries stay alive
    # for the duration of the call
    return a.ctypes.data_as(C.c_void_p)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ref_check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(ref().gsref_last_error().decode())


def _orc_check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(orc().orc_last_error().decode())


class CsrView:
    """Any object with rows, cols, row_ptr, col_idx, val."""

    def __init__(self, rows, cols, row_ptr, col_idx, val):
        self.rows, self.cols = int(rows), int(cols)
        self.row_ptr, self.col_idx, self.val = _i32(row_ptr), _i32(col_idx), _f64(val)

    @property
    def nnz(self):
        return int(self.row_ptr[-1])

    @staticmethod
    def of(m) -> "CsrView":
        return CsrView(m.rows, m.cols, m.row_ptr, m.col_idx, m.val)

    @staticmethod
    def from_scipy(m) -> "CsrView":
        m = m.tocsr()
        m.sort_indices()
        return CsrView(m.shape[0], m.shape[1], m.indptr, m.indices, m.data)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col_idx, self.row_ptr), shape=(self.rows, self.cols))


# ---- reference (compiled) ---------------------------------------------------
def ref_coloring(m) -> Tuple[int, np.ndarray, np.ndarray, np.ndarray]:
    m = CsrView.of(m)
    n = m.rows
    c, v, o = np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n + 2, np.int32)
    nc = C.c_int()
    _ref_check(ref().gsref_coloring(n, _p(m.row_ptr), _p(m.col_idx), _p(c), _p(v), _p(o), C.byref(nc)))
    return nc.value, c, v, o[: nc.value + 1].copy()


def ref_rcm(m) -> Tuple[np.ndarray, np.ndarray]:
    m = CsrView.of(m)
    o2n, n2o = np.empty(m.rows, np.int32), np.empty(m.rows, np.int32)
    _ref_check(ref().gsref_rcm(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(o2n), _p(n2o)))
    return o2n, n2o


def ref_apply_permutation(m, o2n, n2o):
    m = CsrView.of(m)
    rp, ci, v = np.empty(m.rows + 1, np.int32), np.empty(m.nnz, np.int32), np.empty(m.nnz, np.float32)
    _ref_check(ref().gsref_apply_permutation(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(_f32(m.val)),
                                             _p(_i32(o2n)), _p(_i32(n2o)), _p(rp), _p(ci), _p(v)))
    return rp, ci, v


def ref_permute_matrix(m, ro2n, co2n):
    m = CsrView.of(m)
    rp, ci, v = np.empty(m.rows + 1, np.int32), np.empty(m.nnz, np.int32), np.empty(m.nnz, np.float32)
    _ref_check(ref().gsref_permute_matrix(m.rows, m.cols, _p(m.row_ptr), _p(m.col_idx),
                                          _p(_f32(m.val)), _p(_i32(ro2n)), _p(_i32(co2n)), _p(rp),
                                          _p(ci), _p(v)))
    return rp, ci, v


def ref_ell(m, width):
    m = CsrView.of(m)
    n = m.rows
    ec, ev = np.empty(n * width, np.int32), np.empty(n * width, np.float32)
    orp, oc, ov = np.empty(n + 1, np.int32), np.empty(max(m.nnz, 1), np.int32), np.empty(max(m.nnz, 1), np.float32)
    on = C.c_int()
    _ref_check(ref().gsref_ell(n, _p(m.row_ptr), _p(m.col_idx), _p(_f32(m.val)), width, _p(ec), _p(ev),
                               _p(orp), _p(oc), _p(ov), C.byref(on)))
    return ec, ev, orp, oc[: on.value], ov[: on.value]


def ref_block_graph(m):
    m = CsrView.of(m)
    grp, gci = np.empty(m.rows // 3 + 1, np.int32), np.empty(max(m.nnz, 1), np.int32)
    _ref_check(ref().gsref_block_graph(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(_f32(m.val)), _p(grp), _p(gci)))
    return grp, gci[: grp[-1]]


def ref_block_inverses(m):
    m = CsrView.of(m)
    out = np.empty(3 * m.rows, np.float32)
    _ref_check(ref().gsref_block_inverses3x3(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(_f32(m.val)), _p(out)))
    return out


def ref_spmv(m, x):
    m = CsrView.of(m)
    y = np.empty(m.rows, np.float32)
    _ref_check(ref().gsref_spmv(m.rows, m.cols, _p(m.row_ptr), _p(m.col_idx), _p(_f32(m.val)),
                                _p(_f32(x)), _p(y)))
    return y


def ref_gs_color(m, order, start, count, rhs, x, omega):
    m = CsrView.of(m)
    x = _f32(x).copy()
    order = _i32(order)
    _ref_check(ref().gsref_gs_color(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(_f32(m.val)), _p(order),
                                    len(order), start, count, _p(_f32(rhs)), _p(x), omega))
    return x


def ref_sgs_apply(m, rhs, omega=1.0, sweeps=1):
    m = CsrView.of(m)
    z = np.empty(m.rows, np.float32)
    _ref_check(ref().gsref_sgs_apply(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(_f32(m.val)),
                                     _p(_f32(rhs)), _p(z), omega, sweeps))
    return z


def ref_apply_block_inverses(dinv, r):
    c = np.empty(len(r), np.float32)
    _ref_check(ref().gsref_apply_block_inverses3x3(len(r), _p(_f32(dinv)), _p(_f32(r)), _p(c)))
    return c


def ref_dot(x, y) -> float:
    out = C.c_float()
    _ref_check(ref().gsref_dot(len(x), _p(_f32(x)), _p(_f32(y)), C.byref(out)))
    return out.value


def ref_set_threads(n: int) -> None:
    ref().gsref_set_threads(int(n))


def ref_max_threads() -> int:
    return ref().gsref_max_threads()


def _ref_levels(mats):
    keep = []
    arr = (_RefCsr * max(len(mats), 1))()
    for i, m in enumerate(mats):
        m = CsrView.of(m)
        v = _f32(m.val)
        keep += [m, v]
        arr[i] = _RefCsr(m.rows, m.cols, m.row_ptr.ctypes.data, m.col_idx.ctypes.data, v.ctypes.data)
    return arr, keep


def ref_hierarchical_reordering(A: Sequence, P: Sequence, R: Sequence):
    """The reference's HierarchicalReordering::compute (FP32 hierarchy)."""
    L = len(A)
    a, ka = _ref_levels(A)
    p, kp = _ref_levels(P)
    r, kr = _ref_levels(R)
    o2n = [np.empty(CsrView.of(m).rows, np.int32) for m in A]
    n2o = [np.empty(CsrView.of(m).rows, np.int32) for m in A]
    po = (C.c_void_p * L)(*[q.ctypes.data for q in o2n])
    pn = (C.c_void_p * L)(*[q.ctypes.data for q in n2o])
    _ref_check(ref().gsref_hierarchical_reordering(L, a, p, r, po, pn))
    return list(zip(o2n, n2o))


def hierarchical_reordering(A: Sequence, R: Sequence):
    """Independent numpy restatement of HierarchicalReordering::compute
    (src/ReorderingStrategies/HierarchicalReordering.cc:11-278), using the
    reference's RCM (oracle/_ref) for the per-level RCM ranks."""
    L = len(A)
    perms = [None] * L
    perms[L - 1] = ref_rcm(A[L - 1])
    for f in range(L - 2, -1, -1):
        Rm = CsrView.of(R[f])
        nf, nc = CsrView.of(A[f]).rows, Rm.rows
        parent = np.full(nf, -1, np.int64)
        best = np.full(nf, -1.0, np.float32)
        w = np.abs(Rm.val.astype(np.float32))
        for c in range(nc):
            for e in range(Rm.row_ptr[c], Rm.row_ptr[c + 1]):
                j = Rm.col_idx[e]
                if w[e] > best[j]:
                    best[j], parent[j] = w[e], c
        frcm = ref_rcm(A[f])[0]
        crank = perms[f + 1][0]
        prank = np.where(parent >= 0, crank[np.maximum(parent, 0)], nc)
        order = np.lexsort((frcm, prank)).astype(np.int32)
        o2n = np.empty(nf, np.int32)
        o2n[order] = np.arange(nf, dtype=np.int32)
        perms[f] = (o2n, order)
    return perms


def ref_amg_pcg(A: Sequence, P: Sequence, R: Sequence, b, x0=None, perms=None, smoother=0,
                pre=1, post=1, coarse=None, vcycles=1, omega=1.0, tol=1e-6, max_iter=1000):
    """The reference's CGSolver + Multigrid{GaussSeidel,BlockGaussSeidel}Preconditioner
    on its CPUBackend, FP32. Returns (x, iterations, setup_ms, solve_ms)."""
    L = len(A)
    a, ka = _ref_levels(A)
    p, kp = _ref_levels(P)
    r, kr = _ref_levels(R)
    o2n = n2o = None
    keep = []
    if perms is not None:
        po = [_i32(q[0]) for q in perms]
        pn = [_i32(q[1]) for q in perms]
        keep += po + pn
        o2n = (C.c_void_p * L)(*[q.ctypes.data for q in po])
        n2o = (C.c_void_p * L)(*[q.ctypes.data for q in pn])
    if coarse is None:
        coarse = pre + post
    bf = _f32(b)
    x = np.zeros(len(bf), np.float32) if x0 is None else _f32(x0).copy()
    it = C.c_int()
    sm, so = C.c_double(), C.c_double()
    _ref_check(ref().gsref_amg_pcg(L, a, p, r, o2n, n2o, smoother, pre, post, coarse, vcycles,
                                   C.c_float(omega), C.c_float(tol), max_iter, _p(bf), _p(x),
                                   C.byref(it), C.byref(sm), C.byref(so)))
    return x, it.value, sm.value, so.value


def ref_pcg(m, b, preconditioner=0, omega=1.0, sweeps=1, tol=1e-6, max_iter=1000, perm=None):
    m = CsrView.of(m)
    x = np.zeros(m.rows, np.float32)
    it = C.c_int()
    o2n = n2o = None
    if perm is not None:
        o2n, n2o = _i32(perm[0]), _i32(perm[1])
    _ref_check(ref().gsref_pcg(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(_f32(m.val)),
                               None if o2n is None else _p(o2n), None if n2o is None else _p(n2o),
                               preconditioner, omega, sweeps, tol, max_iter, _p(_f32(b)), _p(x),
                               C.byref(it)))
    return x, it.value


# ---- restatement -------------------------------------------------------------
def _orc_levels(mats):
    arr = (_OrcCsr * max(len(mats), 1))()
    keep = []
    for i, m in enumerate(mats):
        m = CsrView.of(m)
        keep.append(m)
        arr[i] = _OrcCsr(m.rows, m.cols, m.row_ptr.ctypes.data, m.col_idx.ctypes.data, m.val.ctypes.data)
    return arr, keep


PREC_F64, PREC_F32, PREC_MIXED = 0, 1, 2


def _colour_arrays(colourings, L, keep):
    """Per-level (color_vertices, color_offsets) or None -> the counts array and
    the two pointer arrays of orc_options (None when no colouring is given)."""
    if colourings is None:
        return None, None, None
    counts = np.array([0 if c is None else len(c[1]) - 1 for c in colourings] + [0] * (L - len(colourings)),
                      np.int32)
    cverts = [None if c is None else _i32(c[0]) for c in colourings]
    coffs = [None if c is None else _i32(c[1]) for c in colourings]
    keep += [counts] + [q for q in cverts + coffs if q is not None]
    ptr = lambda q: None if q is None else q.ctypes.data
    cv = (C.c_void_p * L)(*([ptr(q) for q in cverts] + [None] * (L - len(cverts))))
    co = (C.c_void_p * L)(*([ptr(q) for q in coffs] + [None] * (L - len(coffs))))
    keep += [cv, co]
    return counts, cv, co


def amg_pcg(A, P, R, b, x0=None, perms=None, precision=PREC_F64, smoother=0, pre=1, post=1,
            coarse_steps=None, vcycles=1, omega=1.0, coarse_solver=1, flexible=0, tol=1e-8,
            max_iter=1000, weights: Optional[List[np.ndarray]] = None, alias=0, coarse_smoother=-1,
            node_weights: Optional[List[np.ndarray]] = None, half_sweeps=0, colourings=None, relaxed=0):
    """The restated CGSolver + V-cycle. Returns (x, iterations, status, ratio).
    node_weights: per level, one weight per node (caller order) of the 3x3
    block Gauss-Seidel levels, replacing the colour weights there.
    colourings: per level None or (color_vertices, color_offsets) replacing the
    greedy colouring of a scalar Gauss-Seidel level; relaxed 1: a pass on such
    a level reads its own colour's rows from the iterate its sweep started with."""
    L = len(A)
    a, ka = _orc_levels(A)
    p, kp = _orc_levels(P)
    r, kr = _orc_levels(R)
    o2n = n2o = None
    keep = []
    if perms is not None:
        po = [_i32(q[0]) for q in perms]
        pn = [_i32(q[1]) for q in perms]
        keep += po + pn
        o2n = (C.c_void_p * L)(*[q.ctypes.data for q in po])
        n2o = (C.c_void_p * L)(*[q.ctypes.data for q in pn])
    wv = wo = None
    if weights is not None:
        offs = np.zeros(L + 1, np.int32)
        for k, w in enumerate(weights):
            offs[k + 1] = offs[k] + len(w)
        wv, wo = _f64(np.concatenate(weights)), offs
    nv = no = None
    if node_weights is not None:
        no = np.zeros(L + 1, np.int32)
        for k, w in enumerate(node_weights):
            no[k + 1] = no[k] + len(w)
        nv = _f64(np.concatenate(node_weights))
    cc, cv, co = _colour_arrays(colourings, L, keep)
    opts = _OrcOptions(smoother, pre, post, pre + post if coarse_steps is None else coarse_steps,
                       vcycles, omega, coarse_solver, flexible, tol, max_iter,
                       None if wv is None else wv.ctypes.data,
                       None if wo is None else wo.ctypes.data, alias, coarse_smoother,
                       None if nv is None else nv.ctypes.data, None if no is None else no.ctypes.data,
                       half_sweeps, None if cc is None else cc.ctypes.data,
                       None if cv is None else C.cast(cv, C.c_void_p).value,
                       None if co is None else C.cast(co, C.c_void_p).value, relaxed)
    bb = _f64(b)
    x = np.zeros(len(bb)) if x0 is None else _f64(x0).copy()
    it, st, ratio = C.c_int(), C.c_int(), C.c_double()
    _orc_check(orc().orc_amg_pcg(precision, L, a, p, r, o2n, n2o, C.byref(opts), _p(bb), _p(x),
                                 C.byref(it), C.byref(st), C.byref(ratio)))
    return x, it.value, st.value, ratio.value


def precondition(A, P, R, rvec, perms=None, precision=PREC_F64, smoother=0, pre=1, post=1,
                 coarse_steps=None, vcycles=1, omega=1.0, coarse_solver=1, alias=0, coarse_smoother=-1,
                 half_sweeps=0, colourings=None, relaxed=0):
    """z = M r for r in the level-0 permuted order (colourings / relaxed as in
    amg_pcg)."""
    L = len(A)
    a, ka = _orc_levels(A)
    p, kp = _orc_levels(P)
    r, kr = _orc_levels(R)
    o2n = n2o = None
    keep = []
    if perms is not None:
        po = [_i32(q[0]) for q in perms]
        pn = [_i32(q[1]) for q in perms]
        keep += po + pn
        o2n = (C.c_void_p * L)(*[q.ctypes.data for q in po])
        n2o = (C.c_void_p * L)(*[q.ctypes.data for q in pn])
    cc, cv, co = _colour_arrays(colourings, L, keep)
    opts = _OrcOptions(smoother, pre, post, pre + post if coarse_steps is None else coarse_steps,
                       vcycles, omega, coarse_solver, 0, 1e-8, 1, None, None, alias, coarse_smoother,
                       None, None, half_sweeps, None if cc is None else cc.ctypes.data,
                       None if cv is None else C.cast(cv, C.c_void_p).value,
                       None if co is None else C.cast(co, C.c_void_p).value, relaxed)
    rv = _f64(rvec)
    z = np.empty_like(rv)
    _orc_check(orc().orc_precondition(precision, L, a, p, r, o2n, n2o, C.byref(opts), _p(rv), _p(z)))
    return z


def spmv(m, x, f32=False):
    m = CsrView.of(m)
    if f32:
        y = np.empty(m.rows, np.float32)
        orc().orc_spmv_f32(m.rows, m.cols, _p(m.row_ptr), _p(m.col_idx), _p(m.val), _p(_f32(x)), _p(y))
    else:
        y = np.empty(m.rows, np.float64)
        orc().orc_spmv_f64(m.rows, m.cols, _p(m.row_ptr), _p(m.col_idx), _p(m.val), _p(_f64(x)), _p(y))
    return y


def gs_color(m, order, start, count, rhs, x, omega, f32=False):
    m = CsrView.of(m)
    order = _i32(order)
    if f32:
        x = _f32(x).copy()
        _orc_check(orc().orc_gs_color_f32(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(m.val), _p(order),
                                          start, count, _p(_f32(rhs)), _p(x), omega))
    else:
        x = _f64(x).copy()
        _orc_check(orc().orc_gs_color_f64(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(m.val), _p(order),
                                          start, count, _p(_f64(rhs)), _p(x), omega))
    return x


def block_gs_color(m, order, start, count, dinv, rhs, x, omega):
    m = CsrView.of(m)
    x = _f64(x).copy()
    _orc_check(orc().orc_block_gs_color_f64(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(m.val),
                                            _p(_i32(order)), start, count, _p(_f64(dinv)),
                                            _p(_f64(rhs)), _p(x), omega))
    return x


def block_inverses(m):
    m = CsrView.of(m)
    out = np.empty(3 * m.rows, np.float64)
    _orc_check(orc().orc_block_inverses_f64(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(m.val), _p(out)))
    return out


def dot(x, y, f32=False) -> float:
    if f32:
        return float(orc().orc_dot_f32(len(x), _p(_f32(x)), _p(_f32(y))))
    return float(orc().orc_dot_f64(len(x), _p(_f64(x)), _p(_f64(y))))


def coloring(m):
    m = CsrView.of(m)
    v, o = np.empty(m.rows, np.int32), np.empty(m.rows + 1, np.int32)
    nc = orc().orc_coloring(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(v), _p(o))
    return nc, v, o[: nc + 1].copy()


# ---- smoothed aggregation, numpy restatement ---------------------------------
def node_priority(v: int) -> int:
    """MurmurHash3's 32-bit finaliser (Appleby, public domain): the node
    priority of the independent-set rounds."""
    v &= 0xFFFFFFFF
    v ^= v >> 16
    v = (v * 0x85EBCA6B) & 0xFFFFFFFF
    v ^= v >> 13
    v = (v * 0xC2B2AE35) & 0xFFFFFFFF
    v ^= v >> 16
    return v


def mis2_aggregates(nn, nbr, w, strong):
    """Aggregation from a distance-2 maximal independent set of the strength
    graph by max propagation (Bell, Dalton & Olson, SIAM J. Sci. Comput.
    34(4), 2012), one synchronous round at a time as a GPU runs it: keys
    (state << 32 | priority), state 2 root / 1 undecided / 0 out; the largest
    key over the closed strong neighbourhood, twice; an undecided node that
    sees its own key is a root, one that sees a root's key is out. Roots are
    numbered in index order; a non-root strong neighbour of roots joins the
    lowest-numbered one; every other node joins its strongest strongly
    coupled aggregated neighbour (first in column order on ties); what is
    left becomes singletons after the roots, in index order. Returns (agg with
    -2 for isolated nodes, number of aggregates, rounds)."""
    state = [0 if not any(strong[i]) else 1 for i in range(nn)]
    prio = [node_priority(i) for i in range(nn)]
    rounds = 0
    while any(st == 1 for st in state):
        rounds += 1
        key = [(state[i] << 32) | prio[i] for i in range(nn)]
        t1 = [max([key[i]] + [key[j] for q, j in enumerate(nbr[i]) if strong[i][q]]) for i in range(nn)]
        t2 = [max([t1[i]] + [t1[j] for q, j in enumerate(nbr[i]) if strong[i][q]]) for i in range(nn)]
        for i in range(nn):
            if state[i] != 1:
                continue
            if t2[i] == (1 << 32) | prio[i]:
                state[i] = 2
            elif t2[i] >> 32 == 2:
                state[i] = 0
    agg = np.full(nn, -1, np.int64)
    nagg = 0
    for i in range(nn):
        if not any(strong[i]):
            agg[i] = -2
        elif state[i] == 2:
            agg[i] = nagg
            nagg += 1
    for i in range(nn):
        if state[i] != 2:
            continue
        for q, j in enumerate(nbr[i]):
            if strong[i][q] and agg[j] == -1:
                agg[j] = agg[i]
    agg1 = agg.copy()
    for i in range(nn):
        if agg[i] != -1:
            continue
        best, bw = -1, -1.0
        for q, j in enumerate(nbr[i]):
            if strong[i][q] and agg1[j] >= 0 and w[i][q] > bw:
                bw, best = w[i][q], agg1[j]
        if best >= 0:
            agg[i] = best
    for i in range(nn):
        if agg[i] == -1:
            agg[i] = nagg
            nagg += 1
    return agg, nagg, rounds


def sa_coarsen(a, block: int = 1, eps: float = 0.1, aggregation: int = 0):
    """One smoothed-aggregation step. Returns (agg, P, R, Ac) with P, R, Ac
    as scipy CSR. Loops in natural order so every tie and every floating-point
    sum happens in the documented order. aggregation 0: the sequential three
    steps; 1: mis2_aggregates."""
    import scipy.sparse as sp
    a = CsrView.of(a)
    n = a.rows
    nn = n // block
    rp, ci, v = a.row_ptr, a.col_idx, a.val
    # node couplings (Frobenius norms of the blocks), neighbours sorted
    nbr: List[List[int]] = [[] for _ in range(nn)]
    w: List[List[float]] = [[] for _ in range(nn)]
    d = np.zeros(nn)
    for i in range(nn):
        acc = {}
        dsum = 0.0
        for r in range(block * i, block * i + block):
            for k in range(rp[r], rp[r + 1]):
                j = ci[k] // block
                sq = v[k] * v[k]
                if j == i:
                    dsum += sq
                else:
                    acc[j] = acc.get(j, 0.0) + sq
        d[i] = np.sqrt(dsum)
        for j in sorted(acc):
            nbr[i].append(j)
            w[i].append(float(np.sqrt(acc[j])))
    eps2 = eps * eps
    strong = [[w[i][q] * w[i][q] >= eps2 * d[i] * d[nbr[i][q]] for q in range(len(nbr[i]))]
              for i in range(nn)]
    if aggregation == 1:
        agg, nagg, _ = mis2_aggregates(nn, nbr, w, strong)
    else:
        agg, nagg = _sequential_aggregates(nn, nbr, w, strong)
    return _sa_transfer(a, block, nbr, strong, agg, nagg)


def _sequential_aggregates(nn, nbr, w, strong):
    agg = np.full(nn, -1, np.int64)
    for i in range(nn):
        if not any(strong[i]):
            agg[i] = -2
    nagg = 0
    for i in range(nn):  # step 1
        if agg[i] != -1:
            continue
        if any(strong[i][q] and agg[nbr[i][q]] != -1 for q in range(len(nbr[i]))):
            continue
        agg[i] = nagg
        for q, j in enumerate(nbr[i]):
            if strong[i][q]:
                agg[j] = nagg
        nagg += 1
    agg1 = agg.copy()
    for i in range(nn):  # step 2
        if agg[i] != -1:
            continue
        best, bw = -1, -1.0
        for q, j in enumerate(nbr[i]):
            if strong[i][q] and agg1[j] >= 0 and w[i][q] > bw:
                bw, best = w[i][q], agg1[j]
        if best >= 0:
            agg[i] = best
    for i in range(nn):  # step 3
        if agg[i] != -1:
            continue
        agg[i] = nagg
        for q, j in enumerate(nbr[i]):
            if strong[i][q] and agg[j] == -1:
                agg[j] = nagg
        nagg += 1
    return agg, nagg


def _sa_transfer(a, block, nbr, strong, agg, nagg):
    """Tentative prolongator, filtered matrix, damping, smoothed P, R and the
    Galerkin product from given aggregates."""
    import scipy.sparse as sp
    n = a.rows
    rp, ci, v = a.row_ptr, a.col_idx, a.val
    size = np.bincount(agg[agg >= 0], minlength=nagg)
    nc = nagg * block
    tcol = np.full(n, -1, np.int64)
    tval = np.zeros(n)
    for row in range(n):
        i, comp = divmod(row, block)
        if agg[i] >= 0:
            tcol[row] = agg[i] * block + comp
            tval[row] = 1.0 / np.sqrt(float(size[agg[i]]))
    # filtered matrix: keep same-node and strong-node entries, lump the rest
    keep = np.zeros(a.nnz, bool)
    fdiag = np.zeros(n)
    for row in range(n):
        i = row // block
        sset = {nbr[i][q] for q in range(len(nbr[i])) if strong[i][q]}
        dd, lump = 0.0, 0.0
        for k in range(rp[row], rp[row + 1]):
            j = ci[k] // block
            kp = (j == i) or (j in sset)
            keep[k] = kp
            if ci[k] == row:
                dd += v[k]
            elif not kp:
                lump += v[k]
        fdiag[row] = dd + lump
    rho = 0.0
    for row in range(n):
        s = abs(fdiag[row])
        for k in range(rp[row], rp[row + 1]):
            if keep[k] and ci[k] != row:
                s += abs(v[k])
        if fdiag[row] != 0.0:
            rho = max(rho, s / abs(fdiag[row]))
    omega = (4.0 / 3.0) / rho if rho > 0 else 0.0
    prow, pcol, pval = [0], [], []
    for row in range(n):
        scale = omega / fdiag[row] if fdiag[row] != 0.0 else 0.0
        acc = {}
        for k in range(rp[row], rp[row + 1]):
            if not keep[k]:
                continue
            c = ci[k]
            if tcol[c] < 0:
                continue
            afv = fdiag[row] if c == row else v[k]
            coef = (1.0 if c == row else 0.0) - scale * afv
            acc[tcol[c]] = acc.get(tcol[c], 0.0) + coef * tval[c]
        for c in sorted(acc):
            pcol.append(c)
            pval.append(acc[c])
        prow.append(len(pcol))
    P = sp.csr_matrix((np.array(pval), np.array(pcol, np.int64), np.array(prow, np.int64)), shape=(n, nc))
    R = P.T.tocsr()
    R.sort_indices()
    A = a.to_scipy()
    Ac = (R @ (A @ P)).tocsr()
    Ac.sort_indices()
    agg_out = np.where(agg < 0, -1, agg).astype(np.int32)
    return agg_out, P, R, Ac


def sa_hierarchy(a, block=1, eps=0.1, max_levels=10, min_dofs=1000):
    """The C++ twin of build_hierarchy (sequential aggregation; oracle/sa.cc):
    the same levels at full sizes in seconds. Returns (A, P, R) as CsrView lists."""
    L = orc()
    m = CsrView.of(a)
    h = C.c_void_p()
    if L.orc_sa_build(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(m.val), block, C.c_double(eps),
                      max_levels, min_dofs, C.byref(h)) != 0:
        raise RuntimeError(L.orc_sa_last_error().decode())
    try:
        out = ([], [], [])
        for k in range(L.orc_sa_levels(h)):
            for which in range(3):
                if which > 0 and k == L.orc_sa_levels(h) - 1:
                    continue
                r, c, z = C.c_int(), C.c_int(), C.c_int()
                L.orc_sa_matrix(h, k, which, C.byref(r), C.byref(c), C.byref(z), None, None, None)
                rp, ci, v = np.empty(r.value + 1, np.int32), np.empty(z.value, np.int32), np.empty(z.value)
                L.orc_sa_matrix(h, k, which, C.byref(r), C.byref(c), C.byref(z), _p(rp), _p(ci), _p(v))
                out[which].append(CsrView(r.value, c.value, rp, ci, v))
        return out
    finally:
        L.orc_sa_free(h)


def build_hierarchy(a, block=1, eps=0.1, max_levels=10, min_dofs=1000, aggregation=0):
    """AMGHierarchyBuilder::build semantics with the numpy restatement."""
    A = [CsrView.of(a).to_scipy()]
    P, R, aggs = [], [], []
    for level in range(max_levels):
        cur = A[-1]
        if cur.shape[0] <= min_dofs:
            break
        agg, p, r, ac = sa_coarsen(CsrView.from_scipy(cur), block, eps * 0.5 ** level, aggregation)
        if ac.shape[0] == 0 or ac.shape[0] >= cur.shape[0]:
            break
        aggs.append(agg)
        P.append(p)
        R.append(r)
        A.append(ac)
    return A, P, R, aggs
