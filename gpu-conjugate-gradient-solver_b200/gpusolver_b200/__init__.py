"""Python binding of the gpusolver_b200 C ABI (include/gpusolver_b200.h).

A thin ctypes layer over ``libgpusolver_b200.so`` (built in-tree by the
package Makefile). The names mirror the reference library's C++ API
(theofbraune/GPU-Conjugate-Gradient-Solver): ``GraphColoring``,
``RCMReordering``, ``HostCSRMatrix.applyPermutation``, ``permuteMatrix``,
``HostELLMatrix``, ``AMGHierarchyBuilder``, ``CGSolver`` with a multigrid
Gauss-Seidel preconditioner. There is no CPU fallback: every solve runs the
CUDA kernels, and creating a solver without a GPU raises ``NoDeviceError``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.dirname(_HERE)
LIB_PATH = os.path.join(_PKG, "libgpusolver_b200.so")

GS_OK = 0
GS_ERR_INVALID = 1
GS_ERR_CUDA = 2
GS_ERR_NOT_FINITE = 3
GS_ERR_NO_DEVICE = 4

STATUS_CONVERGED = 1
STATUS_MAX_ITER = 2
STATUS_BREAKDOWN = 4
STATUS_INITIAL_CONVERGED = 5
STATUS_ZERO_RHS = 6

PROBLEM_POISSON7 = 0
PROBLEM_VARCOEF_GRF = 1
PROBLEM_VARCOEF_LOGUNI = 2
PROBLEM_KUHN_P1 = 3
PROBLEM_ELASTICITY_P1 = 4

#: every C entry point declared in include/gpusolver_b200.h
EXPORTED_SYMBOLS = [
    "gs_last_error", "gs_version", "gs_greedy_coloring", "gs_smallest_last_coloring", "gs_relaxed_coloring",
    "gs_relaxed_block_coloring",
    "gs_rcm", "gs_apply_permutation",
    "gs_permute_matrix", "gs_ell_build", "gs_block_graph", "gs_block_inverses3x3",
    "gs_expand_block_permutation", "gs_problem_create", "gs_host_csr_create",
    "gs_host_csr_info", "gs_host_csr_copy", "gs_host_csr_rhs", "gs_host_csr_destroy",
    "gs_uniform_rhs", "gs_set_tune_cache", "gs_hierarchy_build", "gs_hierarchy_from_levels",
    "gs_hierarchy_num_levels", "gs_hierarchy_matrix_info", "gs_hierarchy_matrix",
    "gs_hierarchy_aggregates", "gs_hierarchy_build_ex", "gs_solver_setup_times", "gs_hierarchy_destroy", "gs_hierarchical_reordering", "gs_solver_options_default",
    "gs_solver_create", "gs_solver_solve", "gs_solver_solve_f32", "gs_solver_solve_device",
    "gs_solver_apply_preconditioner", "gs_solver_set_tolerance",
    "gs_solver_set_colour_weights", "gs_solver_num_levels", "gs_solver_level_info",
    "gs_solver_level_format", "gs_solver_level_in_tail", "gs_solver_level_layout", "gs_solver_level_launch",
    "gs_solver_setup_phases",
    "gs_solver_time_kernel", "gs_solver_time_level", "gs_solver_launch_count", "gs_solver_destroy", "gs_dense_spd_inverse",
    "gs_solver_update_matrix",
    "gs_device_csr_create", "gs_device_csr_update_values", "gs_device_csr_destroy", "gs_spmv",
    "gs_gauss_seidel_color", "gs_block_gauss_seidel_color3x3", "gs_apply_block_inverses3x3",
    "gs_dot", "gs_dot_noalloc", "gs_vector_op", "gs_scalar_op",
    "gs_mlp_param_count", "gs_mlp_forward", "gs_mlp_backward", "gs_mlp_adam",
    "gs_solver_colour_features", "gs_solver_error_reduction", "gs_solver_node_features",
    "gs_solver_set_node_weights", "gs_hierarchy_refresh",
    "gs_batch_create", "gs_batch_solve", "gs_batch_solve_device", "gs_batch_set_tolerance",
    "gs_batch_info", "gs_batch_system_rows", "gs_batch_level_info", "gs_batch_launch_count",
    "gs_batch_destroy", "gs_batch_plan_check", "gs_batch_time_kernel",
    "gs_batch_time_level",
    "gs_device_malloc", "gs_device_free", "gs_memcpy", "gs_memset", "gs_stream_create", "gs_stream_destroy",
    "gs_stream_synchronize",
]

F32, F64 = 0, 1
VEC_AXPY, VEC_SCALE, VEC_COPY, VEC_SET_ZERO, VEC_SCALE_BY_VECTOR = 0, 1, 2, 3, 4
SCALAR_DIVIDE, SCALAR_MULTIPLY, SCALAR_SET, SCALAR_COPY, SCALAR_NEGATE, SCALAR_SQRT = range(6)


class SolverError(RuntimeError):
    """A C entry point returned an error status (the reference throws std::runtime_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class NoDeviceError(SolverError):
    pass


class NotFiniteError(SolverError):
    pass


class _Options(C.Structure):
    _fields_ = [
        ("smoother", C.c_int), ("pre_steps", C.c_int), ("post_steps", C.c_int),
        ("coarse_steps", C.c_int), ("vcycles", C.c_int), ("omega", C.c_double),
        ("coarse_solver", C.c_int), ("precision", C.c_int), ("flexible", C.c_int),
        ("use_graph", C.c_int), ("check_every", C.c_int), ("tol", C.c_double),
        ("max_iter", C.c_int), ("reference_vcycle", C.c_int), ("autotune", C.c_int),
        ("coarse_tail", C.c_int), ("lanes", C.c_int), ("sliced_lanes", C.c_int),
        ("coarse_rows", C.c_int), ("coarse_smoother", C.c_int), ("overlap_launch", C.c_int),
        ("packed_rows", C.c_int), ("coloring", C.c_int), ("sweep_launch", C.c_int),
        ("half_sweeps", C.c_int), ("coarse_half", C.c_int),
    ]


class _Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("status", C.c_int), ("spmv", C.c_int),
        ("ratio", C.c_double), ("rhs_norm2", C.c_double), ("solve_ms", C.c_double),
    ]


class _Csr(C.Structure):
    _fields_ = [
        ("rows", C.c_int), ("cols", C.c_int), ("row_ptr", C.c_void_p),
        ("col_idx", C.c_void_p), ("val", C.c_void_p),
    ]


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Loads the shared library (fails loudly when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C {_PKG}` "
                "(there is no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        _lib.gs_last_error.restype = C.c_char_p
        _lib.gs_solver_options_default.restype = None
        _lib.gs_host_csr_destroy.restype = None
        _lib.gs_hierarchy_destroy.restype = None
        _lib.gs_solver_destroy.restype = None
        _lib.gs_batch_destroy.restype = None
        for name in ("gs_hierarchy_build", "gs_problem_create", "gs_host_csr_create",
                     "gs_hierarchy_from_levels", "gs_solver_create"):
            getattr(_lib, name).restype = C.c_int
        _lib.gs_uniform_rhs.argtypes = [C.c_int, C.c_ulonglong, C.c_void_p]
        _lib.gs_problem_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_ulonglong,
                                           C.c_void_p]
        _lib.gs_hierarchy_build.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int,
                                            C.c_void_p]
        _lib.gs_hierarchy_build_ex.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int,
                                               C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        _lib.gs_solver_set_tolerance.argtypes = [C.c_void_p, C.c_double, C.c_int]
        _lib.gs_device_csr_destroy.restype = None
        _lib.gs_device_csr_update_values.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong]
        _lib.gs_gauss_seidel_color.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_longlong,
                                               C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        _lib.gs_block_gauss_seidel_color3x3.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong,
                                                        C.c_longlong, C.c_void_p, C.c_void_p,
                                                        C.c_void_p, C.c_double, C.c_void_p]
        _lib.gs_apply_block_inverses3x3.argtypes = [C.c_longlong, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_int, C.c_void_p]
        _lib.gs_dot.argtypes = [C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        _lib.gs_dot_noalloc.argtypes = [C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                        C.c_void_p]
        _lib.gs_vector_op.argtypes = [C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_double,
                                      C.c_void_p, C.c_int, C.c_void_p]
        _lib.gs_mlp_adam.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                     C.c_void_p]
        _lib.gs_scalar_op.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                      C.c_int, C.c_void_p]
        _lib.gs_solver_node_features.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]
        _lib.gs_solver_set_node_weights.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong]
        _lib.gs_hierarchy_refresh.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    return _lib


def _check(rc: int) -> None:
    if rc != GS_OK:
        msg = lib().gs_last_error().decode(errors="replace")
        if rc == GS_ERR_NO_DEVICE:
            raise NoDeviceError(rc, msg)
        if rc == GS_ERR_NOT_FINITE:
            raise NotFiniteError(rc, msg)
        raise SolverError(rc, msg)


def _p(a: np.ndarray):
    # data_as keeps a reference to the array, so temporaries stay alive
    # for the duration of the call
    return a.ctypes.data_as(C.c_void_p)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class Csr:
    """Host CSR matrix (int32 indices, FP64 values)."""
    rows: int
    cols: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    val: np.ndarray
    rhs: Optional[np.ndarray] = None

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col_idx, self.row_ptr), shape=(self.rows, self.cols))

    @staticmethod
    def from_scipy(m) -> "Csr":
        m = m.tocsr()
        m.sort_indices()
        return Csr(m.shape[0], m.shape[1], _i32(m.indptr), _i32(m.indices), _f64(m.data))

    def matvec(self, x: np.ndarray) -> np.ndarray:
        return self.to_scipy() @ x

    def as_c(self) -> _Csr:
        return _Csr(self.rows, self.cols, self.row_ptr.ctypes.data, self.col_idx.ctypes.data,
                    self.val.ctypes.data)


def _csr_from_handle(h) -> Csr:
    L = lib()
    rows, cols, nnz, has_rhs = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    _check(L.gs_host_csr_info(h, C.byref(rows), C.byref(cols), C.byref(nnz), C.byref(has_rhs)))
    rp = np.empty(rows.value + 1, np.int32)
    ci = np.empty(max(nnz.value, 1), np.int32)
    v = np.empty(max(nnz.value, 1), np.float64)
    _check(L.gs_host_csr_copy(h, _p(rp), _p(ci), _p(v)))
    rhs = None
    if has_rhs.value:
        rhs = np.empty(rows.value, np.float64)
        _check(L.gs_host_csr_rhs(h, _p(rhs)))
    return Csr(rows.value, cols.value, rp, ci[: nnz.value], v[: nnz.value], rhs)


def problem(kind: int, ip: Sequence[int], dp: Sequence[float] = (), seed: int = 0) -> Csr:
    """Synthetic problem generator (the C++ generators in csrc/setup.cc)."""
    L = lib()
    ipa = _i32(list(ip) + [0] * (4 - len(ip)))
    dpa = _f64(list(dp) + [0.0] * (4 - len(dp)))
    h = C.c_void_p()
    _check(L.gs_problem_create(kind, _p(ipa), _p(dpa), C.c_ulonglong(seed), C.byref(h)))
    try:
        return _csr_from_handle(h)
    finally:
        L.gs_host_csr_destroy(h)


def poisson7(nx: int, ny: int = None, nz: int = None) -> Csr:
    return problem(PROBLEM_POISSON7, [nx, ny or nx, nz or nx])


def varcoef_grf(n: int, corr: float = 8.0, sigma: float = 2.3, seed: int = 4) -> Csr:
    return problem(PROBLEM_VARCOEF_GRF, [n, n, n], [corr, sigma], seed)


def varcoef_loguniform(nx: int, ny: int, nz: int, lo=0.1, hi=10.0, seed: int = 3) -> Csr:
    return problem(PROBLEM_VARCOEF_LOGUNI, [nx, ny, nz], [lo, hi], seed)


def kuhn_laplacian(m: int, jitter: float = 0.2, seed: int = 1) -> Csr:
    return problem(PROBLEM_KUHN_P1, [m], [jitter], seed)


def elasticity(v: int, nu: float = 0.3, seed: int = 2) -> Csr:
    return problem(PROBLEM_ELASTICITY_P1, [v], [nu], seed)


def set_tune_cache(path: Optional[str]) -> None:
    """File of cached autotuner decisions for solvers created afterwards."""
    _check(lib().gs_set_tune_cache(None if path is None else path.encode()))


def uniform_rhs(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    _check(lib().gs_uniform_rhs(n, C.c_ulonglong(seed), _p(out)))
    return out


# ---- setup routines (integer work, bit-exact with the reference) ----------
def greedy_coloring(m: Csr) -> Tuple[int, np.ndarray, np.ndarray, np.ndarray]:
    """GraphColoring::compute -> (ncolors, colors, color_vertices, color_offsets)."""
    n = m.rows
    colors = np.empty(n, np.int32)
    verts = np.empty(n, np.int32)
    offs = np.empty(n + 2, np.int32)
    nc = C.c_int()
    _check(lib().gs_greedy_coloring(n, _p(m.row_ptr), _p(m.col_idx), _p(colors), _p(verts),
                                    _p(offs), C.byref(nc)))
    return nc.value, colors, verts, offs[: nc.value + 1].copy()


def smallest_last_coloring(m: Csr) -> Tuple[int, np.ndarray, np.ndarray, np.ndarray]:
    """First-fit colouring in smallest-last order -> (ncolors, colors, color_vertices, color_offsets)."""
    n = m.rows
    colors = np.empty(n, np.int32)
    verts = np.empty(n, np.int32)
    offs = np.empty(n + 2, np.int32)
    nc = C.c_int()
    _check(lib().gs_smallest_last_coloring(n, _p(m.row_ptr), _p(m.col_idx), _p(colors), _p(verts),
                                           _p(offs), C.byref(nc)))
    return nc.value, colors, verts, offs[: nc.value + 1].copy()


def relaxed_coloring(m: Csr, theta: float = 0.05, rho: float = 0.5,
                     block: int = 1) -> Tuple[int, np.ndarray, np.ndarray, np.ndarray]:
    """Colouring of the strong couplings (same-colour weak couplings allowed, each
    row's same-colour mass below rho |a_ii|; block 3: of the 3x3 blocks' nodes)
    -> (ncolors, colors, color_vertices, color_offsets), per row or per node."""
    n = m.rows // block
    colors = np.empty(n, np.int32)
    verts = np.empty(n, np.int32)
    offs = np.empty(n + 2, np.int32)
    nc = C.c_int()
    fn = lib().gs_relaxed_coloring if block == 1 else lib().gs_relaxed_block_coloring
    _check(fn(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(_f64(m.val)), C.c_double(theta), C.c_double(rho),
              _p(colors), _p(verts), _p(offs), C.byref(nc)))
    return nc.value, colors, verts, offs[: nc.value + 1].copy()


def rcm(m: Csr) -> Tuple[np.ndarray, np.ndarray]:
    """RCMReordering::compute -> (old_to_new, new_to_old)."""
    o2n = np.empty(m.rows, np.int32)
    n2o = np.empty(m.rows, np.int32)
    _check(lib().gs_rcm(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(o2n), _p(n2o)))
    return o2n, n2o


def apply_permutation(m: Csr, o2n: np.ndarray, n2o: np.ndarray) -> Csr:
    """HostCSRMatrix::applyPermutation."""
    o2n, n2o = _i32(o2n), _i32(n2o)
    rp = np.empty(m.rows + 1, np.int32)
    ci = np.empty(max(m.nnz, 1), np.int32)
    v = np.empty(max(m.nnz, 1), np.float64)
    _check(lib().gs_apply_permutation(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(m.val), _p(o2n),
                                      _p(n2o), _p(rp), _p(ci), _p(v)))
    return Csr(m.rows, m.cols, rp, ci[: m.nnz], v[: m.nnz])


def permute_matrix(m: Csr, row_o2n: np.ndarray, col_o2n: np.ndarray) -> Csr:
    """permuteMatrix (columns sorted per row)."""
    row_o2n, col_o2n = _i32(row_o2n), _i32(col_o2n)
    rp = np.empty(m.rows + 1, np.int32)
    ci = np.empty(max(m.nnz, 1), np.int32)
    v = np.empty(max(m.nnz, 1), np.float64)
    _check(lib().gs_permute_matrix(m.rows, m.cols, _p(m.row_ptr), _p(m.col_idx), _p(m.val),
                                   _p(row_o2n), _p(col_o2n), _p(rp), _p(ci), _p(v)))
    nnz = int(rp[-1])
    return Csr(m.rows, m.cols, rp, ci[:nnz], v[:nnz])


def ell_build(m: Csr, width: int):
    """HostELLMatrix -> (ell_col, ell_val, ovf_row_ptr, ovf_col, ovf_val)."""
    n = m.rows
    ec = np.empty(n * width, np.int32)
    ev = np.empty(n * width, np.float64)
    orp = np.empty(n + 1, np.int32)
    oc = np.empty(max(m.nnz, 1), np.int32)
    ov = np.empty(max(m.nnz, 1), np.float64)
    on = C.c_int()
    _check(lib().gs_ell_build(n, m.cols, _p(m.row_ptr), _p(m.col_idx), _p(m.val), width, _p(ec),
                              _p(ev), _p(orp), _p(oc), _p(ov), C.byref(on)))
    return ec, ev, orp, oc[: on.value], ov[: on.value]


def block_graph(m: Csr, block: int = 3) -> Tuple[np.ndarray, np.ndarray]:
    """buildBlockGraph -> (row_ptr, col)."""
    nb = m.rows // block if block > 0 else 0  # the library reports a bad block size
    grp = np.empty(nb + 1, np.int32)
    gci = np.empty(max(m.nnz, 1), np.int32)
    gn = C.c_int()
    _check(lib().gs_block_graph(m.rows, _p(m.row_ptr), _p(m.col_idx), block, _p(grp), _p(gci),
                                C.byref(gn)))
    return grp, gci[: gn.value]


def block_inverses3x3(m: Csr) -> np.ndarray:
    """extractInverseDiagonalBlocks3x3 -> 9 doubles per node (row-major)."""
    out = np.empty(3 * m.rows, np.float64)
    _check(lib().gs_block_inverses3x3(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(m.val), _p(out)))
    return out


def expand_block_permutation(node_o2n, node_n2o, block: int = 3):
    node_o2n, node_n2o = _i32(node_o2n), _i32(node_n2o)
    n = len(node_o2n) * block
    o2n = np.empty(n, np.int32)
    n2o = np.empty(n, np.int32)
    _check(lib().gs_expand_block_permutation(len(node_o2n), block, _p(node_o2n), _p(node_n2o),
                                             _p(o2n), _p(n2o)))
    return o2n, n2o


# ---- hierarchy -------------------------------------------------------------
class _SetupStats(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("upload_ms", C.c_double), ("build_ms", C.c_double),
                ("download_ms", C.c_double), ("mis_rounds", C.c_int)]


class Hierarchy:
    """AMGHierarchy: A[k], P[k] (k+1 -> k), R[k] (k -> k+1), aggregates."""

    def __init__(self, handle):
        self._h = handle

    @staticmethod
    def build(a: Csr, block_size: int = 1, eps_strong: float = 0.1, max_levels: int = 10,
              min_dofs: int = 1000) -> "Hierarchy":
        """AMGHierarchyBuilder(SmoothedAggregationCoarsener(block, eps), maxLevels, minDofs)."""
        L = lib()
        m = C.c_void_p()
        _check(L.gs_host_csr_create(a.rows, a.cols, _p(a.row_ptr), _p(a.col_idx), _p(a.val),
                                    C.byref(m)))
        try:
            h = C.c_void_p()
            _check(L.gs_hierarchy_build(m, block_size, eps_strong, max_levels, min_dofs,
                                        C.byref(h)))
        finally:
            L.gs_host_csr_destroy(m)
        return Hierarchy(h)

    @staticmethod
    def build_ex(a: Csr, block_size: int = 1, eps_strong: float = 0.1, max_levels: int = 10,
                 min_dofs: int = 1000, aggregation: int = 1, device: int = -1) -> "Hierarchy":
        """The builder with a choice of aggregation (0 sequential, 1 from a
        distance-2 independent set) and of where it runs (device < 0: host,
        else that GPU, aggregation 1 only). ``.setup_stats`` holds the times."""
        L = lib()
        m = C.c_void_p()
        _check(L.gs_host_csr_create(a.rows, a.cols, _p(a.row_ptr), _p(a.col_idx), _p(a.val),
                                    C.byref(m)))
        st = _SetupStats()
        try:
            h = C.c_void_p()
            _check(L.gs_hierarchy_build_ex(m, block_size, eps_strong, max_levels, min_dofs,
                                           aggregation, device, C.byref(st), C.byref(h)))
        finally:
            L.gs_host_csr_destroy(m)
        out = Hierarchy(h)
        out.setup_stats = dict(total_ms=st.total_ms, upload_ms=st.upload_ms, build_ms=st.build_ms,
                               download_ms=st.download_ms, mis_rounds=st.mis_rounds)
        return out

    def refresh(self, values: np.ndarray, device: int = -1) -> "Hierarchy":
        """DeviceCSRMatrix::updateValues for the whole hierarchy: new finest values
        (same sparsity), every coarser level R_k A_k P_k with the same transfer
        operators; device >= 0 forms the products on that GPU, < 0 on the host."""
        v = _f64(values)
        if len(v) != self.A(0).nnz:
            raise ValueError("refresh: one value per stored entry of the finest level")
        h = C.c_void_p()
        _check(lib().gs_hierarchy_refresh(self._h, _p(v), device, C.byref(h)))
        return Hierarchy(h)

    @staticmethod
    def from_levels(A: List[Csr], P: List[Csr], R: List[Csr], block_size: int = 1) -> "Hierarchy":
        arr = lambda xs: (_Csr * max(len(xs), 1))(*[x.as_c() for x in xs])
        h = C.c_void_p()
        _check(lib().gs_hierarchy_from_levels(len(A), arr(A), arr(P), arr(R), block_size,
                                              C.byref(h)))
        return Hierarchy(h)

    @property
    def levels(self) -> int:
        return lib().gs_hierarchy_num_levels(self._h)

    def matrix(self, level: int, which: int) -> Csr:
        L = lib()
        r, c, nz = C.c_int(), C.c_int(), C.c_int()
        _check(L.gs_hierarchy_matrix_info(self._h, level, which, C.byref(r), C.byref(c),
                                          C.byref(nz)))
        rp = np.empty(r.value + 1, np.int32)
        ci = np.empty(max(nz.value, 1), np.int32)
        v = np.empty(max(nz.value, 1), np.float64)
        _check(L.gs_hierarchy_matrix(self._h, level, which, _p(rp), _p(ci), _p(v)))
        return Csr(r.value, c.value, rp, ci[: nz.value], v[: nz.value])

    def A(self, k: int) -> Csr:
        return self.matrix(k, 0)

    def P(self, k: int) -> Csr:
        return self.matrix(k, 1)

    def R(self, k: int) -> Csr:
        return self.matrix(k, 2)

    def aggregates(self, k: int, block: int = 1) -> np.ndarray:
        out = np.empty(self.A(k).rows // block, np.int32)
        _check(lib().gs_hierarchy_aggregates(self._h, k, _p(out)))
        return out

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.gs_hierarchy_destroy(self._h)
            self._h = None


# ---- solver -----------------------------------------------------------------
@dataclass
class SolverOptions:
    smoother: int = 0           # 0 SGS, 1 3x3 block SGS, 2 damped Jacobi, 3 block Jacobi, 4 identity
    pre_steps: int = 1
    post_steps: int = 1
    coarse_steps: int = 2
    vcycles: int = 1
    omega: float = 1.0
    coarse_solver: int = 1      # 0 smoother (the reference), 1 dense Cholesky
    precision: int = 0          # 0 FP64 V-cycle, 1 FP32 V-cycle
    flexible: int = 0           # 0 rho'/rho (the reference), 1 Polak-Ribiere
    use_graph: int = 0
    check_every: int = 8
    tol: float = 1e-6
    max_iter: int = 1000
    reference_vcycle: int = 0   # 1: the reference's V-cycle incl. its buffer aliasing
    autotune: int = 1           # 1: threads per row picked per level by timing candidates
    coarse_tail: int = 1        # cluster-resident coarse V-cycle: 0 never, 1 if faster, 2 always
    lanes: int = 0              # >0 forces threads per row everywhere; 0 autotuned
    sliced_lanes: int = 0       # >0 forces the sliced layout (SELL/BELL) with 1, 2, 4 or 8 lanes per row
    coarse_rows: int = 0        # >0: dense coarsest solve on the first level with <= this many rows
    coarse_smoother: int = -1   # smoother below the finest level (-1: same as smoother)
    overlap_launch: int = 2     # 2: programmatic dependent launch of V-cycle kernels, graphs too; 1 eager only; 0 off
    packed_rows: int = 8192     # dense coarsest levels above this size store a tiled lower triangle of the inverse
    coloring: int = 0           # 0 the reference's greedy colouring, 1 smallest-last order where it has fewer
                                # colours, 2 and the strong couplings only on the coarse levels
    sweep_launch: int = 1       # SGS steps: 0 a launch per colour, 1 cooperative where faster, 2 always cooperative
    half_sweeps: int = 0        # 1: forward sweeps before, backward sweeps after the coarse correction
    coarse_half: int = 0        # 1: packed dense coarsest inverse in FP16 tiles with a scale per tile

    def to_c(self) -> _Options:
        return _Options(**{f[0]: getattr(self, f[0]) for f in _Options._fields_})


@dataclass
class SolveStats:
    iterations: int
    status: int
    spmv: int
    ratio: float
    rhs_norm2: float
    solve_ms: float


def _stats(s: _Stats) -> SolveStats:
    return SolveStats(s.iterations, s.status, s.spmv, s.ratio, s.rhs_norm2, s.solve_ms)


class Solver:
    """CGSolver + Multigrid{GaussSeidel,BlockGaussSeidel}Preconditioner on one GPU."""

    def __init__(self, h: Hierarchy, opts: SolverOptions = None,
                 permutations: Optional[List[Tuple[np.ndarray, np.ndarray]]] = None,
                 device: int = 0):
        self.opts = opts or SolverOptions()
        L = lib()
        self._keep = []
        o2n = n2o = None
        if permutations is not None:
            if len(permutations) != h.levels:
                raise SolverError(GS_ERR_INVALID, "MultigridSmoother: invalid number of permutations.")
            a = [_i32(p[0]) for p in permutations]
            b = [_i32(p[1]) for p in permutations]
            self._keep += a + b
            o2n = (C.c_void_p * len(a))(*[x.ctypes.data for x in a])
            n2o = (C.c_void_p * len(b))(*[x.ctypes.data for x in b])
        c_opts = self.opts.to_c()
        s = C.c_void_p()
        _check(L.gs_solver_create(h._h, o2n, n2o, C.byref(c_opts), device, C.byref(s)))
        self._s = s
        self.hierarchy = h

    def __del__(self):
        if getattr(self, "_s", None) and _lib is not None:
            _lib.gs_solver_destroy(self._s)
            self._s = None

    def set_tolerance(self, tol: float, max_iter: int = None) -> None:
        _check(lib().gs_solver_set_tolerance(self._s, tol, max_iter or self.opts.max_iter))

    def solve(self, b: np.ndarray, x0: Optional[np.ndarray] = None) -> Tuple[np.ndarray, SolveStats]:
        b = _f64(b)
        x = np.zeros_like(b) if x0 is None else _f64(x0).copy()
        st = _Stats()
        _check(lib().gs_solver_solve(self._s, _p(b), _p(x), C.byref(st)))
        return x, _stats(st)

    def solve_f32(self, b: np.ndarray, x0: Optional[np.ndarray] = None):
        b = np.ascontiguousarray(b, dtype=np.float32)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float32).copy()
        st = _Stats()
        _check(lib().gs_solver_solve_f32(self._s, _p(b), _p(x), C.byref(st)))
        return x, _stats(st)

    def solve_device(self, b_ptr: int, x_ptr: int, stream: int = 0) -> SolveStats:
        """b, x: device addresses of FP64 arrays (e.g. torch tensor data_ptr())."""
        st = _Stats()
        _check(lib().gs_solver_solve_device(self._s, C.c_void_p(b_ptr), C.c_void_p(x_ptr),
                                            C.c_void_p(stream), C.byref(st)))
        return _stats(st)

    def apply_preconditioner_device(self, r_ptr: int, z_ptr: int, stream: int = 0) -> None:
        _check(lib().gs_solver_apply_preconditioner(self._s, C.c_void_p(r_ptr), C.c_void_p(z_ptr),
                                                    C.c_void_p(stream)))

    def update_matrix(self, values: np.ndarray) -> None:
        """New values of the finest matrix (same sparsity, the CSR order the hierarchy was
        built from); coarser levels recomputed as R A P with the transfers kept."""
        v = _f64(values)
        _check(lib().gs_solver_update_matrix(self._s, _p(v)))

    def set_colour_weights(self, weights: Optional[List[np.ndarray]]) -> None:
        """Per-level arrays of per-colour weights in (0, 2); None restores omega."""
        if weights is None:
            _check(lib().gs_solver_set_colour_weights(self._s, None, None, 0))
            return
        offs = np.zeros(len(weights) + 1, np.int32)
        for k, w in enumerate(weights):
            offs[k + 1] = offs[k] + len(w)
        w = _f64(np.concatenate(weights))
        _check(lib().gs_solver_set_colour_weights(self._s, _p(w), _p(offs), len(weights)))

    def level_info(self) -> List[dict]:
        L = lib()
        out = []
        for k in range(L.gs_solver_num_levels(self._s)):
            r, nz, nc, ns, st = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_longlong()
            _check(L.gs_solver_level_info(self._s, k, C.byref(r), C.byref(nz), C.byref(nc),
                                          C.byref(ns), C.byref(st)))
            ln, pl, rl = C.c_int(), C.c_int(), C.c_int()
            _check(L.gs_solver_level_format(self._s, k, C.byref(ln), C.byref(pl), C.byref(rl)))
            out.append(dict(rows=r.value, nnz=nz.value, colors=nc.value, slices=ns.value,
                            stored=st.value, lanes=ln.value, p_lanes=pl.value, r_lanes=rl.value,
                            in_tail=L.gs_solver_level_in_tail(self._s, k),
                            sliced=L.gs_solver_level_layout(self._s, k),
                            launch=L.gs_solver_level_launch(self._s, k)))
        return out

    def launch_count(self) -> int:
        c = C.c_longlong()
        _check(lib().gs_solver_launch_count(self._s, C.byref(c)))
        return c.value

    def solve_host_ptr(self, b_ptr: int, x_ptr: int) -> SolveStats:
        """Host arrays given by address (e.g. pinned torch tensors), FP64."""
        st = _Stats()
        _check(lib().gs_solver_solve(self._s, C.c_void_p(b_ptr), C.c_void_p(x_ptr), C.byref(st)))
        return _stats(st)

    def colour_features(self) -> np.ndarray:
        """The solver's 8 features per (level, colour), level-major (n, 8) FP32."""
        L = lib()
        cnt = C.c_int()
        _check(L.gs_solver_colour_features(self._s, None, 0, C.byref(cnt)))
        out = np.empty(8 * cnt.value, np.float32)
        _check(L.gs_solver_colour_features(self._s, _p(out), len(out), C.byref(cnt)))
        return out.reshape(cnt.value, 8)

    def node_features(self) -> np.ndarray:
        """8 features per node (3x3 block row) of every level, caller order, level
        after level: (nodes, 8) FP32; empty for scalar hierarchies."""
        L = lib()
        cnt = C.c_longlong()
        _check(L.gs_solver_node_features(self._s, None, 0, C.byref(cnt)))
        out = np.empty(8 * cnt.value, np.float32)
        if cnt.value:
            _check(L.gs_solver_node_features(self._s, _p(out), len(out), C.byref(cnt)))
        return out.reshape(cnt.value, 8)

    def set_node_weights(self, weights) -> None:
        """Per-block scalings of the 3x3 block smoother: one array per level (or
        one concatenated array) of weights in (0, 2), the order of node_features;
        None restores the colour weights / omega."""
        if weights is None:
            _check(lib().gs_solver_set_node_weights(self._s, None, 0))
            return
        w = _f64(np.concatenate([np.asarray(x, np.float64).ravel() for x in weights])
                 if isinstance(weights, (list, tuple)) else weights)
        _check(lib().gs_solver_set_node_weights(self._s, _p(w), len(w)))

    def error_reduction(self, e0_ptr: int, stream: int = 0) -> float:
        """||e1||_A / ||e0||_A of one preconditioner step from the device error e0."""
        r = C.c_double()
        _check(lib().gs_solver_error_reduction(self._s, C.c_void_p(e0_ptr), C.c_void_p(stream),
                                               C.byref(r)))
        return r.value

    def time_kernel(self, kind: int, reps: int = 20, stream: int = 0) -> float:
        ms = C.c_double()
        _check(lib().gs_solver_time_kernel(self._s, kind, reps, C.c_void_p(stream), C.byref(ms)))
        return ms.value

    def setup_times(self) -> dict:
        """Wall-clock ms of the solver's setup phases."""
        t = (C.c_double * 4)()
        _check(lib().gs_solver_setup_times(self._s, t))
        return dict(levels_ms=t[0], autotune_ms=t[1], tail_ms=t[2], total_ms=t[3])

    def setup_phases(self) -> dict:
        """setup_times plus where the levels' time went (wall-clock ms)."""
        t = (C.c_double * 10)()
        _check(lib().gs_solver_setup_phases(self._s, t, 10))
        keys = ("levels_ms", "autotune_ms", "tail_ms", "total_ms", "colouring_ms", "permutation_ms",
                "features_ms", "layouts_ms", "transfers_ms", "dense_inverse_ms")
        return {k: round(t[i], 1) for i, k in enumerate(keys)}

    def time_level(self, level: int, op: int, lanes: int = 0, reps: int = 10, stream: int = 0) -> float:
        """op 0 forward GS sweep, 1 residual, 2 restriction, 3 prolongation of `level` (ms)."""
        ms = C.c_double()
        _check(lib().gs_solver_time_level(self._s, level, op, lanes, reps, C.c_void_p(stream),
                                          C.byref(ms)))
        return ms.value


def hierarchical_reordering(h: "Hierarchy") -> List[Tuple[np.ndarray, np.ndarray]]:
    """HierarchicalReordering::compute: one (old_to_new, new_to_old) per level, finest first."""
    o2n = [np.empty(h.A(k).rows, np.int32) for k in range(h.levels)]
    n2o = [np.empty(h.A(k).rows, np.int32) for k in range(h.levels)]
    po = (C.c_void_p * h.levels)(*[q.ctypes.data for q in o2n])
    pn = (C.c_void_p * h.levels)(*[q.ctypes.data for q in n2o])
    _check(lib().gs_hierarchical_reordering(h._h, po, pn))
    return list(zip(o2n, n2o))


def dense_spd_inverse(m: Csr, device: int = 0) -> np.ndarray:
    """Inverse of an SPD matrix on the GPU (the library's tiled Cholesky and inverse; n x n, FP64)."""
    out = np.empty((m.rows, m.rows), np.float64)
    _check(lib().gs_dense_spd_inverse(m.rows, _p(m.row_ptr), _p(m.col_idx), _p(m.val), _p(out), device))
    return out


# ---- batched solves ---------------------------------------------------------
STATUS_NOT_FINITE = 3


def _hier_array(hierarchies) -> "C.Array":
    return (C.c_void_p * len(hierarchies))(*[h._h.value if isinstance(h._h, C.c_void_p) else h._h
                                             for h in hierarchies])


class Batch:
    """Many independent systems (one Hierarchy each) with `nrhs` right-hand
    sides per system, solved together on one GPU (no reference counterpart;
    each pair follows CGSolver::solve). Vectors use the caller layout of
    gs_batch_solve: system after system, right-hand side j of system s a
    contiguous block of n_s values."""

    def __init__(self, hierarchies: List[Hierarchy], nrhs: int = 1, opts: SolverOptions = None,
                 device: int = 0):
        self.opts = opts or SolverOptions()
        self.hierarchies = list(hierarchies)
        arr = _hier_array(self.hierarchies)
        c_opts = self.opts.to_c()
        b = C.c_void_p()
        _check(lib().gs_batch_create(len(self.hierarchies), arr, nrhs, C.byref(c_opts), device,
                                     C.byref(b)))
        self._b = b
        ns, nr, unk, lv = C.c_int(), C.c_int(), C.c_longlong(), C.c_int()
        _check(lib().gs_batch_info(b, C.byref(ns), C.byref(nr), C.byref(unk), C.byref(lv)))
        self.num_systems, self.nrhs, self.unknowns, self.levels = ns.value, nr.value, unk.value, lv.value
        rows = np.empty(self.num_systems, np.int32)
        _check(lib().gs_batch_system_rows(b, _p(rows)))
        self.system_rows = rows

    def __del__(self):
        if getattr(self, "_b", None) and _lib is not None:
            _lib.gs_batch_destroy(self._b)
            self._b = None

    @property
    def size(self) -> int:
        """Values in one caller-layout vector (sum of n_s) * nrhs."""
        return int(self.unknowns) * self.nrhs

    def pack(self, vectors: List[np.ndarray]) -> np.ndarray:
        """[per system an (nrhs, n_s) array] -> caller-layout FP64 vector."""
        return np.concatenate([_f64(v).reshape(-1) for v in vectors])

    def unpack(self, flat: np.ndarray) -> List[np.ndarray]:
        out, o = [], 0
        for n in self.system_rows:
            out.append(flat[o:o + self.nrhs * n].reshape(self.nrhs, n))
            o += self.nrhs * n
        return out

    def set_tolerance(self, tol: float, max_iter: int = None) -> None:
        _check(lib().gs_batch_set_tolerance(self._b, C.c_double(tol), max_iter or self.opts.max_iter))

    def solve(self, b: np.ndarray, x0: Optional[np.ndarray] = None) -> Tuple[np.ndarray, List[SolveStats]]:
        b = _f64(b)
        if b.size != self.size:
            raise SolverError(GS_ERR_INVALID, "batch: right-hand side size does not match the systems")
        x = np.zeros_like(b) if x0 is None else _f64(x0).copy()
        st = (_Stats * (self.num_systems * self.nrhs))()
        _check(lib().gs_batch_solve(self._b, _p(b), _p(x), st))
        return x, [_stats(s) for s in st]

    def solve_host_ptr(self, b_ptr: int, x_ptr: int) -> List[SolveStats]:
        """Host arrays given by address (e.g. pinned torch tensors), caller layout, FP64."""
        st = (_Stats * (self.num_systems * self.nrhs))()
        _check(lib().gs_batch_solve(self._b, C.c_void_p(b_ptr), C.c_void_p(x_ptr), st))
        return [_stats(s) for s in st]

    def solve_device(self, b_ptr: int, x_ptr: int, stream: int = 0) -> List[SolveStats]:
        st = (_Stats * (self.num_systems * self.nrhs))()
        _check(lib().gs_batch_solve_device(self._b, C.c_void_p(b_ptr), C.c_void_p(x_ptr),
                                           C.c_void_p(stream), st))
        return [_stats(s) for s in st]

    def level_info(self) -> List[dict]:
        out = []
        for k in range(self.levels):
            r, sy, mc, ln, pl, rl = (C.c_int() for _ in range(6))
            nz = C.c_longlong()
            _check(lib().gs_batch_level_info(self._b, k, C.byref(r), C.byref(nz), C.byref(sy),
                                             C.byref(mc), C.byref(ln), C.byref(pl), C.byref(rl)))
            out.append(dict(rows=r.value, nnz=nz.value, systems=sy.value, max_colors=mc.value,
                            lanes=ln.value, p_lanes=pl.value, r_lanes=rl.value))
        return out

    def launch_count(self) -> int:
        c = C.c_longlong()
        _check(lib().gs_batch_launch_count(self._b, C.byref(c)))
        return c.value

    def time_kernel(self, kind: int, reps: int = 20, stream: int = 0) -> float:
        """kind 0 outer FP64 SpMV, 1 level-0 forward GS sweep, 2 one V-cycle (ms)."""
        ms = C.c_double()
        _check(lib().gs_batch_time_kernel(self._b, kind, reps, C.c_void_p(stream), C.byref(ms)))
        return ms.value

    def time_level(self, level: int, op: int, lanes: int = 0, reps: int = 10, stream: int = 0) -> float:
        """op 0 forward GS sweep, 1 residual, 2 restriction, 3 prolongation of `level` (ms)."""
        ms = C.c_double()
        _check(lib().gs_batch_time_level(self._b, level, op, lanes, reps, C.c_void_p(stream),
                                         C.byref(ms)))
        return ms.value


def batch_plan_check(hierarchies: List[Hierarchy]) -> dict:
    """Host-only check of the batch work lists (see gs_batch_plan_check)."""
    arr = _hier_array(list(hierarchies))
    lv, ps, it = C.c_int(), C.c_int(), C.c_longlong()
    _check(lib().gs_batch_plan_check(len(hierarchies), arr, C.byref(lv), C.byref(ps), C.byref(it)))
    return dict(levels=lv.value, passes=ps.value, items=it.value)


# ---- kernel-level Backend operations (device arrays given by address) -------
class DeviceCsr:
    """Backend::createCSRMatrix: a CSR matrix on the device (FP32 or FP64)."""

    def __init__(self, m: Csr, dtype: int = F64):
        L = lib()
        vals = np.ascontiguousarray(m.val, dtype=np.float32 if dtype == F32 else np.float64)
        h = C.c_void_p()
        _check(L.gs_device_csr_create(m.rows, m.cols, _p(m.row_ptr), _p(m.col_idx), _p(vals),
                                      dtype, C.byref(h)))
        self._h, self.rows, self.cols, self.nnz, self.dtype = h, m.rows, m.cols, m.nnz, dtype

    def update_values(self, values: np.ndarray) -> None:
        vals = np.ascontiguousarray(values, dtype=np.float32 if self.dtype == F32 else np.float64)
        _check(lib().gs_device_csr_update_values(self._h, _p(vals), len(vals)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.gs_device_csr_destroy(self._h)
            self._h = None


def spmv(A: DeviceCsr, x_ptr: int, y_ptr: int, stream: int = 0) -> None:
    _check(lib().gs_spmv(A._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), C.c_void_p(stream)))


def gauss_seidel_color(A: DeviceCsr, order_ptr: int, start: int, count: int, rhs_ptr: int,
                       x_ptr: int, omega: float, stream: int = 0) -> None:
    _check(lib().gs_gauss_seidel_color(A._h, C.c_void_p(order_ptr), start, count,
                                       C.c_void_p(rhs_ptr), C.c_void_p(x_ptr), omega,
                                       C.c_void_p(stream)))


def block_gauss_seidel_color3x3(A: DeviceCsr, order_ptr: int, start: int, count: int,
                                dinv_ptr: int, rhs_ptr: int, x_ptr: int, omega: float,
                                stream: int = 0) -> None:
    _check(lib().gs_block_gauss_seidel_color3x3(A._h, C.c_void_p(order_ptr), start, count,
                                                C.c_void_p(dinv_ptr), C.c_void_p(rhs_ptr),
                                                C.c_void_p(x_ptr), omega, C.c_void_p(stream)))


def apply_block_inverses3x3(n: int, dinv_ptr: int, r_ptr: int, c_ptr: int, dtype: int,
                            stream: int = 0) -> None:
    _check(lib().gs_apply_block_inverses3x3(n, C.c_void_p(dinv_ptr), C.c_void_p(r_ptr),
                                            C.c_void_p(c_ptr), dtype, C.c_void_p(stream)))


def dot(n: int, x_ptr: int, y_ptr: int, result_ptr: int, dtype: int, stream: int = 0) -> None:
    _check(lib().gs_dot(n, C.c_void_p(x_ptr), C.c_void_p(y_ptr), C.c_void_p(result_ptr), dtype,
                        C.c_void_p(stream)))


def dot_noalloc(n: int, x_ptr: int, y_ptr: int, result_ptr: int, dtype: int,
                stream: int = 0) -> None:
    """gs_dot without allocating: scratch in a fixed array of the library
    (n <= 8,388,608; calls that overlap on the GPU race on that array)."""
    _check(lib().gs_dot_noalloc(n, C.c_void_p(x_ptr), C.c_void_p(y_ptr), C.c_void_p(result_ptr),
                                dtype, C.c_void_p(stream)))


def vector_op(op: int, n: int, x_ptr: int, y_ptr: int, alpha: float = 0.0,
              alpha_ptr: Optional[int] = None, dtype: int = F64, stream: int = 0) -> None:
    _check(lib().gs_vector_op(op, n, C.c_void_p(x_ptr), C.c_void_p(y_ptr), alpha,
                              None if alpha_ptr is None else C.c_void_p(alpha_ptr), dtype,
                              C.c_void_p(stream)))


def scalar_op(op: int, a_ptr: Optional[int], b_ptr: Optional[int], out_ptr: int,
              value: float = 0.0, dtype: int = F64, stream: int = 0) -> None:
    _check(lib().gs_scalar_op(op, None if a_ptr is None else C.c_void_p(a_ptr),
                              None if b_ptr is None else C.c_void_p(b_ptr), C.c_void_p(out_ptr),
                              value, dtype, C.c_void_p(stream)))


# ---- learned relaxation weights: MLP kernels (device arrays by address) ------
def mlp_param_count() -> int:
    return lib().gs_mlp_param_count()


def mlp_forward(params_ptr: int, feats_ptr: int, n: int, omega_ptr: int,
                cache_ptr: Optional[int] = None, stream: int = 0) -> None:
    _check(lib().gs_mlp_forward(C.c_void_p(params_ptr), C.c_void_p(feats_ptr), n,
                                C.c_void_p(omega_ptr),
                                None if cache_ptr is None else C.c_void_p(cache_ptr),
                                C.c_void_p(stream)))


def mlp_backward(params_ptr: int, feats_ptr: int, n: int, cache_ptr: int, upstream_ptr: int,
                 delta_ptr: int, grad_ptr: int, stream: int = 0) -> None:
    _check(lib().gs_mlp_backward(C.c_void_p(params_ptr), C.c_void_p(feats_ptr), n,
                                 C.c_void_p(cache_ptr), C.c_void_p(upstream_ptr),
                                 C.c_void_p(delta_ptr), C.c_void_p(grad_ptr), C.c_void_p(stream)))


def mlp_adam(params_ptr: int, grad_ptr: int, m_ptr: int, v_ptr: int, n_params: int, lr: float,
             step: int, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
             stream: int = 0) -> None:
    _check(lib().gs_mlp_adam(C.c_void_p(params_ptr), C.c_void_p(grad_ptr), C.c_void_p(m_ptr),
                             C.c_void_p(v_ptr), n_params, lr, beta1, beta2, eps, step,
                             C.c_void_p(stream)))
