"""The C ABI library loads and exports every entry point include/gpusolver_b200.h declares."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT, cuda_available


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "gpusolver_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gs_[a-z0-9_]+)\s*\(", text)))


def test_header_lists_match(gs):
    assert declared_symbols() == sorted(gs.EXPORTED_SYMBOLS)


def test_loaded_library_matches_the_header(gs):
    """The library reports the ABI version its header declares (a library
    built from older sources fails here)."""
    text = open(os.path.join(ROOT, "include", "gpusolver_b200.h")).read()
    declared = int(re.search(r"#define GS_VERSION (\d+)", text).group(1))
    assert C.CDLL(gs.LIB_PATH).gs_version() == declared


def test_every_declared_symbol_is_exported(gs):
    lib = C.CDLL(gs.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_solver_without_device_fails_loudly(gs):
    if cuda_available():
        pytest.skip("a CUDA device is present")
    H = gs.Hierarchy.build(gs.poisson7(6), 1, 0.1, 10, 50)
    with pytest.raises(gs.NoDeviceError):
        gs.Solver(H)


def test_invalid_inputs_raise(gs):
    with pytest.raises(gs.SolverError):
        gs.rcm(gs.Csr(0, 0, __import__("numpy").zeros(1, "int32"), __import__("numpy").zeros(0, "int32"),
                      __import__("numpy").zeros(0)))
    import numpy as np
    m = gs.poisson7(3)
    bad = np.arange(m.rows, dtype=np.int32)
    bad[0] = 1
    with pytest.raises(gs.SolverError, match="not inverses|invalid"):
        gs.apply_permutation(m, bad, np.arange(m.rows))


def _csr(gs, n, rp, ci):
    import numpy as np
    rp = np.asarray(rp, np.int32)
    ci = np.asarray(ci, np.int32)
    return gs.Csr(n, n, rp, ci, np.ones(len(ci)))


def test_graph_entry_points_reject_bad_graphs(gs):
    """Column indices outside [0, n) and decreasing row pointers are errors,
    not out-of-bounds reads (colourings, RCM, node graph)."""
    out_of_range = _csr(gs, 2, [0, 2, 3], [0, 2, 1])
    decreasing = _csr(gs, 2, [0, 2, 1], [0, 1])
    for m in (out_of_range, decreasing):
        for f in (gs.greedy_coloring, gs.smallest_last_coloring, gs.rcm):
            with pytest.raises(gs.SolverError, match="out of range|decreases"):
                f(m)
    with pytest.raises(gs.SolverError, match="block size must be positive"):
        gs.block_graph(gs.poisson7(2), 0)
    with pytest.raises(gs.SolverError, match="out of range"):
        gs.block_graph(_csr(gs, 3, [0, 1, 2, 3], [0, 1, 5]), 3)


def test_permute_matrix_requires_permutations(gs):
    import numpy as np
    m = gs.poisson7(2)
    ident = np.arange(m.rows, dtype=np.int32)
    twice = ident.copy()
    twice[1] = 0
    high = ident.copy()
    high[-1] = m.rows
    for bad in (twice, high):
        with pytest.raises(gs.SolverError, match="not a permutation"):
            gs.permute_matrix(m, bad, ident)
        with pytest.raises(gs.SolverError, match="not a permutation"):
            gs.permute_matrix(m, ident, bad)
    p = gs.permute_matrix(m, ident[::-1].copy(), ident)
    assert p.nnz == m.nnz


def test_problem_sizes_and_parameters_are_checked(gs):
    for make in (lambda: gs.poisson7(0), lambda: gs.poisson7(4, -1, 4), lambda: gs.poisson7(1300),
                 lambda: gs.varcoef_grf(4, corr=0.0), lambda: gs.varcoef_loguniform(2, 2, 2, lo=1.0, hi=0.5),
                 lambda: gs.kuhn_laplacian(1), lambda: gs.kuhn_laplacian(4, jitter=-0.1),
                 lambda: gs.elasticity(1), lambda: gs.elasticity(3, nu=0.5)):
        with pytest.raises(gs.SolverError):
            make()
    assert gs.poisson7(2).rows == 8


def test_null_arguments_are_errors(gs):
    """Entry points given a null output or handle return GS_ERR_INVALID with a
    message instead of writing through it."""
    import numpy as np
    lib = C.CDLL(gs.LIB_PATH)
    lib.gs_last_error.restype = C.c_char_p
    m = gs.poisson7(2)
    rp = m.row_ptr.ctypes.data_as(C.c_void_p)
    ci = m.col_idx.ctypes.data_as(C.c_void_p)
    v = m.val.ctypes.data_as(C.c_void_p)
    buf = np.zeros(64, np.int32)
    b = buf.ctypes.data_as(C.c_void_p)
    nc = C.c_int()
    calls = {
        "greedy": lambda: lib.gs_greedy_coloring(m.rows, rp, ci, None, b, b, C.byref(nc)),
        "smallest_last": lambda: lib.gs_smallest_last_coloring(m.rows, rp, ci, b, None, b, C.byref(nc)),
        "rcm": lambda: lib.gs_rcm(m.rows, rp, ci, b, None),
        "rcm_ci": lambda: lib.gs_rcm(m.rows, rp, None, b, b),
        "permute": lambda: lib.gs_permute_matrix(m.rows, m.cols, rp, ci, v, None, b, b, b, b),
        "block_graph": lambda: lib.gs_block_graph(m.rows, rp, ci, 2, None, b, C.byref(nc)),
        "problem": lambda: lib.gs_problem_create(0, None, None, C.c_ulonglong(0), C.byref(C.c_void_p())),
        "problem_out": lambda: lib.gs_problem_create(0, b, None, C.c_ulonglong(0), None),
        "rhs": lambda: lib.gs_uniform_rhs(4, C.c_ulonglong(0), None),
        "rhs_n": lambda: lib.gs_uniform_rhs(-1, C.c_ulonglong(0), b),
        "host_csr": lambda: lib.gs_host_csr_create(m.rows, m.cols, rp, ci, v, None),
        "host_csr_rp": lambda: lib.gs_host_csr_create(m.rows, m.cols, None, ci, v, C.byref(C.c_void_p())),
        "hierarchy": lambda: lib.gs_hierarchy_build(None, 1, C.c_double(0.1), 10, 10, C.byref(C.c_void_p())),
        "from_levels": lambda: lib.gs_hierarchy_from_levels(2, None, None, None, 1, C.byref(C.c_void_p())),
    }
    for name, call in calls.items():
        assert call() == gs.GS_ERR_INVALID, name
        assert lib.gs_last_error(), name


def test_device_csr_is_validated_before_upload(gs):
    """A device CSR whose indices would send the kernels out of bounds is
    refused on the host, before any device is touched (so also without one)."""
    import numpy as np
    cases = {
        "column index out of range": _csr(gs, 2, [0, 2, 3], [0, 2, 1]),
        "row pointer decreases": _csr(gs, 2, [0, 2, 1], [0, 1]),
        "row pointer must start at 0": gs.Csr(2, 2, np.array([1, 2, 3], np.int32), np.array([0, 1, 1], np.int32),
                                              np.ones(3)),
    }
    for msg, m in cases.items():
        for dtype in (gs.F32, gs.F64):
            with pytest.raises(gs.SolverError, match=msg) as e:
                gs.DeviceCsr(m, dtype)
            assert not isinstance(e.value, gs.NoDeviceError)


@pytest.mark.parametrize("field, value", [
    ("smoother", 5), ("smoother", -1), ("coarse_smoother", 7), ("pre_steps", 0), ("post_steps", 0),
    ("vcycles", 0), ("omega", 0.0), ("omega", 2.0), ("omega", float("nan")), ("coarse_solver", 2),
    ("precision", 2), ("flexible", -1), ("use_graph", 3), ("reference_vcycle", 2), ("autotune", 2),
    ("coloring", 3), ("coloring", -1), ("tol", 0.0), ("tol", float("inf")), ("max_iter", 0), ("coarse_tail", 3),
    ("overlap_launch", 3), ("lanes", 3), ("lanes", 64), ("sliced_lanes", 16), ("coarse_rows", -1),
    ("packed_rows", -5), ("sweep_launch", 3), ("sweep_launch", -1),
    ("half_sweeps", 2), ("coarse_half", 3),
])
def test_solver_options_are_checked_before_the_device(gs, field, value):
    """Every option outside its documented range is refused on the host, before
    any device is looked for (so the same error with or without a GPU), for the
    single-system solver and the batch alike."""
    H = gs.Hierarchy.build(gs.poisson7(6), 1, 0.1, 10, 50)
    opts = gs.SolverOptions()
    setattr(opts, field, value)
    for make in (lambda: gs.Solver(H, opts), lambda: gs.Batch([H], 1, opts)):
        with pytest.raises(gs.SolverError, match="solver options") as e:
            make()
        assert not isinstance(e.value, gs.NoDeviceError)
    # coarse_steps only matters when the coarsest level is smoothed
    opts = gs.SolverOptions(coarse_solver=0, coarse_steps=0)
    with pytest.raises(gs.SolverError, match="coarse_steps"):
        gs.Solver(H, opts)


def test_batch_refuses_options_it_does_not_implement(gs):
    """Half sweeps and the strong-coupling colouring are single-system options:
    the batched solver refuses them on the host, before any device is looked for."""
    H = gs.Hierarchy.build(gs.poisson7(6), 1, 0.1, 10, 50)
    for field, msg in (("half_sweeps", "half_sweeps"), ("coloring", "coloring 2")):
        opts = gs.SolverOptions()
        setattr(opts, field, 1 if field == "half_sweeps" else 2)
        with pytest.raises(gs.SolverError, match=msg) as e:
            gs.Batch([H], 1, opts)
        assert not isinstance(e.value, gs.NoDeviceError)


def test_default_options_pass_the_check(gs):
    if cuda_available():
        pytest.skip("a CUDA device is present")
    H = gs.Hierarchy.build(gs.poisson7(6), 1, 0.1, 10, 50)
    for opts in (gs.SolverOptions(), gs.SolverOptions(tol=1e-8, precision=1, flexible=1, use_graph=1, coarse_solver=1,
                                                      coarse_rows=24576, coloring=1)):
        with pytest.raises(gs.NoDeviceError):
            gs.Solver(H, opts)


def test_kernel_level_entry_points_check_before_launch(gs):
    """Arguments that would send a kernel through memory of the wrong size or
    through a null pointer are refused on the host, before any launch: an
    unknown dtype (read as FP64 it would double the bytes read), a missing
    scalar operand, a negative length."""
    import numpy as np
    lib = C.CDLL(gs.LIB_PATH)
    buf = np.zeros(64, np.float64)
    p = C.c_void_p(buf.ctypes.data)
    calls = {
        "dot_dtype": lambda: lib.gs_dot(C.c_longlong(4), p, p, p, 7, None),
        "dot_noalloc_dtype": lambda: lib.gs_dot_noalloc(C.c_longlong(4), p, p, p, -1, None),
        "dot_noalloc_negative": lambda: lib.gs_dot_noalloc(C.c_longlong(-1), p, p, p, gs.F64, None),
        "node_weights_null_solver": lambda: lib.gs_solver_set_node_weights(None, p, C.c_longlong(4)),
        "node_features_null_solver": lambda: lib.gs_solver_node_features(None, None, C.c_longlong(0), p),
        "dot_noalloc_oversize": lambda: lib.gs_dot_noalloc(C.c_longlong(8_388_609), p, p, p, gs.F64, None),
        "vector_dtype": lambda: lib.gs_vector_op(gs.VEC_AXPY, C.c_longlong(4), p, p, C.c_double(1.0), None, 2, None),
        "scalar_dtype": lambda: lib.gs_scalar_op(gs.SCALAR_COPY, p, None, p, C.c_double(0.0), 5, None),
        "scalar_divide_null_b": lambda: lib.gs_scalar_op(gs.SCALAR_DIVIDE, p, None, p, C.c_double(0.0), gs.F64, None),
        "scalar_sqrt_null_a": lambda: lib.gs_scalar_op(gs.SCALAR_SQRT, None, None, p, C.c_double(0.0), gs.F64, None),
        "block_apply_negative": lambda: lib.gs_apply_block_inverses3x3(C.c_longlong(-3), p, p, p, gs.F64, None),
        "block_apply_dtype": lambda: lib.gs_apply_block_inverses3x3(C.c_longlong(3), p, p, p, 9, None),
        "adam_np": lambda: lib.gs_mlp_adam(p, p, p, p, 0, C.c_double(1e-3), C.c_double(0.9), C.c_double(0.999),
                                           C.c_double(1e-8), 1, None),
    }
    for name, call in calls.items():
        assert call() == gs.GS_ERR_INVALID, name


def test_product_never_uses_the_oracle():
    """The library, its binding and its headers neither import nor load
    anything from oracle/ (the oracle is the checker, not the product)."""
    import re
    roots = [os.path.join(ROOT, "gpu-conjugate-gradient-solver_b200"), os.path.join(ROOT, "include")]
    pattern = re.compile(r"(import\s+oracle|from\s+oracle|liboracle|libgsref|oracle/)")
    hits = []
    for root in roots:
        for dirpath, _, files in os.walk(root):
            for f in files:
                if f.endswith((".py", ".h", ".cuh", ".cu", ".cc", ".cpp")) or f == "Makefile":
                    path = os.path.join(dirpath, f)
                    with open(path, errors="replace") as fh:
                        for i, line in enumerate(fh, 1):
                            if pattern.search(line):
                                hits.append(f"{os.path.relpath(path, ROOT)}:{i}: {line.strip()}")
    assert not hits, hits


def test_binding_fails_loudly_without_the_library(monkeypatch):
    """No CPU fallback: without the built library the binding raises."""
    import gpusolver_b200 as gsm
    monkeypatch.setattr(gsm, "_lib", None)
    monkeypatch.setattr(gsm, "LIB_PATH", os.path.join(ROOT, "no-such-dir", "libgpusolver_b200.so"))
    with pytest.raises(ImportError, match="no CPU fallback"):
        gsm.lib()
