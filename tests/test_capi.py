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
