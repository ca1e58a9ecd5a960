"""The C++ API mirror (include/GPUSolver/*.h): programs written the way the
reference's examples use gpuSolver:: classes compile against these headers,
link libgpusolver_b200.so and give the same results as the Python binding
(which calls the same C ABI) and the oracle.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT, cuda_available

CPP = os.path.join(ROOT, "tests", "cpp")


def compile_program(src, out_dir):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = os.path.join(str(out_dir), os.path.splitext(src)[0])
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(CPP, src), "-L", PKG, "-lgpusolver_b200", f"-Wl,-rpath,{PKG}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def parse(lines):
    return {ln.split(" ", 1)[0]: ln.split(" ", 1)[1] if " " in ln else "" for ln in lines}


def test_host_side_validation_and_setup(gs, tmp_path):
    exe = compile_program("api_host_checks.cpp", tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    kv = parse(out.splitlines())
    # the reference's messages and throw points
    assert kv["perm_size0"] == "throws: Permutation: size must be nonzero."
    assert kv["perm_null"] == "throws: Permutation: input pointers must not be null."
    assert kv["perm_range"] == "throws: Permutation: oldToNew contains invalid index."
    assert kv["perm_inverse"] == "throws: Permutation: mappings are not inverses."
    assert kv["coloring_uninit"] == "throws:  the coloring was not initialized"
    assert kv["builder_levels"].startswith("throws:")
    assert kv["pc_perm_count"].startswith("throws:")
    assert kv["solver_wrong_matrix"].startswith("throws:")
    # the MultigridGaussSeidelPreconditioner defaults: coarsest level pre + post steps, reference V-cycle
    assert kv["coarse_steps"] == "2 smoother 0 reference_vcycle 1"
    # the hierarchy, RCM and colouring agree with the Python binding of the same C ABI
    a = gs.poisson7(12)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 50)
    assert int(kv["levels"]) == H.levels
    # build(matrix, nearNullspace): no modes is build(matrix); modes are refused loudly
    assert int(kv["null_nullspace_levels"]) == H.levels
    assert kv["nullspace_modes"] == "throws: AMGHierarchyBuilder: near-nullspace modes are not supported by this library."
    level_lines = [ln for ln in out.splitlines() if ln.startswith("level ")]
    for k, ln in enumerate(level_lines):
        f = ln.split()
        assert int(f[3]) == H.A(k).rows and int(f[5]) == H.A(k).nnz
    sig = 0
    for k in range(H.levels):
        o2n, _ = gs.rcm(H.A(k))
        for v in o2n:
            sig = (sig * 31 + int(v)) % 1000000007
    assert int(kv["rcm_signature"]) == sig
    hsig = 0
    for o2n, _ in gs.hierarchical_reordering(H):
        for v in o2n:
            hsig = (hsig * 31 + int(v)) % 1000000007
    assert int(kv["hierarchical_signature"]) == hsig
    colors = gs.greedy_coloring(a)
    assert kv["colors"] == f"{colors[0]} offsets {colors[0] + 1}"
    # C ABI extensions: host build of the independent-set aggregation, colouring, errors
    Hm = gs.Hierarchy.build_ex(a, 1, 0.1, 10, 50, aggregation=1, device=-1)
    f = kv["mis2_rc"].split()
    assert f[0] == "0" and int(f[2]) == Hm.levels
    assert [int(v) for v in f[3:]] == [Hm.A(k).rows for k in range(Hm.levels)]
    rc, msg = kv["gpu_sequential_rc"].split(" ", 1)
    assert int(rc) != 0 and "aggregation 1" in msg
    assert int(kv["smallest_last_colors"]) == gs.smallest_last_coloring(a)[0]
    assert int(kv["setup_times_null"]) != 0
    if "device_solve" in kv and kv["device_solve"].startswith("throws:"):
        assert "no CUDA device" in kv["device_solve"]


@pytest.mark.gpu
def test_reference_style_program_solves_on_gpu(gs, orc, device, tmp_path):
    """mainTetmeshPoisson's call sequence in C++: SA hierarchy, per-level RCM,
    MultigridGaussSeidelPreconditioner(1, 1, 1 V-cycle, omega 1), CGSolver
    with tolerance 1e-6 on an FP32 right-hand side."""
    exe = compile_program("reference_style_solve.cpp", tmp_path)
    side = 24
    a = gs.poisson7(side)
    b = gs.uniform_rhs(a.rows, 3).astype(np.float32)
    rhs, xout = tmp_path / "b.bin", tmp_path / "x.bin"
    b.tofile(rhs)
    out = subprocess.run([exe, str(side), str(rhs), str(xout)], check=True, capture_output=True, text=True,
                         timeout=300).stdout.split()
    levels, iterations = int(out[1]), int(out[3])
    x = np.fromfile(xout, dtype=np.float32)

    H = gs.Hierarchy.build(a, 1, 0.1, 10, 200)
    assert levels == H.levels
    perms = [gs.rcm(H.A(k)) for k in range(H.levels)]
    opts = gs.SolverOptions(tol=1e-6, max_iter=100, reference_vcycle=1, coarse_solver=0, coarse_steps=2)
    xp, st = gs.Solver(H, opts, permutations=perms, device=device).solve_f32(b)
    assert iterations == st.iterations
    # same library and options; each solver autotunes its lanes per row by timing, so the
    # summation order (and the last bits of the FP64 iterate) may differ between instances
    assert np.linalg.norm(x - xp) / np.linalg.norm(xp) <= 1e-6

    A = [H.A(k) for k in range(H.levels)]
    P = [H.P(k) for k in range(H.levels - 1)]
    R = [H.R(k) for k in range(H.levels - 1)]
    xo, it, status, _ = orc.amg_pcg(A, P, R, b.astype(np.float64), perms=perms, tol=1e-6, max_iter=100,
                                    alias=1, coarse_solver=0, coarse_steps=2)
    assert status == 1 and abs(iterations - it) <= 1
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-6  # FP32 output of an FP64 solve


@pytest.mark.gpu
def test_reference_style_program_gpu_setup(gs, device, tmp_path):
    """The same program with AMGHierarchyBuilder::buildOnDevice: the levels of the
    C ABI's GPU build and the solve's iteration count of that hierarchy."""
    exe = compile_program("reference_style_solve.cpp", tmp_path)
    side = 24
    a = gs.poisson7(side)
    b = gs.uniform_rhs(a.rows, 3).astype(np.float32)
    rhs, xout = tmp_path / "b.bin", tmp_path / "x.bin"
    b.tofile(rhs)
    out = subprocess.run([exe, str(side), str(rhs), str(xout), "gpu-setup"], check=True, capture_output=True,
                         text=True, timeout=300).stdout.split()
    levels, iterations = int(out[1]), int(out[3])
    x = np.fromfile(xout, dtype=np.float32)
    H = gs.Hierarchy.build_ex(a, 1, 0.1, 10, 200, aggregation=1, device=device)
    assert levels == H.levels
    perms = [gs.rcm(H.A(k)) for k in range(H.levels)]
    opts = gs.SolverOptions(tol=1e-6, max_iter=100, reference_vcycle=1, coarse_solver=0, coarse_steps=2)
    xp, st = gs.Solver(H, opts, permutations=perms, device=device).solve_f32(b)
    assert iterations == st.iterations
    assert np.linalg.norm(x - xp) / np.linalg.norm(xp) <= 1e-6


@pytest.mark.gpu
def test_reference_style_program_single_level_jacobi(gs, orc, device, tmp_path):
    """cantileverBeam's DampedJacobiPreconditioner(4, 0.9) through the C++ mirror; the CG
    permutes its matrix by the RCM permutation it is given, as the reference does."""
    exe = compile_program("reference_style_solve.cpp", tmp_path)
    side = 16
    a = gs.poisson7(side)
    b = gs.uniform_rhs(a.rows, 5).astype(np.float32)
    rhs, xout = tmp_path / "b.bin", tmp_path / "x.bin"
    b.tofile(rhs)
    out = subprocess.run([exe, str(side), str(rhs), str(xout), "jacobi"], check=True, capture_output=True,
                         text=True, timeout=300).stdout.split()
    iterations = int(out[3])
    x = np.fromfile(xout, dtype=np.float32)
    perm = gs.rcm(a)
    xo, it, status, _ = orc.amg_pcg([a], [], [], b.astype(np.float64), perms=[perm], smoother=2,
                                    coarse_solver=0, coarse_steps=4, omega=0.9, tol=1e-6, max_iter=1000)
    assert status == 1 and abs(iterations - it) <= 1
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-6


def test_host_containers_and_block_helpers(gs, tmp_path):
    """HostCSRMatrix, HostELLMatrix, permuteMatrix, the block helpers and the
    reordering strategies of the mirror: each property is checked inside the
    program; the errors carry the reference's messages (src/HostSparseMatrix.cc,
    src/HostELLMatrix.cc, src/BlockUtils.cc)."""
    exe = compile_program("host_matrix_checks.cpp", tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    kv = parse(out.splitlines())
    assert "FAIL" not in out
    assert kv["csr_dims"] == "throws: HostCSRMatrix: matrix dimensions must be nonzero."
    assert kv["csr_null"] == "throws: HostCSRMatrix: input pointers must not be null."
    assert kv["csr_square"] == "throws: HostCSRMatrix::applyPermutation: matrix must be square."
    assert kv["csr_perm_size"] == ("throws: HostCSRMatrix::applyPermutation: permutation size does not match "
                                   "matrix dimensions.")
    for key in ("csr_unpermuted", "csr_from_container", "permute_matrix", "block_graph_host",
                "expand_block_permutation", "identity_reordering"):
        assert kv[key] == "ok", key
    assert kv["csr_permuted"] == "ok originals_kept ok"
    assert kv["ell_width0"] == "throws: HostELLMatrix: ELL width must be nonzero."
    f = kv["ell"].split()
    assert f[0] == "ok" and int(f[2]) > 0
    assert kv["permute_matrix_not_bijective"].startswith("throws:") and "not a permutation" in kv[
        "permute_matrix_not_bijective"]
    # path of 5 nodes: neighbours only, the diagonal block makes no edge
    assert kv["block_graph"] == "0:1,;1:0,2,;2:1,3,;3:2,4,;4:3,;"
    assert kv["block_graph_divisible"] == "throws: buildBlockGraph: matrix size is not divisible by block size."
    assert "more entries than the matrix" in kv["block_graph_unsymmetric"]
    assert float(kv["block_inverse_residual"]) < 1e-6
    assert kv["block_inverse_not_spd"] == "throws: Block diagonal is not SPD."


def test_block_graph_of_unsymmetric_pattern_is_refused(gs):
    """The symmetrised node graph of an unsymmetric pattern can outgrow nnz;
    the entry point reports it instead of writing past the caller's array."""
    import scipy.sparse as sp
    u = sp.csr_matrix(np.triu(np.ones((4, 4))))
    with pytest.raises(gs.SolverError, match="more entries than the matrix"):
        gs.block_graph(gs.Csr.from_scipy(u), 1)
    # a symmetric pattern of the same size is fine
    s = sp.csr_matrix(np.ones((4, 4)))
    grp, gci = gs.block_graph(gs.Csr.from_scipy(s), 1)
    assert list(grp) == [0, 3, 6, 9, 12] and len(gci) == 12


def test_backend_without_device_fails_loudly(gs, tmp_path):
    """The mirror's CudaBackend has no CPU fallback: its first device object
    raises the library's no-device error."""
    if cuda_available():
        pytest.skip("a CUDA device is present")
    exe = compile_program("backend_checks.cpp", tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    assert parse(out.splitlines())["no_device"].startswith("no CUDA device is available")


@pytest.mark.gpu
def test_backend_known_answers_and_smoothers(gs, device, tmp_path):
    """Backend / Device* / encoder mirror on the GPU: the reference's CUDA test
    answers (tests/cuda/testCuda{GaussSeidel,Spmv,BlockOps,VectorOps,ScalarOps}.cc)
    and the four single-level smoothers within 1e-5 of FP32 host loops (the
    reference's own GPU-vs-CPU smoother tolerance,
    tests/metal/gaussSeidelSymmUnittest.cc:300)."""
    exe = compile_program("backend_checks.cpp", tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    kv = parse(out.splitlines())
    assert "no_device" not in kv, out
    assert kv["gs_color0"] == "1 0 3 0"
    assert kv["gs_sweep"] == "1 3 3 4.75"
    assert kv["gs_range"] == "throws: encodeGaussSeidelColor: invalid color range."
    assert kv["spmv"] == "6 13 19"
    assert kv["spmv_updated"] == "8 14"
    assert kv["spmv_shape"] == "throws: encodeSpmv: dimension mismatch."
    assert kv["update_count"].startswith("throws:")
    assert kv["dot"] == "32"
    assert kv["block_apply"] == "2 6 12 9 10 18"
    assert kv["axpy_scale"] == "6 12 18"
    assert kv["axpy_dev_scale_vector"] == "9 36 81"
    assert kv["copy"] == "1 2 3"
    assert kv["set_zero"] == "0 0 0"
    assert kv["resized"] == "2 10 20"
    assert kv["scalars"] == "1.5 -6 4"
    for key in ("sgs_smoother", "block_gs_smoother"):
        f = kv[key].split()
        assert float(f[0]) <= 1e-5 and int(f[2]) == 2, key
    for key in ("jacobi_smoother", "block_jacobi_smoother"):
        assert float(kv[key]) <= 1e-5, key
    assert kv["sgs_omega"] == "throws: SymmetricGaussSeidelSmoother: invalid omega."
    assert kv["sgs_twice"] == "throws: SymmetricGaussSeidelSmoother: already initialized."
    assert kv["ell"] == "18 18 4 72"


def test_smoothers_on_a_host_backend(gs, tmp_path):
    """The smoother classes drive any implementation of the abstract Backend:
    on a host-memory test backend they issue the reference's encode sequences
    (src/Smoothers/SymmetricGaussSeidelSmoother.cc:80-128: colours forward then
    backward as (colorStart, colorCount); DampedJacobiSmoother.cc:72-89 and
    BlockJacobiSmoother.cc:36-87: spmv, copy, axpy, scale, axpy) and reduce the
    residual."""
    exe = compile_program("host_backend_smoothers.cpp", tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    kv = parse(out.splitlines())
    # 1-D path of 6 rows: greedy colours {0, 2, 4} and {1, 3, 5}; 2 steps
    assert kv["sgs_sequence"] == ",".join(["gs 0 3", "gs 3 3", "gs 3 3", "gs 0 3"] * 2)
    assert kv["sgs_reduces"] == "1"
    assert kv["jacobi_sequence"] == "spmv,copy,axpy,scale_vector,axpy"
    # path of 4 nodes: node colours {0, 2} and {1, 3}
    assert kv["bgs_sequence"] == "bgs 0 2,bgs 2 2,bgs 2 2,bgs 0 2"
    assert kv["bgs_reduces"] == "1"
    assert kv["block_jacobi_sequence"] == "spmv,copy,axpy,block_apply,axpy"
    assert float(kv["block_jacobi_first_step"]) == 0.0
    assert kv["sgs_uninitialized"] == "throws: SymmetricGaussSeidelSmoother: not initialized."


@pytest.mark.parametrize("kind, smoother, pre, post, coarse, omega", [
    ("sgs", 0, 1, 1, 2, 1.0),      # MultigridGaussSeidelSmoother(1, 1, 2, 1.0)
    ("jacobi", 2, 2, 2, 4, 0.7),   # MultigridDampedJacobiSmoother(2, 2, 4, 0.7)
])
def test_multigrid_smoother_matches_reference_vcycle(gs, orc, tmp_path, kind, smoother, pre, post, coarse, omega):
    """The mirror's MultigridSmoother (built on any Backend; here the host test
    backend) applies the reference's V-cycle (src/Smoothers/MultigridSmoother.cc:337-420)
    including its correction/solution buffer aliasing on the coarse levels: one
    V-cycle from z = 0 equals the oracle's FP32 restatement bit for bit."""
    exe = compile_program("multigrid_smoother_host.cpp", tmp_path)
    side = 10
    a = gs.poisson7(side)
    H = gs.Hierarchy.build(a, 1, 0.1, 10, 50)
    perms = [gs.rcm(H.A(k)) for k in range(H.levels)]
    r = np.random.default_rng(7).uniform(-1, 1, a.rows).astype(np.float32)
    rb, zb = tmp_path / "r.bin", tmp_path / "z.bin"
    r.tofile(rb)
    out = subprocess.run([exe, str(side), kind, str(rb), str(zb)], check=True, capture_output=True, text=True,
                         timeout=120).stdout.split()
    assert int(out[1]) == H.levels >= 3
    z = np.fromfile(zb, dtype=np.float32)
    A = [H.A(k) for k in range(H.levels)]
    P = [H.P(k) for k in range(H.levels - 1)]
    R = [H.R(k) for k in range(H.levels - 1)]
    args = dict(perms=perms, smoother=smoother, pre=pre, post=post, coarse_steps=coarse, omega=omega, coarse_solver=0)
    zo = orc.precondition(A, P, R, r.astype(np.float64), precision=orc.PREC_F32, alias=1, **args)
    assert np.array_equal(z, zo.astype(np.float32))
    # the aliasing is observable: the textbook V-cycle differs by percents
    zt = orc.precondition(A, P, R, r.astype(np.float64), precision=orc.PREC_F64, alias=0, **args)
    assert np.linalg.norm(z - zt) / np.linalg.norm(zt) > 1e-3


def test_preconditioner_apply_on_a_backend(gs, orc, tmp_path):
    """Preconditioner::initialize / apply of the mirror (any Backend; here the
    host test backend), as the reference's CGSolver drives them: the single-level
    SGS preconditioner against the reference's own SymmetricGaussSeidelPreconditioner
    on its CPUBackend (1e-6; FP32 rounding of the update differs in the last bit),
    Jacobi z = D^-1 r and identity exactly, damped Jacobi against FP32 numpy, and
    MultigridGaussSeidelPreconditioner bit-equal to the oracle's reference V-cycle."""
    exe = compile_program("preconditioner_apply_host.cpp", tmp_path)
    side = 8
    a = gs.poisson7(side)
    r = np.random.default_rng(3).uniform(-1, 1, a.rows).astype(np.float32)
    rb = tmp_path / "r.bin"
    r.tofile(rb)
    prefix = str(tmp_path / "out_")
    subprocess.run([exe, "single", str(side), "1.3", "2", str(rb), prefix], check=True, timeout=120)
    load = lambda name: np.fromfile(prefix + name + ".bin", np.float32)
    if orc.ref_available():
        zr = orc.ref_sgs_apply(a, r, 1.3, 2)
        assert np.abs(load("sgs") - zr).max() <= 1e-6 * np.abs(zr).max()
    rows = np.repeat(np.arange(a.rows), np.diff(a.row_ptr))
    d = np.zeros(a.rows, np.float32)
    d[rows[a.col_idx == rows]] = a.val[a.col_idx == rows]
    inv = np.float32(1) / d
    assert np.array_equal(load("jacobi"), r * inv)
    assert np.array_equal(load("identity"), r)
    A = a.to_scipy().astype(np.float32)
    x = np.zeros_like(r)
    for _ in range(2):
        x = x + np.float32(1.3) * ((r - A @ x) * inv)
    assert np.abs(load("damped") - x).max() <= 1e-6 * np.abs(x).max()

    H = gs.Hierarchy.build(a, 1, 0.1, 10, 50)
    perms = [gs.rcm(H.A(k)) for k in range(H.levels)]
    zb = tmp_path / "zm.bin"
    subprocess.run([exe, "multigrid", str(side), str(rb), str(zb)], check=True, timeout=120)
    Al = [H.A(k) for k in range(H.levels)]
    P = [H.P(k) for k in range(H.levels - 1)]
    R = [H.R(k) for k in range(H.levels - 1)]
    zo = orc.precondition(Al, P, R, r.astype(np.float64), perms=perms, precision=orc.PREC_F32, smoother=0, pre=1,
                          post=1, coarse_steps=2, omega=1.0, coarse_solver=0, alias=1)
    assert H.levels >= 3 and np.array_equal(np.fromfile(zb, np.float32), zo.astype(np.float32))


def test_every_header_compiles_alone(tmp_path):
    """Each header of the C++ mirror compiles as the only include of a
    translation unit (-Wall -Wextra -Werror), and the C ABI header compiles as
    C99 with -pedantic."""
    import concurrent.futures as cf
    import glob
    if shutil.which("g++") is None or shutil.which("gcc") is None:
        pytest.skip("g++/gcc not available")
    inc = os.path.join(ROOT, "include")
    headers = sorted(glob.glob(os.path.join(inc, "GPUSolver", "**", "*.h"), recursive=True))
    assert len(headers) >= 45

    def compile_alone(h):
        rel = os.path.relpath(h, inc)
        r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-x", "c++", "-I", inc,
                            "-"], input=f"#include <{rel}>\n", capture_output=True, text=True, timeout=120)
        return rel, r.returncode, r.stderr[:400]

    with cf.ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1))) as ex:
        failed = [(rel, err) for rel, rc, err in ex.map(compile_alone, headers) if rc]
    assert not failed, failed
    # all of them in one unit (no conflicting definitions), with a preconditioner a caller writes
    unit = "".join(f"#include <{os.path.relpath(h, inc)}>\n" for h in headers) + (
        "struct Mine : gpuSolver::Preconditioner {\n"
        "  void initialize(gpuSolver::Backend &, const gpuSolver::HostCSRMatrix &,\n"
        "                  const gpuSolver::DeviceCSRMatrix &) override {}\n"
        "  void apply(gpuSolver::Backend &b, gpuSolver::BackendEncoder &e, const gpuSolver::DeviceVector &i,\n"
        "             gpuSolver::DeviceVector &o) override { b.encodeCopy(e, i, o); }\n"
        "};\n"
        "int main() { Mine m; return m.custom() ? 0 : 1; }\n")
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-x", "c++", "-I", inc, "-"],
                       input=unit, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[:2000]
    c_unit = "#include <gpusolver_b200.h>\nint main(void) { gs_solver_options o; gs_solver_options_default(&o); return 0; }\n"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-fsyntax-only", "-x", "c", "-I",
                        inc, "-"], input=c_unit, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("kind, code, omega, sweeps", [("jacobi", 1, 1.0, 1), ("sgs", 2, 1.2, 2)])
@pytest.mark.parametrize("rcm", [0, 1])
def test_cg_with_a_caller_written_preconditioner(gs, ref, tmp_path, kind, code, omega, sweeps, rcm):
    """CGSolver with a preconditioner the caller wrote against the reference's
    interface runs the reference's CG loop on the Backend (here the host test
    backend): with a Jacobi preconditioner it equals the reference's CGSolver +
    JacobiPreconditioner bit for bit, with an SGS one the reference's iteration
    count and iterate within 1e-6 (the Gauss-Seidel update rounds differently in
    the last bit); with and without an RCM permutation of the CG's matrix."""
    exe = compile_program("custom_preconditioner_host.cpp", tmp_path)
    side = 10
    a = gs.poisson7(side)
    rows = np.repeat(np.arange(a.rows), np.diff(a.row_ptr))
    v = a.val.copy()
    d = a.col_idx == rows
    v[d] = 6 + 0.05 * (rows[d] % 7)  # the program's matrix
    a = gs.Csr(a.rows, a.cols, a.row_ptr, a.col_idx, v)
    b = np.random.default_rng(1).uniform(-1, 1, a.rows).astype(np.float32)
    bb, xb = tmp_path / "b.bin", tmp_path / "x.bin"
    b.tofile(bb)
    out = subprocess.run([exe, str(side), kind, str(rcm), str(bb), str(xb)], check=True, capture_output=True,
                         text=True, timeout=120).stdout.split()
    assert out[3] == "1"  # a caller-written preconditioner
    x = np.fromfile(xb, np.float32)
    xr, itr = ref.ref_pcg(a, b, preconditioner=code, omega=omega, sweeps=sweeps, tol=1e-5, max_iter=500,
                          perm=gs.rcm(a) if rcm else None)
    assert int(out[1]) == itr
    if kind == "jacobi":
        assert np.array_equal(x, xr)
    else:
        assert np.abs(x - xr).max() <= 1e-6 * np.abs(xr).max()


def test_integration_examples_compile():
    """The C++ examples of the integration guide (the reference's call sequence
    and a caller-written preconditioner), kept in tests/cpp/integration_examples.cpp,
    compile against the mirror."""
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    src = os.path.join(ROOT, "tests", "cpp", "integration_examples.cpp")
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I",
                        os.path.join(ROOT, "include"), src], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[:3000]
