"""The host setup code built with AddressSanitizer and UndefinedBehaviorSanitizer
(tests/cpp/setup_sanitizer_driver.cc + csrc/setup.cc): no out-of-bounds access,
use after free, leak or undefined behaviour on four problem families, with
the row-parallel loops on one host thread and on four."""
import os
import shutil
import subprocess

import pytest

from conftest import PKG, ROOT


def test_host_setup_is_clean_under_address_and_ub_sanitizers(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "setup_sanitizer_driver")
    src = os.path.join(ROOT, "tests", "cpp", "setup_sanitizer_driver.cc")
    build = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
                            "-I", os.path.join(PKG, "csrc"), src, os.path.join(PKG, "csrc", "setup.cc"), "-o", exe,
                            "-lpthread"], capture_output=True, text=True, timeout=600)
    if build.returncode != 0 and "sanitize" in build.stderr:
        pytest.skip("the compiler has no sanitizer runtime: " + build.stderr[:200])
    assert build.returncode == 0, build.stderr[:2000]
    for threads in ("1", "4"):
        env = dict(os.environ, GS_HOST_THREADS=threads, ASAN_OPTIONS="detect_leaks=1:halt_on_error=1",
                   UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
        run = subprocess.run([exe], capture_output=True, text=True, timeout=600, env=env)
        assert run.returncode == 0, (threads, run.stderr[-3000:])
        assert run.stdout.count("levels") == 8


def test_oracle_is_clean_under_address_and_ub_sanitizers(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "oracle_sanitizer_driver")
    build = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
                            "-I", os.path.join(PKG, "csrc"), os.path.join(ROOT, "tests", "cpp", "oracle_sanitizer_driver.cc"),
                            os.path.join(ROOT, "oracle", "oracle.cc"), os.path.join(PKG, "csrc", "setup.cc"), "-o", exe,
                            "-lpthread"], capture_output=True, text=True, timeout=600)
    if build.returncode != 0 and "sanitize" in build.stderr:
        pytest.skip("the compiler has no sanitizer runtime: " + build.stderr[:200])
    assert build.returncode == 0, build.stderr[:2000]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:halt_on_error=1", UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
    run = subprocess.run([exe], capture_output=True, text=True, timeout=900, env=env)
    assert run.returncode == 0, run.stderr[-3000:]
    lines = run.stdout.splitlines()
    # 4 problems x 12 option sets, plus 4 strong-coupling colouring runs for
    # each of the two Gauss-Seidel problems without a coarse smoother of its own
    assert len(lines) == 56 and all(" rc 0 " in ln and ln.endswith("st 1") for ln in lines), run.stdout[-2000:]


def test_host_entry_points_are_clean_under_address_and_ub_sanitizers(tmp_path):
    """The C ABI's host entry points, malformed inputs included, under the two
    sanitizers (the CUDA parts of the library are not linked: no host entry
    point reaches them)."""
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    if shutil.which("g++") is None or not os.path.exists(os.path.join(cuda, "lib64", "libcudart.so")):
        pytest.skip("g++ or the CUDA runtime library not available")
    exe = str(tmp_path / "capi_sanitizer_driver")
    build = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
                            "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc"),
                            "-I", os.path.join(cuda, "include"),
                            os.path.join(ROOT, "tests", "cpp", "capi_sanitizer_driver.cc"),
                            os.path.join(PKG, "csrc", "capi.cc"), os.path.join(PKG, "csrc", "setup.cc"),
                            "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,--unresolved-symbols=ignore-all",
                            f"-Wl,-rpath,{os.path.join(cuda, 'lib64')}", "-o", exe, "-lpthread"],
                           capture_output=True, text=True, timeout=600)
    if build.returncode != 0 and "sanitize" in build.stderr:
        pytest.skip("the compiler has no sanitizer runtime: " + build.stderr[:200])
    assert build.returncode == 0, build.stderr[:2000]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:halt_on_error=1", UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
    run = subprocess.run([exe], capture_output=True, text=True, timeout=900, env=env)
    assert run.returncode == 0, run.stderr[-3000:]
    ok, refused = (int(v) for v in run.stdout.split()[1::2])
    assert ok > 5000 and refused > 5000
