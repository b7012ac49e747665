"""The C++ host API (include/cie_cuda/linalg.hpp) over the C-ABI.

CPU: the test program compiles and links against libciecu.so, and -- where the
reference sources are present -- the wrapper compiles against the reference's own
LinearOperator / LinalgSpaceLike headers with CUDASpace satisfying the concept.
GPU: the program runs the solveSYCLCG-style driver and checks SpMV, both CG paths,
Jacobi and the mixed solver against the oracle."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOURCE = os.path.join(ROOT, "tests", "cpp", "cie_cuda_test.cpp")
REFERENCE = "/root/reference/libraries"


def _compile(out, extra=()):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    lib, ora = os.path.join(ROOT, "cie_b200"), os.path.join(ROOT, "oracle")
    if not os.path.exists(os.path.join(lib, "libciecu.so")) or not os.path.exists(os.path.join(ora, "liboracle.so")):
        pytest.skip("libciecu.so / liboracle.so not built")
    cmd = [cxx, "-std=c++20", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), SOURCE,
           "-L" + lib, "-lciecu", "-L" + ora, "-loracle", "-Wl,-rpath," + lib, "-Wl,-rpath," + ora, "-o", out,
           *extra]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


def test_cpp_api_compiles_and_links(tmp_path):
    _compile(str(tmp_path / "cie_cuda_test"))


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="reference sources not present")
def test_cpp_api_is_a_linalg_space_of_the_reference():
    r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-Werror", "-DCIE_CUDA_WITH_CIE_LINALG",
                        "-I" + os.path.join(ROOT, "include"), "-I" + REFERENCE + "/cieutils",
                        "-I" + REFERENCE + "/cieutils/inc", "-I" + REFERENCE + "/linalg", SOURCE],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


@pytest.mark.gpu
def test_cpp_api_solves_like_the_reference(tmp_path):
    exe = str(tmp_path / "cie_cuda_test")
    _compile(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0 and "ALL OK" in r.stdout, r.stdout[-4000:] + r.stderr[-2000:]
