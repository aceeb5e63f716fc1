"""The C++ drop-in header include/blockdaglu/solver.h.

CPU: the header compiles (strict warnings) and links against libbdlu, both
for this repository's C++ API test and for the reference's own test program
(apps/tests/main.cpp) when it was built against the header under oracle/_ref.
GPU: both programs run on the engine and pass.  The reference's test program
is used unmodified: its cases (apps/tests/main.cpp:93-204) -- input errors,
the 3x3 golden solution with duplicates, the BLOCK route on two patterns and
scaled values, the P*A*Q = L*U export identity and two solvers on two
threads -- then run on the GPU engine through the drop-in class.
"""
import os
import subprocess

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "block-daglu_b200", "lib")
SRC = os.path.join(ROOT, "tests", "cpp", "solver_api_test.cpp")
REF_TESTS = os.path.join(ROOT, "oracle", "_ref", "blockdaglu_tests_b200")


def _compile(out):
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"), SRC,
           "-L" + LIB, "-lbdlu", "-Wl,-rpath," + LIB, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def test_header_compiles_and_links(tmp_path):
    _compile(str(tmp_path / "api_test"))


def test_reference_tests_link_against_header():
    if not os.path.exists(REF_TESTS):
        pytest.skip("oracle/_ref/blockdaglu_tests_b200 not built (needs the reference sources)")
    r = subprocess.run(["ldd", REF_TESTS], capture_output=True, text=True)
    assert "libbdlu.so" in r.stdout and "libbdlu_ref" not in r.stdout


@pytest.mark.gpu
def test_cpp_api_on_gpu(cuda_device, tmp_path):
    exe = _compile(str(tmp_path / "api_test"))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


@pytest.mark.gpu
def test_reference_test_program_on_gpu(cuda_device):
    if not os.path.exists(REF_TESTS):
        pytest.skip("oracle/_ref/blockdaglu_tests_b200 not built (needs the reference sources)")
    r = subprocess.run([REF_TESTS], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "All BlockDAGLU tests passed" in r.stdout, r.stdout + r.stderr
