"""The header-only C++ drop-in layer (include/qmb/qmbcuda.hpp): a program
written against the reference's class names and constructor signatures
(tests/cpp/dropin_check.cpp) compiles with g++ against libqmb_b200.so, and
on a GPU reproduces the known ground energies (the checks are listed in the
program)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_check.cpp")
CUDA = "/usr/local/cuda"


def _build(tmp_path):
    exe = str(tmp_path / "dropin_check")
    lib_dir = os.path.join(ROOT, "qmbcuda_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), SRC, "-o", exe, "-L", lib_dir, "-lqmb_b200",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{lib_dir}",
           f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_program_compiles(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_dropin_program_energies(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASSED" in r.stdout
