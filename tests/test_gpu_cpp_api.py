"""The reference's known-answer tests as a C++ program against the C++ API."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "trotter-suzuki-mpi_b200", "trottersuzuki_b200")
SRC = os.path.join(REPO, "tests", "cpp", "kerneltest_b200.cpp")


def build(tmp_path):
    exe = str(tmp_path / "kerneltest_b200")
    subprocess.check_call([
        "g++", "-O2", "-std=c++17", SRC,
        "-I" + os.path.join(REPO, "trotter-suzuki-mpi_b200", "host"),
        "-I" + os.path.join(REPO, "include"),
        "-L" + PKG, "-ltrottersuzuki_b200", "-ltsb200", "-Wl,-rpath," + PKG, "-o", exe])
    return exe


def test_cpp_program_compiles_against_the_api(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
@pytest.mark.parametrize("kernel_type", ["gpu", "gpu_fp32"])
def test_cpp_known_answer_tests(tmp_path, kernel_type):
    exe = build(tmp_path)
    r = subprocess.run([exe, kernel_type], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
