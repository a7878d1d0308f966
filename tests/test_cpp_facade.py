"""The C++ facade (include/stardust_sim.hpp): a C++ program with the reference's
sim_tests checks for the PM path builds against it (CPU) and passes (GPU)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "sim_facade_test.cpp")
LIBDIR = os.path.join(ROOT, "stardust_b200")


def _build(out_dir):
    exe = os.path.join(out_dir, "sim_facade_test")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-L", LIBDIR,
           "-lstardust_pm", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_facade_program_builds(lib, tmp_path):
    assert os.path.exists(_build(str(tmp_path)))


@pytest.mark.gpu
def test_facade_program_passes(cuda, tmp_path):
    exe = _build(str(tmp_path))
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
