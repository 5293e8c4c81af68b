"""The C++ drop-in (include/rsg_rmatrixsolver.hpp) compiles against the C ABI,
and on a GPU runs the reference's own matrix-solver tests through it."""
import os
import subprocess

import pytest

from conftest import REPO

LIBDIR = os.path.join(REPO, "range-solver-lib_b200", "lib")


def _build(tmp_path):
    exe = str(tmp_path / "test_dropin")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I" + os.path.join(REPO, "include"),
           os.path.join(REPO, "tests", "cpp", "test_dropin.cpp"), "-L" + LIBDIR, "-lrsg", "-Wl,-rpath," + LIBDIR,
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_compiles(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_dropin_runs_reference_tests(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all passed" in r.stdout
