"""The C++20 drop-in header (include/fpx/fastpoly.hpp): reference-style code
compiles against it (CPU), and runs bit-exactly on the GPU library (gpu)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "test_dropin.cpp")
LIBDIR = os.path.join(ROOT, "fastpoly_b200")


def _compile(out_dir):
    exe = os.path.join(out_dir, "test_dropin")
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-std=c++20", "-O2", "-I" + os.path.join(ROOT, "include"), SRC, "-L" + LIBDIR, "-lfpx_b200",
                    "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    return exe


def test_dropin_compiles(tmp_path):
    assert os.path.exists(_compile(str(tmp_path)))


@pytest.mark.gpu
def test_dropin_runs_on_gpu(tmp_path):
    exe = _compile(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all drop-in checks passed" in r.stdout
