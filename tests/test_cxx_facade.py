"""The C++ facade (include/kate_b200/Kate.hpp) compiles a reference-style
program (Kate::Circuit / Gate / Matrix / Simulator, gate-id macros) and links
against libkate_b200.so."""
import os
import subprocess

import numpy as np
import pytest

from kate_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def facade_exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cxx") / "facade_main")
    libdir = os.path.dirname(_lib.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cxx",
           "facade_main.cpp"), "-L" + libdir, "-lkate_b200", "-Wl,-rpath," + libdir, "-o", out]
    # the library is named libkate_b200.so in the package directory
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_facade_builds_and_runs_the_passes(facade_exe):
    r = subprocess.run([facade_exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "gates" in r.stdout


@pytest.mark.gpu
def test_facade_simulates_on_the_gpu(facade_exe, oracle):
    r = subprocess.run([facade_exe, "sim"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("Qbit ") == 10
