"""The C++ facade (include/kate_b200/Kate.hpp) compiles a reference-style
program (Kate::Circuit / Gate / Matrix / Simulator, gate-id macros) and links
against libkate_b200.so."""
import os
import subprocess

import numpy as np
import pytest

from kate_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path_factory, name):
    out = str(tmp_path_factory.mktemp("cxx") / name)
    libdir = os.path.dirname(_lib.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cxx",
           name + ".cpp"), "-L" + libdir, "-lkate_b200", "-Wl,-rpath," + libdir, "-o", out]
    # the library is named libkate_b200.so in the package directory
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.fixture(scope="module")
def facade_exe(tmp_path_factory):
    return _build(tmp_path_factory, "facade_main")


@pytest.fixture(scope="module")
def bench_exe(tmp_path_factory):
    return _build(tmp_path_factory, "bench_main")


def test_facade_builds_and_runs_the_passes(facade_exe):
    r = subprocess.run([facade_exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "gates" in r.stdout
    # H*H = I (x2 after the scale), (1+2i)/(3+4i) = 0.44+0.08i, +1, *i, *2
    vals = [float(x) for x in r.stdout.split("arith ")[1].split()[:5]]
    assert vals == pytest.approx([2.0, 0.0, -0.16, 2.88, np.pi / 4], abs=1e-6)  # printed to 6 digits


def facade_circuit(n=10):
    """The circuit tests/cxx/facade_main.cpp builds, as gate tuples."""
    x = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    g = []
    for i in range(n):
        g += [(2, [i], 0, None), (2, [i], 0, None)]
    g += [(3, [i, (i + 1) % n], 0, None) for i in range(n)]
    g += [(4, [1, 3], 3, None), (0, [4], 0, x), (2, [5], 0, None)]
    return g


@pytest.mark.gpu
def test_facade_simulates_on_the_gpu(facade_exe, oracle):
    r = subprocess.run([facade_exe, "sim"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("Qbit ")]
    assert len(lines) == 10
    # "Qbit i : teta=T , phi=P", printed with 6 significant digits.
    got = np.array([[float(ln.split("teta=")[1].split(",")[0]), float(ln.split("phi=")[1])] for ln in lines])
    n = 10
    want = oracle.measure(n, oracle.simulate(n, facade_circuit(n)))
    assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())


def test_reference_main_builds_with_bench_circuits(bench_exe):
    # The reference's main.cpp pattern: printGpuInfo, QulacsBench, QFT,
    # randomCircuit (BenchCircuits.hpp), the compile passes.
    n = 12
    r = subprocess.run([bench_exe, "plan", str(n)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"qulacs gates {41 * n}" in r.stdout
    assert f"qft gates {n * (n + 1) // 2}" in r.stdout
    assert "random gates 50" in r.stdout
    assert "CPU Info:" in r.stdout and "done" in r.stdout


@pytest.mark.gpu
def test_reference_main_simulates_with_displaytime(bench_exe, oracle):
    from kate_b200 import circuits
    n = 12
    r = subprocess.run([bench_exe, "sim", str(n)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "GPU 0 : " in r.stdout
    assert "Initialization/Measurement : " in r.stdout and "Total computing time : " in r.stdout
    got = []
    for line in r.stdout.splitlines():
        if line.startswith("Qbit "):
            t, p = line.split(":", 1)[1].split(",")
            got.append((float(t.split("=")[1]), float(p.split("=")[1])))
    ref = oracle.measure(n, oracle.simulate(n, circuits.qulacs_bench(n)))
    assert np.abs(np.array(got) - ref).max() <= 1e-5  # printed with 6 significant digits


def test_circuit_print_matches_between_cxx_and_python(bench_exe):
    # QuantumCircuit::print (QuantumCircuit.hpp:38-123) from the C++ facade
    # and the Python mirror: grouped gate list, a program with swaps and
    # permutation tables, a program without swaps.
    import kate_b200 as K
    from kate_b200 import circuits
    n = 6
    r = subprocess.run([bench_exe, "print", str(n)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    want = K.Circuit(n, circuits.qulacs_bench(n)[:3 * n]).program_text()
    assert want.startswith("gate 0 is Identifier : 2")
    c = K.Circuit(n, circuits.qulacs_bench(n))
    c.gateScheduling()
    c.gateGrouping(3)
    want += c.program_text()
    s = c.copy()
    s.allocate(1)
    swapped = s.program_text(True)
    assert "SWAP " in swapped and "Permutation table (subjective to real) : " in swapped
    want += swapped
    c.compileDefault(0)
    want += c.program_text(False)
    assert r.stdout == want
    assert want.count("EXEC Group") == 2 * len(c.groups)


def test_circuit_print_matches_the_reference_golden(bench_exe):
    # tests/golden/print_qulacs4.txt is the reference's own print output
    # (tests/golden/make_golden.py).
    golden = open(os.path.join(ROOT, "tests", "golden", "print_qulacs4.txt")).read()
    r = subprocess.run([bench_exe, "print", "4"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout == golden
