"""Complex64 path: 5-qubit dense blocks on the tensor cores (split-BF16
products, FP32 accumulation) and the complex64 generic kernel, against the
oracle's FP64 states. Bar: infidelity 1 - |<psi64|psi128>|^2 <= 1e-6 per
circuit; amplitudes and <Z> within 1e-4 (about 16 bits kept per operand)."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits
from common import random_circuit

pytestmark = pytest.mark.gpu


def infidelity(a, b):
    a = a / np.linalg.norm(a)
    b = b / np.linalg.norm(b)
    return 1.0 - abs(np.vdot(a, b)) ** 2


@pytest.mark.parametrize("n", [3, 8, 11, 12, 13, 15])
def test_c64_random_circuits(oracle, n):
    rng = np.random.default_rng(900 + n)
    kinds = ("h", "cnot", "crk", "toff", "d1", "d2", "d3", "diag1", "diag2", "d5")
    gates = random_circuit(n, 80, rng, kinds=kinds)
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C64)
    sim.execute()
    ref = oracle.simulate(n, gates)
    got = sim.state()
    assert infidelity(got, ref) <= 1e-6
    assert np.abs(got - ref).max() <= 1e-4


@pytest.mark.parametrize("fuse", [False, True])
def test_c64_brickwork_su4_fused_blocks(oracle, fuse):
    n = 16
    gates = circuits.brickwork_su4(n, 8, seed=3)
    c = K.Circuit(n, gates)
    if fuse:
        c.gateScheduling()
        c.gateFusion(5, 1e-6)
    sim = K.Simulator(c, 1, K.C64)
    assert all(k == 3 for k in sim.pass_kernels())  # every pass on the tensor cores
    sim.execute()
    assert infidelity(sim.state(), oracle.simulate(n, gates)) <= 1e-6


def test_c64_layered_and_measurements(oracle):
    n = 14
    gates = circuits.layered(n, 4, seed=5)
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C64)
    res = sim.execute()
    ref = oracle.simulate(n, gates)
    assert infidelity(sim.state(), ref) <= 1e-6
    assert np.abs(res.as_array() - oracle.measure(n, ref)).max() <= 1e-4
    p = np.abs(ref) ** 2
    z = np.array([p[((np.arange(1 << n) >> q) & 1) == 0].sum() - p[((np.arange(1 << n) >> q) & 1) == 1].sum()
                  for q in range(n)])
    assert np.abs(sim.expect_z() - z).max() <= 1e-4
