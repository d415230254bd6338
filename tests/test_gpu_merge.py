"""Gate merging on the GPU (kate_merge_gates_device, kate_circuit_fuse_device;
the reference's mergeGate, HIPcode/GateMerger.hpp:12-109) against the host
merger (CPUmergeGate arithmetic, CPUcode/GateMerger.hpp:8-55), which the
reference's own CPU merger pins bit for bit (tests/test_passes.py): the
device matrices must be identical, not merely close."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits
from common import random_circuit
from golden_io import merge_cases, same_gates

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [1, 2, 3, 5, 7, 10])
def test_device_merge_is_bit_identical(k):
    rng = np.random.default_rng(40 + k)
    kinds = ("h", "cnot", "crk", "toff", "d1", "d2", "d3", "diag1", "diag2", "d5")
    gates = random_circuit(k, 12 * k, rng, kinds=kinds)
    host = K.mergeGate(gates)
    dev = K.mergeGate(gates, device=0)
    assert dev.qbits == host.qbits
    assert np.array_equal(dev.densecontent, host.densecontent)


def test_device_merge_of_scattered_qubits_and_reference_golden():
    # Qubits far apart (the merged gate's local bits are their ranks), and
    # every merge the reference's own CPU merger produced for the fixtures.
    rng = np.random.default_rng(7)
    gates = [(g[0], [3 * q + 1 for q in g[1]], g[2], g[3]) for g in random_circuit(6, 60, rng)]
    host, dev = K.mergeGate(gates), K.mergeGate(gates, device=0)
    assert dev.qbits == host.qbits == [1, 4, 7, 10, 13, 16]
    assert np.array_equal(dev.densecontent, host.densecontent)
    for name, gl, qbits, mat in merge_cases():
        got = K.mergeGate(gl, device=0)
        assert got.qbits == qbits, name
        assert np.array_equal(got.densecontent, mat), name


@pytest.mark.parametrize("limit", [3, 5, 8])
def test_fusion_with_device_merges_equals_host_fusion(limit):
    n = 14
    rng = np.random.default_rng(100 + limit)
    gates = circuits.layered(n, 3, seed=limit) + random_circuit(n, 80, rng)
    a, b = K.Circuit(n, gates), K.Circuit(n, gates)
    for c in (a, b):
        c.gateScheduling()
    a.gateFusion(limit, 1e-6)
    b.gateFusion(limit, 1e-6, device=0)
    assert same_gates(a.gate_set_ordered, b.gate_set_ordered, exact=True)


def test_device_merge_on_a_stream():
    torch = pytest.importorskip("torch")
    s = torch.cuda.Stream()
    gates = circuits.qft(6)
    host = K.mergeGate(gates)
    dev = K.mergeGate(gates, device=0, stream=s.cuda_stream)
    assert np.array_equal(dev.densecontent, host.densecontent)
