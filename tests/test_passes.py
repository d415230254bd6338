"""The product's host compile passes reproduce the reference's decisions:
schedules, fusion intervals (bit-identical merged matrices), groups, swap
instructions and permutations (backendagnosticcode/Circuit.hpp,
QuantumCircuit.hpp, CPUcode/GateMerger.hpp)."""
import numpy as np
import pytest

import kate_b200 as K
from common import random_circuit
from golden_io import merge_cases, pass_cases, same_gates


@pytest.mark.parametrize("case", list(pass_cases()), ids=lambda c: c["name"])
def test_passes_match_golden(case):
    c = K.Circuit(case["n"], case["gates"])
    c.gateScheduling()
    assert same_gates(c.gate_set_ordered, case["sched"])
    c.gateFusion(case["k"], case["mtm"])
    assert same_gates(c.gate_set_ordered, case["fused"])
    c.gateGrouping(case["m"])
    assert [list(g) for g in c.groups] == [list(g) for g in case["groups"]]
    if case["alloc"]:
        c.allocate(0)
    else:
        c.compileDefault(0)
    assert same_gates(c.gate_set_ordered, case["compiled"])
    assert [list(i) for i in c.instructions] == [list(i) for i in case["instructions"]]
    a, b = c.permutations()
    assert [list(a), list(b)] == case["perms"]


@pytest.mark.parametrize("case", list(merge_cases()), ids=lambda c: c[0])
def test_merge_matches_golden(case):
    name, gates, qbits, mat = case
    g = K.mergeGate(gates)
    assert g.qbits == qbits
    assert np.array_equal(g.densecontent, mat)


@pytest.mark.parametrize("seed", range(10))
def test_passes_match_reference_fresh(ref, seed):
    rng = np.random.default_rng(500 + seed)
    n = int(rng.integers(3, 12))
    gates = random_circuit(n, int(rng.integers(1, 80)), rng)
    a, b = K.Circuit(n, gates), ref.circuit(n, gates)
    a.gateScheduling(); b.schedule()
    assert same_gates(a.gate_set_ordered, b.gates())
    k, mtm = int(rng.integers(2, 6)), [0.0, 1e-6, 1.0][seed % 3]
    a.gateFusion(k, mtm); b.fuse(k, mtm)
    assert same_gates(a.gate_set_ordered, b.gates())
    m = int(rng.integers(5, 10))
    a.gateGrouping(m); b.group(m)
    assert a.groups == b.groups()
    a.allocate(0); b.allocate(0)
    assert same_gates(a.gate_set_ordered, b.gates())
    assert a.instructions == b.instructions()
    assert a.permutations() == b.perms()


def test_compile_opt_equals_the_four_passes(ref):
    rng = np.random.default_rng(3)
    n = 9
    gates = random_circuit(n, 50, rng)
    a = K.Circuit(n, gates)
    a.compileOPT(4, 1e-6, 7, 0, 300)
    b = ref.circuit(n, gates)
    b.schedule(); b.fuse(4, 1e-6); b.group(7); b.allocate(0, 300)
    assert same_gates(a.gate_set_ordered, b.gates())
    assert a.groups == b.groups()


def test_layered_fusion_counts_match_reference(ref):
    from kate_b200 import circuits
    n = 20
    gates = circuits.layered(n, 10, seed=1234)
    a = K.Circuit(n, gates)
    a.gateScheduling(); a.gateFusion(5, 1e-6); a.gateGrouping(12)
    b = ref.circuit(n, gates)
    b.schedule(); b.fuse(5, 1e-6); b.group(12)
    assert same_gates(a.gate_set_ordered, b.gates())
    assert a.groups == b.groups()


def test_schedule_reproduces_size_t_weight(ref):
    # Two ready gates, one adding new qubits and one not: the reference's
    # size_t score makes the new-qubit gate win (Circuit.hpp:69-75).
    gates = [(2, [0], 0, None), (3, [0, 1], 0, None), (2, [2], 0, None), (2, [0], 0, None)]
    a, b = K.Circuit(3, gates), ref.circuit(3, gates)
    a.gateScheduling(); b.schedule()
    assert same_gates(a.gate_set_ordered, b.gates())
