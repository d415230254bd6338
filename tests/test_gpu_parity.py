"""Parity of the CUDA path with the oracle (Kate's CPU double-precision
arithmetic), through the C ABI. Bar: max-abs amplitude error <= 1e-12."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits
from common import random_circuit

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run(n, gates, **kw):
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    res = sim.execute(**kw) if kw else sim.execute()
    return sim, res


def test_layered_n20_10_layers_matches_oracle(oracle):
    n = 20
    gates = circuits.layered(n, 10, seed=1234)
    assert len(gates) == 590
    sim, res = run(n, gates)
    ref = oracle.simulate(n, gates)
    assert np.abs(sim.state() - ref).max() <= TOL
    assert np.abs(res.as_array() - oracle.measure(n, ref)).max() <= 1e-9


def test_qulacs_bench_n20_matches_oracle(oracle):
    # The reference's own benchmark circuit (BenchCircuits.hpp:8-42).
    n = 20
    gates = circuits.qulacs_bench(n)
    sim, res = run(n, gates)
    ref = oracle.simulate(n, gates)
    assert np.abs(sim.state() - ref).max() <= TOL
    assert np.abs(res.as_array() - oracle.measure(n, ref)).max() <= 1e-9


def test_execute_displaytime_times_the_phases(oracle, capsys):
    # execute(true) prints the reference's three timing lines
    # (HIPcode/simulator.hpp:346-350) and returns the same proba_state.
    n = 16
    gates = circuits.qulacs_bench(n)
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    res = sim.execute(True)
    out = capsys.readouterr().out
    assert "Initialization/Measurement : " in out and "Total computing time : " in out
    init_ms, passes_ms, meas_ms, npass = sim.last_times
    assert npass == len(sim.passes()) and passes_ms > 0 and init_ms >= 0 and meas_ms > 0
    assert np.abs(res.as_array() - oracle.measure(n, oracle.simulate(n, gates))).max() <= 1e-9
    names = [d[0] for d in K.devices()]
    assert names and "B200" in names[0]


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 9, 12, 13, 16])
def test_random_circuits_all_gate_kinds(oracle, n):
    rng = np.random.default_rng(100 + n)
    gates = random_circuit(n, 120, rng)
    sim, _ = run(n, gates)
    assert np.abs(sim.state() - oracle.simulate(n, gates)).max() <= TOL


def test_many_passes_with_remap_n22(oracle):
    n = 22
    rng = np.random.default_rng(7)
    gates = circuits.layered(n, 3, seed=9) + random_circuit(n, 150, rng)
    sim, _ = run(n, gates)
    assert len(sim.passes()) > 3
    assert np.abs(sim.state() - oracle.simulate(n, gates)).max() <= TOL


def test_execute_from_product_state(oracle):
    n = 14
    rng = np.random.default_rng(3)
    gates = random_circuit(n, 60, rng)
    tp = np.stack([rng.uniform(0, 1, n), rng.uniform(-np.pi, np.pi, n)], axis=1)
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    res = sim.execute(K.proba_state(tp))
    ref = oracle.simulate(n, gates, proba_in=tp)
    assert np.abs(sim.state() - ref).max() <= TOL
    assert np.abs(res.as_array() - oracle.measure(n, ref)).max() <= 1e-9


def test_compiled_with_allocate_matches_reference(ref):
    n = 12
    rng = np.random.default_rng(11)
    gates = random_circuit(n, 80, rng)
    c = K.Circuit(n, gates)
    c.gateScheduling()
    c.gateFusion(4, 1e-6)
    c.gateGrouping(8)
    c.allocate(0)
    rc = ref.circuit(n, gates)
    rc.schedule(); rc.fuse(4, 1e-6); rc.group(8); rc.allocate(0)
    rst, rpr, _ = rc.simulate()
    sim = K.Simulator(c, 1, K.C128, 0)
    pr = sim.execute()
    assert np.abs(sim.state() - rst).max() <= TOL
    assert np.abs(pr.as_array() - rpr).max() <= 1e-9


def test_expect_z_and_probabilities(oracle):
    n = 13
    rng = np.random.default_rng(5)
    gates = random_circuit(n, 50, rng)
    sim, _ = run(n, gates)
    st = oracle.simulate(n, gates)
    p = np.abs(st) ** 2
    z = np.array([p[((np.arange(1 << n) >> q) & 1) == 0].sum() - p[((np.arange(1 << n) >> q) & 1) == 1].sum()
                  for q in range(n)])
    assert np.abs(sim.expect_z() - z).max() <= 1e-12
    assert np.abs(sim.probabilities() - p).max() <= 1e-12


def test_factored_rotations_at_edge_angles_complex128_and_complex64(oracle):
    """RX / RY at angles where a rotation's factor vanishes or dominates run as
    factored register ops on the GPU: the complex128 simulator within 1e-12
    of the oracle's amplitudes, a complex64 batch (register stages in packed
    FP32) within 2e-5 on <Z>."""
    n = 14
    angles = [0.0, np.pi / 2, np.pi, 1.5 * np.pi, 2 * np.pi, 1e-9, np.pi - 1e-9]
    rng = np.random.default_rng(78)
    angles += list(rng.uniform(0, 2 * np.pi, 20))
    g = []
    for i, th in enumerate(angles):
        q = i % n
        g.append((0, [q], 0, circuits.rx(th)))
        g.append((0, [(q + 5) % n], 0, circuits.ry(th)))
        g.append((3, [q, (q + 1) % n], 0, None))
    ref = oracle.simulate(n, g)
    s128, _ = run(n, g)
    assert np.abs(s128.state() - ref).max() <= TOL
    b = K.Batch([K.Circuit(n, g)], precision=K.C64)
    b.run()
    p = np.abs(ref) ** 2
    idx = np.arange(1 << n)
    zref = np.array([p[((idx >> q) & 1) == 0].sum() - p[((idx >> q) & 1) == 1].sum() for q in range(n)])
    assert np.abs(b.expect_z()[0] - zref).max() <= 2e-5
    b.close()
