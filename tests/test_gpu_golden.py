"""The CUDA path against the reference's own outputs, with no oracle in
between: the committed golden fixtures (tests/golden/states.npz, made by
the reference's CPU simulator through tests/golden/make_golden.py) hold
each case's final state and proba_state. Bar: 1e-12 max-abs amplitude
error, 1e-9 on (theta, phi); complex64 to 2e-5 on the state."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits
from golden_io import state_cases

pytestmark = pytest.mark.gpu


def _angle_diff(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    d[:, 1] = np.minimum(d[:, 1], 2 * np.pi - d[:, 1])
    return d.max()


@pytest.mark.parametrize("case", list(state_cases()), ids=lambda c: c[0])
def test_golden_state_complex128(case):
    name, n, gates, state, proba, pin = case
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    res = sim.execute(K.proba_state(pin)) if pin is not None else sim.execute()
    assert np.abs(sim.state() - state).max() <= 1e-12, name
    assert _angle_diff(res.as_array(), proba) <= 1e-9, name
    sim.close()


@pytest.mark.parametrize("case", list(state_cases()), ids=lambda c: c[0])
def test_golden_state_complex64(case):
    name, n, gates, state, proba, pin = case
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C64, 0)
    if pin is not None:
        sim.execute(K.proba_state(pin))
    else:
        sim.execute()
    assert np.abs(sim.state() - state).max() <= 2e-5, name
    sim.close()


@pytest.mark.parametrize("n", [1, 5, 12, 13, 20])
def test_empty_circuit_is_the_zero_state(oracle, n):
    sim = K.Simulator(K.Circuit(n), 1, K.C128, 0)
    res = sim.execute()
    st = sim.state()
    want = np.zeros(1 << n, dtype=np.complex128)
    want[0] = 1
    assert np.array_equal(st, want)
    assert np.abs(res.as_array() - oracle.measure(n, want)).max() <= 1e-12
    sim.close()


def test_qft_n16_matches_oracle(oracle):
    # Controlled phases of every order CRk(k = 2..16): the diagonal path.
    n = 16
    gates = [(2, [q], 0, None) for q in range(0, n, 3)] + circuits.qft(n)
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    res = sim.execute()
    ref = oracle.simulate(n, gates)
    assert np.abs(sim.state() - ref).max() <= 1e-12
    assert np.abs(res.as_array() - oracle.measure(n, ref)).max() <= 1e-9
    sim.close()
