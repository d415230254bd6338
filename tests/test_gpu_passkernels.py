"""Pass-specialised kernels on the GPU: they run every pass of complex128
plans, give the interpreter's amplitudes (<= 1e-12; both are checked
against the oracle elsewhere), and a run from |0...0> needs no separate
initialisation pass."""
import os

import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits
from common import random_circuit

pytestmark = pytest.mark.gpu
TOL = 1e-12


def sim_with(n, gates, jit):
    old = os.environ.get("KATE_JIT")
    os.environ["KATE_JIT"] = "1" if jit else "0"
    try:
        return K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    finally:
        if old is None:
            del os.environ["KATE_JIT"]
        else:
            os.environ["KATE_JIT"] = old


@pytest.mark.parametrize("n,seed", [(16, 1), (20, 2), (22, 3)])
def test_layered_passes_run_specialised_and_match_interpreter(n, seed, oracle):
    gates = circuits.layered(n, 6, seed=seed)
    a = sim_with(n, gates, True)
    assert all(k == 2 for k in a.pass_kernels())
    # The first pass generates |0...0>: no initialisation launch.
    assert a.launches_per_run() == len(a.pass_kernels())
    a.execute()
    b = sim_with(n, gates, False)
    assert all(k == 1 for k in b.pass_kernels())
    b.execute()
    sa, sb = a.state(), b.state()
    assert np.abs(sa - sb).max() <= TOL
    if n <= 20:
        assert np.abs(sa - oracle.simulate(n, gates)).max() <= TOL


def test_random_circuits_specialised_vs_oracle(oracle):
    rng = np.random.default_rng(77)
    for n in (12, 13, 15, 18):
        gates = random_circuit(n, 120, rng, kinds=("h", "cnot", "crk", "toff", "d1", "diag1", "diag2"))
        s = sim_with(n, gates, True)
        s.execute()
        assert np.abs(s.state() - oracle.simulate(n, gates)).max() <= TOL


def test_from_zero_first_pass_equals_product_state_start():
    # execute() starts from |0...0> inside the first pass; execute(proba_state)
    # with every theta = 0 initialises the same state in a separate kernel.
    n = 20
    gates = circuits.layered(n, 4, seed=9)
    s = sim_with(n, gates, True)
    s.execute()
    a = s.state().copy()
    s.execute(K.proba_state(np.zeros((n, 2))))
    b = s.state()
    assert np.abs(a - b).max() <= TOL


@pytest.mark.parametrize("n,kind", [(16, "layered"), (20, "qulacs"), (13, "qft"), (22, "hea")])
def test_product_state_start_matches_oracle(oracle, n, kind):
    """execute(proba_state&) on a plan whose first pass has a specialised
    kernel: that pass computes the product state itself (no initialisation
    pass); amplitudes against the oracle at 1e-12, proba_state at 1e-9, and a
    later run from |0...0> on the same simulator is unaffected."""
    gates = {"layered": lambda: circuits.layered(n, 4, seed=n), "qulacs": lambda: circuits.qulacs_bench(n),
             "qft": lambda: circuits.qft(n), "hea": lambda: circuits.hea(n, 6, seed=n)}[kind]()
    rng = np.random.default_rng(50 + n)
    tp = np.stack([rng.uniform(0, 1, n), rng.uniform(-np.pi, np.pi, n)], axis=1)
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    assert sim.pass_kernels()[0] == 2
    res = sim.execute(K.proba_state(tp))
    ref = oracle.simulate(n, gates, proba_in=tp)
    assert np.abs(sim.state() - ref).max() <= 1e-12
    assert np.abs(res.as_array() - oracle.measure(n, ref)).max() <= 1e-9
    sim.execute()
    assert np.abs(sim.state() - oracle.simulate(n, gates)).max() <= 1e-12
    sim.close()


def test_remap_search_plan_runs_specialised_and_matches_oracle(oracle):
    # The planner's remap and gate-cap search, forced at a size the oracle
    # checks quickly: fewer passes, every one pass-specialised, same state.
    n = 20
    gates = circuits.layered(n, 12, seed=7)
    old = os.environ.get("KATE_REMAP_SEARCH")
    try:
        os.environ["KATE_REMAP_SEARCH"] = "1"
        a = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
        os.environ["KATE_REMAP_SEARCH"] = "0"
        b = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    finally:
        if old is None:
            del os.environ["KATE_REMAP_SEARCH"]
        else:
            os.environ["KATE_REMAP_SEARCH"] = old
    assert len(a.pass_kernels()) < len(b.pass_kernels())
    assert all(k == 2 for k in a.pass_kernels())
    a.execute()
    ref = oracle.simulate(n, gates)
    assert np.abs(a.state() - ref).max() <= TOL


def test_pass_work_counts():
    # HBM bytes, FP64 instructions and shared-memory bytes per amplitude of
    # each pass-specialised pass: 32 B of HBM; a layered pass applies
    # rotations (FP64 > 0); shared memory moves 32 B per round trip.
    n = 22
    s = K.Simulator(K.Circuit(n, circuits.layered(n, 6, seed=3)), 1, K.C128, 0)
    work = s.pass_work()
    assert len(work) == len(s.pass_kernels())
    for w, k in zip(work, s.pass_kernels()):
        assert (w is not None) == (k == 2)
        if w is not None:
            hbm, fp64, smem = w
            assert hbm == 32.0 and fp64 >= 0.0 and smem >= 0.0 and smem % 32.0 == 0.0
    assert any(w[1] > 0 for w in work if w is not None)
