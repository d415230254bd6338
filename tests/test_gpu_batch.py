"""Batch engine (one persistent launch for many circuits): <Z_q> of every
circuit of a mixed batch against the oracle's state, through the C ABI.
Bars: complex128 1e-12; complex64 (FP32 arithmetic) 2e-5."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import _lib, circuits
from common import random_circuit

pytestmark = pytest.mark.gpu


def zexp(n, st):
    p = np.abs(st) ** 2
    idx = np.arange(1 << n)
    return np.array([p[((idx >> q) & 1) == 0].sum() - p[((idx >> q) & 1) == 1].sum() for q in range(n)])


def mixed(seed):
    rng = np.random.default_rng(seed)
    specs = []
    for n in [1, 2, 3, 5, 8, 11, 12, 13, 14, 16, 18]:
        specs.append((n, random_circuit(n, 60, rng)))
    for n in [10, 12, 13, 17]:
        specs.append((n, circuits.hea(n, 2 * n, seed=n)))
    specs.append((5, []))
    specs.append((14, []))
    return specs


@pytest.mark.parametrize("prec,tol", [(K.C128, 1e-12), (K.C64, 2e-5)])
def test_mixed_batch_matches_oracle(oracle, prec, tol):
    specs = mixed(1)
    b = K.Batch([K.Circuit(n, g) for n, g in specs], precision=prec)
    b.run()
    got = b.expect_z()
    for (n, g), z in zip(specs, got):
        ref = zexp(n, oracle.simulate(n, g))
        assert np.abs(z - ref).max() <= tol, (n, len(g), np.abs(z - ref).max())


def test_runs_repeat_and_options_do_not_change_results(oracle):
    specs = mixed(2)
    circs = [K.Circuit(n, g) for n, g in specs]
    b = K.Batch(circs, precision=K.C128)
    b.run()
    z1 = b.expect_z_flat().copy()
    b.run()
    b.run()
    assert np.abs(b.expect_z_flat() - z1).max() <= 1e-13
    o = _lib.BatchOptions()
    K._lib.lib().kate_batch_options_default(ctypes_ref(o))
    o.chunk = 1
    o.zchunks = 1
    o.window_bytes = 1 << 20  # one large state per window
    for n in range(K._lib.KATE_BATCH_MAX_QUBITS + 1):
        o.tune[n].fusion = 3
        o.tune[n].max_gates = 40
    b2 = K.Batch(circs, precision=K.C128, options=o)
    b2.run()
    assert b2.info()["tasks"] > b.info()["tasks"]
    assert np.abs(b2.expect_z_flat() - z1).max() <= 1e-12


def ctypes_ref(x):
    import ctypes
    return ctypes.byref(x)


def test_compiled_circuits_match_simulator():
    rng = np.random.default_rng(9)
    circs = []
    for n in (9, 14):
        c = K.Circuit(n, random_circuit(n, 80, rng))
        c.gateScheduling()
        c.gateFusion(3, 1e-6)
        c.gateGrouping(6)
        c.allocate(0)
        circs.append(c)
    b = K.Batch(circs, precision=K.C128)
    b.run()
    for c, z in zip(circs, b.expect_z()):
        sim = K.Simulator(c, 1, K.C128, 0)
        sim.execute()
        assert np.abs(sim.expect_z() - z).max() <= 1e-12


@pytest.mark.parametrize("m,c", [(10, 3), (11, 5), (12, 4), (10, 5), (12, 3)])
def test_every_grouping_and_coalesce_choice_matches_oracle(oracle, m, c):
    """The autotuner's search space beyond fusion width and gates per pass:
    the grouping size m (qubits one pass's gates span; the 12-qubit tile is
    filled up) and the coalesce width c (low physical bits every tile keeps).
    Each choice gives the oracle's <Z> (complex128, 1e-12)."""
    specs = mixed(3)
    o = _lib.BatchOptions()
    K._lib.lib().kate_batch_options_default(ctypes_ref(o))
    for n in range(K._lib.KATE_BATCH_MAX_QUBITS + 1):
        o.tune[n].fusion = 2
        o.tune[n].max_gates = 96
        o.tune[n].group_qubits = m
        o.tune[n].coalesce = c
    b = K.Batch([K.Circuit(n, g) for n, g in specs], precision=K.C128, options=o)
    b.run()
    for (n, g), z in zip(specs, b.expect_z()):
        assert np.abs(z - zexp(n, oracle.simulate(n, g))).max() <= 1e-12, (n, m, c)


def test_autotune_then_run(oracle):
    specs = [(n, circuits.hea(n, 2 * n, seed=100 + i)) for i, n in enumerate([10, 11, 13, 13, 15])]
    b = K.Batch([K.Circuit(n, g) for n, g in specs], precision=K.C64, autotune=True)
    for n in (10, 11, 13, 15):
        t = b.options.tune[n]
        assert t.fusion >= 1 and t.max_gates >= 1
        assert 10 <= t.group_qubits <= 12 and 3 <= t.coalesce <= 5
    b.run()
    for (n, g), z in zip(specs, b.expect_z()):
        assert np.abs(z - zexp(n, oracle.simulate(n, g))).max() <= 2e-5


def test_hea_batch_of_many_circuits(oracle):
    rng = np.random.default_rng(4)
    ns = [int(x) for x in rng.integers(10, 17, 300)]
    specs = [(n, circuits.hea(n, 2 * n, seed=1000 + i)) for i, n in enumerate(ns)]
    b = K.Batch([K.Circuit(n, g) for n, g in specs], precision=K.C64)
    b.run()
    got = b.expect_z()
    for i in range(0, len(specs), 37):
        n, g = specs[i]
        assert np.abs(got[i] - zexp(n, oracle.simulate(n, g))).max() <= 2e-5


def test_dependency_wait_runs_out_and_reports(oracle):
    """A task made (on the host) to wait for a count its circuit never
    reaches: the kernel's bounded wait gives up after wait_ms, every CTA stops
    at its next task, the run reports the timeout, and the device stays
    usable for the next batch."""
    specs = [(14, circuits.hea(14, 8, seed=3)), (16, circuits.hea(16, 8, seed=4)), (10, circuits.hea(10, 4, seed=5))]
    circs = [K.Circuit(n, g) for n, g in specs]
    o = _lib.BatchOptions()
    K._lib.lib().kate_batch_options_default(ctypes_ref(o))
    o.wait_ms = 200
    b = K.Batch(circs, precision=K.C64, options=o)
    ntasks = b.info()["tasks"]
    b.close()
    o.fault_task = ntasks  # 1-based: the last task, a <Z> reduction that waits on the passes
    bad = K.Batch(circs, precision=K.C64, options=o)
    with pytest.raises(K.KateError, match="timed out") as err:
        bad.run()
    assert err.value.status == K.KATE_ETIMEDOUT
    bad.close()
    o.fault_task = 0
    good = K.Batch(circs, precision=K.C64, options=o)
    good.run()
    for (n, g), z in zip(specs, good.expect_z()):
        assert np.abs(z - zexp(n, oracle.simulate(n, g))).max() <= 2e-5
    good.close()


def test_batch_state_readback_matches_complex128():
    """kate_batch_get_state returns a resident circuit's final state in its
    labels: the complex64 batch arithmetic within 1e-6 infidelity of the
    complex128 simulator; circuits run in shared memory have no state."""
    circs = [K.Circuit(n, circuits.hea(n, n, seed=n)) for n in (10, 14, 17)]
    b = K.Batch(circs, precision=K.C64)
    b.run()
    progs, res = b.circuit_info()
    assert res[0] == 0 and res[1] == 14 and res[2] == 17
    with pytest.raises(K.KateError):
        b.state(0)
    for i in (1, 2):
        psi64 = b.state(i)
        s = K.Simulator(circs[i], 1, K.C128, 0)
        s.execute()
        psi128 = s.state()
        s.close()
        assert 1.0 - abs(np.vdot(psi128, psi64)) ** 2 <= 1e-6
    b.close()


def _block_options(nmin=13, blocks=1):
    o = _lib.BatchOptions()
    K._lib.lib().kate_batch_options_default(ctypes_ref(o))
    for n in range(nmin, K._lib.KATE_BATCH_MAX_QUBITS + 1):
        o.tune[n].blocks = blocks
    return o


def test_tensor_core_block_passes_match_oracle(oracle):
    """Complex64 circuits kept in device memory with tensor-core block
    passes (the batch kernel's block tasks: split-BF16 products, FP32
    accumulation), mixed in one launch with register-staged and
    shared-memory circuits: <Z> of every circuit against the oracle
    (2e-5), and the block passes' states within 1e-6 infidelity of
    complex128."""
    specs = mixed(5) + [(15, circuits.brickwork_su4(15, 6, seed=9)), (13, [])]
    circs = [K.Circuit(n, g) for n, g in specs]
    b = K.Batch(circs, precision=K.C64, options=_block_options())
    nres = sum(1 for n, g in specs if n >= 13 and len(g) > 0)
    assert b.info()["block_programs"] >= nres  # every resident circuit with gates plans to block passes
    b.run()
    got = b.expect_z()
    for (n, g), z in zip(specs, got):
        assert np.abs(z - zexp(n, oracle.simulate(n, g))).max() <= 2e-5, (n, len(g))
    b.run()  # a second run of the same graph gives the same outputs
    for z1, z2 in zip(got, b.expect_z()):
        assert np.abs(z1 - z2).max() <= 1e-12
    _, res = b.circuit_info()
    for i, (n, g) in enumerate(specs):
        if res[i] >= 13 and len(g) > 0:
            psi = b.state(i)
            ref = oracle.simulate(n, g)
            assert 1.0 - abs(np.vdot(ref, psi)) ** 2 / np.vdot(psi, psi).real <= 1e-6, n
    b.close()


def test_block_and_register_batches_agree():
    """The same HEA circuits with and without tensor-core block passes: the
    two complex64 forms agree on <Z> to 2e-5."""
    rng = np.random.default_rng(11)
    ns = [int(x) for x in rng.integers(13, 19, 24)]
    circs = [K.Circuit(n, circuits.hea(n, 2 * n, seed=50 + i)) for i, n in enumerate(ns)]
    a = K.Batch(circs, precision=K.C64, options=_block_options(blocks=0))
    a.run()
    b = K.Batch(circs, precision=K.C64, options=_block_options(blocks=1))
    assert a.info()["block_programs"] == 0 and b.info()["block_programs"] == b.info()["programs"]
    b.run()
    assert np.abs(a.expect_z_flat() - b.expect_z_flat()).max() <= 2e-5
    a.close()
    b.close()
