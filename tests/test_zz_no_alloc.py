"""kate_proba_state_noalloc: the reference's per-qubit measurement of a
state the caller already holds on the GPU, computed without allocating any
device memory (its scratch is a fixed __device__ array inside the library).

It exists for callers that cannot allocate once running - a serving loop
that reserved the GPU's memory for resident states, a caller inside a fixed
budget or someone else's memory pool, a language binding that cannot own
device buffers. These tests check it, through the C ABI, against the
existing measurement entry point (kate_sim_proba_state) on the same states,
on two calls in a row (the scratch keeps the previous call's contents). The
file is collected last so a failure here never hides the other tests.
"""
import ctypes

import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import _lib, circuits
from common import random_circuit

pytestmark = pytest.mark.gpu
TOL = 1e-10  # the two reductions add in different orders

_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


def noalloc(sim, final_inv=None, nqbits=None):
    ptr, phys = sim.state_device()
    n = sim.nqbits if nqbits is None else nqbits
    ph = np.array(phys + list(range(len(phys), n)), dtype=np.int32)
    fi = None if final_inv is None else np.array(final_inv, dtype=np.int32)
    out = np.zeros(2 * n, dtype=np.float64)
    st = _lib.lib().kate_proba_state_noalloc(ctypes.c_void_p(ptr), n, ph.ctypes.data_as(_ip),
                                             None if fi is None else fi.ctypes.data_as(_ip),
                                             out.ctypes.data_as(_dp), None)
    return st, out.reshape(n, 2)


@pytest.mark.parametrize("n", [9, 18, 26])
def test_noalloc_matches_existing_measurement_twice(n):
    rng = np.random.default_rng(40 + n)
    gates = circuits.layered(n, 3, seed=n) + random_circuit(n, 60, rng)
    sim = K.Simulator(K.Circuit(n, gates))
    ref = sim.execute().as_array()
    for _ in range(2):
        st, got = noalloc(sim)
        assert st == K.KATE_OK, _lib.last_error()
        assert np.abs(got - ref).max() <= TOL
        assert np.abs(sim.proba().as_array() - ref).max() <= TOL


def test_noalloc_with_final_permutation():
    n = 14
    rng = np.random.default_rng(8)
    c = K.Circuit(n, random_circuit(n, 70, rng))
    c.gateScheduling()
    c.gateGrouping(8)
    c.allocate(0)
    _, finv = c.permutations()
    sim = K.Simulator(c)
    ref = sim.execute().as_array()
    for _ in range(2):
        st, got = noalloc(sim, finv)
        assert st == K.KATE_OK, _lib.last_error()
        assert np.abs(got - ref).max() <= TOL


def test_noalloc_rejects_sizes_above_its_fixed_scratch():
    sim = K.Simulator(K.Circuit(4, [(2, [0], 0, None)]))
    sim.execute()
    st, _ = noalloc(sim, nqbits=31)
    assert st == K.KATE_EINVAL
    assert "30 qubits" in _lib.last_error()
