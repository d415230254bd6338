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

TOL = 1e-10  # the two reductions add in different orders

_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


def call(ptr, nbytes, n, phys=None, final_inv=None):
    ph = None if phys is None else np.array(phys, dtype=np.int32)
    fi = None if final_inv is None else np.array(final_inv, dtype=np.int32)
    out = np.zeros(2 * n, dtype=np.float64)
    st = _lib.lib().kate_proba_state_noalloc(ctypes.c_void_p(ptr), nbytes, n,
                                             None if ph is None else ph.ctypes.data_as(_ip),
                                             None if fi is None else fi.ctypes.data_as(_ip),
                                             out.ctypes.data_as(_dp), None)
    return st, out.reshape(n, 2)


def noalloc(sim, final_inv=None, nqbits=None, nbytes=None):
    ptr, phys = sim.state_device()
    n = sim.nqbits if nqbits is None else nqbits
    ph = phys + list(range(len(phys), n))
    return call(ptr, (16 << n) if nbytes is None else nbytes, n, ph, final_inv)


# ---- host-side argument checks (no GPU needed: refused before any CUDA call) ----

def test_noalloc_refuses_a_buffer_smaller_than_a_complex128_state():
    st, _ = call(4096, 8 << 10, 10)  # a complex64-sized buffer
    assert st == K.KATE_EINVAL
    assert "complex128" in _lib.last_error()


def test_noalloc_refuses_misaligned_pointers_and_bad_permutations():
    st, _ = call(4096 + 8, 16 << 10, 10)
    assert st == K.KATE_EINVAL and "aligned" in _lib.last_error()
    st, _ = call(4096, 16 << 4, 4, phys=[0, 1, 1, 3])
    assert st == K.KATE_EINVAL and "phys_of_label" in _lib.last_error()
    st, _ = call(4096, 16 << 4, 4, final_inv=[0, 1, 2, 4])
    assert st == K.KATE_EINVAL and "final_inverse_permutation" in _lib.last_error()
    st, _ = call(4096, 16 << 4, 4, final_inv=[3, 3, 2, 1])
    assert st == K.KATE_EINVAL and "final_inverse_permutation" in _lib.last_error()


# ---- on the GPU, against kate_sim_proba_state ----

@pytest.mark.gpu
@pytest.mark.parametrize("n", [9, 12, 13, 18, 26, 30])
def test_noalloc_matches_existing_measurement_twice(n):
    # n = 12 / 13: the reduction's grid switches from one CTA to two; n = 30:
    # the scratch is used up to its fixed size.
    rng = np.random.default_rng(40 + n)
    gates = circuits.layered(n, 3, seed=n) + random_circuit(n, 60 if n <= 26 else 20, rng)
    sim = K.Simulator(K.Circuit(n, gates))
    ref = sim.execute().as_array()
    for _ in range(2):
        st, got = noalloc(sim)
        assert st == K.KATE_OK, _lib.last_error()
        assert np.abs(got - ref).max() <= TOL
        assert np.abs(sim.proba().as_array() - ref).max() <= TOL


@pytest.mark.gpu
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


@pytest.mark.gpu
def test_noalloc_rejects_sizes_above_its_fixed_scratch():
    sim = K.Simulator(K.Circuit(4, [(2, [0], 0, None)]))
    sim.execute()
    st, _ = noalloc(sim, nqbits=31)
    assert st == K.KATE_EINVAL
    assert "30 qubits" in _lib.last_error()


@pytest.mark.gpu
def test_noalloc_refuses_host_memory_and_complex64_states():
    host = np.zeros(1 << 10, dtype=np.complex128)
    st, _ = call(host.ctypes.data, host.nbytes, 10)
    assert st == K.KATE_EINVAL and "device memory" in _lib.last_error()
    # A complex64 state (8 bytes per amplitude, its own allocation of that
    # size) claimed as complex128: the state would not fit its allocation.
    K.release_cached_memory(0)
    n = 20
    s64 = K.Simulator(K.Circuit(n, circuits.layered(n, 1, seed=3)), 1, K.C64, 0)
    s64.execute()
    ptr, phys = s64.state_device()
    st, _ = call(ptr, 16 << n, n, phys)
    assert st == K.KATE_EINVAL and "does not fit" in _lib.last_error()
    st, _ = call(ptr, 8 << n, n, phys)
    assert st == K.KATE_EINVAL and "complex128" in _lib.last_error()
