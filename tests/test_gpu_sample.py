"""Sampling on the device (kate_sim_sample): the probabilities never leave
the GPU. Shot k draws u_k = (splitmix64 output k of the seed >> 11) * 2^-53
and takes the first basis index whose cumulative probability exceeds u_k
times the total, so the samples can be recomputed exactly on the host from
the oracle's state (numpy cumsum + searchsorted); a histogram follows the
probabilities; and states beyond the host-copy range (32 qubits) sample
with only the shots crossing PCIe."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits
from common import random_circuit

pytestmark = pytest.mark.gpu


def uniforms(seed, shots):
    g = circuits.SplitMix64(seed)
    return np.array([(g.next() >> 11) * (1.0 / (1 << 53)) for _ in range(shots)])


def expected_samples(p, seed, shots):
    cdf = np.cumsum(p)
    y = uniforms(seed, shots) * cdf[-1]
    return np.minimum(np.searchsorted(cdf, y, side="right"), p.size - 1)


@pytest.mark.parametrize("n,prec", [(10, K.C128), (17, K.C128), (18, K.C64)])
def test_samples_equal_the_host_recomputation(n, prec, oracle):
    rng = np.random.default_rng(n)
    gates = random_circuit(n, 60, rng, kinds=("h", "cnot", "crk", "d1", "d2", "diag1"))
    sim = K.Simulator(K.Circuit(n, gates), 1, prec, 0)
    sim.execute()
    st = sim.state()
    p = st.real ** 2 + st.imag ** 2  # the simulator's own probabilities (label order), as the device forms them
    for seed in (1, 99):
        got = sim.sample(4096, seed=seed).astype(np.int64)
        assert np.array_equal(got, expected_samples(p, seed, 4096))
    if prec == K.C128:
        assert np.abs(p - np.abs(oracle.simulate(n, gates)) ** 2).max() <= 1e-12


def test_sample_histogram_follows_probabilities(oracle):
    n = 6
    rng = np.random.default_rng(2)
    gates = random_circuit(n, 30, rng)
    sim = K.Simulator(K.Circuit(n, gates))
    sim.execute()
    p = np.abs(oracle.simulate(n, gates)) ** 2
    s = sim.sample(200000, seed=42)
    hist = np.bincount(s.astype(np.int64), minlength=1 << n) / len(s)
    assert np.abs(hist - p).max() < 0.01
    assert np.array_equal(s[:100], sim.sample(100, seed=42))
    # Zero-probability states are never drawn.
    assert np.all(p[np.unique(s.astype(np.int64))] > 0)


def test_sampling_32_qubits_complex64():
    # RX(theta_q) on every qubit: a product state with P(bit q = 1) =
    # sin^2(theta_q / 2); 4096 shots from a 32 GiB state.
    n = 32
    th = np.linspace(0.3, 2.8, n)
    gates = [(0, [q], 0, circuits.rx(t)) for q, t in enumerate(th)]
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C64, 0)
    sim.execute()
    s = sim.sample(4096, seed=7).astype(np.uint64)
    freq = np.array([((s >> np.uint64(q)) & np.uint64(1)).mean() for q in range(n)])
    want = np.sin(th / 2) ** 2
    sigma = np.sqrt(want * (1 - want) / 4096)
    assert np.all(np.abs(freq - want) <= 6 * sigma + 1e-3), np.abs(freq - want).max()
    sim.close()
