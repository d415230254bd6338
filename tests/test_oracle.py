"""The oracle (oracle/kate_oracle.c) pinned against the reference's own CPU
path: the committed golden fixtures made from it, and - where the reference
harness is built - fresh seeded circuits. The bar is bit-exactness: the C
restatement follows the reference's operation order."""
import numpy as np
import pytest

from common import random_circuit
from golden_io import merge_cases, state_cases


@pytest.mark.parametrize("case", list(state_cases()), ids=lambda c: c[0])
def test_oracle_matches_golden_states_bit_exact(oracle, case):
    name, n, gates, state, proba, pin = case
    st = oracle.simulate(n, gates, proba_in=pin)
    assert np.array_equal(st.view(np.float64), state.view(np.float64)), name
    assert np.array_equal(oracle.measure(n, st), proba), name


@pytest.mark.parametrize("case", list(merge_cases()), ids=lambda c: c[0])
def test_oracle_merge_matches_golden(oracle, case):
    name, gates, qbits, mat = case
    q, m = oracle.merge(gates)
    assert q == qbits
    assert np.array_equal(m, mat)


@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_reference_fresh(oracle, ref, seed):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(2, 12))
    gates = random_circuit(n, 60, rng)
    st, pr, _ = ref.circuit(n, gates).simulate()
    mine = oracle.simulate(n, gates)
    assert np.array_equal(mine.view(np.float64), st.view(np.float64))
    assert np.array_equal(oracle.measure(n, mine), pr)


def test_reference_thread_count_is_pinned_to_a_power_of_two(ref):
    t = ref.hw_threads()
    assert t >= 1 and (t & (t - 1)) == 0


def test_reference_drops_no_group_at_n16(oracle, ref):
    # 2^(16-14) = 4 groups: with a power-of-two thread count none is dropped
    # (the reference skips groups mod threads, CPUcode/simulator.hpp:284-287).
    n = 16
    gates = [(2, [q], 0, None) for q in range(n)]
    st, _, _ = ref.circuit(n, gates).simulate()
    assert np.allclose(np.abs(st), 2 ** (-n / 2))
    assert np.array_equal(st, oracle.simulate(n, gates))
