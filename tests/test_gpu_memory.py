"""Device buffers kept for reuse: a destroyed simulator's state (>= 64 MiB)
is handed to the next simulator or batch it covers, and results do not
depend on it (every run initialises the state it uses)."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits

pytestmark = pytest.mark.gpu


def run(n, gates, prec=K.C128):
    sim = K.Simulator(K.Circuit(n, gates), 1, prec, 0)
    sim.execute()
    st = sim.state()
    sim.close()
    return st


def test_reused_state_gives_identical_results():
    n = 24  # 256 MiB complex128: kept for reuse
    g = circuits.layered(n, 3, seed=21)
    a = run(n, g)
    b = run(n, circuits.layered(n, 2, seed=22))  # reuses a's buffer, leaves other contents in it
    c = run(n, g)                                # reuses it again
    assert np.array_equal(a, c)
    assert not np.array_equal(a, b)
    K.release_cached_memory(0)
    d = run(n, g)                                # fresh allocation
    assert np.array_equal(a, d)
    K.release_cached_memory()


def test_batch_after_simulator_reuse(oracle):
    run(24, circuits.layered(24, 1, seed=3))  # leaves a 256 MiB buffer for reuse
    # complex64 arena of 128 + 32 MiB (+ a small state): covered by that buffer
    specs = [(24, circuits.hea(24, 1, seed=1)), (22, circuits.hea(22, 1, seed=2)), (14, circuits.hea(14, 8, seed=3))]
    b = K.Batch([K.Circuit(n, g) for n, g in specs], precision=K.C64)
    b.run()
    for (n, g), z in zip(specs, b.expect_z()):
        st = oracle.simulate(n, g)
        p = np.abs(st) ** 2
        idx = np.arange(1 << n)
        ref = np.array([p[((idx >> q) & 1) == 0].sum() - p[((idx >> q) & 1) == 1].sum() for q in range(n)])
        assert np.abs(z - ref).max() <= 2e-5
    b.close()
    K.release_cached_memory()
