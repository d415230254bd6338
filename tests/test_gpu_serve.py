"""Serving engine: requests through kate_server_* against the oracle, the
same request alone and inside a mix, and admission under a small budget."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits

pytestmark = pytest.mark.gpu


def zexp(n, st):
    p = np.abs(st) ** 2
    idx = np.arange(1 << n)
    return np.array([p[((idx >> q) & 1) == 0].sum() - p[((idx >> q) & 1) == 1].sum() for q in range(n)])


def layered(n, seed):
    return circuits.layered(n, n, seed=seed)


@pytest.mark.parametrize("prec,tol,blocks", [(K.C128, 1e-12, 0), (K.C64, 2e-5, 0), (K.C64, 2e-5, 1)])
def test_requests_match_oracle(oracle, prec, tol, blocks):
    # blocks=1: complex64 requests run their passes as tensor-core blocks.
    srv = K.Server(prec, budget_bytes=1 << 30, aux_bytes=256 << 20, tensor_blocks=blocks)
    specs = [(n, layered(n, 10 + n)) for n in (12, 13, 14, 16, 17)]
    ids = [srv.submit(K.Circuit(n, g), shots=4096, seed=7 + n) for n, g in specs]
    for (n, g), rid in zip(specs, ids):
        z, s, t = srv.wait(rid, timeout=120)
        st = oracle.simulate(n, g)
        assert np.abs(z - zexp(n, st)).max() <= tol
        assert t[0] <= t[1] <= t[2]
        # Samples follow |amplitude|^2: per-qubit sample means of Z agree
        # with <Z> within 5 standard errors.
        assert s.shape == (4096,) and int(s.max()) < (1 << n)
        bits = (s[:, None] >> np.arange(n)[None, :].astype(np.uint64)) & np.uint64(1)
        zs = 1.0 - 2.0 * bits.astype(np.float64).mean(axis=0)
        assert np.all(np.abs(zs - z) <= 5.0 / np.sqrt(4096) + 1e-9)
        # Heavy outputs: the most likely basis state is sampled about as often as expected.
        p = np.abs(st) ** 2
        top = int(np.argmax(p))
        assert abs((s == top).mean() - p[top]) <= 5 * np.sqrt(p[top] / 4096) + 1e-3
    srv.close()


def test_same_result_alone_and_in_a_mix():
    n = 15
    x = K.Circuit(n, layered(n, 99))
    a = K.Server(K.C64, budget_bytes=1 << 30, aux_bytes=256 << 20)
    za, sa, _ = a.wait(a.submit(x, shots=1024, seed=1234))
    a.close()
    b = K.Server(K.C64, budget_bytes=1 << 30, aux_bytes=256 << 20, step_tiles=64)
    rng = np.random.default_rng(3)
    ids = []
    for i in range(12):
        m = int(rng.integers(12, 19))
        ids.append(b.submit(K.Circuit(m, layered(m, i)), shots=1024, seed=i))
        if i == 5:
            mine = b.submit(x, shots=1024, seed=1234)
    zb, sb, _ = b.wait(mine)
    for r in ids:
        b.wait(r)
    b.close()
    assert np.array_equal(sa, sb)
    assert np.abs(za - zb).max() <= 1e-12


def test_admission_respects_the_budget(oracle):
    # 32 MiB budget, 8 MiB complex64 states at n = 20: at most four resident.
    srv = K.Server(K.C64, budget_bytes=32 << 20, aux_bytes=128 << 20)
    gates = layered(20, 5)
    ids = [srv.submit(K.Circuit(20, gates), shots=256, seed=i) for i in range(10)]
    res = [srv.wait(r, timeout=300) for r in ids]
    st = srv.stats()
    assert st["completed"] == 10 and st["failed"] == 0
    assert st["peak_resident_bytes"] <= 32 << 20
    z0 = zexp(20, oracle.simulate(20, gates))
    for z, s, _ in res:
        assert np.abs(z - z0).max() <= 2e-5
    # Same circuit and seed: same samples.
    srv2 = K.Server(K.C64, budget_bytes=32 << 20, aux_bytes=128 << 20)
    z, s, _ = srv2.wait(srv2.submit(K.Circuit(20, gates), shots=256, seed=0), timeout=300)
    assert np.array_equal(s, res[0][1])
    srv2.close()
    srv.close()


def test_request_above_budget_fails_cleanly():
    srv = K.Server(K.C64, budget_bytes=16 << 20, aux_bytes=64 << 20)
    rid = srv.submit(K.Circuit(22, layered(22, 1)), shots=8, seed=0)  # 32 MiB state
    with pytest.raises(K.KateError):
        srv.wait(rid, timeout=60)
    ok = srv.submit(K.Circuit(12, layered(12, 1)), shots=8, seed=0)
    srv.wait(ok, timeout=60)
    srv.close()
