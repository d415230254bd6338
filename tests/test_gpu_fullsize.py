"""Full-size checks through a size-independent property: a circuit followed
by its inverse returns the state to |0...0>, so every <Z_q> is 1 and every
sample is 0. Run at the workloads' full sizes (30 qubits complex128, 32
qubits complex64 on the tensor cores, 4096-circuit batch, served requests),
where the oracle cannot follow."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits

pytestmark = pytest.mark.gpu


def inverse(gates):
    """The inverse circuit: reversed order, each gate's inverse (dense: the
    conjugate transpose; H, CNOT, TOFFOLI are their own inverses)."""
    out = []
    for gid, q, opt, d in reversed(gates):
        if gid == K.DENSE:
            out.append((gid, list(q), 0, np.ascontiguousarray(np.conj(np.asarray(d)).T)))
        elif gid in (K.Hadamard, K.CNOT, K.TOFFOLI):
            out.append((gid, list(q), opt, None))
        else:
            raise ValueError("no inverse for gate id %d" % gid)
    return out


def with_inverse_flat(ids, nqs, qb, opt, dense):
    """Flat arrays (as circuits.hea_flat) of a dense-gate circuit followed by
    its inverse."""
    qo = np.concatenate([[0], np.cumsum(nqs)])
    dims = 1 << nqs.astype(np.int64)
    do = np.concatenate([[0], np.cumsum(dims * dims)])
    rq, rd = [], []
    for k in range(len(ids) - 1, -1, -1):
        rq.append(qb[qo[k]:qo[k + 1]])
        d = dims[k]
        rd.append(np.conj(dense[do[k]:do[k + 1]].reshape(d, d)).T.ravel())
    return (np.concatenate([ids, ids[::-1]]), np.concatenate([nqs, nqs[::-1]]), np.concatenate([qb] + rq),
            np.concatenate([opt, opt[::-1]]), np.concatenate([dense] + rd))


def test_layered_n30_complex128_round_trip():
    n = 30
    g = circuits.layered(n, 6, seed=11)
    sim = K.Simulator(K.Circuit(n, g + inverse(g)), 1, K.C128, 0)
    sim.execute()
    z = sim.expect_z()
    assert np.all(np.abs(z - 1.0) <= 1e-9), np.abs(z - 1.0).max()
    sim.close()


def test_brickwork_n32_complex64_tensor_cores_round_trip():
    n = 32
    g = circuits.brickwork_su4(n, 6, seed=5)
    c = K.Circuit(n, g + inverse(g))
    c.gateScheduling()
    c.gateFusion(5, 1e-6)
    sim = K.Simulator(c, 1, K.C64, 0)
    sim.execute()
    z = sim.expect_z()
    assert np.all(np.abs(z - 1.0) <= 1e-4), np.abs(z - 1.0).max()
    sim.close()


def test_batch_of_4096_round_trips():
    rng = np.random.default_rng(2024)
    ns = [int(x) for x in rng.integers(10, 23, 4096)]
    circs = []
    for i, n in enumerate(ns):
        c = K.Circuit(n)  # depth n, then its inverse: 2n layers in all
        c.appendFlat(*with_inverse_flat(*circuits.hea_flat(n, n, seed=i)))
        circs.append(c)
    b = K.Batch(circs, precision=K.C64)
    b.run()
    z = b.expect_z_flat()
    assert z.size == sum(ns)
    assert np.all(np.abs(z - 1.0) <= 1e-4), np.abs(z - 1.0).max()
    b.close()


def test_served_round_trips_sample_zero():
    srv = K.Server(K.C64, budget_bytes=8 << 30, aux_bytes=512 << 20)
    ids = []
    for i, n in enumerate([12, 14, 18, 22, 26]):
        g = circuits.layered(n, n, seed=i)
        ids.append(srv.submit(K.Circuit(n, g + inverse(g)), shots=1024, seed=i))
    for rid in ids:
        z, s, _ = srv.wait(rid, timeout=300)
        assert np.all(np.abs(z - 1.0) <= 1e-4)
        assert np.all(s == 0)
    srv.close()
