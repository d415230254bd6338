"""The reference's own GPU path (its HIPcode headers under nvcc, in
oracle/_ref/libkate_ref_gpu.so) as a second check: on a GPU its states must
match the oracle and this library's; on CPU the harness must refuse every
circuit its group kernel cannot hold (groups above 9 qubits)."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits
from common import random_circuit

ref_gpu = pytest.importorskip("oracle.ref_gpu")
pytestmark = pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libkate_ref_gpu.so not built")


def compiled(n, gates, fuse=5, group=9):
    c = ref_gpu.RefGpuCircuit(n, gates)
    c.compile(fuse=fuse, group=group)
    return c


def test_harness_accepts_groups_up_to_9_qubits():
    c = compiled(20, circuits.layered(20, 2, seed=3))
    assert c.max_group() <= 9
    assert c.check() == 0


def test_harness_refuses_larger_groups_and_uncompiled_circuits():
    c = compiled(20, circuits.layered(20, 2, seed=3), group=12)
    assert c.max_group() > 9
    assert c.check() == 2
    with pytest.raises(ref_gpu.RefGpuRefused, match="more than 9 qubits"):
        c.session()
    u = ref_gpu.RefGpuCircuit(10, circuits.layered(10, 1, seed=3))
    assert u.check() == 1
    with pytest.raises(ref_gpu.RefGpuRefused, match="not compiled"):
        u.session()


def test_harness_without_gpu_refuses_instead_of_falling_back():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    c = compiled(12, circuits.layered(12, 1, seed=3))
    with pytest.raises(ref_gpu.RefGpuRefused, match="no GPU"):
        c.session()


@pytest.mark.gpu
def test_layered_n20_matches_oracle_and_kate_b200(oracle):
    n = 20
    gates = circuits.layered(n, 10, seed=1234)
    s = compiled(n, gates).session()
    s.run()
    st = s.state()
    pr = s.proba_state()
    s.close()
    ref = oracle.simulate(n, gates)
    assert np.abs(st - ref).max() <= 1e-12
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    res = sim.execute()
    assert np.abs(sim.state() - st).max() <= 1e-12
    assert np.abs(res.as_array() - pr).max() <= 1e-9
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,fuse", [(5, 0), (9, 5), (14, 0), (14, 3)])
def test_random_circuits_all_gate_kinds(oracle, n, fuse):
    rng = np.random.default_rng(300 + n + fuse)
    gates = random_circuit(n, 100, rng)
    s = compiled(n, gates, fuse=fuse).session()
    s.run()
    st = s.state()
    s.close()
    assert np.abs(st - oracle.simulate(n, gates)).max() <= 1e-12
