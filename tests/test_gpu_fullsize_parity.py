"""Amplitude-level parity at the workloads' full sizes, where the CPU oracle
cannot follow:

* the 30-qubit, 20-layer complex128 layered circuit (16 GiB state) against
  Kate's own GPU path (its HIPcode headers built by nvcc, oracle/ref_gpu.py)
  run on the same GPU with gateScheduling + gateFusion(5) + gateGrouping(9)
  + compileDefault(0): max-abs amplitude difference <= 1e-12. The reference
  GPU path is itself checked against the CPU oracle at n <= 20
  (tests/test_ref_gpu.py), and this library against the oracle there too;
* the complex64 tensor-core form against the complex128 path on the
  28-qubit, 20-layer brickwork of Haar SU(4) gates: infidelity <= 1e-6.

Both states are copied to host memory and compared in chunks."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits

pytestmark = pytest.mark.gpu
CHUNK = 1 << 24


def test_layered_n30_20_layers_matches_kate_gpu_path_amplitudes():
    from oracle import ref_gpu as RG
    if not RG.available():
        pytest.skip("oracle/_ref/libkate_ref_gpu.so not built")
    n, L = 30, 20
    gates = circuits.layered(n, L, seed=1234)
    sim = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    sim.execute()
    ours = sim.state()
    sim.close()
    del sim
    K.release_cached_memory(0)
    rc = RG.RefGpuCircuit(n, gates)
    rc.compile(fuse=5, group=RG.MAX_GROUP_QUBITS)
    s = rc.session()
    try:
        s.run()
        theirs = s.state()
    finally:
        s.close()
    worst = 0.0
    for i in range(0, ours.size, CHUNK):
        worst = max(worst, float(np.abs(ours[i:i + CHUNK] - theirs[i:i + CHUNK]).max()))
    norm = sum(float(np.vdot(ours[i:i + CHUNK], ours[i:i + CHUNK]).real) for i in range(0, ours.size, CHUNK))
    assert abs(norm - 1.0) <= 1e-10
    assert worst <= 1e-12, worst


@pytest.mark.parametrize("fuse", [False, True])
def test_brickwork_n28_complex64_tensor_cores_infidelity(fuse):
    # fuse=False is the precision workload's plan (the planner forms the
    # 5-qubit blocks); fuse=True first runs the reference's gateFusion(5).
    n, L = 28, 20
    gates = circuits.brickwork_su4(n, L, seed=1234)
    f = K.Circuit(n, gates)
    if fuse:
        f.gateScheduling()
        f.gateFusion(5, 1e-6)
    a = K.Simulator(f, 1, K.C64, 0)
    assert all(k == 3 for k in a.pass_kernels())  # every pass on the tensor cores
    a.execute()
    psi64 = a.state()
    a.close()
    b = K.Simulator(K.Circuit(n, gates), 1, K.C128, 0)
    b.execute()
    psi128 = b.state()
    b.close()
    ov = 0j
    n64 = n128 = 0.0
    for i in range(0, psi64.size, CHUNK):
        x, y = psi64[i:i + CHUNK], psi128[i:i + CHUNK]
        ov += np.vdot(y, x)
        n64 += float(np.vdot(x, x).real)
        n128 += float(np.vdot(y, y).real)
    infid = 1.0 - abs(ov) ** 2 / (n64 * n128)
    assert infid <= 1e-6, infid
