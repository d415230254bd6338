"""Renormalisation of complex64 states (the tensor-core precision form).

The split-BF16 products of the 5-qubit blocks do not keep ||psi|| = 1
exactly; at the end of every run a complex64 simulator reduces ||psi||^2
in FP64 on the device and rescales the state (each product formed in FP64,
rounded once to FP32). After the rescale the only departure from norm 1 is
the FP32 rounding of the rescaled amplitudes themselves, |d_i| <= 2^-24
relative per amplitude; when the scale is within a few FP32 ulps of 1 most
of those roundings fall the same way (an amplitude times 1 + e, e below
half an ulp, rounds back to itself), so a state stored in FP32 is held to
about 1e-10, not 1e-12: the bar is 1e-9. The infidelity against complex128
must stay <= 1e-6."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits

pytestmark = pytest.mark.gpu
CHUNK = 1 << 24


def fused(n, L, seed):
    c = K.Circuit(n, circuits.brickwork_su4(n, L, seed=seed))
    c.gateScheduling()
    c.gateFusion(5, 1e-6)
    return c


def norm2(psi):
    return sum(float(np.vdot(psi[i:i + CHUNK], psi[i:i + CHUNK]).real) for i in range(0, psi.size, CHUNK))


def test_complex64_run_is_renormalised_n28_20_layers():
    n, L = 28, 20
    a = K.Simulator(fused(n, L, 1234), 1, K.C64, 0)
    a.execute()
    before = a.norm2_before_renorm()
    psi64 = a.state()
    a.close()
    drift_before, drift_after = abs(before - 1.0), abs(norm2(psi64) - 1.0)
    assert drift_before < 1e-3, drift_before   # the drift the rescale removed
    assert drift_after <= 1e-9, (drift_before, drift_after)
    b = K.Simulator(K.Circuit(n, circuits.brickwork_su4(n, L, seed=1234)), 1, K.C128, 0)
    b.execute()
    psi128 = b.state()
    b.close()
    ov = sum(np.vdot(psi128[i:i + CHUNK], psi64[i:i + CHUNK]) for i in range(0, psi64.size, CHUNK))
    assert 1.0 - abs(ov) ** 2 <= 1e-6


def test_renormalisation_is_deterministic_and_repeats():
    n = 20
    s = K.Simulator(fused(n, 6, 7), 1, K.C64, 0)
    s.execute()
    a = s.state().copy()
    na = s.norm2_before_renorm()
    s.execute()
    assert s.norm2_before_renorm() == na
    assert np.array_equal(s.state(), a)
    assert abs(norm2(a) - 1.0) <= 1e-9


def test_complex128_is_not_rescaled():
    s = K.Simulator(K.Circuit(14, circuits.layered(14, 2, seed=1)), 1, K.C128, 0)
    s.execute()
    with pytest.raises(K.KateError):
        s.norm2_before_renorm()
