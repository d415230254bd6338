"""The C ABI: every declared symbol is exported, errors are reported as
status codes with messages (the reference prints and continues), and the
Python mirror keeps the reference's names."""
import ctypes
import os
import re

import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"KATE_API\s+[\w\s\*]+?\b(kate_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_declares_every_symbol():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_version():
    assert b"sm_100a" in _lib.lib().kate_version()


@pytest.mark.parametrize("gate,msg", [
    ((2, [5], 0, None), "outside"),
    ((3, [1, 1], 0, None), "twice"),
    ((2, [0, 1], 0, None), "exactly 1"),
    ((5, [0, 1], 0, None), "exactly 3"),
    ((9, [0], 0, None), "unknown"),
])
def test_bad_gates_rejected(gate, msg):
    c = K.Circuit(3)
    with pytest.raises(K.KateError) as e:
        c.appendGate(gate)
    assert e.value.status == K.KATE_EINVAL
    assert msg in str(e.value)
    assert c.num_gates() == 0


def test_dense_dimension_mismatch_rejected():
    c = K.Circuit(3)
    L = _lib.lib()
    m = np.zeros(2 * 16)
    q = np.array([0], dtype=np.int32)
    # a 4x4 matrix on one qubit: dimension mismatch, 2x2 expected
    st = L.kate_circuit_append_dense(c.handle, m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     q.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 1)
    assert st == K.KATE_OK  # reads exactly 2*4 doubles for one qubit: the size is implied by nq
    with pytest.raises(K.KateError):
        K.Circuit(2).appendGate(K.Gate(np.eye(4), [0]))


def test_append_after_grouping_is_a_state_error():
    c = K.Circuit(3, [(2, [0], 0, None)])
    c.gateGrouping(3)
    with pytest.raises(K.KateError) as e:
        c.appendGate((2, [1], 0, None))
    assert e.value.status == K.KATE_ESTATE


def test_group_size_below_a_gate_is_rejected():
    c = K.Circuit(4, [(5, [0, 1, 2], 0, None)])
    with pytest.raises(K.KateError):
        c.gateGrouping(2)


def test_fusion_failure_leaves_circuit_unchanged():
    # an RX (id 6) gate alone has no single-gate cost edge in the reference's
    # fusion graph, and a 2-qubit neighbour makes the merge window too wide
    c = K.Circuit(4, [(6, [0], 0, None), (0, [1, 2], 0, np.eye(4))])
    before = c.gate_set_ordered
    with pytest.raises(K.KateError):
        c.gateFusion(1, 0.0)
    assert len(c.gate_set_ordered) == len(before)


def test_rx_rz_identifiers_are_no_ops_like_the_reference(oracle):
    gates = [(6, [0], 0, None), (7, [1], 0, None), (2, [0], 0, None)]
    st = oracle.simulate(2, gates)
    assert np.allclose(st, [2 ** -0.5, 2 ** -0.5, 0, 0])


def test_qcx_export_matches_reference_text(tmp_path):
    from golden_io import GOLDEN
    c = K.Circuit(5, [(2, [0], 0, None), (3, [1, 2], 0, None), (4, [3, 0], 3, None), (5, [0, 1, 4], 0, None),
                      (0, [2, 3], 0, np.eye(4, dtype=np.complex128))])
    p = str(tmp_path / "c.qcx")
    c.exportqcx(p)
    assert open(p).read() == open(os.path.join(GOLDEN, "circuit.qcx")).read()


def test_clone_is_deep():
    c = K.Circuit(3, [(2, [0], 0, None)])
    d = c.copy()
    d.appendGate((2, [1], 0, None))
    assert c.num_gates() == 1 and d.num_gates() == 2


def test_merge_range_errors():
    c = K.Circuit(3, [(2, [0], 0, None)])
    with pytest.raises(K.KateError):
        c.merge(0, 5)


def test_simulator_without_device_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(K.KateError) as e:
        K.Simulator(K.Circuit(3, [(2, [0], 0, None)]))
    assert e.value.status in (K.KATE_ECUDA, K.KATE_ENOMEM)


def test_plan_requires_valid_tile():
    c = K.Circuit(3, [(2, [0], 0, None)])
    h = ctypes.c_void_p()
    assert _lib.lib().kate_plan_create(c.handle, 0, 0, 0, ctypes.byref(h)) == K.KATE_EINVAL
    assert _lib.lib().kate_plan_create(c.handle, 15, 0, 0, ctypes.byref(h)) == K.KATE_EINVAL


def test_device_queries_without_a_gpu_report_zero_devices():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    assert K.devices() == []
    L = _lib.lib()
    with pytest.raises(K.KateError, match="no such CUDA device"):
        K._check(L.kate_device_properties(0, None, 0, None, None, None))


def test_device_merger_without_a_gpu_fails_loudly():
    # The device merger has no silent host fallback (the host merger is a
    # separate entry point).
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    gates = [(2, [0], 0, None), (3, [1, 0], 0, None)]
    with pytest.raises(K.KateError, match="no such CUDA device"):
        K.mergeGate(gates, device=0)
    c = K.Circuit(2, gates)
    with pytest.raises(K.KateError, match="no such CUDA device"):
        c.gateFusion(2, 1e-6, device=0)
    assert c.num_gates() == 2
