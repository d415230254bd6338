"""Test and measurement infrastructure only: ctypes access to the reference
simulator's own GPU path (``oracle/_ref/libkate_ref_gpu.so``, built from the
reference's ``HIPcode/*`` headers under nvcc by ``oracle/Makefile``).

It is a baseline and a full-size cross-check, not the oracle: the oracle is
the CPU path (``oracle.oracle``). Only ``tests/`` and ``bench.py``'s
reference-GPU leg import this module; the product never does.

``RefGpuCircuit.session()`` refuses (``RefGpuRefused``) any circuit whose
groups exceed 9 qubits, whose gates exceed 5 qubits or that needs swaps: the
reference's group kernel only stays inside its 12 KiB of shared memory under
those limits (HIPcode/simulator.hpp:785-793, HIPcode/GPUGate.hpp:153-196).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_GPU_SO = os.path.join(HERE, "_ref", "libkate_ref_gpu.so")

MAX_GROUP_QUBITS = 9

_REFUSALS = {
    1: "the circuit is not compiled (gateGrouping + compileDefault)",
    2: "a group has more than 9 qubits",
    3: "a gate has more than 5 qubits",
    4: "the program has swap instructions",
    5: "a gate lies outside its group",
    10: "no GPU",
}

_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


class RefGpuRefused(RuntimeError):
    pass


def available() -> bool:
    return os.path.exists(REF_GPU_SO)


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise FileNotFoundError(f"{REF_GPU_SO} was not built (make -C oracle refgpu)")
        lib = ctypes.CDLL(REF_GPU_SO)
        lib.krefg_circuit_new.restype = _vp
        lib.krefg_circuit_new.argtypes = [ctypes.c_int]
        lib.krefg_free.argtypes = [_vp]
        lib.krefg_append.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int, _dp]
        for f in ("krefg_schedule", "krefg_ngates", "krefg_ngroups", "krefg_max_group", "krefg_check"):
            getattr(lib, f).argtypes = [_vp]
        for f in ("krefg_ngates", "krefg_ngroups", "krefg_max_group", "krefg_check"):
            getattr(lib, f).restype = ctypes.c_int
        lib.krefg_fuse.argtypes = [_vp, ctypes.c_int, ctypes.c_double]
        lib.krefg_group.argtypes = [_vp, ctypes.c_int]
        lib.krefg_compile_default.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
        lib.krefg_session_new.restype = _vp
        lib.krefg_session_new.argtypes = [_vp, _ip]
        lib.krefg_session_run.restype = ctypes.c_int
        lib.krefg_session_run.argtypes = [_vp, _dp]
        lib.krefg_session_measure.restype = ctypes.c_int
        lib.krefg_session_measure.argtypes = [_vp, _dp]
        lib.krefg_session_state.restype = ctypes.c_int
        lib.krefg_session_state.argtypes = [_vp, _dp]
        lib.krefg_session_free.argtypes = [_vp]
        _LIB = lib
    return _LIB


class RefGpuCircuit:
    """A reference ``Kate::Circuit`` inside libkate_ref_gpu.so."""

    def __init__(self, n: int, gates=()):
        self.lib = _lib()
        self.n = n
        self.h = self.lib.krefg_circuit_new(n)
        for g in gates:
            self.append(g)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.krefg_free(h)
            self.h = None

    def append(self, gate):
        gid, qbits, optarg, dense = gate
        q = np.array(qbits, dtype=np.int32)
        d = None
        if gid == 0:
            d = np.ascontiguousarray(dense, dtype=np.complex128).view(np.float64).ravel()
        self.lib.krefg_append(self.h, gid, len(qbits), q.ctypes.data_as(_ip), optarg,
                              None if d is None else d.ctypes.data_as(_dp))

    def compile(self, fuse=5, mtm=1e-6, group=MAX_GROUP_QUBITS, schedule=True):
        """The reference's pipeline: gateScheduling, gateFusion(fuse, mtm),
        gateGrouping(group), compileDefault(0)."""
        if schedule:
            self.lib.krefg_schedule(self.h)
        if fuse:
            self.lib.krefg_fuse(self.h, fuse, mtm)
        self.lib.krefg_group(self.h, group)
        self.lib.krefg_compile_default(self.h, 0, 300)

    def num_gates(self):
        return self.lib.krefg_ngates(self.h)

    def num_groups(self):
        return self.lib.krefg_ngroups(self.h)

    def max_group(self):
        return self.lib.krefg_max_group(self.h)

    def check(self) -> int:
        return self.lib.krefg_check(self.h)

    def session(self) -> "RefGpuSession":
        st = ctypes.c_int(0)
        s = self.lib.krefg_session_new(self.h, ctypes.byref(st))
        if not s:
            why = _REFUSALS.get(st.value, f"CUDA error {-st.value}")
            raise RefGpuRefused(why)
        return RefGpuSession(self, s)


class RefGpuSession:
    """A reference GPU ``Simulator`` (device 0) on a compiled circuit."""

    def __init__(self, circ: RefGpuCircuit, s):
        self.circ = circ
        self.lib = circ.lib
        self.s = s
        self.n = circ.n

    def close(self):
        if self.s:
            self.lib.krefg_session_free(self.s)
            self.s = None

    def __del__(self):
        self.close()

    def run(self) -> float:
        """|0..0> then the whole gate phase; returns its wall time in ms."""
        ms = ctypes.c_double(0)
        e = self.lib.krefg_session_run(self.s, ctypes.byref(ms))
        if e != 0:
            raise RuntimeError(f"reference GPU run failed: CUDA error {-e}")
        return ms.value

    def proba_state(self):
        out = np.empty(2 * self.n, dtype=np.float64)
        e = self.lib.krefg_session_measure(self.s, out.ctypes.data_as(_dp))
        if e != 0:
            raise RuntimeError(f"reference GPU measurement failed: CUDA error {-e}")
        return out.reshape(self.n, 2)

    def state(self):
        out = np.empty(2 << self.n, dtype=np.float64)
        e = self.lib.krefg_session_state(self.s, out.ctypes.data_as(_dp))
        if e != 0:
            raise RuntimeError(f"reference GPU state copy failed: CUDA error {-e}")
        return out.view(np.complex128)
