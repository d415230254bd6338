"""Test infrastructure only: ctypes access to the two CPU checkers.

* ``Ref`` wraps ``oracle/_ref/libkate_ref.so``: the reference simulator's own
  CPU path (Line-fr/Kate, ``CPUcode/simulator.hpp``, ``CPUcode/GateMerger.hpp``,
  ``backendagnosticcode/Circuit.hpp``), compiled from its headers by
  ``oracle/Makefile``.
* ``Oracle`` wraps ``oracle/libkate_oracle.so``: the plain-C restatement of
  the same arithmetic in ``oracle/kate_oracle.c``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module; the product never does.

Gate lists are Python tuples ``(id, qbits, optarg, dense)`` where ``dense`` is
a complex128 numpy array of shape (2^k, 2^k) for id 0 and None otherwise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libkate_ref.so")
ORACLE_SO = os.path.join(HERE, "libkate_oracle.so")

_i = ctypes.c_int
_d = ctypes.c_double
_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


def _iptr(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _dptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def flatten(gates):
    """Flat arrays (ids, nqs, qbits, optargs, dense) for a gate list."""
    ids = np.array([g[0] for g in gates], dtype=np.int32)
    nqs = np.array([len(g[1]) for g in gates], dtype=np.int32)
    qb = np.array([q for g in gates for q in g[1]], dtype=np.int32)
    opt = np.array([g[2] for g in gates], dtype=np.int32)
    dense_parts = [np.ascontiguousarray(g[3], dtype=np.complex128).view(np.float64).ravel()
                   for g in gates if g[0] == 0]
    dense = np.concatenate(dense_parts) if dense_parts else np.zeros(2, dtype=np.float64)
    if qb.size == 0:
        qb = np.zeros(1, dtype=np.int32)
    return ids, nqs, qb, opt, dense


class Oracle:
    """The C restatement (kate_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        lib = ctypes.CDLL(path)
        lib.ko_simulate.argtypes = [_i, _i, _ip, _ip, _ip, _ip, _dp, _dp, _ip, _dp]
        lib.ko_apply.argtypes = [_i, _dp, _i, _i, _ip, _i, _dp]
        lib.ko_merge.argtypes = [_i, _ip, _ip, _ip, _ip, _dp, _ip, _dp]
        lib.ko_merge.restype = _i
        lib.ko_measure.argtypes = [_i, _dp, _ip, _dp]
        self.lib = lib

    def simulate(self, n, gates, proba_in=None, initial_permutation=None):
        ids, nqs, qb, opt, dense = flatten(gates)
        out = np.empty(2 << n, dtype=np.float64)
        pin = None if proba_in is None else np.ascontiguousarray(proba_in, dtype=np.float64).ravel()
        perm = None if initial_permutation is None else np.ascontiguousarray(initial_permutation, dtype=np.int32)
        self.lib.ko_simulate(n, len(gates), _iptr(ids), _iptr(nqs), _iptr(qb), _iptr(opt), _dptr(dense),
                             _dptr(pin), _iptr(perm), _dptr(out))
        return out.view(np.complex128)

    def apply(self, n, state, gate):
        st = np.ascontiguousarray(state, dtype=np.complex128).copy()
        ids, nqs, qb, opt, dense = flatten([gate])
        self.lib.ko_apply(n, _dptr(st.view(np.float64)), int(ids[0]), int(nqs[0]), _iptr(qb), int(opt[0]),
                          _dptr(dense))
        return st

    def merge(self, gates):
        ids, nqs, qb, opt, dense = flatten(gates)
        oq = np.zeros(64, dtype=np.int32)
        od = np.zeros(2 * 4 ** 10, dtype=np.float64)
        k = self.lib.ko_merge(len(gates), _iptr(ids), _iptr(nqs), _iptr(qb), _iptr(opt), _dptr(dense), _iptr(oq),
                              _dptr(od))
        if k < 0:
            raise ValueError("merge covers more than 5 qubits")
        dim = 1 << k
        return list(oq[:k]), od[: 2 * dim * dim].view(np.complex128).reshape(dim, dim).copy()

    def measure(self, n, state, final_inverse_permutation=None):
        st = np.ascontiguousarray(state, dtype=np.complex128)
        out = np.empty(2 * n, dtype=np.float64)
        perm = None if final_inverse_permutation is None else np.ascontiguousarray(final_inverse_permutation,
                                                                                   dtype=np.int32)
        self.lib.ko_measure(n, _dptr(st.view(np.float64)), _iptr(perm), _dptr(out))
        return out.reshape(n, 2)


class RefCircuit:
    """A reference ``Kate::Circuit`` living inside libkate_ref.so."""

    def __init__(self, ref: "Ref", n: int, gates=()):
        self.ref = ref
        self.lib = ref.lib
        self.n = n
        self.h = self.lib.kref_circuit_new(n)
        for g in gates:
            self.append(g)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.kref_free(h)
            self.h = None

    def append(self, gate):
        gid, qbits, optarg, dense = gate
        q = np.array(qbits, dtype=np.int32)
        d = None
        if gid == 0:
            d = np.ascontiguousarray(dense, dtype=np.complex128).view(np.float64).ravel()
        self.lib.kref_append(self.h, gid, len(qbits), _iptr(q), optarg, _dptr(d))

    def schedule(self):
        self.lib.kref_schedule(self.h)

    def fuse(self, k=5, mtm=1e-6):
        self.lib.kref_fuse(self.h, k, mtm)

    def group(self, m=8):
        self.lib.kref_group(self.h, m)

    def allocate(self, g=0, maxlocal=300):
        self.lib.kref_allocate(self.h, g, maxlocal)

    def compile_default(self, g=0, maxlocal=300):
        self.lib.kref_compile_default(self.h, g, maxlocal)

    def gates(self):
        out = []
        q = np.zeros(64, dtype=np.int32)
        d = np.zeros(2 * 4 ** 10, dtype=np.float64)
        gid, nq, opt = _i(), _i(), _i()
        for i in range(self.lib.kref_ngates(self.h)):
            self.lib.kref_gate(self.h, i, ctypes.byref(gid), ctypes.byref(nq), _iptr(q), ctypes.byref(opt), _dptr(d))
            k = nq.value
            dense = None
            if gid.value == 0:
                dim = 1 << k
                dense = d[: 2 * dim * dim].view(np.complex128).reshape(dim, dim).copy()
            out.append((gid.value, [int(x) for x in q[:k]], opt.value, dense))
        return out

    def groups(self):
        out = []
        q = np.zeros(64, dtype=np.int32)
        end, nq = _i(), _i()
        for i in range(self.lib.kref_ngroups(self.h)):
            self.lib.kref_group_get(self.h, i, ctypes.byref(end), ctypes.byref(nq), _iptr(q))
            out.append((end.value, [int(x) for x in q[: nq.value]]))
        return out

    def instructions(self):
        out = []
        q = np.zeros(256, dtype=np.int32)
        kind, nq = _i(), _i()
        for i in range(self.lib.kref_ninstr(self.h)):
            self.lib.kref_instr(self.h, i, ctypes.byref(kind), ctypes.byref(nq), _iptr(q))
            out.append((kind.value, [int(x) for x in q[: nq.value]]))
        return out

    def perms(self):
        a = np.zeros(self.n, dtype=np.int32)
        b = np.zeros(self.n, dtype=np.int32)
        if not self.lib.kref_perms(self.h, _iptr(a), _iptr(b)):
            return None, None
        return list(a), list(b)

    def merge(self, b, e):
        q = np.zeros(64, dtype=np.int32)
        d = np.zeros(2 * 4 ** 10, dtype=np.float64)
        k = self.lib.kref_merge(self.h, b, e, _iptr(q), _dptr(d))
        dim = 1 << k
        return [int(x) for x in q[:k]], d[: 2 * dim * dim].view(np.complex128).reshape(dim, dim).copy()

    def simulate(self, proba_in=None, want_state=True):
        st = np.empty(2 << self.n, dtype=np.float64) if want_state else None
        pr = np.empty(2 * self.n, dtype=np.float64)
        ms = _d()
        pin = None if proba_in is None else np.ascontiguousarray(proba_in, dtype=np.float64).ravel()
        self.lib.kref_simulate(self.h, _dptr(pin), _dptr(st), _dptr(pr), ctypes.byref(ms))
        return (st.view(np.complex128) if want_state else None), pr.reshape(self.n, 2), ms.value

    def session(self):
        """Gate-phase timing session (see kref_session_new)."""
        return RefSession(self)

    def export_qcx(self, path):
        self.lib.kref_export_qcx(self.h, path.encode())

    def print_to(self, path, permutationtable=False):
        """QuantumCircuit::print, appended to the file at path."""
        if self.lib.kref_print(self.h, int(permutationtable), path.encode()) != 0:
            raise OSError(f"cannot append to {path}")


class RefSession:
    def __init__(self, circ: RefCircuit):
        self.lib = circ.lib
        self.s = self.lib.kref_session_new(circ.h)
        if not self.s:
            raise MemoryError("reference simulator could not allocate its state")

    def run(self) -> float:
        """Runs every compute group once; returns ms."""
        return float(self.lib.kref_session_run(self.s))

    def close(self):
        if self.s:
            self.lib.kref_session_free(self.s)
            self.s = None

    def __del__(self):
        self.close()


class Ref:
    """The reference's own CPU path (libkate_ref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference is present")
        lib = ctypes.CDLL(path)
        lib.kref_circuit_new.restype = _vp
        lib.kref_circuit_new.argtypes = [_i]
        lib.kref_free.argtypes = [_vp]
        lib.kref_append.argtypes = [_vp, _i, _i, _ip, _i, _dp]
        lib.kref_schedule.argtypes = [_vp]
        lib.kref_fuse.argtypes = [_vp, _i, _d]
        lib.kref_group.argtypes = [_vp, _i]
        lib.kref_allocate.argtypes = [_vp, _i, _i]
        lib.kref_compile_default.argtypes = [_vp, _i, _i]
        lib.kref_ngates.argtypes = [_vp]
        lib.kref_gate.argtypes = [_vp, _i, _ip, _ip, _ip, _ip, _dp]
        lib.kref_ngroups.argtypes = [_vp]
        lib.kref_group_get.argtypes = [_vp, _i, _ip, _ip, _ip]
        lib.kref_ninstr.argtypes = [_vp]
        lib.kref_instr.argtypes = [_vp, _i, _ip, _ip, _ip]
        lib.kref_perms.argtypes = [_vp, _ip, _ip]
        lib.kref_merge.argtypes = [_vp, _i, _i, _ip, _dp]
        lib.kref_merge.restype = _i
        lib.kref_simulate.argtypes = [_vp, _dp, _dp, _dp, ctypes.POINTER(_d)]
        lib.kref_export_qcx.argtypes = [_vp, ctypes.c_char_p]
        lib.kref_print.argtypes = [_vp, ctypes.c_int, ctypes.c_char_p]
        lib.kref_print.restype = ctypes.c_int
        lib.kref_session_new.argtypes = [_vp]
        lib.kref_session_new.restype = _vp
        lib.kref_session_run.argtypes = [_vp]
        lib.kref_session_run.restype = _d
        lib.kref_session_free.argtypes = [_vp]
        self.lib = lib

    def hw_threads(self) -> int:
        return int(self.lib.kref_hw_threads())

    def circuit(self, n, gates=()):
        return RefCircuit(self, n, gates)


def available_ref() -> bool:
    return os.path.exists(REF_SO)
