"""CPU emulation of group-pass plans (test helper, numpy).

Reads a plan through the C ABI (kate_plan_*), applies each pass to a host
state vector with the same semantics as the device kernels (gather the tile
of every coset, apply the ops in order, scatter with the tile bits permuted),
and returns the state in the program's label order. It checks the planner's
logic (tile choice, op lowering, remap bookkeeping) without a GPU; the
kernels themselves are checked on the GPU against the oracle.
"""
from __future__ import annotations

import ctypes

import numpy as np

from kate_b200 import _lib

_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def _deposit(vals: np.ndarray, positions) -> np.ndarray:
    out = np.zeros_like(vals, dtype=np.int64)
    for i, p in enumerate(positions):
        out |= ((vals >> i) & 1) << int(p)
    return out


class PlanView:
    def __init__(self, circuit, max_tile=12, coalesce=4, flags=0):
        L = _lib.lib()
        self.L = L
        h = ctypes.c_void_p()
        st = L.kate_plan_create(circuit.handle, max_tile, coalesce, flags, ctypes.byref(h))
        if st != 0:
            raise RuntimeError(_lib.last_error())
        self.h = h
        self.n = circuit.nqbits
        v = ctypes.c_int()
        L.kate_plan_num_passes(h, ctypes.byref(v))
        self.passes = []
        for i in range(v.value):
            info = np.zeros(4, dtype=np.int32)
            tp = np.zeros(16, dtype=np.uint8)
            os_ = np.zeros(16, dtype=np.uint8)
            L.kate_plan_get_pass(h, i, info.ctypes.data_as(_ip), tp.ctypes.data_as(_u8p), os_.ctypes.data_as(_u8p))
            m = int(info[0])
            self.passes.append(dict(m=m, nops=int(info[1]), op0=int(info[2]), tphys=[int(x) for x in tp[:m]],
                                    outsrc=[int(x) for x in os_[:m]]))
        L.kate_plan_num_ops(h, ctypes.byref(v))
        self.ops = []
        for i in range(v.value):
            ints = np.zeros(18, dtype=np.int32)
            pm = ctypes.c_uint64()
            vals = np.zeros(2 + 2 * 1024, dtype=np.float64)
            L.kate_plan_get_op(h, i, ints.ctypes.data_as(_ip), ctypes.byref(pm), vals.ctypes.data_as(_dp))
            kind, k = int(ints[0]), int(ints[1])
            op = dict(kind=kind, k=k, tb=[int(x) for x in ints[2:7]], ftb=[int(x) for x in ints[7:12]],
                      fpos=[int(x) for x in ints[12:17]], tmask=int(ints[17]) & 0xFFFFFFFF, pmask=pm.value,
                      phase=complex(vals[0], vals[1]))
            if kind == 0:
                d = 1 << k
                op["mat"] = vals[2:2 + 2 * d * d].view(np.complex128).reshape(d, d).copy()
            elif kind == 4:
                op["tab"] = vals[2:2 + 2 * (1 << k)].view(np.complex128).copy()
            self.ops.append(op)
        phys = np.zeros(self.n, dtype=np.int32)
        l2l = np.zeros(self.n, dtype=np.int32)
        L.kate_plan_final_layout(h, phys.ctypes.data_as(_ip), l2l.ctypes.data_as(_ip))
        self.final_phys = [int(x) for x in phys]
        self.label_to_logical = [int(x) for x in l2l]

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.kate_plan_destroy(self.h)
            self.h = None

    def run(self, state: np.ndarray) -> np.ndarray:
        n = self.n
        st = state.astype(np.complex128).copy()
        for p in self.passes:
            m = p["m"]
            T = 1 << m
            tphys = p["tphys"]
            cphys = [b for b in range(n) if b not in tphys]
            toff = _deposit(np.arange(T, dtype=np.int64), tphys)
            bases = _deposit(np.arange(1 << (n - m), dtype=np.int64), cphys)
            idx = bases[:, None] + toff[None, :]
            tile = st[idx]
            for op in self.ops[p["op0"]:p["op0"] + p["nops"]]:
                self._apply(tile, bases, m, op)
            o = np.arange(T, dtype=np.int64)
            src = np.zeros(T, dtype=np.int64)
            for b in range(m):
                src |= ((o >> b) & 1) << p["outsrc"][b]
            st[idx] = tile[:, src]
        # physical -> label order
        x = np.arange(1 << n, dtype=np.int64)
        phys_of_label = [self.final_phys[self.label_to_logical[b]] for b in range(n)]
        return st[_deposit(x, phys_of_label)]

    @staticmethod
    def _apply(tile, bases, m, op):
        T = 1 << m
        ar = np.arange(T, dtype=np.int64)
        kind = op["kind"]
        if kind == 0 or kind == 1:
            k = op["k"] if kind == 0 else 1
            tb = op["tb"][:k]
            mat = op["mat"] if kind == 0 else np.array([[1, 1], [1, -1]]) / np.sqrt(2.0)
            free = np.ones(T, dtype=bool)
            for t in tb:
                free &= ((ar >> t) & 1) == 0
            base = ar[free]
            D = 1 << k
            sub = np.zeros((base.size, D), dtype=np.int64)
            for s in range(D):
                sub[:, s] = base | sum(((s >> i) & 1) << tb[i] for i in range(k))
            x = tile[:, sub]
            tile[:, sub] = np.einsum("rc,gnc->gnr", mat, x)
        elif kind == 2:
            ok_c = (bases & op["pmask"]) == op["pmask"]
            t = op["tb"][0]
            i0 = ar[(((ar >> t) & 1) == 0) & ((ar & op["tmask"]) == op["tmask"])]
            i1 = i0 | (1 << t)
            rows = np.nonzero(ok_c)[0]
            a = tile[np.ix_(rows, i0)].copy()
            tile[np.ix_(rows, i0)] = tile[np.ix_(rows, i1)]
            tile[np.ix_(rows, i1)] = a
        elif kind == 3:
            ok_c = (bases & op["pmask"]) == op["pmask"]
            cols = ar[(ar & op["tmask"]) == op["tmask"]]
            rows = np.nonzero(ok_c)[0]
            tile[np.ix_(rows, cols)] *= op["phase"]
        elif kind == 4:
            k = op["k"]
            d = np.zeros((bases.size, T), dtype=np.int64)
            for i in range(k):
                if op["ftb"][i] >= 0:
                    d |= (((ar >> op["ftb"][i]) & 1) << i)[None, :]
                else:
                    d |= (((bases >> op["fpos"][i]) & 1) << i)[:, None]
            tile *= op["tab"][d]
        else:
            raise ValueError(kind)
