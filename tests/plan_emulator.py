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


SOP_DTYPE = np.dtype([("kind", "u1"), ("a", "u1"), ("src", "u1"), ("creg", "u1"), ("cthr", "u1"), ("pad", "u1"),
                      ("idx", "<u2"), ("ccos", "<u8")])
PROG_DTYPE = np.dtype([("m", "<i4"), ("ncb", "<i4"), ("nops", "<i4"), ("nmats", "<i4"), ("tphys", "u1", 16),
                       ("outsrc", "u1", 16), ("cphys", "u1", 48), ("ops", SOP_DTYPE, 160), ("mats", "<f8", (640, 2)),
                       ("stab", "<u2", (40, 44)), ("srb", "u1", (40, 4)), ("stb", "u1", (40, 8)),
                       ("nstages", "<i4"), ("sop0", "<i4")])


BLOCK_DTYPE = np.dtype([("m", "<i4"), ("ncb", "<i4"), ("nblocks", "<i4"), ("pad", "<i4"), ("tphys", "u1", 16),
                        ("outsrc", "u1", 16), ("cphys", "u1", 48), ("btb", "u1", (2, 8)), ("bimg", "<u8", 2),
                        ("smask", "<u2", 4)], align=True)


def _sw128_offsets_bf16(rows):
    """Byte offset of (row, k) in a K-major SWIZZLE_128B image of 64 BF16 columns."""
    r = np.arange(rows)[:, None]
    k = np.arange(64)[None, :]
    chunk, w = k >> 3, k & 7
    return (r >> 3) * 1024 + (r & 7) * 128 + ((chunk ^ (r & 7)) << 4) + w * 2


def _swz(i):
    return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7)


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

        # register-staged programs
        self.smem_ops = []
        L.kate_plan_num_smem_ops(h, ctypes.byref(v))
        for i in range(v.value):
            self.smem_ops.append(self._read_op(L.kate_plan_get_smem_op, i))
        self.programs = []
        for i in range(len(self.passes)):
            size, has = ctypes.c_size_t(), ctypes.c_int()
            L.kate_plan_get_program(h, i, None, 0, ctypes.byref(size), ctypes.byref(has))
            if not has.value:
                self.programs.append(None)
                continue
            buf = np.zeros(size.value, dtype=np.uint8)
            L.kate_plan_get_program(h, i, buf.ctypes.data_as(ctypes.c_void_p), size.value, ctypes.byref(size),
                                    ctypes.byref(has))
            self.programs.append(buf.view(PROG_DTYPE)[0])

        # complex64 tensor-core block programs
        self.block_programs = []
        for i in range(len(self.passes)):
            size, has = ctypes.c_size_t(), ctypes.c_int()
            L.kate_plan_get_block_program(h, i, None, 0, ctypes.byref(size), ctypes.byref(has))
            if not has.value:
                self.block_programs.append(None)
                continue
            buf = np.zeros(size.value, dtype=np.uint8)
            L.kate_plan_get_block_program(h, i, buf.ctypes.data_as(ctypes.c_void_p), size.value, ctypes.byref(size),
                                          ctypes.byref(has))
            self.block_programs.append(buf.view(BLOCK_DTYPE)[0])
        size = ctypes.c_size_t()
        L.kate_plan_block_images(h, None, 0, ctypes.byref(size))
        self.bimg = np.zeros(max(size.value, 16), dtype=np.uint8)
        L.kate_plan_block_images(h, self.bimg.ctypes.data_as(ctypes.c_void_p), self.bimg.size, ctypes.byref(size))

    def block_matrix(self, off):
        """The real 64x64 W = hi + lo read back from a block's BF16 operand images."""
        o = _sw128_offsets_bf16(64)
        def dec(b):
            return (b.view(np.uint16).astype(np.uint32) << 16).view(np.float32)
        hi = dec(self.bimg[off:off + 8192])
        lo = dec(self.bimg[off + 8192:off + 16384])
        return hi[o // 2].astype(np.float64) + lo[o // 2].astype(np.float64)

    def run_blocks(self, state):
        """Executes complex64 block programs (the others generically): each
        block multiplies the 128 x 64 real rows of the tile by W^T read back
        from the operand images, as the tensor-core kernel does."""
        n = self.n
        st = state.astype(np.complex128).copy()
        for p, bp in zip(self.passes, self.block_programs):
            m = p["m"]
            T = 1 << m
            tphys = p["tphys"]
            cphys = [b for b in range(n) if b not in tphys]
            toff = _deposit(np.arange(T, dtype=np.int64), tphys)
            bases = _deposit(np.arange(1 << (n - m), dtype=np.int64), cphys)
            idx = bases[:, None] + toff[None, :]
            tile = st[idx]
            if bp is None:
                for op in self.ops[p["op0"]:p["op0"] + p["nops"]]:
                    self._apply(tile, bases, m, op)
            else:
                for b in range(int(bp["nblocks"])):
                    btb = [int(x) for x in bp["btb"][b][:5]]
                    nb = [i for i in range(m) if i not in btb]
                    rows = _deposit(np.arange(128, dtype=np.int64), nb)
                    cols = _deposit(np.arange(32, dtype=np.int64), btb)
                    sel = rows[:, None] | cols[None, :]          # (128, 32) tile indices
                    x = tile[:, sel]                            # (C, 128, 32) complex
                    xr = np.stack([x.real, x.imag], axis=-1).reshape(x.shape[0], 128, 64)
                    W = self.block_matrix(int(bp["bimg"][b]))
                    y = xr @ W.T
                    tile[:, sel] = y[..., 0::2] + 1j * y[..., 1::2]
            o = np.arange(T, dtype=np.int64)
            src = np.zeros(T, dtype=np.int64)
            for b in range(m):
                src |= ((o >> b) & 1) << p["outsrc"][b]
            st[idx] = tile[:, src]
        x = np.arange(1 << n, dtype=np.int64)
        phys_of_label = [self.final_phys[self.label_to_logical[b]] for b in range(n)]
        return st[_deposit(x, phys_of_label)]

    def _read_op(self, fn, i):
        ints = np.zeros(18, dtype=np.int32)
        pm = ctypes.c_uint64()
        vals = np.zeros(2 + 2 * 1024, dtype=np.float64)
        fn(self.h, i, ints.ctypes.data_as(_ip), ctypes.byref(pm), vals.ctypes.data_as(_dp))
        kind, k = int(ints[0]), int(ints[1])
        op = dict(kind=kind, k=k, tb=[int(x) for x in ints[2:7]], ftb=[int(x) for x in ints[7:12]],
                  fpos=[int(x) for x in ints[12:17]], tmask=int(ints[17]) & 0xFFFFFFFF, pmask=pm.value,
                  phase=complex(vals[0], vals[1]))
        if kind == 0:
            d = 1 << k
            op["mat"] = vals[2:2 + 2 * d * d].view(np.complex128).reshape(d, d).copy()
        elif kind == 4:
            op["tab"] = vals[2:2 + 2 * (1 << k)].view(np.complex128).copy()
        return op

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.kate_plan_destroy(self.h)
            self.h = None

    def run_staged(self, state: np.ndarray) -> np.ndarray:
        """Executes passes that have a register-staged program with the tile
        kernel's semantics (256 threads x 16 registers), the others with the
        generic semantics."""
        n = self.n
        st = state.astype(np.complex128).copy()
        t = np.arange(256, dtype=np.int64)
        jj = np.arange(16, dtype=np.int64)
        for p, prog in zip(self.passes, self.programs):
            m = p["m"]
            T = 1 << m
            tphys = p["tphys"]
            cphys = [b for b in range(n) if b not in tphys]
            toff = _deposit(np.arange(T, dtype=np.int64), tphys)
            bases = _deposit(np.arange(1 << (n - m), dtype=np.int64), cphys)
            idx = bases[:, None] + toff[None, :]
            tile = st[idx]
            if prog is None:
                for op in self.ops[p["op0"]:p["op0"] + p["nops"]]:
                    self._apply(tile, bases, m, op)
            else:
                assert int(prog["m"]) == 12
                mats = prog["mats"][:, 0] + 1j * prog["mats"][:, 1]
                a = None
                sidx = None   # (C, 256, 16) store indices of the open stage
                lflip = np.zeros((tile.shape[0], 256), dtype=np.int64)

                def store():
                    rows = np.arange(tile.shape[0])[:, None, None]
                    tile[rows, sidx] = a

                for k in range(int(prog["nops"])):
                    op = prog["ops"][k]
                    kind = int(op["kind"])
                    if kind == 12:  # XL: flip the next stage's load offset
                        cthr, ccos = int(op["cthr"]), int(op["ccos"])
                        cond = (((t & cthr) == cthr)[None, :]) & (((bases & ccos) == ccos)[:, None])
                        lflip = np.where(cond, lflip ^ int(op["idx"]), lflip)
                        continue
                    if kind == 1:  # STAGE
                        if a is not None:
                            store()
                        si = int(op["idx"])
                        nidx = _deposit(t, prog["stb"][si])[:, None] | _deposit(jj, prog["srb"][si])[None, :]
                        tab = prog["stab"][si].astype(np.int64)
                        s0 = tab[t & 15] ^ tab[16 + (t >> 4)]
                        wl = np.zeros(16, dtype=np.int64)
                        ws = np.zeros(16, dtype=np.int64)
                        wn = np.zeros(16, dtype=np.int64)
                        for i in range(4):
                            bit = ((jj >> i) & 1) == 1
                            wl ^= np.where(bit, tab[32 + i], 0)
                            ws ^= np.where(bit, tab[36 + i], 0)
                            wn ^= np.where(bit, tab[40 + i], 0)
                        # the natural-layout table agrees with the stage's layout
                        assert np.array_equal(_swz((s0[:, None] ^ wn[None, :]) >> 4), nidx)
                        lidx = _swz(((s0[None, :] ^ lflip)[:, :, None] ^ wl[None, None, :]) >> 4)
                        rows = np.arange(tile.shape[0])[:, None, None]
                        a = tile[rows, lidx].copy()
                        lflip = np.zeros((tile.shape[0], 256), dtype=np.int64)
                        s0s = np.broadcast_to(s0[None, :], (tile.shape[0], 256)).copy()
                        sidx = _swz((s0s[:, :, None] ^ ws[None, None, :]) >> 4)
                    elif kind == 11:  # XF: flip the store offset
                        cthr, ccos = int(op["cthr"]), int(op["ccos"])
                        cond = (((t & cthr) == cthr)[None, :]) & (((bases & ccos) == ccos)[:, None])
                        s0s = np.where(cond, s0s ^ int(op["idx"]), s0s)
                        sidx = _swz((s0s[:, :, None] ^ ws[None, None, :]) >> 4)
                    elif kind == 2:  # SMEM
                        if a is not None:
                            store()
                            a = None
                        self._apply(tile, bases, m, self.smem_ops[int(prog["sop0"]) + int(op["idx"])])
                    else:
                        cthr = int(op["cthr"])
                        ccos = int(op["ccos"])
                        creg = int(op["creg"])
                        cond = (((t & cthr) == cthr)[None, :]) & (((bases & ccos) == ccos)[:, None])
                        B = int(op["a"])
                        if kind == 10:  # DR: diagonal over the register bits
                            a *= mats[int(op["idx"]):int(op["idx"]) + 16][None, None, :]
                            continue
                        if kind == 17:  # U2: 4x4 on register bits a (index bit 0) and src (bit 1)
                            A, Bb = 1 << int(op["a"]), 1 << int(op["src"])
                            assert int(op["a"]) < int(op["src"])
                            u = mats[int(op["idx"]):int(op["idx"]) + 16].reshape(4, 4)
                            base = jj[((jj & A) == 0) & ((jj & Bb) == 0)]
                            cols = [base, base | A, base | Bb, base | A | Bb]
                            x = np.stack([a[:, :, c] for c in cols], axis=-1)  # (C, 256, 4 groups, 4)
                            y = x @ u.T
                            for r in range(4):
                                a[:, :, cols[r]] = y[..., r]
                            continue
                        if kind in (8, 9):  # real / RX-form 2x2: same arithmetic as U here
                            kind = 3
                        if kind in (13, 14, 15, 16):  # rotations with their factor taken out
                            tt = mats[int(op["idx"])]
                            t0, t1 = tt.real, tt.imag
                            lo = jj[((jj >> B) & 1) == 0]
                            hi = lo | (1 << B)
                            x, y = a[:, :, lo].copy(), a[:, :, hi].copy()
                            if kind == 13:
                                a[:, :, lo], a[:, :, hi] = x + t0 * y, t1 * x + y
                            elif kind == 14:
                                a[:, :, lo], a[:, :, hi] = t0 * x + y, t1 * y - x
                            elif kind == 15:
                                a[:, :, lo], a[:, :, hi] = x + 1j * t0 * y, y + 1j * t1 * x
                            else:
                                a[:, :, lo], a[:, :, hi] = y - 1j * t0 * x, x - 1j * t1 * y
                            continue
                        if kind in (3, 4, 5):
                            lo = jj[((jj >> B) & 1) == 0]
                            if kind == 5:
                                lo = lo[(lo & creg) == creg]
                            hi = lo | (1 << B)
                            x, y = a[:, :, lo].copy(), a[:, :, hi].copy()
                            if kind == 3:
                                u = mats[int(op["idx"]):int(op["idx"]) + 4]
                                a[:, :, lo] = u[0] * x + u[1] * y
                                a[:, :, hi] = u[2] * x + u[3] * y
                            elif kind == 4:
                                s2 = 1 / np.sqrt(2)
                                a[:, :, lo] = (x + y) * s2
                                a[:, :, hi] = (x - y) * s2
                            else:
                                c3 = cond[:, :, None]
                                a[:, :, lo] = np.where(c3, y, x)
                                a[:, :, hi] = np.where(c3, x, y)
                        elif kind == 6:
                            sel = jj[(jj & creg) == creg]
                            ph = mats[int(op["idx"])]
                            a[:, :, sel] = np.where(cond[:, :, None], a[:, :, sel] * ph, a[:, :, sel])
                        elif kind == 7:
                            d0, d1 = mats[int(op["idx"])], mats[int(op["idx"]) + 1]
                            src = int(op["src"])
                            if src == 0:
                                a *= np.where(((jj >> B) & 1) == 1, d1, d0)[None, None, :]
                            elif src == 1:
                                a *= np.where(((t >> B) & 1) == 1, d1, d0)[None, :, None]
                            else:
                                a *= np.where(((bases >> B) & 1) == 1, d1, d0)[:, None, None]
                        else:
                            raise ValueError(kind)
                if a is not None:
                    store()
            o = np.arange(T, dtype=np.int64)
            src = np.zeros(T, dtype=np.int64)
            for b in range(m):
                src |= ((o >> b) & 1) << p["outsrc"][b]
            st[idx] = tile[:, src]
        x = np.arange(1 << n, dtype=np.int64)
        phys_of_label = [self.final_phys[self.label_to_logical[b]] for b in range(n)]
        return st[_deposit(x, phys_of_label)]

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
