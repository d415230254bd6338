"""Python mirror of Kate's circuit/simulator API over libkate_b200.so.

The names and argument meanings follow the reference's C++ API (Line-fr/Kate):
``Gate`` (backendagnosticcode/basic_host_types.hpp:190-296), ``Circuit``
(backendagnosticcode/Circuit.hpp, QuantumCircuit.hpp), ``Simulator``
(HIPcode/simulator.hpp:220-811), ``mergeGate`` (CPUcode/GateMerger.hpp:8-55)
and ``proba_state`` (basic_host_types.hpp:319-336). Every call goes through
the C ABI declared in include/kate_b200.h; nothing here computes amplitudes.
Failures raise ``KateError`` (the reference prints and continues).
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib

Hadamard = 2
CNOT = 3
CRk = 4
TOFFOLI = 5
RX = 6
RZ = 7
DENSE = 0

C128 = 0
C64 = 1

KATE_OK, KATE_EINVAL, KATE_ENOMEM, KATE_ECUDA, KATE_ETIMEDOUT, KATE_ESTATE = range(6)


class KateError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[kate status {status}] {msg}")
        self.status = status


def _check(st: int):
    if st != KATE_OK:
        raise KateError(st, _lib.last_error())


_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def _iarr(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32))


class Gate:
    """Gate(identifier, qbits, optarg=0) or Gate(matrix, qbits) for a dense gate.

    ``matrix`` is a 2^k x 2^k complex array, row-major; bit i of its local
    index is ``qbits[i]``.
    """

    def __init__(self, what, qbits: Sequence[int], optarg: int = 0):
        self.qbits = [int(q) for q in qbits]
        if isinstance(what, (int, np.integer)):
            self.identifier = int(what)
            self.optarg = int(optarg)
            self.densecontent = None
        else:
            m = np.ascontiguousarray(np.asarray(what, dtype=np.complex128))
            self.identifier = DENSE
            self.optarg = 0
            self.densecontent = m

    def as_tuple(self):
        return (self.identifier, list(self.qbits), self.optarg, self.densecontent)

    def __repr__(self):
        return f"Gate(id={self.identifier}, qbits={self.qbits}, optarg={self.optarg})"


class proba_state:
    """Per-qubit (theta, phi) pairs, as in the reference."""

    def __init__(self, val):
        self.val = [(float(a), float(b)) for a, b in val]

    def as_array(self) -> np.ndarray:
        return np.array(self.val, dtype=np.float64).reshape(-1, 2)

    def print(self):
        for i, (t, p) in enumerate(self.val):
            print(f"Qbit {i} : teta={t} , phi={p}")


class Circuit:
    """Kate::Circuit: gate list plus the compile passes."""

    def __init__(self, nqbits: int, gates: Sequence = (), _handle=None):
        self._lib = _lib.lib()
        if _handle is not None:
            self._h = _handle
        else:
            h = ctypes.c_void_p()
            _check(self._lib.kate_circuit_create(int(nqbits), ctypes.byref(h)))
            self._h = h
        gates = list(gates)
        if gates:
            self.appendGates(gates)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.kate_circuit_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def nqbits(self) -> int:
        v = ctypes.c_int()
        _check(self._lib.kate_circuit_nqbits(self._h, ctypes.byref(v)))
        return v.value

    def copy(self) -> "Circuit":
        h = ctypes.c_void_p()
        _check(self._lib.kate_circuit_clone(self._h, ctypes.byref(h)))
        return Circuit(0, _handle=h)

    def appendGate(self, gate):
        if isinstance(gate, tuple):
            gate = Gate(gate[3] if gate[0] == DENSE else gate[0], gate[1], gate[2])
        q = _iarr(gate.qbits)
        if gate.identifier == DENSE:
            dim = 1 << len(gate.qbits)
            if gate.densecontent is None or gate.densecontent.shape != (dim, dim):
                raise KateError(KATE_EINVAL, "size mismatch: dense matrix dimension must be 2^k for k qubits")
            d = np.ascontiguousarray(gate.densecontent, dtype=np.complex128).view(np.float64).ravel()
            _check(self._lib.kate_circuit_append_dense(self._h, d.ctypes.data_as(_dp), q.ctypes.data_as(_ip),
                                                       len(gate.qbits)))
        else:
            _check(self._lib.kate_circuit_append_gate(self._h, gate.identifier, q.ctypes.data_as(_ip),
                                                      len(gate.qbits), gate.optarg))

    def appendGates(self, gates: Sequence):
        """Appends many gates (Gate objects or (id, qbits, optarg, dense)
        tuples) in one call; all or nothing."""
        ids, nqs, qb, opt, dense = [], [], [], [], []
        for g in gates:
            if isinstance(g, Gate):
                g = g.as_tuple()
            gid, q, o, d = g
            ids.append(int(gid))
            nqs.append(len(q))
            qb.extend(int(x) for x in q)
            opt.append(int(o))
            if gid == DENSE:
                dim = 1 << len(q)
                m = np.asarray(d, dtype=np.complex128) if d is not None else None
                if m is None or m.shape != (dim, dim):
                    raise KateError(KATE_EINVAL, "size mismatch: dense matrix dimension must be 2^k for k qubits")
                dense.append(m.ravel())
        self.appendFlat(ids, nqs, qb, opt, np.concatenate(dense) if dense else None)

    def appendFlat(self, ids, nqs, qbits, optargs, dense=None):
        """Appends gates given as flat arrays (kate_circuit_append_many):
        ids[i], nqs[i] qubits taken in order from qbits, optargs[i]; dense
        gates' 4^nq complex entries in order in ``dense``."""
        ids_a, nqs_a, qb_a, opt_a = (_iarr(x) for x in (ids, nqs, qbits, optargs))
        d = (np.ascontiguousarray(np.asarray(dense, dtype=np.complex128)).view(np.float64) if dense is not None
             else np.zeros(2, dtype=np.float64))
        _check(self._lib.kate_circuit_append_many(self._h, len(ids_a), ids_a.ctypes.data_as(_ip),
                                                  nqs_a.ctypes.data_as(_ip), qb_a.ctypes.data_as(_ip),
                                                  opt_a.ctypes.data_as(_ip), d.ctypes.data_as(_dp)))

    # --- passes (backendagnosticcode/Circuit.hpp) ---
    def gateScheduling(self):
        _check(self._lib.kate_circuit_schedule(self._h))

    def gateFusion(self, qbitsizelimit: int = 5, merge_time_matters: float = 0.000001, device: Optional[int] = None):
        """gateFusion; with `device`, every merge of the pass runs on that
        CUDA device in one launch (same intervals, bit-identical matrices)."""
        if device is None:
            _check(self._lib.kate_circuit_fuse(self._h, int(qbitsizelimit), float(merge_time_matters)))
        else:
            _check(self._lib.kate_circuit_fuse_device(self._h, int(qbitsizelimit), float(merge_time_matters),
                                                      int(device)))

    def gateGrouping(self, qbitgroupsize: int = 8):
        _check(self._lib.kate_circuit_group(self._h, int(qbitgroupsize)))

    def allocate(self, numberofgpulog2: int = 0, maxlocalqbitnumber: int = 300):
        _check(self._lib.kate_circuit_allocate(self._h, int(numberofgpulog2), int(maxlocalqbitnumber)))

    def compileDefault(self, numberofgpulog2: int = 0, maxlocalqbitnumber: int = 300):
        _check(self._lib.kate_circuit_compile_default(self._h, int(numberofgpulog2), int(maxlocalqbitnumber)))

    def compileOPT(self, qbit_matrix_merge_size_limit=5, merge_time_matters=0.000001, groupsize=10,
                   numberofgpulog2=0, maxlocalqbitnumber=300):
        _check(self._lib.kate_circuit_compile_opt(self._h, int(qbit_matrix_merge_size_limit),
                                                  float(merge_time_matters), int(groupsize), int(numberofgpulog2),
                                                  int(maxlocalqbitnumber)))

    def exportqcx(self, filename: str):
        _check(self._lib.kate_circuit_export_qcx(self._h, filename.encode()))

    # --- introspection ---
    def num_gates(self) -> int:
        v = ctypes.c_int()
        _check(self._lib.kate_circuit_num_gates(self._h, ctypes.byref(v)))
        return v.value

    @property
    def gate_set_ordered(self) -> List[Tuple]:
        out = []
        q = np.zeros(64, dtype=np.int32)
        d = np.zeros(2 * 4 ** 10, dtype=np.float64)
        gid, nq, opt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        for i in range(self.num_gates()):
            _check(self._lib.kate_circuit_get_gate(self._h, i, ctypes.byref(gid), q.ctypes.data_as(_ip),
                                                   ctypes.byref(nq), ctypes.byref(opt), d.ctypes.data_as(_dp)))
            k = nq.value
            dense = None
            if gid.value == DENSE:
                dim = 1 << k
                dense = d[: 2 * dim * dim].view(np.complex128).reshape(dim, dim).copy()
            out.append((gid.value, [int(x) for x in q[:k]], opt.value, dense))
        return out

    @property
    def groups(self):
        n = ctypes.c_int()
        _check(self._lib.kate_circuit_num_groups(self._h, ctypes.byref(n)))
        out = []
        q = np.zeros(64, dtype=np.int32)
        end, nq = ctypes.c_int(), ctypes.c_int()
        for i in range(n.value):
            _check(self._lib.kate_circuit_get_group(self._h, i, ctypes.byref(end), q.ctypes.data_as(_ip),
                                                    ctypes.byref(nq)))
            out.append((end.value, [int(x) for x in q[: nq.value]]))
        return out

    @property
    def instructions(self):
        n = ctypes.c_int()
        _check(self._lib.kate_circuit_num_instructions(self._h, ctypes.byref(n)))
        out = []
        q = np.zeros(256, dtype=np.int32)
        kind, nq = ctypes.c_int(), ctypes.c_int()
        for i in range(n.value):
            _check(self._lib.kate_circuit_get_instruction(self._h, i, ctypes.byref(kind), q.ctypes.data_as(_ip),
                                                          ctypes.byref(nq)))
            out.append((kind.value, [int(x) for x in q[: nq.value]]))
        return out

    def permutations(self):
        n = self.nqbits
        a = np.zeros(n, dtype=np.int32)
        b = np.zeros(n, dtype=np.int32)
        v = ctypes.c_int()
        _check(self._lib.kate_circuit_get_permutations(self._h, a.ctypes.data_as(_ip), b.ctypes.data_as(_ip),
                                                       ctypes.byref(v)))
        return (list(a), list(b)) if v.value else (None, None)

    def print(self, permutationtable: bool = False):
        """Kate's QuantumCircuit::print (QuantumCircuit.hpp:38-123): the gate
        list (by group once grouped) before compilation, the program
        (swaps, then each group with its gates; with permutationtable the
        label-to-qubit table before each group) after it."""
        print(self.program_text(permutationtable), end="")

    def program_text(self, permutationtable: bool = False) -> str:
        """The text ``print`` writes."""
        gates = self.gate_set_ordered
        groups = self.groups
        instr = self.instructions

        def gate_line(g):
            return "Identifier : " + str(g[0]) + ", Qbits affected : " + "".join(f"{q} " for q in g[1]) + "\n"

        def group_head(label, k):
            return f"{label} {k} with qbits " + "".join(f"{q} " for q in groups[k][1]) + " : \n"

        out = ""
        if not instr:
            group = 0
            if groups:
                out += group_head("Group", 0)
            for i, g in enumerate(gates):
                if groups:
                    if group >= len(groups):
                        return out + "ERROR while printing the circuit, group vector is bad\n"
                    if groups[group][0] == i:
                        group += 1
                        out += group_head("Group", group)
                    out += "   " + gate_line(g)
                else:
                    out += f"gate {i} is " + gate_line(g)
            return out
        perm, _ = self.permutations()
        n = self.nqbits
        inv = [0] * n
        for m in range(n):
            inv[perm[m]] = m
        out += "-------Quantum-Program-------\n"
        i, group = 0, 0
        for kind, q in instr:
            if kind == 0:
                out += "SWAP "
                for m in range(len(q) // 2):
                    a, b = q[2 * m], q[2 * m + 1]
                    out += f"{a} and {b}, "
                    inv[a], inv[b] = inv[b], inv[a]
            else:
                if permutationtable:
                    out += "Permutation table (subjective to real) : \n"
                    out += "".join(f"{m} " + (" " if m < 10 else "") for m in range(n)) + "\n"
                    out += "".join(f"{inv[m]} " + (" " if inv[m] < 10 else "") for m in range(n)) + "\n\n"
                out += group_head("EXEC Group", group)
                for j in range(i, groups[group][0]):
                    out += "   " + gate_line(gates[j])
                i = groups[group][0]
                group += 1
            out += "\n\n"
        return out + "-----------------------------\n"

    def merge(self, begin: int, end: int, device: Optional[int] = None, stream: int = 0) -> Gate:
        """mergeGate of gates [begin, end) of this circuit; on CUDA device
        `device` (on `stream`, a cudaStream_t value) when given."""
        q = np.zeros(64, dtype=np.int32)
        d = np.zeros(2 * 4 ** 10, dtype=np.float64)
        k = ctypes.c_int()
        if device is None:
            _check(self._lib.kate_merge_gates(self._h, int(begin), int(end), q.ctypes.data_as(_ip), ctypes.byref(k),
                                              d.ctypes.data_as(_dp)))
        else:
            _check(self._lib.kate_merge_gates_device(self._h, int(begin), int(end), int(device),
                                                     ctypes.c_void_p(int(stream)), q.ctypes.data_as(_ip),
                                                     ctypes.byref(k), d.ctypes.data_as(_dp)))
        dim = 1 << k.value
        return Gate(d[: 2 * dim * dim].view(np.complex128).reshape(dim, dim).copy(), [int(x) for x in q[: k.value]])


def release_cached_memory(device: int = -1):
    """Frees the device buffer kept for reuse after a simulator or batch was
    destroyed (kate_release_cached_memory); device -1: every device."""
    _check(_lib.lib().kate_release_cached_memory(int(device)))


def devices():
    """The CUDA devices: a list of (name, global memory bytes, shared memory
    per block, SM count); empty when no device answers."""
    L = _lib.lib()
    n = ctypes.c_int()
    _check(L.kate_device_count(ctypes.byref(n)))
    out = []
    for i in range(n.value):
        name = ctypes.create_string_buffer(256)
        gm, sm = ctypes.c_size_t(), ctypes.c_size_t()
        cnt = ctypes.c_int()
        _check(L.kate_device_properties(i, name, 256, ctypes.byref(gm), ctypes.byref(sm), ctypes.byref(cnt)))
        out.append((name.value.decode(), gm.value, sm.value, cnt.value))
    return out


def printGpuInfo():
    """printGpuInfo (HIPcode/DeviceInfo.hpp:10-35): host threads, the CUDA
    devices, device 0's memory in qubits of complex128 state."""
    import math
    print(f"CPU Info: {os.cpu_count()} threads")
    devs = devices()
    if not devs:
        print("couldnt detect devices, check permissions")
        return
    for i, d in enumerate(devs):
        print(f"GPU {i} : {d[0]}")
    print("-----------------------")
    name, gm, sm, cnt = devs[0]
    print(f"current GPU: \n{name} ({cnt} SMs)\n")
    print(f"Global memory: {gm} ({int(math.log2(gm / 16))} qbits)")
    print(f"Shared memory per block : {sm}\n")


def mergeGate(gates: Sequence[Gate], device: Optional[int] = None, stream: int = 0) -> Gate:
    """CPUmergeGate / mergeGate (CPUcode/GateMerger.hpp:8-55,
    HIPcode/GateMerger.hpp:43-109): FP64 product of the gates on the sorted
    union of their qubits; on CUDA device `device` when given (the same
    matrix, bit for bit)."""
    gs = [g if isinstance(g, Gate) else Gate(g[3] if g[0] == DENSE else g[0], g[1], g[2]) for g in gates]
    n = 1 + max(q for g in gs for q in g.qbits)
    c = Circuit(n, gs)
    return c.merge(0, len(gs), device=device, stream=stream)


class Simulator:
    """Kate::Simulator on one B200 (HIPcode/simulator.hpp:220-811)."""

    def __init__(self, circuit: Circuit, number_of_gpu: int = 1, precision: int = C128, device: int = 0):
        self._lib = _lib.lib()
        h = ctypes.c_void_p()
        _check(self._lib.kate_sim_create(circuit.handle, int(precision), int(device), ctypes.byref(h)))
        self._h = h
        v = ctypes.c_int()
        _check(self._lib.kate_sim_nqbits(self._h, ctypes.byref(v)))
        self.nqbits = v.value
        self.precision = precision

    def __del__(self):
        self.close()

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.kate_sim_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def execute(self, arg=False, displaytime: bool = False) -> proba_state:
        """execute(displaytime) or execute(proba_state_in, displaytime).
        With displaytime the phases the reference prints are timed and
        printed (HIPcode/simulator.hpp:346-350); ``last_times`` keeps them
        (init_ms, passes_ms, measure_ms, passes)."""
        out = np.zeros(2 * self.nqbits, dtype=np.float64)
        pin = None
        if isinstance(arg, proba_state):
            pin = arg.as_array().ravel().copy()
        else:
            displaytime = bool(arg) or displaytime
        if displaytime:
            ms = np.zeros(4, dtype=np.float64)
            _check(self._lib.kate_sim_execute_timed(self._h, None if pin is None else pin.ctypes.data_as(_dp),
                                                    out.ctypes.data_as(_dp), ms.ctypes.data_as(_dp)))
            self.last_times = tuple(float(x) for x in ms)
            print(f"Initialization/Measurement : {ms[0]:g} / {ms[2]:g} ms")
            print(f"Total computing time : {ms[1]:g} ms with swap% : 0%")
            print(f"Average swap time : 0 ms and average group time : {ms[1] / max(ms[3], 1):g} ms")
        elif pin is not None:
            _check(self._lib.kate_sim_execute_from(self._h, pin.ctypes.data_as(_dp), out.ctypes.data_as(_dp)))
        else:
            _check(self._lib.kate_sim_execute(self._h, out.ctypes.data_as(_dp)))
        return proba_state(out.reshape(-1, 2))

    def run_async(self, stream: int = 0):
        _check(self._lib.kate_sim_run_async(self._h, ctypes.c_void_p(stream or None)))

    def synchronize(self):
        _check(self._lib.kate_sim_synchronize(self._h))

    def proba(self) -> proba_state:
        out = np.zeros(2 * self.nqbits, dtype=np.float64)
        _check(self._lib.kate_sim_proba_state(self._h, out.ctypes.data_as(_dp)))
        return proba_state(out.reshape(-1, 2))

    def state(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The state in the reference's amplitude order (complex128)."""
        if out is None:
            out = np.empty(1 << self.nqbits, dtype=np.complex128)
        _check(self._lib.kate_sim_get_state(self._h, out.view(np.float64).ctypes.data_as(_dp)))
        return out

    def set_state(self, st: np.ndarray):
        a = np.ascontiguousarray(st, dtype=np.complex128)
        _check(self._lib.kate_sim_set_state(self._h, a.view(np.float64).ctypes.data_as(_dp)))

    def expect_z(self) -> np.ndarray:
        out = np.zeros(self.nqbits, dtype=np.float64)
        _check(self._lib.kate_sim_expect_z(self._h, out.ctypes.data_as(_dp)))
        return out

    def probabilities(self) -> np.ndarray:
        out = np.zeros(1 << self.nqbits, dtype=np.float64)
        _check(self._lib.kate_sim_probabilities(self._h, out.ctypes.data_as(_dp)))
        return out

    def sample(self, shots: int, seed: int = 0) -> np.ndarray:
        out = np.zeros(max(1, shots), dtype=np.uint64)
        _check(self._lib.kate_sim_sample(self._h, int(shots), ctypes.c_uint64(seed),
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out[:shots]

    def state_device(self):
        """(device pointer, physical bit of each qubit label)."""
        p = ctypes.c_void_p()
        phys = np.zeros(self.nqbits, dtype=np.int32)
        _check(self._lib.kate_sim_state_device(self._h, ctypes.byref(p), phys.ctypes.data_as(_ip)))
        return p.value, list(phys)

    def profile_passes(self):
        """(init_ms, [ms per pass]) from CUDA events between launches."""
        n = ctypes.c_int()
        _check(self._lib.kate_sim_num_passes(self._h, ctypes.byref(n)))
        ms = (ctypes.c_float * max(1, n.value))()
        init = ctypes.c_float()
        _check(self._lib.kate_sim_profile_passes(self._h, ms, ctypes.byref(init)))
        return init.value, [ms[i] for i in range(n.value)]

    def norm2_before_renorm(self) -> float:
        """Complex64: ||psi||^2 of the last run before it was rescaled to 1."""
        v = ctypes.c_double()
        _check(self._lib.kate_sim_norm2_before_renorm(self._h, ctypes.byref(v)))
        return v.value

    def pass_kernels(self) -> List[int]:
        """Kernel per pass: 0 generic, 1 interpreter, 2 pass-specialised, 3 complex64 blocks."""
        n = ctypes.c_int()
        _check(self._lib.kate_sim_num_passes(self._h, ctypes.byref(n)))
        out = []
        for i in range(n.value):
            k = ctypes.c_int()
            _check(self._lib.kate_sim_pass_kernel(self._h, i, ctypes.byref(k)))
            out.append(k.value)
        return out

    def pass_work(self) -> List[Optional[Tuple[float, float, float]]]:
        """Per pass, when its pass-specialised kernel runs it: (HBM bytes,
        FP64 instructions, shared-memory bytes) per amplitude; else None."""
        n = ctypes.c_int()
        _check(self._lib.kate_sim_num_passes(self._h, ctypes.byref(n)))
        out = []
        for i in range(n.value):
            v = (ctypes.c_double * 3)()
            st = self._lib.kate_sim_pass_work(self._h, i, v)
            out.append((v[0], v[1], v[2]) if st == 0 else None)
        return out

    def launches_per_run(self) -> int:
        v = ctypes.c_int()
        _check(self._lib.kate_sim_launches_per_run(self._h, ctypes.byref(v)))
        return v.value

    def passes(self):
        n = ctypes.c_int()
        _check(self._lib.kate_sim_num_passes(self._h, ctypes.byref(n)))
        out = []
        q = np.zeros(16, dtype=np.int32)
        m, ng = ctypes.c_int(), ctypes.c_int()
        for i in range(n.value):
            _check(self._lib.kate_sim_get_pass(self._h, i, q.ctypes.data_as(_ip), ctypes.byref(m), ctypes.byref(ng)))
            out.append(([int(x) for x in q[: m.value]], ng.value))
        return out


__all__ = ["Gate", "Circuit", "Simulator", "mergeGate", "release_cached_memory", "devices", "printGpuInfo", "proba_state", "KateError", "Hadamard", "CNOT", "CRk",
           "TOFFOLI", "RX", "RZ", "DENSE", "C128", "C64"]


class Batch:
    """Many independent circuits in one persistent-kernel launch (one CUDA
    graph). Outputs <Z_q> per qubit of every circuit.

    ``options``: a ``_lib.BatchOptions`` (``None``: defaults); with
    ``autotune=True`` the options are first tuned on the device for the qubit
    counts present (``self.options`` holds the result).
    """

    def __init__(self, circuits: Sequence[Circuit], precision: int = C64, device: int = 0, options=None,
                 autotune: bool = False):
        self._lib = _lib.lib()
        self._h = None
        self.circuits = list(circuits)
        self.nqbits = [c.nqbits for c in self.circuits]
        arr = (ctypes.c_void_p * len(self.circuits))(*[c.handle.value for c in self.circuits])
        if options is None:
            options = _lib.BatchOptions()
            _check(self._lib.kate_batch_options_default(ctypes.byref(options)))
        if autotune:
            _check(self._lib.kate_batch_autotune(arr, len(self.circuits), int(precision), int(device),
                                                 ctypes.byref(options)))
        self.options = options
        h = ctypes.c_void_p()
        _check(self._lib.kate_batch_create(arr, len(self.circuits), int(precision), int(device),
                                           ctypes.byref(options), ctypes.byref(h)))
        self._h = h
        v = ctypes.c_longlong()
        _check(self._lib.kate_batch_num_outputs(self._h, ctypes.byref(v)))
        self.num_outputs = v.value

    def __del__(self):
        self.close()

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.kate_batch_destroy(h)
            self._h = None

    def run_async(self, stream: int = 0):
        _check(self._lib.kate_batch_run_async(self._h, ctypes.c_void_p(stream or None)))

    def synchronize(self):
        _check(self._lib.kate_batch_synchronize(self._h))

    def run(self):
        _check(self._lib.kate_batch_run(self._h))

    def expect_z_flat(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.zeros(self.num_outputs, dtype=np.float64)
        _check(self._lib.kate_batch_expect_z(self._h, out.ctypes.data_as(_dp)))
        return out

    def expect_z(self) -> List[np.ndarray]:
        flat = self.expect_z_flat()
        res, o = [], 0
        for n in self.nqbits:
            res.append(flat[o:o + n].copy())
            o += n
        return res

    def info(self) -> dict:
        v = (ctypes.c_longlong * 4)()
        _check(self._lib.kate_batch_info(self._h, v))
        nb = ctypes.c_longlong()
        _check(self._lib.kate_batch_block_programs(self._h, ctypes.byref(nb)))
        return {"tasks": v[0], "programs": v[1], "arena_bytes": v[2], "ctas": v[3], "block_programs": nb.value}

    def create_times(self) -> dict:
        """Host wall time of the batch's creation, in ms, per phase."""
        v = (ctypes.c_double * 4)()
        _check(self._lib.kate_batch_create_times(self._h, v))
        return {"plan": v[0], "assemble": v[1], "upload": v[2], "graph": v[3]}

    def upload_bytes(self) -> int:
        """Host-to-device bytes copied when the batch was created."""
        v = ctypes.c_longlong()
        _check(self._lib.kate_batch_upload_bytes(self._h, ctypes.byref(v)))
        return v.value

    def state(self, i: int) -> np.ndarray:
        """Final state of circuit i (resident circuits only) in its qubit labels, complex128."""
        n = self.nqbits[i]
        out = np.empty(1 << n, dtype=np.complex128)
        _check(self._lib.kate_batch_get_state(self._h, int(i), out.view(np.float64).ctypes.data_as(_dp)))
        return out

    def circuit_info(self):
        """(pass programs, resident qubits) per circuit; resident qubits is 0
        for circuits run in shared memory."""
        n = len(self.circuits)
        p = np.zeros(n, dtype=np.int32)
        r = np.zeros(n, dtype=np.int32)
        _check(self._lib.kate_batch_circuit_info(self._h, p.ctypes.data_as(_ip), r.ctypes.data_as(_ip)))
        return p, r

    def time(self, runs: int = 1) -> float:
        ms = ctypes.c_float()
        _check(self._lib.kate_batch_time(self._h, int(runs), ctypes.byref(ms)))
        return ms.value


class Server:
    """Continuous-batching request server on one GPU (see kate_server_* in
    include/kate_b200.h). ``submit`` returns a request id at once; ``wait``
    returns ``(z, samples, times)`` with times = (submitted, admitted, done)
    in seconds on the server's clock."""

    def __init__(self, precision: int = C64, device: int = 0, options=None, **kw):
        self._lib = _lib.lib()
        self._h = None
        if options is None:
            options = _lib.ServerOptions()
            _check(self._lib.kate_server_options_default(ctypes.byref(options)))
        for k, v in kw.items():
            setattr(options, k, v)
        self.options = options
        h = ctypes.c_void_p()
        _check(self._lib.kate_server_create(int(precision), int(device), ctypes.byref(options), ctypes.byref(h)))
        self._h = h
        self._meta = {}

    def __del__(self):
        self.close()

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.kate_server_destroy(h)
            self._h = None

    def submit(self, circuit: Circuit, shots: int = 1024, seed: int = 0) -> int:
        v = ctypes.c_longlong()
        _check(self._lib.kate_server_submit(self._h, circuit.handle, int(shots), ctypes.c_uint64(seed & (2**64 - 1)),
                                            ctypes.byref(v)))
        self._meta[v.value] = (circuit.nqbits, int(shots))
        return v.value

    def wait(self, rid: int, timeout: float = 60.0):
        n, shots = self._meta[rid]
        z = np.zeros(n, dtype=np.float64)
        s = np.zeros(max(1, shots), dtype=np.uint64)
        t = np.zeros(3, dtype=np.float64)
        nq = ctypes.c_int()
        _check(self._lib.kate_server_wait(self._h, int(rid), float(timeout), ctypes.byref(nq), z.ctypes.data_as(_dp),
                                          s.ctypes.data_as(_u64p), t.ctypes.data_as(_dp)))
        del self._meta[rid]
        return z, s[:shots], tuple(t)

    def stats(self) -> dict:
        v = (ctypes.c_longlong * 12)()
        _check(self._lib.kate_server_stats(self._h, v))
        keys = ("submitted", "completed", "live", "queued", "steps", "resident_bytes", "peak_resident_bytes", "failed",
                "us_admit", "us_build", "us_kernel", "us_collect")
        return dict(zip(keys, list(v)))

    def now(self) -> float:
        t = ctypes.c_double()
        _check(self._lib.kate_server_now(self._h, ctypes.byref(t)))
        return t.value

