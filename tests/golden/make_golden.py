"""Generates the committed golden fixtures from the reference's own CPU path.

Run where the reference headers exist (they are compiled into
oracle/_ref/libkate_ref.so by oracle/Makefile):

    make -C oracle ref && python tests/golden/make_golden.py

Outputs (small, committed):
  states.npz   per case: gate list, final state (CPUSimulator::qbitstate)
               and proba_state of the reference, for execute() and
               execute(proba_state&)
  passes.npz   gate lists, groups, instructions and permutations after the
               reference's gateScheduling / gateFusion / gateGrouping /
               allocate / compileDefault on seeded circuits
  merge.npz    CPUmergeGate results
  circuit.qcx  exportqcx output of a small circuit
  print_qulacs4.txt  QuantumCircuit::print output (grouped, with swaps,
               compiled); ``make_golden.py print`` rewrites only this file
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from common import random_circuit  # noqa: E402
from kate_b200 import circuits  # noqa: E402
from oracle.oracle import Ref, flatten  # noqa: E402


def pack(prefix, gates, out):
    ids, nqs, qb, opt, dense = flatten(gates)
    out[prefix + "ids"] = ids
    out[prefix + "nqs"] = nqs
    out[prefix + "qbits"] = qb
    out[prefix + "optargs"] = opt
    out[prefix + "dense"] = dense


def unpack(prefix, d):
    ids, nqs, qb, opt, dense = (d[prefix + k] for k in ("ids", "nqs", "qbits", "optargs", "dense"))
    gates, qi, di = [], 0, 0
    for g in range(len(ids)):
        k = int(nqs[g])
        q = [int(x) for x in qb[qi:qi + k]]
        qi += k
        m = None
        if ids[g] == 0:
            dim = 1 << k
            m = dense[di:di + 2 * dim * dim].view(np.complex128).reshape(dim, dim).copy()
            di += 2 * dim * dim
        gates.append((int(ids[g]), q, int(opt[g]), m))
    return gates


def state_cases():
    rng = np.random.default_rng(2024)
    return {
        "layered_n10_l3": (10, circuits.layered(10, 3, seed=1234), None),
        "qft_n8": (8, circuits.qft(8), None),
        "qulacs_n9": (9, circuits.qulacs_bench(9), None),
        "random_n8": (8, random_circuit(8, 70, rng), None),
        "random_n11": (11, random_circuit(11, 90, rng), None),
        "hea_n9": (9, circuits.hea(9, 4, seed=5), None),
        "brick_n8": (8, circuits.brickwork_su4(8, 4, seed=5), None),
        "product_n7": (7, random_circuit(7, 40, rng),
                       np.stack([rng.uniform(0, 1, 7), rng.uniform(-np.pi, np.pi, 7)], axis=1)),
    }


def main():
    ref = Ref()
    st = {}
    names = []
    for name, (n, gates, pin) in state_cases().items():
        c = ref.circuit(n, gates)
        state, proba, _ = c.simulate(proba_in=pin)
        pack(name + "/", gates, st)
        st[name + "/n"] = np.int32(n)
        st[name + "/state"] = state
        st[name + "/proba"] = proba
        if pin is not None:
            st[name + "/proba_in"] = pin
        names.append(name)
    st["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "states.npz"), **st)

    ps = {}
    pnames = []
    rng = np.random.default_rng(77)
    for i in range(8):
        n = int(rng.integers(3, 11))
        gates = random_circuit(n, int(rng.integers(5, 40)), rng)
        k = int(rng.integers(2, 6))
        mtm = [0.0, 1e-6, 1.0][i % 3]
        m = int(rng.integers(5, 10))
        alloc = i % 2 == 1
        c = ref.circuit(n, gates)
        name = f"case{i}"
        pack(name + "/in/", gates, ps)
        c.schedule()
        pack(name + "/sched/", c.gates(), ps)
        c.fuse(k, mtm)
        pack(name + "/fused/", c.gates(), ps)
        c.group(m)
        ps[name + "/groups"] = np.array(json.dumps(c.groups()))
        if alloc:
            c.allocate(0)
        else:
            c.compile_default(0)
        pack(name + "/compiled/", c.gates(), ps)
        ps[name + "/instructions"] = np.array(json.dumps(c.instructions()))
        a, b = c.perms()
        ps[name + "/perms"] = np.array(json.dumps([[int(x) for x in a], [int(x) for x in b]]))
        ps[name + "/params"] = np.array([n, k, m, int(alloc)], dtype=np.int64)
        ps[name + "/mtm"] = np.float64(mtm)
        pnames.append(name)
    ps["names"] = np.array(pnames)
    np.savez_compressed(os.path.join(HERE, "passes.npz"), **ps)

    mg = {}
    rng = np.random.default_rng(99)
    mnames = []
    for i in range(6):
        n = 6
        gates = random_circuit(n, 8, rng, kinds=("h", "cnot", "crk", "toff", "d1", "d2"))
        c = ref.circuit(n, gates)
        q, m = c.merge(0, len(gates))
        if len(q) > 5:
            continue
        name = f"merge{i}"
        pack(name + "/gates/", gates, mg)
        mg[name + "/qbits"] = np.array(q, dtype=np.int32)
        mg[name + "/mat"] = m
        mnames.append(name)
    mg["names"] = np.array(mnames)
    np.savez_compressed(os.path.join(HERE, "merge.npz"), **mg)

    c = ref.circuit(5, [(2, [0], 0, None), (3, [1, 2], 0, None), (4, [3, 0], 3, None), (5, [0, 1, 4], 0, None),
                        (0, [2, 3], 0, np.eye(4, dtype=np.complex128))])
    c.export_qcx(os.path.join(HERE, "circuit.qcx"))
    write_print_golden(ref)
    print("golden fixtures written to", HERE)


def write_print_golden(ref):
    """print_qulacs4.txt: QuantumCircuit::print of the first 12 gates of the
    4-qubit QulacsBench circuit as appended, of the whole circuit after
    gateScheduling + gateGrouping(3), then with permutation
    tables after allocate(1) (swap instructions), then after
    compileDefault(0)."""
    path = os.path.join(HERE, "print_qulacs4.txt")
    if os.path.exists(path):
        os.remove(path)
    gates = circuits.qulacs_bench(4)
    ref.circuit(4, gates[:12]).print_to(path)  # the first 3n gates, ungrouped: "gate i is ..."

    def grouped():
        c = ref.circuit(4, gates)
        c.schedule()
        c.group(3)
        return c

    grouped().print_to(path)
    s = grouped()
    s.allocate(1)
    s.print_to(path, True)
    c = grouped()
    c.compile_default(0)
    c.print_to(path, False)


if __name__ == "__main__" and sys.argv[1:] == ["print"]:
    from oracle.oracle import Ref as _Ref  # noqa: E402
    write_print_golden(_Ref())
elif __name__ == "__main__":
    main()
