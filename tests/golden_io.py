"""Readers for the committed golden fixtures (tests/golden/*.npz)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


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


def load(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def state_cases():
    d = load("states.npz")
    for name in d["names"]:
        name = str(name)
        pin = d[name + "/proba_in"] if (name + "/proba_in") in d.files else None
        yield name, int(d[name + "/n"]), unpack(name + "/", d), d[name + "/state"], d[name + "/proba"], pin


def pass_cases():
    d = load("passes.npz")
    for name in d["names"]:
        name = str(name)
        n, k, m, alloc = (int(x) for x in d[name + "/params"])
        yield dict(name=name, n=n, k=k, m=m, alloc=bool(alloc), mtm=float(d[name + "/mtm"]),
                   gates=unpack(name + "/in/", d), sched=unpack(name + "/sched/", d),
                   fused=unpack(name + "/fused/", d), groups=json.loads(str(d[name + "/groups"])),
                   compiled=unpack(name + "/compiled/", d),
                   instructions=json.loads(str(d[name + "/instructions"])),
                   perms=json.loads(str(d[name + "/perms"])))


def merge_cases():
    d = load("merge.npz")
    for name in d["names"]:
        name = str(name)
        yield name, unpack(name + "/gates/", d), [int(x) for x in d[name + "/qbits"]], d[name + "/mat"]


def same_gates(a, b, exact=True):
    """Gate lists equal: ids, qubits, optargs (not for dense gates, whose
    optarg the reference leaves uninitialised) and matrices (bit-exact)."""
    if len(a) != len(b):
        return False
    for x, y in zip(a, b):
        if x[0] != y[0] or list(x[1]) != list(y[1]):
            return False
        if x[0] != 0 and x[2] != y[2]:
            return False
        if x[0] == 0:
            if exact and not np.array_equal(x[3], y[3]):
                return False
            if not exact and not np.allclose(x[3], y[3], atol=1e-13):
                return False
    return True
