"""Seeded workload circuits, as gate tuples ``(id, qbits, optarg, dense)``.

Angles come from splitmix64 (a named, portable PRNG): u = (x >> 11) * 2^-53,
angle = 2*pi*u. Rotations are passed as dense gates, because the reference's
RX/RZ identifiers have no arithmetic (CPUcode/GateComputing.hpp:7-128).

* ``layered``: per layer RX(theta_q) on every qubit, RZ(phi_q) on every qubit,
  then the CNOT ladder Gate(CNOT, {q, q+1}) for q = 0..n-2 (Kate's order:
  qbits[0] = q is the target, qbits[1] = q+1 the control). 3n-1 gates/layer.
* ``brickwork_su4``: Haar-random SU(4) (QR of a seeded complex Gaussian with
  the diagonal-phase correction) on pairs (2i, 2i+1) in even layers and
  (2i+1, 2i+2) in odd layers.
* ``hea``: hardware-efficient ansatz, per layer RY(theta), RZ(phi) on every
  qubit then CZ brickwork, depth given.
* ``qulacs_bench``: the reference's benchmark circuit structure
  (BenchCircuits.hpp:8-42): H/CNOT-ring layers, 41*n gates.
* ``qft``: the reference's QFT structure (BenchCircuits.hpp:44-58).
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / (1 << 53))

    def angle(self) -> float:
        return 2.0 * math.pi * self.uniform()


def rx(t: float) -> np.ndarray:
    c, s = math.cos(t / 2), math.sin(t / 2)
    return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)


def ry(t: float) -> np.ndarray:
    c, s = math.cos(t / 2), math.sin(t / 2)
    return np.array([[c, -s], [s, c]], dtype=np.complex128)


def rz(p: float) -> np.ndarray:
    return np.array([[complex(math.cos(-p / 2), math.sin(-p / 2)), 0], [0, complex(math.cos(p / 2), math.sin(p / 2))]],
                    dtype=np.complex128)


CZ = np.diag([1, 1, 1, -1]).astype(np.complex128)


def layered(n: int, layers: int, seed: int = 1234) -> List[Tuple]:
    rng = SplitMix64(seed)
    gates = []
    for _ in range(layers):
        th = [rng.angle() for _ in range(n)]
        ph = [rng.angle() for _ in range(n)]
        for q in range(n):
            gates.append((0, [q], 0, rx(th[q])))
        for q in range(n):
            gates.append((0, [q], 0, rz(ph[q])))
        for q in range(n - 1):
            gates.append((3, [q, q + 1], 0, None))
    return gates


def haar_su4(rng: np.random.Generator) -> np.ndarray:
    z = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    q = q * (d / np.abs(d))
    q = q / np.linalg.det(q) ** 0.25
    return np.ascontiguousarray(q)


def brickwork_su4(n: int, layers: int, seed: int = 1234) -> List[Tuple]:
    rng = np.random.default_rng(seed)
    gates = []
    for l in range(layers):
        start = l % 2
        for a in range(start, n - 1, 2):
            gates.append((0, [a, a + 1], 0, haar_su4(rng)))
    return gates


def splitmix_angles(seed: int, count: int) -> np.ndarray:
    """The first `count` SplitMix64(seed).angle() values, vectorised."""
    k = np.arange(1, count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & MASK64) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return 2.0 * math.pi * ((z >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53)))


def hea_flat(n: int, depth: int, seed: int = 1234):
    """``hea`` as flat arrays (ids, nqs, qbits, optargs, dense) for
    Circuit.appendFlat: per layer RY(theta_q) for every q, RZ(phi_q) for
    every q, then CZ on (a, a+1), a = l % 2, l % 2 + 2, ..."""
    ang = splitmix_angles(seed, 2 * n * depth).reshape(depth, 2, n)
    ids, nqs, qb, dense = [], [], [], []
    cz = CZ.ravel()
    for l in range(depth):
        t = ang[l, 0] / 2
        c, s_ = np.cos(t), np.sin(t)
        ryd = np.stack([c, -s_, s_, c], axis=1).astype(np.complex128)
        p = ang[l, 1] / 2
        rzd = np.zeros((n, 4), dtype=np.complex128)
        rzd[:, 0] = np.cos(-p) + 1j * np.sin(-p)
        rzd[:, 3] = np.cos(p) + 1j * np.sin(p)
        pairs = list(range(l % 2, n - 1, 2))
        ids += [0] * (2 * n + len(pairs))
        nqs += [1] * (2 * n) + [2] * len(pairs)
        qb += list(range(n)) + list(range(n))
        for a in pairs:
            qb += [a, a + 1]
        dense += [ryd.ravel(), rzd.ravel()] + [cz] * len(pairs)
    nops = len(ids)
    return (np.array(ids, np.int32), np.array(nqs, np.int32), np.array(qb, np.int32), np.zeros(nops, np.int32),
            np.concatenate(dense))


def hea(n: int, depth: int, seed: int = 1234) -> List[Tuple]:
    ids, nqs, qb, _, dense = hea_flat(n, depth, seed)
    gates, qo, do = [], 0, 0
    for k in range(len(ids)):
        q = [int(x) for x in qb[qo:qo + nqs[k]]]
        dim = 1 << int(nqs[k])
        gates.append((0, q, 0, dense[do:do + dim * dim].reshape(dim, dim).copy()))
        qo += int(nqs[k])
        do += dim * dim
    return gates


def qulacs_bench(n: int) -> List[Tuple]:
    g = []
    for i in range(n):
        g += [(2, [i], 0, None), (2, [i], 0, None)]
    for i in range(n):
        g.append((3, [i, (i + 1) % n], 0, None))
    for _ in range(9):
        for i in range(n):
            g += [(2, [i], 0, None)] * 3
        for i in range(n):
            g.append((3, [i, (i + 1) % n], 0, None))
    for i in range(n):
        g += [(2, [i], 0, None), (2, [i], 0, None)]
    return g


def qft(n: int) -> List[Tuple]:
    g = []
    for i in range(n):
        g.append((2, [i], 0, None))
        for j in range(i + 1, n):
            g.append((4, [j, i], j - i + 1, None))
    return g
