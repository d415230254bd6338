"""Seeded circuit generators for the tests (unitary gates only)."""
import numpy as np


def haar(dim, rng):
    z = (rng.standard_normal((dim, dim)) + 1j * rng.standard_normal((dim, dim))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return np.ascontiguousarray(q * (d / np.abs(d)))


def random_circuit(n, G, rng, kinds=("h", "cnot", "crk", "toff", "d1", "d2", "d3", "diag1", "diag2", "d5")):
    gates = []
    kinds = [k for k in kinds if not (k in ("toff", "d3") and n < 3) and not (k in ("cnot", "crk", "d2", "diag2") and n < 2)
             and not (k == "d5" and n < 5)]
    for _ in range(G):
        k = kinds[int(rng.integers(len(kinds)))]
        if k == "h":
            gates.append((2, [int(rng.integers(n))], 0, None))
        elif k == "cnot":
            a, b = rng.choice(n, 2, replace=False)
            gates.append((3, [int(a), int(b)], 0, None))
        elif k == "crk":
            a, b = rng.choice(n, 2, replace=False)
            gates.append((4, [int(a), int(b)], int(rng.integers(1, 8)), None))
        elif k == "toff":
            a, b, c = rng.choice(n, 3, replace=False)
            gates.append((5, [int(a), int(b), int(c)], 0, None))
        elif k in ("d1", "d2", "d3", "d5"):
            kk = int(k[1])
            q = [int(x) for x in rng.choice(n, kk, replace=False)]
            gates.append((0, q, 0, haar(1 << kk, rng)))
        elif k in ("diag1", "diag2"):
            kk = int(k[4])
            q = [int(x) for x in rng.choice(n, kk, replace=False)]
            gates.append((0, q, 0, np.diag(np.exp(1j * rng.uniform(0, 2 * np.pi, 1 << kk)))))
    return gates
