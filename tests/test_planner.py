"""The group-pass planner, checked on the CPU: plans are executed by a numpy
emulation of the kernel semantics (tests/plan_emulator.py) and compared with
the oracle; structural invariants are checked directly."""
import numpy as np
import pytest

import kate_b200 as K
from kate_b200 import circuits
from common import random_circuit
from plan_emulator import PlanView

NO_REMAP, NO_FUSE1Q, REMAP_SEARCH = 1, 2, 16


def zero_state(n):
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1
    return s


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("opts", [(6, 2, 0), (8, 3, NO_REMAP), (5, 4, NO_FUSE1Q), (12, 4, 0), (4, 1, 0),
                                  (12, 4, REMAP_SEARCH), (6, 2, REMAP_SEARCH)])
def test_emulated_plan_matches_oracle(oracle, seed, opts):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 12))
    mt, co, fl = opts
    mt = min(mt, n)
    kinds = ("h", "cnot", "crk", "toff", "d1", "d2", "d3", "diag1", "diag2", "d5")
    kinds = tuple(k for k in kinds if not (k == "d5" and mt < 5) and not (k == "d3" and mt < 3))
    gates = random_circuit(n, int(rng.integers(1, 70)), rng, kinds=kinds)
    pv = PlanView(K.Circuit(n, gates), mt, min(co, mt), fl)
    out = pv.run(zero_state(n))
    assert np.abs(out - oracle.simulate(n, gates)).max() <= 1e-12


def test_layered_n20_plan_matches_oracle(oracle):
    n = 20
    gates = circuits.layered(n, 10, seed=1234)
    pv = PlanView(K.Circuit(n, gates), 12, 4, 0)
    assert np.abs(pv.run(zero_state(n)) - oracle.simulate(n, gates)).max() <= 1e-12


def test_qulacs_bench_ring_plan_matches_oracle(oracle):
    # The reference's benchmark circuit closes its CNOT ring with
    # (n-1, 0): the tile of that gate holds the lowest and highest qubit.
    n = 16
    gates = circuits.qulacs_bench(n)
    pv = PlanView(K.Circuit(n, gates), 12, 4, 0)
    assert np.abs(pv.run(zero_state(n)) - oracle.simulate(n, gates)).max() <= 1e-12


def test_every_pass_keeps_the_low_bits_in_the_tile():
    n = 24
    pv = PlanView(K.Circuit(n, circuits.layered(n, 4)), 12, 4, 0)
    for p in pv.passes:
        assert p["tphys"][:4] == [0, 1, 2, 3]
        assert sorted(p["outsrc"]) == list(range(p["m"]))
        assert p["tphys"] == sorted(p["tphys"])
    assert sorted(pv.final_phys) == list(range(n))


def test_headline_plan_pass_count():
    # 30 qubits, 20 layers of RX/RZ/CNOT ladder with 12-qubit tiles: about
    # three passes per layer (each pass advances the ladder by ~11 qubits).
    pv = PlanView(K.Circuit(30, circuits.layered(30, 20)), 12, 4, 0)
    assert len(pv.passes) <= 62
    ops = sum(p["nops"] for p in pv.passes)
    # RX and RZ stay separate (an RX-form 2x2 plus a diagonal that merges
    # into the stage's register diagonal is cheaper than one general 2x2).
    assert ops == 20 * (3 * 30 - 1)


def test_remap_search_packs_the_headline_into_fewer_passes():
    # Trying every 4-subset of the tile for the low bits lets each pass hold
    # the qubits the next one works on, and the gate cap is chosen among
    # 96..144: the 20-layer ladder takes 20 passes instead of 58, with the
    # same ops, every low bit still a tile bit, every pass register-staged.
    base = PlanView(K.Circuit(30, circuits.layered(30, 20)), 12, 4, 0)
    pv = PlanView(K.Circuit(30, circuits.layered(30, 20)), 12, 4, REMAP_SEARCH)
    assert len(pv.passes) <= 21 < len(base.passes)
    assert sum(p["nops"] for p in pv.passes) == sum(p["nops"] for p in base.passes)
    assert all(p is not None for p in pv.programs)
    for p in pv.passes:
        assert p["tphys"][:4] == [0, 1, 2, 3]
        assert p["nops"] <= 144


def test_remap_search_keeps_dense_two_qubit_gates_in_registers():
    # A pass that packs more SU(4)s than the register program's matrix pool
    # holds is planned again with fewer gates instead of falling back to
    # shared-memory ops (which the pass-specialised kernels do not run).
    SOP_SMEM = 2
    pv = PlanView(K.Circuit(32, circuits.brickwork_su4(32, 20)), 12, 4, REMAP_SEARCH)
    base = PlanView(K.Circuit(32, circuits.brickwork_su4(32, 20)), 12, 4, 0)
    assert len(pv.passes) < len(base.passes)
    for prog in pv.programs:
        assert prog is not None
        kinds = prog["ops"]["kind"][: int(prog["nops"])]
        assert not (kinds == SOP_SMEM).any()


def test_remap_search_layered_matches_oracle(oracle):
    n = 22
    gates = circuits.layered(n, 8, seed=5)
    pv = PlanView(K.Circuit(n, gates), 12, 4, REMAP_SEARCH)
    assert np.abs(pv.run_staged(zero_state(n)) - oracle.simulate(n, gates)).max() <= 1e-12


def test_single_qubit_chains_are_fused_when_cheaper(oracle):
    rx, rz, ry = circuits.rx, circuits.rz, circuits.ry
    gates = [(0, [0], 0, rx(0.3)), (0, [0], 0, rx(0.4)),      # RX.RX -> RX form: fused
             (0, [1], 0, rz(0.3)), (0, [1], 0, rz(0.9)),      # diagonal: fused
             (0, [2], 0, rx(0.3)), (0, [2], 0, rz(0.9)),      # general product: kept apart
             (2, [3], 0, None), (2, [3], 0, None)]            # H.H = identity: fused
    pv = PlanView(K.Circuit(4, gates), 4, 2, 0)
    assert sum(p["nops"] for p in pv.passes) == 1 + 1 + 2 + 1
    pv2 = PlanView(K.Circuit(4, gates), 4, 2, NO_FUSE1Q)
    assert sum(p["nops"] for p in pv2.passes) == 8
    assert np.abs(pv.run(zero_state(4)) - oracle.simulate(4, gates)).max() <= 1e-12


def test_diagonal_gates_may_sit_outside_the_tile(oracle):
    # CRk and diagonal dense gates act as free qubits: one pass suffices even
    # when they touch qubits outside a 4-qubit tile.
    n = 10
    gates = [(2, [q], 0, None) for q in range(4)] + [(4, [0, 9], 3, None), (4, [8, 7], 2, None),
                                                      (0, [9], 0, np.diag([1, 1j]))]
    pv = PlanView(K.Circuit(n, gates), 4, 2, 0)
    assert len(pv.passes) == 1
    assert np.abs(pv.run(zero_state(n)) - oracle.simulate(n, gates)).max() <= 1e-12


def test_swap_instructions_become_relabelings(oracle, ref):
    # allocate(g > 0) emits swap instructions (Circuit.hpp:207-348). On one
    # GPU a swap of positions p1, p2 is a relabeling; its meaning is a SWAP
    # gate on those positions in the program's label space.
    n = 8
    rng = np.random.default_rng(4)
    gates = random_circuit(n, 40, rng, kinds=("h", "cnot", "d1", "d2", "crk"))
    c = K.Circuit(n, gates)
    c.gateGrouping(5)
    c.allocate(2)
    ins = c.instructions
    assert any(k == 0 for k, _ in ins)
    swap = np.eye(4)[[0, 2, 1, 3]].astype(np.complex128)
    seq, gi, k0 = [], 0, 0
    comp = c.gate_set_ordered
    groups = c.groups
    for kind, qs in ins:
        if kind == 0:
            for a, b in zip(qs[::2], qs[1::2]):
                seq.append((0, [a, b], 0, swap))
        else:
            end = groups[gi][0]
            seq += comp[k0:end]
            k0, gi = end, gi + 1
    pv = PlanView(c, 6, 2, 0)
    assert np.abs(pv.run(zero_state(n)) - oracle.simulate(n, seq)).max() <= 1e-12


@pytest.mark.parametrize("seed", range(8))
def test_register_staged_programs_match_oracle(oracle, seed):
    rng = np.random.default_rng(300 + seed)
    n = int(rng.integers(12, 15))
    gates = random_circuit(n, 90, rng)
    pv = PlanView(K.Circuit(n, gates), 12, 4, 0)
    assert all(p is not None for p in pv.programs)
    assert np.abs(pv.run_staged(zero_state(n)) - oracle.simulate(n, gates)).max() <= 1e-12


def test_register_staged_layered_matches_oracle(oracle):
    n = 14
    gates = circuits.layered(n, 6, seed=3)
    pv = PlanView(K.Circuit(n, gates), 12, 4, 0)
    assert np.abs(pv.run_staged(zero_state(n)) - oracle.simulate(n, gates)).max() <= 1e-12


@pytest.mark.parametrize("seed", range(4))
def test_multi_qubit_diagonals_become_register_ops(oracle, seed):
    """k-qubit diagonals (CZ, random diagonal tables) lower to one-qubit
    diagonals and controlled phases, not shared-memory ops."""
    rng = np.random.default_rng(500 + seed)
    n = 13 + seed % 3
    gates = circuits.hea(n, 4, seed=seed) + random_circuit(n, 60, rng, kinds=("diag2", "diag1", "d1", "cnot"))
    pv = PlanView(K.Circuit(n, gates), 12, 4, 0)
    assert all(p is not None for p in pv.programs)
    assert pv.smem_ops == [] or len(pv.smem_ops) == 0
    assert np.abs(pv.run_staged(zero_state(n)) - oracle.simulate(n, gates)).max() <= 1e-12


@pytest.mark.parametrize("fuse", [True, False])
@pytest.mark.parametrize("seed", range(3))
def test_c64_block_programs_match_oracle(oracle, seed, fuse):
    """Complex64 plans: each pass's 5-qubit blocks, read back from their BF16
    hi/lo operand images and applied as the tensor-core kernel does, give the
    oracle's state (the image split keeps about 16 bits per entry); with and
    without the reference's gateFusion before planning."""
    rng = np.random.default_rng(700 + seed)
    n = 13 + seed
    gates = circuits.brickwork_su4(n, 6, seed=seed) + random_circuit(n, 40, rng, kinds=("h", "cnot", "crk", "d1", "d2"))
    c = K.Circuit(n, gates)
    if fuse:
        c.gateScheduling()
        c.gateFusion(5, 1e-6)
    pv = PlanView(c, 12, 4, 4)
    assert any(bp is not None for bp in pv.block_programs)
    got = pv.run_blocks(zero_state(n))
    ref = oracle.simulate(n, gates)
    a, b = got / np.linalg.norm(got), ref / np.linalg.norm(ref)
    assert 1 - abs(np.vdot(a, b)) ** 2 <= 1e-8
    assert np.abs(got - ref).max() <= 1e-4


def test_c64_block_selector_packs_light_cones():
    # 32-qubit SU(4) brickwork, 20 layers (310 gates): blocks of at most five
    # qubits, two per pass. Program-order prefixes gave 42 passes of 83
    # blocks; the light-cone selector 27 passes of 54 blocks.
    n = 32
    pv = PlanView(K.Circuit(n, circuits.brickwork_su4(n, 20, seed=1234)), 12, 4, 4)
    assert all(bp is not None for bp in pv.block_programs)
    nblocks = sum(int(bp["nblocks"]) for bp in pv.block_programs)
    assert len(pv.passes) <= 28 and nblocks <= 56, (len(pv.passes), nblocks)


def _warp_local_violations(prog):
    """Stage boundaries marked warp-local (STAGE op src = 1) must give the
    warp index (thread bits 5..7) the same tile bits in both stages, those
    bits must be register bits in neither, and no shared-memory op may sit
    between the two stages."""
    bad = []
    prev = None
    for k in range(int(prog["nops"])):
        op = prog["ops"][k]
        kind = int(op["kind"])
        if kind == 2:
            prev = None
        elif kind == 1:
            si = int(op["idx"])
            if int(op["src"]) == 1:
                if prev is None:
                    bad.append((k, "no open stage before"))
                else:
                    w0 = [int(x) for x in prog["stb"][prev][5:8]]
                    w1 = [int(x) for x in prog["stb"][si][5:8]]
                    regs = set(int(x) for x in prog["srb"][prev]) | set(int(x) for x in prog["srb"][si])
                    if w0 != w1 or regs & set(w1):
                        bad.append((k, w0, w1, sorted(regs)))
            prev = si
    return bad


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_warp_local_stage_boundaries_are_safe(oracle, seed):
    rng = np.random.default_rng(900 + seed)
    n = 18
    g = random_circuit(n, 200, rng)
    for c in (K.Circuit(n, g), K.Circuit(30, circuits.layered(30, 20, 1234))):
        pv = PlanView(c)
        marked = 0
        for prog in pv.programs:
            if prog is None:
                continue
            assert _warp_local_violations(prog) == []
            marked += sum(1 for k in range(int(prog["nops"])) if int(prog["ops"][k]["kind"]) == 1 and
                          int(prog["ops"][k]["src"]) == 1)
        if c.nqbits == 30:
            assert marked > 0
    st0 = np.zeros(1 << n, dtype=np.complex128)
    st0[0] = 1
    assert np.abs(PlanView(K.Circuit(n, g)).run_staged(st0) - oracle.simulate(n, g)).max() <= 1e-12


def test_factored_rotations_at_edge_angles(oracle):
    """RX / RY at angles where one factor vanishes or dominates (0, pi/2,
    pi, 3pi/2, and a random spread) run as factored rotations; the emulated
    program matches the oracle."""
    n = 13
    angles = [0.0, np.pi / 2, np.pi, 1.5 * np.pi, 2 * np.pi, 1e-9, np.pi - 1e-9]
    rng = np.random.default_rng(77)
    angles += list(rng.uniform(0, 2 * np.pi, 12))
    g = []
    for i, th in enumerate(angles):
        q = i % n
        g.append((0, [q], 0, circuits.rx(th)))
        g.append((0, [(q + 5) % n], 0, circuits.ry(th)))
        g.append((3, [q, (q + 1) % n], 0, None))
    pv = PlanView(K.Circuit(n, g))
    kinds = set()
    for prog in pv.programs:
        if prog is not None:
            kinds |= {int(prog["ops"][k]["kind"]) for k in range(int(prog["nops"]))}
    assert kinds & {13, 14, 15, 16}
    st0 = np.zeros(1 << n, dtype=np.complex128)
    st0[0] = 1
    assert np.abs(pv.run_staged(st0) - oracle.simulate(n, g)).max() <= 1e-12
