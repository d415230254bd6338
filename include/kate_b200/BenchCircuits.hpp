// BenchCircuits.hpp - the reference's benchmark circuit generators
// (Line-fr/Kate: BenchCircuits.hpp:8-123) over the kate_b200 facade, so a
// program that includes "BenchCircuits.hpp" next to "Kate.hpp" builds
// unchanged against this library. The gate sequences are the reference's
// (they define the benchmarks); the code is this library's.
#ifndef KATE_B200_BENCHCIRCUITS_HPP
#define KATE_B200_BENCHCIRCUITS_HPP

#include <cstdlib>
#include <ctime>
#include <vector>

#include "Kate.hpp"

namespace Kate {

namespace bench_detail {
inline void one(Circuit& c, int id, int q) {
    std::vector<int> v{q};
    c.appendGate(Gate(id, v, 0));
}
inline void ring(Circuit& c, int n) {
    for (int i = 0; i < n; i++) {
        std::vector<int> v{i, (i + 1) % n};
        c.appendGate(Gate(CNOT, v));
    }
}
}  // namespace bench_detail

// QulacsBench (BenchCircuits.hpp:8-42): H twice on every qubit and a CNOT
// ring, nine rounds of H three times and a ring, then H twice: 41 n gates.
inline Circuit QulacsBench(int qbitsNum) {
    Circuit c(qbitsNum);
    for (int i = 0; i < qbitsNum; i++)
        for (int r = 0; r < 2; r++) bench_detail::one(c, Hadamard, i);
    bench_detail::ring(c, qbitsNum);
    for (int round = 0; round < 9; round++) {
        for (int i = 0; i < qbitsNum; i++)
            for (int r = 0; r < 3; r++) bench_detail::one(c, Hadamard, i);
        bench_detail::ring(c, qbitsNum);
    }
    for (int i = 0; i < qbitsNum; i++)
        for (int r = 0; r < 2; r++) bench_detail::one(c, Hadamard, i);
    return c;
}

// QFT (BenchCircuits.hpp:44-58): H on qubit i, then CRk(j - i + 1) with
// control j for every j > i.
inline Circuit QFT(int qbitsNum) {
    Circuit c(qbitsNum);
    for (int i = 0; i < qbitsNum; i++) {
        bench_detail::one(c, Hadamard, i);
        for (int j = i + 1; j < qbitsNum; j++) {
            std::vector<int> v{j, i};
            c.appendGate(Gate(CRk, v, j - i + 1));
        }
    }
    return c;
}

// randomCircuit (BenchCircuits.hpp:60-118): depth gates, each with equal
// odds an H, a 2-qubit gate (CNOT or an all-ones 4x4) or a 3-qubit gate
// (TOFFOLI or an all-ones 8x8) on distinct random qubits; the matrices only
// serve timing. Seeded from the clock like the reference. Below 3 (2)
// qubits the 3-qubit (2-qubit) kinds are not drawn: the reference's draw
// of distinct qubits would never end there.
inline Circuit randomCircuit(int qbitsNum, int depth) {
    std::srand((unsigned)std::time(nullptr));
    Circuit c(qbitsNum);
    Matrix<Complex> m2(4), m3(8);
    m2.fill(Complex(1.0));
    m3.fill(Complex(1.0));
    auto pick_other = [&](const std::vector<int>& used) {
        int q;
        bool clash;
        do {
            q = std::rand() % qbitsNum;
            clash = false;
            for (int u : used) clash = clash || u == q;
        } while (clash);
        return q;
    };
    for (int d = 0; d < depth; d++) {
        const int kind = std::rand() % (qbitsNum < 3 ? qbitsNum : 3);
        std::vector<int> q{std::rand() % qbitsNum};
        if (kind == 0) {
            c.appendGate(Gate(Hadamard, q));
            continue;
        }
        q.push_back(pick_other(q));
        if (kind == 2) q.push_back(pick_other(q));
        const bool sparse = std::rand() % 2 == 1;
        if (sparse) c.appendGate(Gate(kind == 1 ? CNOT : TOFFOLI, q));
        else c.appendGate(Gate(kind == 1 ? m2 : m3, q));
    }
    return c;
}

}  // namespace Kate

#endif  // KATE_B200_BENCHCIRCUITS_HPP
