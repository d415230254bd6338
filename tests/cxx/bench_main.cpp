// The reference's main.cpp, without MPI, compiled against the kate_b200
// facade: printGpuInfo, QulacsBench, gateScheduling, gateGrouping(12),
// compileDefault, Simulator(circuit, 1).execute(true), res.print(). Without
// a GPU (argv[1] != "sim") it stops before the Simulator.
#include <kate_b200/BenchCircuits.hpp>
#include <kate_b200/Kate.hpp>

#include <algorithm>
#include <cstring>

using namespace Kate;

int main(int argc, char** argv) {
    const bool sim = argc > 1 && std::strcmp(argv[1], "sim") == 0;
    const int n = argc > 2 ? std::atoi(argv[2]) : 12;
    if (argc > 1 && std::strcmp(argv[1], "print") == 0) {
        // Circuit::print of plain gates, before compilation (grouped), then of two programs:
        // one with swap instructions (allocate(1)), one without.
        Circuit c = QulacsBench(n);
        Circuit head(n);  // the first 3n gates (H pairs, one CNOT ring), ungrouped
        for (int q = 0; q < n; q++) {
            std::vector<int> v{q};
            head.appendGate(Gate(Hadamard, v, 0));
            head.appendGate(Gate(Hadamard, v, 0));
        }
        for (int q = 0; q < n; q++) {
            std::vector<int> v{q, (q + 1) % n};
            head.appendGate(Gate(CNOT, v));
        }
        head.print();
        c.gateScheduling();
        c.gateGrouping(3);
        c.print();
        Circuit swapped = c;
        swapped.allocate(1);
        swapped.print(true);
        c.compileDefault(0);
        c.print(false);
        return last_status() == KATE_OK ? 0 : 1;
    }
    printGpuInfo();
    Circuit circuit = QulacsBench(n);
    std::cout << "qulacs gates " << circuit.gateCount() << std::endl;
    std::cout << "qft gates " << QFT(n).gateCount() << std::endl;
    std::cout << "random gates " << randomCircuit(n, 50).gateCount() << std::endl;
    circuit.gateScheduling();
    circuit.gateGrouping(std::min(12, n));
    circuit.compileDefault(0);
    if (sim) {
        auto res = Simulator(circuit, 1).execute(true);
        res.print();
    }
    std::cout << "done" << std::endl;
    return last_status() == KATE_OK ? 0 : 1;
}
