// Reference-style user program (cf. the reference's main.cpp) compiled
// against the kate_b200 facade. Without a GPU it exercises the circuit API
// and passes; with one it also simulates (argv[1] == "sim").
#include <kate_b200/Kate.hpp>

#include <cmath>
#include <cstring>

using namespace Kate;

int main(int argc, char** argv) {
    // The reference's Complex / Matrix arithmetic (basic_host_types.hpp).
    const double r = 1.0 / std::sqrt(2.0);
    Matrix<Complex> h(2);
    h(0, 0, Complex(r));
    h(0, 1, Complex(r));
    h(1, 0, Complex(r));
    h(1, 1, Complex(-r));
    Matrix<Complex> hh = h * h;
    hh.transpose();
    hh *= 2.0;
    Matrix<Complex> d = hh - h;
    d += h;
    Complex z = Complex(1, 2) / Complex(3, 4);
    z += Complex(1);
    z *= Complex(0, 1);
    z *= 2.0;
    std::cout << "arith " << d(0, 0).a << " " << d(0, 1).a << " " << z.a << " " << z.b << " "
              << Complex(1, 1).angle() << std::endl;
    int n = 10;
    Circuit circuit(n);
    std::vector<int> qbits;
    for (int i = 0; i < n; i++) {
        qbits = {i};
        circuit.appendGate(Gate(Hadamard, qbits, 0));
        circuit.appendGate(Gate(Hadamard, qbits, 0));
    }
    for (int i = 0; i < n; i++) {
        qbits = {i, (i + 1) % n};
        circuit.appendGate(Gate(CNOT, qbits));
    }
    qbits = {1, 3};
    circuit.appendGate(Gate(CRk, qbits, 3));
    Matrix<Complex> m(2);
    m(0, 0, Complex(0.0));
    m(0, 1, Complex(1.0));
    m(1, 0, Complex(1.0));
    m(1, 1, Complex(0.0));
    qbits = {4};
    circuit.appendGate(Gate(m, qbits));
    qbits = {5};
    circuit.appendGate(Gate(Hadamard, m, qbits));  // the id decides: a Hadamard
    circuit.gateScheduling();
    circuit.gateFusion(5, 1e-6);
    circuit.gateGrouping(8);
    circuit.compileDefault(0);
    std::cout << "gates " << circuit.gateCount() << std::endl;
    if (argc > 1 && std::strcmp(argv[1], "sim") == 0) {
        auto res = Simulator(circuit, 1).execute(true);
        res.print();
    }
    return last_status() == KATE_OK ? 0 : 1;
}
