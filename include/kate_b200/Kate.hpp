// Kate.hpp - C++ facade of kate_b200 with the reference's class and method
// names (Line-fr/Kate: Kate.hpp, backendagnosticcode/basic_host_types.hpp,
// QuantumCircuit.hpp, Circuit.hpp, HIPcode/simulator.hpp), so that code
// written against `#include "Kate.hpp"` compiles against this library
// instead: replace the include with `#include <kate_b200/Kate.hpp>` and link
// with -lkate_b200. Header-only; every call goes through the C ABI of
// kate_b200.h.
//
// Like the reference, failures are printed to std::cout and execution
// continues; Kate::last_status() returns the status of the last call.
#ifndef KATE_B200_KATE_HPP
#define KATE_B200_KATE_HPP

#include <cmath>
#include <iostream>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../kate_b200.h"

#ifndef Hadamard
#define Hadamard 2
#define CNOT 3
#define CRk 4
#define TOFFOLI 5
#define RX 6
#define RZ 7
#endif

namespace Kate {

inline kate_status& last_status() {
    static thread_local kate_status s = KATE_OK;
    return s;
}

inline bool check(kate_status s) {
    last_status() = s;
    if (s != KATE_OK) std::cout << "kate_b200: " << kate_last_error() << std::endl;
    return s == KATE_OK;
}

class Complex {
public:
    double a = 0, b = 0;
    Complex() = default;
    Complex(double a_) : a(a_), b(0) {}
    Complex(double a_, double b_) : a(a_), b(b_) {}
    Complex operator+(Complex o) const { return Complex(a + o.a, b + o.b); }
    Complex operator-(Complex o) const { return Complex(a - o.a, b - o.b); }
    Complex operator*(Complex o) const { return Complex(a * o.a - b * o.b, a * o.b + b * o.a); }
    Complex operator*(double d) const { return Complex(a * d, b * d); }
    Complex operator*(int d) const { return Complex(a * d, b * d); }
    Complex operator/(Complex o) const {
        const double n = o.a * o.a + o.b * o.b;
        return Complex((a * o.a + b * o.b) / n, (o.a * b - a * o.b) / n);
    }
    void operator+=(Complex o) { a += o.a, b += o.b; }
    void operator-=(Complex o) { a -= o.a, b -= o.b; }
    void operator*=(Complex o) { *this = *this * o; }
    void operator*=(double d) { a *= d, b *= d; }
    double norm() const { return std::sqrt(a * a + b * b); }
    // atan(b / a), as the reference computes it (not atan2).
    double angle() const { return std::atan(b / a); }
    void print() const { std::cout << a << " + " << b << "i"; }
};

namespace detail {
inline void print_entry(const Complex& c) { c.print(); }
template <typename T>
void print_entry(const T& v) {
    std::cout << v;
}
}  // namespace detail

// printGpuInfo (HIPcode/DeviceInfo.hpp:10-35): host threads, the CUDA
// devices, and device 0's memory in qubits of complex128 state.
inline void printGpuInfo() {
    std::cout << "CPU Info: " << std::thread::hardware_concurrency() << " threads" << std::endl;
    int count = 0;
    kate_device_count(&count);
    if (count == 0) {
        std::cout << "couldnt detect devices, check permissions" << std::endl;
        return;
    }
    char name[256];
    size_t gmem = 0, smem = 0;
    int sms = 0;
    for (int i = 0; i < count; i++)
        if (check(kate_device_properties(i, name, (int)sizeof(name), nullptr, nullptr, nullptr)))
            std::cout << "GPU " << i << " : " << name << std::endl;
    std::cout << "-----------------------" << std::endl;
    if (!check(kate_device_properties(0, name, (int)sizeof(name), &gmem, &smem, &sms))) return;
    std::cout << "current GPU: " << std::endl << name << " (" << sms << " SMs)" << std::endl << std::endl;
    std::cout << "Global memory: " << gmem << " (" << (int)std::log2((double)gmem / 16.0) << " qbits)" << std::endl;
    std::cout << "Shared memory per block : " << smem << std::endl << std::endl;
}

// Square row-major matrix (basic_host_types.hpp:86-186).
template <typename T>
class Matrix {
public:
    int n = 0;
    std::vector<T> storage;
    T* data = nullptr;
    Matrix() = default;
    explicit Matrix(int n_) : n(n_), storage((size_t)n_ * n_), data(storage.data()) {}
    Matrix(const Matrix& o) : n(o.n), storage(o.storage), data(storage.data()) {}
    Matrix& operator=(const Matrix& o) {
        n = o.n;
        storage = o.storage;
        data = storage.data();
        return *this;
    }
    T operator()(int r, int c) const { return data[(size_t)r * n + c]; }
    void operator()(int r, int c, T v) { data[(size_t)r * n + c] = v; }
    void fill(T v) {
        for (auto& x : storage) x = v;
    }
    void copy(const Matrix& o) { storage = o.storage, data = storage.data(); }
    void print() const {
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < n; j++) {
                detail::print_entry(data[(size_t)i * n + j]);
                std::cout << " | ";
            }
            std::cout << std::endl;
        }
    }
    Matrix operator+(const Matrix& o) const {
        Matrix r(*this);
        r += o;
        return r;
    }
    Matrix operator-(const Matrix& o) const {
        Matrix r(*this);
        r -= o;
        return r;
    }
    void operator+=(const Matrix& o) {
        for (size_t i = 0; i < storage.size(); i++) storage[i] += o.storage[i];
    }
    void operator-=(const Matrix& o) {
        for (size_t i = 0; i < storage.size(); i++) storage[i] -= o.storage[i];
    }
    // Matrix product (this * o), summed in k order like the reference.
    Matrix operator*(const Matrix& o) const {
        Matrix r(n);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                T sum = T(0);
                for (int k = 0; k < n; k++) sum += data[(size_t)i * n + k] * o(k, j);
                r(i, j, sum);
            }
        return r;
    }
    void operator*=(double d) {
        for (auto& x : storage) x *= d;
    }
    void transpose() {
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++) std::swap(data[(size_t)i * n + j], data[(size_t)j * n + i]);
    }
};

// Gate (basic_host_types.hpp:190-296).
class Gate {
public:
    int identifier = -1;
    int optarg = 0;
    double optarg2 = 0;
    Complex optarg3;
    std::vector<int> qbits;
    Matrix<Complex> densecontent;
    Gate(int id, std::vector<int>& q, int opt = 0, double opt2 = 0, Complex opt3 = 0)
        : identifier(id), optarg(opt), optarg2(opt2), optarg3(opt3), qbits(q) {}
    Gate(Matrix<Complex>& m, std::vector<int>& q) : identifier(0), qbits(q), densecontent(m) {}
    // A gate id carrying a matrix (basic_host_types.hpp:246-262): the id
    // decides what is applied, as in the reference.
    Gate(int id, Matrix<Complex>& m, std::vector<int>& q) : identifier(id), qbits(q), densecontent(m) {}
    void print() const {
        std::cout << "Identifier : " << identifier << ", Qbits affected : ";
        for (int q : qbits) std::cout << q << " ";
        std::cout << std::endl;
    }
};

// proba_state (basic_host_types.hpp:319-336).
class proba_state {
public:
    std::vector<std::pair<double, double>> val;
    explicit proba_state(int n) : val(n, {0.0, 0.0}) {}
    explicit proba_state(std::vector<std::pair<double, double>>& v) : val(v) {}
    void print() const {
        for (size_t i = 0; i < val.size(); i++)
            std::cout << "Qbit " << i << " : teta=" << val[i].first << " , phi=" << val[i].second << std::endl;
    }
};

// Circuit (QuantumCircuit.hpp + Circuit.hpp).
class Circuit {
public:
    int nqbits = 0;
    explicit Circuit(int n) : nqbits(n) { check(kate_circuit_create(n, &h_)); }
    Circuit(const Circuit& o) : nqbits(o.nqbits) { check(kate_circuit_clone(o.h_, &h_)); }
    Circuit& operator=(const Circuit& o) {
        if (this != &o) {
            kate_circuit_destroy(h_);
            nqbits = o.nqbits;
            check(kate_circuit_clone(o.h_, &h_));
        }
        return *this;
    }
    ~Circuit() { kate_circuit_destroy(h_); }

    void appendGate(const Gate& g) {
        if (g.identifier == 0) {
            std::vector<double> m(2 * g.densecontent.storage.size());
            for (size_t i = 0; i < g.densecontent.storage.size(); i++) {
                m[2 * i] = g.densecontent.storage[i].a;
                m[2 * i + 1] = g.densecontent.storage[i].b;
            }
            check(kate_circuit_append_dense(h_, m.data(), g.qbits.data(), (int)g.qbits.size()));
        } else {
            check(kate_circuit_append_gate(h_, g.identifier, g.qbits.data(), (int)g.qbits.size(), g.optarg));
        }
    }
    void gateScheduling() { check(kate_circuit_schedule(h_)); }
    void gateFusion(int qbitsizelimit = 5, double merge_time_matters = 0.000001) {
        check(kate_circuit_fuse(h_, qbitsizelimit, merge_time_matters));
    }
    // gateFusion with every merge of the pass on CUDA device `device` (one
    // launch; the same gates, bit for bit).
    void gateFusion(int qbitsizelimit, double merge_time_matters, int device) {
        check(kate_circuit_fuse_device(h_, qbitsizelimit, merge_time_matters, device));
    }
    void gateGrouping(int qbitgroupsize = 8) { check(kate_circuit_group(h_, qbitgroupsize)); }
    void allocate(int numberofgpulog2 = 0, int maxlocalqbitnumber = 300) {
        check(kate_circuit_allocate(h_, numberofgpulog2, maxlocalqbitnumber));
    }
    void compileDefault(int numberofgpulog2 = 0, int maxlocalqbitnumber = 300) {
        check(kate_circuit_compile_default(h_, numberofgpulog2, maxlocalqbitnumber));
    }
    void compileOPT(int k = 5, double mtm = 0.000001, int groupsize = 10, int numberofgpulog2 = 0,
                    int maxlocalqbitnumber = 300) {
        check(kate_circuit_compile_opt(h_, k, mtm, groupsize, numberofgpulog2, maxlocalqbitnumber));
    }
    void exportqcx(const std::string& filename) { check(kate_circuit_export_qcx(h_, filename.c_str())); }
    // QuantumCircuit::print (QuantumCircuit.hpp:38-123): the gate list (by
    // group once grouped) before compilation; after it the program: swaps,
    // then each group with its gates, with permutationtable the
    // label-to-qubit table before each group.
    void print(bool permutationtable = false) const {
        int ng = 0, ngr = 0, ni = 0;
        kate_circuit_num_gates(h_, &ng);
        kate_circuit_num_groups(h_, &ngr);
        kate_circuit_num_instructions(h_, &ni);
        std::vector<int> q(256);
        auto gate_line = [&](int i) {
            int id = 0, nq = 0, opt = 0;
            kate_circuit_get_gate(h_, i, &id, q.data(), &nq, &opt, nullptr);
            std::cout << "Identifier : " << id << ", Qbits affected : ";
            for (int k = 0; k < nq; k++) std::cout << q[k] << " ";
            std::cout << std::endl;
        };
        auto group_head = [&](const char* label, int g, int* end) {
            int nq = 0;
            kate_circuit_get_group(h_, g, end, q.data(), &nq);
            std::cout << label << " " << g << " with qbits ";
            for (int k = 0; k < nq; k++) std::cout << q[k] << " ";
            std::cout << " : " << std::endl;
        };
        if (ni == 0) {
            int group = 0, end = -1;
            if (ngr) group_head("Group", 0, &end);
            for (int i = 0; i < ng; i++) {
                if (ngr) {
                    if (group >= ngr) {
                        std::cout << "ERROR while printing the circuit, group vector is bad" << std::endl;
                        return;
                    }
                    if (end == i) group_head("Group", ++group, &end);
                    std::cout << "   ";
                    gate_line(i);
                } else {
                    std::cout << "gate " << i << " is ";
                    gate_line(i);
                }
            }
            return;
        }
        std::vector<int> perm(nqbits), fin(nqbits), inv(nqbits);
        int valid = 0;
        kate_circuit_get_permutations(h_, perm.data(), fin.data(), &valid);
        for (int m = 0; m < nqbits; m++) inv[perm[m]] = m;
        std::cout << "-------Quantum-Program-------" << std::endl;
        int i = 0, group = 0;
        for (int k = 0; k < ni; k++) {
            int kind = 0, nq = 0;
            kate_circuit_get_instruction(h_, k, &kind, q.data(), &nq);
            if (kind == 0) {
                std::cout << "SWAP ";
                for (int m = 0; m < nq / 2; m++) {
                    std::cout << q[2 * m] << " and " << q[2 * m + 1] << ", ";
                    std::swap(inv[q[2 * m]], inv[q[2 * m + 1]]);
                }
            } else {
                if (permutationtable) {
                    std::cout << "Permutation table (subjective to real) : " << std::endl;
                    for (int m = 0; m < nqbits; m++) std::cout << m << " " << (m < 10 ? " " : "");
                    std::cout << std::endl;
                    for (int m = 0; m < nqbits; m++) std::cout << inv[m] << " " << (inv[m] < 10 ? " " : "");
                    std::cout << std::endl << std::endl;
                }
                int end = 0;
                group_head("EXEC Group", group, &end);
                for (int j = i; j < end; j++) {
                    std::cout << "   ";
                    gate_line(j);
                }
                i = end;
                group++;
            }
            std::cout << std::endl << std::endl;
        }
        std::cout << "-----------------------------" << std::endl;
    }
    int gateCount() const {
        int n = 0;
        kate_circuit_num_gates(h_, &n);
        return n;
    }
    const kate_circuit* handle() const { return h_; }

private:
    kate_circuit* h_ = nullptr;
};
using QuantumCircuit = Circuit;

namespace detail {
inline Gate merge_gates(const std::vector<Gate>& gates, bool on_device, void* stream, int device) {
    int n = 0;
    for (auto& g : gates)
        for (int q : g.qbits) n = q + 1 > n ? q + 1 : n;
    Circuit c(n);
    for (auto& g : gates) c.appendGate(g);
    std::vector<int> q(64);
    int k = 0;
    std::vector<double> m(2 * 1024 * 1024);
    if (on_device)
        check(kate_merge_gates_device(c.handle(), 0, (int)gates.size(), device, stream, q.data(), &k, m.data()));
    else
        check(kate_merge_gates(c.handle(), 0, (int)gates.size(), q.data(), &k, m.data()));
    q.resize(k);
    Matrix<Complex> mat(1 << k);
    for (size_t i = 0; i < mat.storage.size(); i++) mat.storage[i] = Complex(m[2 * i], m[2 * i + 1]);
    return Gate(mat, q);
}
}  // namespace detail

// mergeGate / CPUmergeGate (CPUcode/GateMerger.hpp:8-55): on the host.
inline Gate mergeGate(std::vector<Gate> gates) { return detail::merge_gates(gates, false, nullptr, 0); }
inline Gate CPUmergeGate(std::vector<Gate> gates) { return detail::merge_gates(gates, false, nullptr, 0); }
// mergeGate(to_merge, stream) of the GPU build (HIPcode/GateMerger.hpp:43-109):
// on CUDA device `device`, on `stream` (a cudaStream_t), bit-identical to
// the host merger.
inline Gate mergeGate(std::vector<Gate> gates, void* stream, int device = 0) {
    return detail::merge_gates(gates, true, stream, device);
}

// Simulator (HIPcode/simulator.hpp:220-811) on one B200. number_of_gpu and
// swapBufferSizeLog2 are accepted for source compatibility; one GPU is used.
class Simulator {
public:
    Simulator(const Circuit& c, int number_of_gpu = 1, int swapBufferSizeLog2 = 24,
              kate_precision precision = KATE_C128, int device = 0)
        : n_(c.nqbits) {
        (void)number_of_gpu;
        (void)swapBufferSizeLog2;
        check(kate_sim_create(c.handle(), precision, device, &s_));
    }
    Simulator(const Simulator&) = delete;
    Simulator& operator=(const Simulator&) = delete;
    ~Simulator() { kate_sim_destroy(s_); }

    // displaytime prints the phases the reference prints (device time of
    // the initialisation and of the group passes, host time of the
    // measurement). Qubit relabelings replace the reference's swaps, so the
    // swap share is 0.
    proba_state execute(bool displaytime = false) { return run(nullptr, displaytime); }
    proba_state execute(proba_state& in, bool displaytime = false) {
        std::vector<double> tin(2 * n_);
        for (int i = 0; i < n_ && i < (int)in.val.size(); i++) {
            tin[2 * i] = in.val[i].first;
            tin[2 * i + 1] = in.val[i].second;
        }
        return run(tin.data(), displaytime);
    }
    // The state in the reference's amplitude order.
    std::vector<Complex> state() {
        std::vector<double> d(2 * ((size_t)1 << n_));
        check(kate_sim_get_state(s_, d.data()));
        std::vector<Complex> r((size_t)1 << n_);
        for (size_t i = 0; i < r.size(); i++) r[i] = Complex(d[2 * i], d[2 * i + 1]);
        return r;
    }
    kate_sim* handle() { return s_; }

private:
    proba_state run(const double* tin, bool displaytime) {
        std::vector<double> tp(2 * n_);
        if (!displaytime) {
            check(tin ? kate_sim_execute_from(s_, tin, tp.data()) : kate_sim_execute(s_, tp.data()));
            return to_proba(tp);
        }
        double ms[4] = {0, 0, 0, 0};
        if (check(kate_sim_execute_timed(s_, tin, tp.data(), ms))) {
            std::cout << "Initialization/Measurement : " << ms[0] << " / " << ms[2] << " ms" << std::endl;
            std::cout << "Total computing time : " << ms[1] << " ms with swap% : 0%" << std::endl;
            std::cout << "Average swap time : 0 ms and average group time : " << (ms[3] > 0 ? ms[1] / ms[3] : 0.0)
                      << " ms" << std::endl;
        }
        return to_proba(tp);
    }
    proba_state to_proba(const std::vector<double>& tp) {
        std::vector<std::pair<double, double>> v(n_);
        for (int i = 0; i < n_; i++) v[i] = {tp[2 * i], tp[2 * i + 1]};
        return proba_state(v);
    }
    int n_;
    kate_sim* s_ = nullptr;
};

}  // namespace Kate

#endif  // KATE_B200_KATE_HPP
