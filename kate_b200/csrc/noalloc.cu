// Measurement entry point that allocates no memory.
//
// Who needs it: code that must not call cudaMalloc or any allocating library
// routine once it is running - a serving loop that reserved the device's
// memory for resident state vectors up front, a caller working under a
// fixed memory budget or inside a memory pool it does not own, or a host
// language binding that cannot manage the lifetime of device buffers. Such a
// caller already holds the state vector on the device and only needs the
// reference's per-qubit (theta, phi) measurement of it
// (HIPcode/simulator.hpp:483-543).
//
// The per-CTA partial sums of the reduction live in a file-scope
// __device__ array of a fixed size (KATE_NOALLOC_SCRATCH_BYTES, about 660 KB
// on every GPU that loads the library, held until the process exits), so
// the call is limited to states of at most KATE_NOALLOC_MAX_QUBITS qubits.
// The array is shared by every call and keeps the last call's contents;
// every slot a call reads is written by the same call first, so nothing
// needs clearing. Calls that overlap on the GPU (on different streams, or
// from different threads) race on the array and must be serialised by the
// caller.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "kate_b200.h"
#include "launch.hpp"

namespace kate {
void set_last_error(const std::string& msg);  // capi.cpp: the message kate_last_error() returns
}

namespace kate {
namespace {

constexpr int kGridBits = 10;                   // 1024 CTAs
constexpr int kMaxRoundBits = 8;                // rounds per thread (k_bitsums)
constexpr int kPartsPerCta = 1 + 2 * (12 + kMaxRoundBits);
constexpr int kPartials = (1 << kGridBits) * kPartsPerCta;
constexpr int kFinal = 2 * KATE_NOALLOC_MAX_QUBITS;

// Partials of the reduction, then the final (sum over bit = 0, sum over
// bit = 1) pair of every physical bit.
static __device__ __align__(256) double2 g_scratch[kPartials + kFinal];
static_assert(sizeof(g_scratch) <= KATE_NOALLOC_SCRATCH_BYTES, "scratch size");

// Adds the per-CTA partials of k_bitsums into one (bit 0, bit 1) sum pair
// per physical bit, in CTA order. One thread per output.
__global__ void k_finish(const double2* __restrict__ part, int n, int g, int nout, double2* __restrict__ out) {
    const int o = threadIdx.x;
    if (o >= 2 * n) return;
    const int b = o / 2, one = o & 1;
    double2 s = make_double2(0.0, 0.0);
    const int grid = 1 << g;
    for (int c = 0; c < grid; c++) {
        const double2* pc = part + (size_t)c * nout;
        double2 v;
        if (b < 12) v = pc[1 + 2 * b + one];
        else if (b < 12 + g) v = ((((c >> (b - 12)) & 1) == one) ? pc[0] : make_double2(0.0, 0.0));
        else v = pc[1 + 2 * (12 + (b - 12 - g)) + one];
        s.x += v.x;
        s.y += v.y;
    }
    out[o] = s;
}

std::mutex g_mu;
void* g_addr[64] = {nullptr};

kate_status fail(kate_status st, const std::string& m) {
    set_last_error(m);
    return st;
}

}  // namespace
}  // namespace kate

extern "C" kate_status kate_proba_state_noalloc(const void* d_state, int nqbits, const int* phys_of_label,
                                                const int* final_inverse_permutation, double* theta_phi,
                                                void* stream) {
    using namespace kate;
    if (!d_state || !theta_phi) return fail(KATE_EINVAL, "null state or output pointer");
    if (nqbits < 1 || nqbits > KATE_NOALLOC_MAX_QUBITS)
        return fail(KATE_EINVAL, "kate_proba_state_noalloc handles 1 to " +
                                     std::to_string(KATE_NOALLOC_MAX_QUBITS) + " qubits (fixed scratch size)");
    const int n = nqbits;
    int phys[KATE_NOALLOC_MAX_QUBITS];
    bool seen[KATE_NOALLOC_MAX_QUBITS] = {false};
    for (int x = 0; x < n; x++) {
        phys[x] = phys_of_label ? phys_of_label[x] : x;
        if (phys[x] < 0 || phys[x] >= n || seen[phys[x]]) return fail(KATE_EINVAL, "phys_of_label is not a permutation");
        seen[phys[x]] = true;
    }
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return fail(KATE_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    if (dev < 0 || dev >= 64) return fail(KATE_EINVAL, "device index above 63");
    void* scratch = nullptr;
    {
        // Set-up, once per device: the device address of the scratch array.
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            ce = cudaGetSymbolAddress(&g_addr[dev], g_scratch);
            if (ce != cudaSuccess) {
                g_addr[dev] = nullptr;
                return fail(KATE_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
            }
        }
        scratch = g_addr[dev];
    }
    double2* part = (double2*)scratch;
    double2* fin = part + kPartials;
    const int g = n <= 12 ? 0 : (n - 12 < kGridBits ? n - 12 : kGridBits);
    const int nr = n <= 12 ? 0 : n - 12 - g;
    const int nout = 1 + 2 * (12 + nr);
    cudaStream_t s = (cudaStream_t)stream;
    ce = launch_bitsums_c128_shape(d_state, n, g, nr, part, s);
    if (ce == cudaSuccess) {
        k_finish<<<1, 64, 0, s>>>(part, n, g, nout, fin);
        ce = cudaGetLastError();
    }
    double2 sums[kFinal];
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(sums, fin, sizeof(double2) * 2 * n, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return fail(KATE_ECUDA, std::string("measurement: ") + cudaGetErrorString(ce));
    // The reference's formula (HIPcode/simulator.hpp:519-535), its Complex
    // division, norm and angle (backendagnosticcode/basic_host_types.hpp:28-57).
    const double kPi = 3.1415926535897932384626433;
    const double p = std::pow(1.4142135623730951, (double)n);
    auto cdiv = [](double ar, double ai, double br, double bi, double& rr, double& ri) {
        double d = br * br + bi * bi;
        rr = (ar * br + ai * bi) / d;
        ri = (br * ai - ar * bi) / d;
    };
    for (int x = 0; x < n; x++) {
        const int b = phys[x];
        double v0r, v0i, v1r, v1i;
        cdiv(sums[2 * b].x, sums[2 * b].y, p, 0.0, v0r, v0i);
        cdiv(sums[2 * b + 1].x, sums[2 * b + 1].y, p, 0.0, v1r, v1i);
        const double n0 = std::sqrt(v0r * v0r + v0i * v0i), n1 = std::sqrt(v1r * v1r + v1i * v1i);
        double teta, phi;
        if (n0 < 0.0000000000001) {
            teta = 1;
            phi = 0;
        } else if (n1 < 0.00000000000001) {
            teta = 0;
            phi = 0;
        } else {
            teta = std::atan(n1 / n0) / (kPi / 2);
            double qr, qi;
            cdiv(v1r, v1i, v0r, v0i, qr, qi);
            phi = std::atan(qi / qr);
        }
        const int o = final_inverse_permutation ? final_inverse_permutation[x] : x;
        theta_phi[2 * o] = teta;
        theta_phi[2 * o + 1] = phi;
    }
    return KATE_OK;
}
