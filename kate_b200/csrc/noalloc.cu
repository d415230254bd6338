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
// on every GPU where the library's device code is loaded, held until the
// process exits), so the call is limited to states of at most
// KATE_NOALLOC_MAX_QUBITS qubits. Under CUDA's lazy module loading the
// device code (and this array) is loaded on a device by the first kernel
// launch or symbol lookup there, which can itself need device memory: a
// caller that reserves all of a device's memory makes one call (or runs any
// simulator) on it first. The array is shared by every call and keeps the
// last call's contents; every slot a call reads is written by the same call
// first, so nothing needs clearing. Calls that overlap on the GPU (on
// different streams, or from different threads) race on the array and must
// be serialised by the caller.
//
// The caller's pointer is checked before anything is launched: it must be
// device memory of the current device (cudaPointerGetAttributes), 16-byte
// aligned, and the complex128 state of 16 * 2^nqbits bytes must fit both
// the caller's stated buffer size and the allocation the pointer lies in
// (cuMemGetAddressRange); a complex64 or short buffer is refused instead of
// being read past its end.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
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

kate_status fail(kate_status st, const std::string& m) {
    set_last_error(m);
    return st;
}

// Checks that [p, p + bytes) lies inside one device allocation (driver
// cuMemGetAddressRange, resolved at run time). True when the range fits or
// the driver call is unavailable.
bool fits_allocation(const void* p, size_t bytes) {
    using Fn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
    static Fn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (Fn) nullptr;
        return (Fn)f;
    }();
    if (!fn) return true;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (fn(&base, &size, (CUdeviceptr)(uintptr_t)p) != CUDA_SUCCESS) return false;
    return (uint64_t)(uintptr_t)p + bytes <= (uint64_t)base + size;
}

}  // namespace
}  // namespace kate

extern "C" kate_status kate_proba_state_noalloc(const void* d_state, size_t state_bytes, int nqbits,
                                                const int* phys_of_label, const int* final_inverse_permutation,
                                                double* theta_phi, void* stream) {
    using namespace kate;
    if (!d_state || !theta_phi) return fail(KATE_EINVAL, "null state or output pointer");
    if (nqbits < 1 || nqbits > KATE_NOALLOC_MAX_QUBITS)
        return fail(KATE_EINVAL, "kate_proba_state_noalloc handles 1 to " +
                                     std::to_string(KATE_NOALLOC_MAX_QUBITS) + " qubits (fixed scratch size)");
    const int n = nqbits;
    const size_t need = (size_t)16 << n;
    if (state_bytes < need)
        return fail(KATE_EINVAL, "state_bytes " + std::to_string(state_bytes) + " is below the " +
                                     std::to_string(need) + " bytes of a complex128 state of " + std::to_string(n) +
                                     " qubits (complex64 states are not accepted)");
    if (((uintptr_t)d_state & 15u) != 0) return fail(KATE_EINVAL, "d_state is not 16-byte aligned");
    int phys[KATE_NOALLOC_MAX_QUBITS];
    bool seen[KATE_NOALLOC_MAX_QUBITS] = {false};
    for (int x = 0; x < n; x++) {
        phys[x] = phys_of_label ? phys_of_label[x] : x;
        if (phys[x] < 0 || phys[x] >= n || seen[phys[x]]) return fail(KATE_EINVAL, "phys_of_label is not a permutation");
        seen[phys[x]] = true;
    }
    if (final_inverse_permutation) {
        bool out_seen[KATE_NOALLOC_MAX_QUBITS] = {false};
        for (int x = 0; x < n; x++) {
            const int o = final_inverse_permutation[x];
            if (o < 0 || o >= n || out_seen[o]) return fail(KATE_EINVAL, "final_inverse_permutation is not a permutation");
            out_seen[o] = true;
        }
    }
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return fail(KATE_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    cudaPointerAttributes attr;
    ce = cudaPointerGetAttributes(&attr, d_state);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        return fail(KATE_EINVAL, std::string("d_state is not a CUDA pointer: ") + cudaGetErrorString(ce));
    }
    if ((attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) || attr.device != dev)
        return fail(KATE_EINVAL, "d_state is not device memory of the current device");
    if (!fits_allocation(d_state, need))
        return fail(KATE_EINVAL, "the " + std::to_string(need) + "-byte state does not fit the allocation d_state lies in");
    // The scratch array's device address on this device (looked up on every
    // call: no allocation once the module is loaded, and it stays valid
    // across a cudaDeviceReset).
    void* scratch = nullptr;
    ce = cudaGetSymbolAddress(&scratch, g_scratch);
    if (ce != cudaSuccess) return fail(KATE_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
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
