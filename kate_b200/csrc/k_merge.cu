// Gate merging on the GPU: the FP64 product of a list of gates as one dense
// gate on the sorted union of their qubits (the reference's mergeGate,
// HIPcode/GateMerger.hpp:12-109, whose CPU form is CPUmergeGate,
// CPUcode/GateMerger.hpp:8-55).
//
// Every merge job (a block of gates) contributes 2^k CTAs, one per basis
// column: the CTA starts from the basis state |col> in shared memory, applies
// the block's gates one by one (a barrier between gates) and writes the
// resulting column into the job's row-major output, transposed on the way
// (entry (r, col) = amplitude r). All jobs of a fusion pass run in one
// launch. The arithmetic is the host merger's operation for operation, each
// product and sum rounded on its own (__dmul_rn / __dadd_rn / __dsub_rn, so
// nothing is contracted into an FMA), the CRk phase is computed on the host
// and passed in, and a dense gate's outputs are summed over its columns in
// ascending order: the matrices are bit-identical to the host merger's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "circuit.hpp"
#include "launch.hpp"

namespace kate {

namespace {

constexpr int MAXK = 10;  // the merger's limit (2^10 x 2^10 matrices)
constexpr int NT = 256;

struct MGate {
    int32_t id, nq;
    int32_t lb[MAXK];      // local bit of qbits[i]
    int32_t sorted[MAXK];  // local bits ascending (for the line deposit)
    int64_t mat;           // dense: offset of the row-major 2^nq x 2^nq matrix in the pool
    double ph_re, ph_im;   // CRk: the phase e^{2 pi i / 2^k}
};

struct MJob {
    int32_t k;        // qubits of the merged gate
    int32_t g0, ng;   // its gates: gates[g0 .. g0 + ng)
    int32_t cta0;     // first CTA of the job (one CTA per column)
    int64_t out;      // offset of its output matrix (complex elements)
};

// Inserts a zero bit at each of the `cnt` ascending positions `s`.
__device__ __forceinline__ uint32_t deposit(uint32_t v, const int32_t* s, int cnt) {
    for (int i = 0; i < cnt; i++) {
        const uint32_t p = (uint32_t)s[i];
        v = ((v >> p) << (p + 1)) | (v & ((1u << p) - 1u));
    }
    return v;
}

__global__ void __launch_bounds__(NT) k_merge(const MJob* __restrict__ jobs, int njobs, const MGate* __restrict__ gates,
                                              const double2* __restrict__ pool, double2* __restrict__ out) {
    extern __shared__ double2 sm[];
    // The job of this CTA: the last one whose first CTA is <= blockIdx.x.
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].cta0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const MJob J = jobs[lo];
    const uint32_t dim = 1u << J.k;
    const uint32_t col = blockIdx.x - (uint32_t)J.cta0;
    double2* A = sm;
    double2* B = sm + dim;
    for (uint32_t i = threadIdx.x; i < dim; i += NT) A[i] = make_double2(i == col ? 1.0 : 0.0, 0.0);
    __syncthreads();
    const double S2 = 1.4142135623730951, S2I = 0.7071067811865475;
    for (int gi = 0; gi < J.ng; gi++) {
        const MGate& g = gates[J.g0 + gi];
        switch (g.id) {
        case G_TOFFOLI:
            for (uint32_t line = threadIdx.x; line < (dim >> 3); line += NT) {
                const uint32_t a = deposit(line, g.sorted, 3) + (1u << g.lb[0]) + (1u << g.lb[1]);
                const uint32_t b = a + (1u << g.lb[2]);
                const double2 x = A[a];
                A[a] = A[b];
                A[b] = x;
            }
            break;
        case G_CNOT:
            for (uint32_t line = threadIdx.x; line < (dim >> 2); line += NT) {
                const uint32_t a = deposit(line, g.sorted, 2) + (1u << g.lb[1]);
                const uint32_t b = a + (1u << g.lb[0]);
                const double2 x = A[a];
                A[a] = A[b];
                A[b] = x;
            }
            break;
        case G_CRK:
            for (uint32_t line = threadIdx.x; line < (dim >> 2); line += NT) {
                const uint32_t a = deposit(line, g.sorted, 2) + (1u << g.lb[1]) + (1u << g.lb[0]);
                const double2 x = A[a];
                A[a] = make_double2(__dsub_rn(__dmul_rn(x.x, g.ph_re), __dmul_rn(x.y, g.ph_im)),
                                    __dadd_rn(__dmul_rn(x.x, g.ph_im), __dmul_rn(x.y, g.ph_re)));
            }
            break;
        case G_H:
            for (uint32_t line = threadIdx.x; line < (dim >> 1); line += NT) {
                const uint32_t a = deposit(line, g.sorted, 1);
                const uint32_t b = a + (1u << g.lb[0]);
                const double2 x = A[a], y = A[b];
                const double2 n0 = make_double2(__dmul_rn(__dadd_rn(x.x, y.x), S2I), __dmul_rn(__dadd_rn(x.y, y.y), S2I));
                A[a] = n0;
                A[b] = make_double2(__dsub_rn(n0.x, __dmul_rn(y.x, S2)), __dsub_rn(n0.y, __dmul_rn(y.y, S2)));
            }
            break;
        case G_DENSE: {
            // Out of place: output (line, r) reads the line's old amplitudes.
            const uint32_t gd = 1u << g.nq;
            const double2* U = pool + g.mat;
            for (uint32_t o = threadIdx.x; o < dim; o += NT) {
                const uint32_t r = o & (gd - 1u);
                const uint32_t base = deposit(o >> g.nq, g.sorted, g.nq);
                double2 sum = make_double2(0.0, 0.0);
                for (uint32_t c = 0; c < gd; c++) {
                    uint32_t idx = base;
                    for (int i = 0; i < g.nq; i++) idx += ((c >> i) & 1u) << g.lb[i];
                    const double2 u = U[(size_t)r * gd + c], x = A[idx];
                    sum.x = __dadd_rn(sum.x, __dsub_rn(__dmul_rn(u.x, x.x), __dmul_rn(u.y, x.y)));
                    sum.y = __dadd_rn(sum.y, __dadd_rn(__dmul_rn(u.x, x.y), __dmul_rn(u.y, x.x)));
                }
                uint32_t idx = base;
                for (int i = 0; i < g.nq; i++) idx += ((r >> i) & 1u) << g.lb[i];
                B[idx] = sum;
            }
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < dim; i += NT) A[i] = B[i];
            break;
        }
        default:
            break;  // RX / RZ: no arithmetic, as in the reference
        }
        __syncthreads();
    }
    double2* M = out + J.out;
    for (uint32_t r = threadIdx.x; r < dim; r += NT) M[(size_t)r * dim + col] = A[r];
}

}  // namespace

std::string merge_gates_device(const std::vector<std::vector<Gate>>& blocks, int device, cudaStream_t stream,
                               std::vector<Gate>* out) {
    out->clear();
    if (blocks.empty()) return "";
    std::vector<MJob> jobs;
    std::vector<MGate> gates;
    std::vector<double2> pool;
    std::vector<std::vector<int>> covs;
    int64_t out_elems = 0, ctas = 0;
    int kmax = 0;
    for (const auto& blk : blocks) {
        std::vector<int> all;
        for (const auto& g : blk) all.insert(all.end(), g.qbits.begin(), g.qbits.end());
        std::sort(all.begin(), all.end());
        all.erase(std::unique(all.begin(), all.end()), all.end());
        const int k = (int)all.size();
        if (k > MAXK) return "merged gate would cover more than 10 qubits";
        MJob j{};
        j.k = k;
        j.g0 = (int32_t)gates.size();
        j.ng = (int32_t)blk.size();
        j.cta0 = (int32_t)ctas;
        j.out = out_elems;
        for (const auto& g : blk) {
            MGate d{};
            d.id = g.id;
            d.nq = (int32_t)g.qbits.size();
            if (d.nq > MAXK) return "a gate has more than 10 qubits";
            for (int i = 0; i < d.nq; i++)
                d.lb[i] = (int32_t)(std::lower_bound(all.begin(), all.end(), g.qbits[i]) - all.begin());
            std::copy(d.lb, d.lb + d.nq, d.sorted);
            std::sort(d.sorted, d.sorted + d.nq);
            if (g.id == G_CRK) {
                const double t = ((double)2 * 3.1415926535897932384626433) / (double)(1ull << g.optarg);
                d.ph_re = std::cos(t);
                d.ph_im = std::sin(t);
            }
            if (g.id == G_DENSE) {
                const size_t dd = (size_t)1 << (2 * d.nq);
                if (g.dense.size() != dd) return "dense gate matrix has the wrong size";
                d.mat = (int64_t)pool.size();
                for (const Cx& x : g.dense) pool.push_back(make_double2(x.re, x.im));
            }
            gates.push_back(d);
        }
        jobs.push_back(j);
        covs.push_back(std::move(all));
        out_elems += (int64_t)1 << (2 * k);
        ctas += (int64_t)1 << k;
        kmax = std::max(kmax, k);
    }
    if (ctas > 0x7fffffff) return "too many merge columns for one launch";
    if (pool.empty()) pool.push_back(make_double2(0.0, 0.0));
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return "cuda: cannot select the device";
    const size_t jb = jobs.size() * sizeof(MJob), gb = gates.size() * sizeof(MGate),
                 pb = pool.size() * sizeof(double2), ob = (size_t)out_elems * sizeof(double2);
    const size_t off_g = (jb + 255) & ~(size_t)255, off_p = (off_g + gb + 255) & ~(size_t)255,
                 off_o = (off_p + pb + 255) & ~(size_t)255, total = off_o + ob;
    std::vector<double2> host((size_t)out_elems);
    void* d = nullptr;
    std::vector<uint8_t> in(off_o);
    std::memcpy(in.data(), jobs.data(), jb);
    std::memcpy(in.data() + off_g, gates.data(), gb);
    std::memcpy(in.data() + off_p, pool.data(), pb);
    const size_t smem = ((size_t)2 << kmax) * sizeof(double2);
    cudaError_t e = cudaMallocAsync(&d, total, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, in.data(), off_o, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        if (smem > 48 * 1024) e = cudaFuncSetAttribute(k_merge, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) {
            k_merge<<<(unsigned)ctas, NT, smem, stream>>>((const MJob*)d, (int)jobs.size(),
                                                           (const MGate*)((uint8_t*)d + off_g),
                                                           (const double2*)((uint8_t*)d + off_p),
                                                           (double2*)((uint8_t*)d + off_o));
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), (uint8_t*)d + off_o, ob, cudaMemcpyDeviceToHost, stream);
    if (d) {
        const cudaError_t f = cudaFreeAsync(d, stream);
        if (e == cudaSuccess) e = f;
    }
    const cudaError_t s = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = s;
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) return std::string("cuda: ") + cudaGetErrorString(e) + " (device gate merger)";
    out->resize(blocks.size());
    for (size_t b = 0; b < blocks.size(); b++) {
        Gate& g = (*out)[b];
        g.id = G_DENSE;
        g.qbits = covs[b];
        g.optarg = 0;
        const size_t n = (size_t)1 << (2 * jobs[b].k);
        g.dense.resize(n);
        const double2* src = host.data() + jobs[b].out;
        for (size_t i = 0; i < n; i++) g.dense[i] = Cx(src[i].x, src[i].y);
    }
    return "";
}

}  // namespace kate
