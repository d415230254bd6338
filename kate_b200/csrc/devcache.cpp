// Reuse of large device buffers. See devcache.hpp.
#include "devcache.hpp"

#include <mutex>
#include <unordered_map>

namespace kate {

namespace {

struct Block {
    void* p = nullptr;
    size_t bytes = 0;
};

constexpr int kMaxDevices = 64;
std::mutex g_mu;
Block g_cached[kMaxDevices];                   // one released buffer per device
std::unordered_map<void*, size_t> g_live;      // buffers handed out, with their real size

void free_cached_locked(int device) {
    Block& c = g_cached[device];
    if (!c.p) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    cudaFree(c.p);
    if (cur != device) cudaSetDevice(cur);
    c = Block{};
}

}  // namespace

cudaError_t cached_malloc(void** p, size_t bytes, int device) {
    *p = nullptr;
    if (bytes < kCacheMinBytes || device < 0 || device >= kMaxDevices) return cudaMalloc(p, bytes);
    std::lock_guard<std::mutex> lk(g_mu);
    Block& c = g_cached[device];
    if (c.p && c.bytes >= bytes && c.bytes / 4 <= bytes) {
        *p = c.p;
        g_live[c.p] = c.bytes;
        c = Block{};
        return cudaSuccess;
    }
    free_cached_locked(device);
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return e;
    g_live[*p] = bytes;
    return cudaSuccess;
}

void cached_free(void* p, int device) {
    if (!p) return;
    std::unique_lock<std::mutex> lk(g_mu);
    auto it = g_live.find(p);
    if (it == g_live.end() || device < 0 || device >= kMaxDevices) {
        lk.unlock();
        cudaFree(p);
        return;
    }
    const size_t bytes = it->second;
    g_live.erase(it);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return;
    }
    free_cached_locked(device);
    g_cached[device] = Block{p, bytes};
}

void release_cached(int device) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (device >= 0 && device < kMaxDevices) {
        free_cached_locked(device);
        return;
    }
    for (int d = 0; d < kMaxDevices; d++) free_cached_locked(d);
}

}  // namespace kate
