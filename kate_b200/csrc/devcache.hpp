// Reuse of large device buffers (simulator states, batch arenas).
//
// A caller that loops `Simulator(circuit).execute()` (the reference's usage,
// HIPcode/simulator.hpp:243-300 allocates the state in every constructor and
// frees it in the destructor) would pay cudaMalloc and cudaFree of the whole
// state on every iteration: hundreds of milliseconds for tens of GB. The most
// recently released large buffer of each device is kept instead and handed
// to the next request it covers (up to 4x its size). The cached buffer stays
// allocated until a request it does not cover, the creation of a server
// (which takes its budget in one allocation) or kate_release_cached_memory
// frees it.
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

namespace kate {

// Buffers below this size are allocated and freed directly.
constexpr size_t kCacheMinBytes = size_t(64) << 20;

// Allocates at least `bytes` on the current device (`device`), reusing the
// cached buffer when it covers the request.
cudaError_t cached_malloc(void** p, size_t bytes, int device);
// Releases a buffer from cached_malloc (the current device is `device`).
// Waits for the device first, so no kernel still uses it when it is reused.
void cached_free(void* p, int device);
// Frees the cached buffer of `device` (-1: of every device).
void release_cached(int device);

}  // namespace kate
