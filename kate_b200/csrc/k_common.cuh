// Small device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace kate {

#define KATE_SQRT2 1.4142135623730951
#define KATE_SQRT2INV 0.7071067811865475

// Inserts a zero bit at position b of v.
__device__ __forceinline__ uint32_t ins0(uint32_t v, int b) {
    return ((v >> b) << (b + 1)) | (v & ((1u << b) - 1u));
}

// (a.x*b.x - a.y*b.y, a.x*b.y + a.y*b.x): the reference's Complex product.
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// acc += a * b (complex), as four FMAs.
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return cmulf(a, b); }
// Complex products for the register stages: complex64 in packed FP32
// (sm_100), b.re * a + b.im * (i a); complex128 as cmul.
__device__ __forceinline__ float2 cmul_r(float2 a, float2 b) {
    return __ffma2_rn(make_float2(b.y, b.y), make_float2(-a.y, a.x), __fmul2_rn(make_float2(b.x, b.x), a));
}
__device__ __forceinline__ double2 cmul_r(double2 a, double2 b) { return cmul(a, b); }
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
}

// A complex double from the matrix pool, as the tile's element type.
template <typename C2>
__device__ __forceinline__ C2 from_pool(double2 v);
template <>
__device__ __forceinline__ double2 from_pool<double2>(double2 v) { return v; }
template <>
__device__ __forceinline__ float2 from_pool<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

__device__ __forceinline__ double2 dadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

}  // namespace kate
