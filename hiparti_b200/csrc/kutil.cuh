// kutil.cuh -- small device helpers shared by the kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace pti {

// Four consecutive factor entries of a row as FP32 (read-only path).
__device__ __forceinline__ float4 load4(const float *row, uint32_t col)
{
    return __ldg(reinterpret_cast<const float4 *>(row + col));
}
__device__ __forceinline__ float4 load4(const __nv_bfloat16 *row, uint32_t col)
{
    uint2 raw = __ldg(reinterpret_cast<const uint2 *>(row + col));
    __nv_bfloat162 lo = *reinterpret_cast<__nv_bfloat162 *>(&raw.x);
    __nv_bfloat162 hi = *reinterpret_cast<__nv_bfloat162 *>(&raw.y);
    float2 a = __bfloat1622float2(lo), b = __bfloat1622float2(hi);
    return make_float4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ float4 mul4(float4 a, float4 b)
{
    return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
}
__device__ __forceinline__ float4 add4(float4 a, float4 b)
{
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 scale4(float4 a, float s)
{
    return make_float4(a.x * s, a.y * s, a.z * s, a.w * s);
}

// One 16-byte vector atomic add into global memory (sm_90+).
__device__ __forceinline__ void red_add4(float *dst, float4 v)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(dst), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w)
                 : "memory");
}

// Zeroes the components of v whose column index (col, col+1, ...) is >= R, so
// pad columns of the output are never written with anything but zero.
__device__ __forceinline__ float4 mask4(float4 v, uint32_t col, uint32_t R)
{
    if (col + 4 <= R) return v;
    return make_float4(col < R ? v.x : 0.f, col + 1 < R ? v.y : 0.f, col + 2 < R ? v.z : 0.f,
                       col + 3 < R ? v.w : 0.f);
}

// Exact FP32 products of the two BF16 halves of a and b (a mixed-precision
// FMA with a zero addend; a product of two BF16 values is exact in FP32).
__device__ __forceinline__ float2 bf16x2_mul(uint32_t a, uint32_t b)
{
    float lo, hi;
    asm("{\n\t.reg .b16 al, ah, bl, bh;\n\t"
        "mov.b32 {al, ah}, %2;\n\t"
        "mov.b32 {bl, bh}, %3;\n\t"
        "fma.rn.f32.bf16 %0, al, bl, 0f00000000;\n\t"
        "fma.rn.f32.bf16 %1, ah, bh, 0f00000000;\n\t}"
        : "=f"(lo), "=f"(hi)
        : "r"(a), "r"(b));
    return make_float2(lo, hi);
}

}  // namespace pti
