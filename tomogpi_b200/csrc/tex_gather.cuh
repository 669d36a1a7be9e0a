// tex_gather.cuh -- 4-texel gathers (tld4) from 2D layered textures, used by the RS
// projector (one layer per z slice) and the VI backprojector (one layer per view).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace tomo {

// Four texels of layer `layer` around the 2x2 footprint centred at (x, y), from a 2D
// layered texture (border colour 0 in x and y): tld4 returns
// (T[i][j+1], T[i+1][j+1], T[i+1][j], T[i][j]) for i = floor(x - 0.5), j = floor(y - 0.5).
// FP32 textures gather floats; 16-bit textures hold raw BF16 / FP16 bits as unsigned
// shorts, gathered as integers and widened exactly.
template <typename Tt>
__device__ __forceinline__ float4 gather_layer(unsigned long long tex, int layer, float x, float y);

template <>
__device__ __forceinline__ float4 gather_layer<float>(unsigned long long tex, int layer, float x, float y) {
    float4 r;
    asm("tld4.r.a2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %7}];"
                 : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
                 : "l"(tex), "r"(layer), "f"(x), "f"(y));
    return r;
}

__device__ __forceinline__ uint4 gather_layer_raw(unsigned long long tex, int layer, float x, float y) {
    uint4 r;
    asm("tld4.r.a2d.v4.u32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %7}];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(tex), "r"(layer), "f"(x), "f"(y));
    return r;
}

template <>
__device__ __forceinline__ float4 gather_layer<__nv_bfloat16>(unsigned long long tex, int layer, float x, float y) {
    const uint4 r = gather_layer_raw(tex, layer, x, y);  // BF16 = the high half of an FP32
    return make_float4(__uint_as_float(r.x << 16), __uint_as_float(r.y << 16), __uint_as_float(r.z << 16),
                       __uint_as_float(r.w << 16));
}

template <>
__device__ __forceinline__ float4 gather_layer<__half>(unsigned long long tex, int layer, float x, float y) {
    const uint4 r = gather_layer_raw(tex, layer, x, y);
    return make_float4(__half2float(__ushort_as_half((unsigned short)r.x)),
                       __half2float(__ushort_as_half((unsigned short)r.y)),
                       __half2float(__ushort_as_half((unsigned short)r.z)),
                       __half2float(__ushort_as_half((unsigned short)r.w)));
}

}  // namespace tomo
