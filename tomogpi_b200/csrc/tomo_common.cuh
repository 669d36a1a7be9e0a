// tomo_common.cuh -- shared device/host definitions of the tomogpi_b200 library.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/tomogpi_b200.h"

namespace tomo {

// ---------------------------------------------------------------------------------
// Geometry as uploaded for the kernels (the values of the reference's __constant__
// symbols, GPUConstant.cuh:23-72), plus per-view tables in device memory.
// ---------------------------------------------------------------------------------
struct DevGeom {
    float fod, fdd, gamma, du, dv, uc, vc, dx, xc, yc, zc;
    float inv_gamma_f;   // 1/gamma in float  (backprojection3D_kernel_16reg.cuh:464)
    double inv_gamma_d;  // 1.0/gamma in double (backprojection3D_kernel_16reg.cuh:404)
    float fdk_alpha;     // FDK weight constants alphaC, betaC (BackProjector.cu:34-35) as float
    float fdk_beta;
    float fdd_du;        // fdd / du in float (FDK3D_kernel_16reg.cuh:78)
    int nx, ny, nz, nu, nv, np;
    int p0;                           // acquisition index of view 0 (a view range of a larger acquisition)
    int rs_wlog;                      // RS launch shape: a warp's rays span 2^rs_wlog u x 2^(5-rs_wlog) v
    int rs_tlog;                      // ... and a block's 2^rs_tlog u x 2^(8-rs_tlog) v (rs_wlog <= rs_tlog)
    const float* __restrict__ alpha;  // cos(phi_p) as float
    const float* __restrict__ beta;   // sin(phi_p) as float
    const float4* __restrict__ vi;    // per view: (-beta*dx)*(fdd/du), (alpha*dx)*(fdd/du), alpha*dx, beta*dx
    // The views ordered by the direction of their rays: first the view_cols views whose rays
    // run mostly along x (|cos phi| > |sin phi|), then the others (null: no such table).
    const int* __restrict__ view_order;
    int view_cols;
};

// Exact IEEE single/double operations: never contracted into FMA, correctly rounded.
// The geometry prologues use these so that their results are bit-identical to the
// reference's host-compiled arithmetic.
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }
// 1 / a correctly rounded: the same value as the IEEE division 1.0f / a, by the reciprocal.
__device__ __forceinline__ float frcp(float a) { return __frcp_rn(a); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Storage <-> FP32.
template <typename T>
__device__ __forceinline__ float ld(const T* p);
template <>
__device__ __forceinline__ float ld<float>(const float* p) { return __ldg(p); }
template <>
__device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
template <>
__device__ __forceinline__ float ld<__half>(const __half* p) { return __half2float(__ldg(p)); }

template <typename T>
__device__ __forceinline__ float ldp(const T* p);  // plain (coherent) load
template <>
__device__ __forceinline__ float ldp<float>(const float* p) { return *p; }
template <>
__device__ __forceinline__ float ldp<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(*p); }
template <>
__device__ __forceinline__ float ldp<__half>(const __half* p) { return __half2float(*p); }

template <typename T>
__device__ __forceinline__ T cvt(float v);
template <>
__device__ __forceinline__ float cvt<float>(float v) { return v; }
template <>
__device__ __forceinline__ __nv_bfloat16 cvt<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <>
__device__ __forceinline__ __half cvt<__half>(float v) { return __float2half_rn(v); }

// FP16 range guard. A gradient dJ = -2 H^T r reaches magnitudes of order 2 * views *
// max|r|, beyond FP16's largest finite value (65504). Before a volume is stored in FP16 it
// is multiplied by 2^-k, the smallest k >= 0 with max|v| * 2^-k < 2^14; the operators are
// linear, so the squared norm of a projection is multiplied back by 2^2k. Scaling by a
// power of two is exact. `amax` holds the FP32 bits of max|v| (non-negative floats order
// like their bit patterns, so atomicMax on the bits computes it); a null pointer means 1.
__host__ __device__ __forceinline__ int fp16_scale_exp(unsigned amax_bits) {
    const int e = (int)((amax_bits >> 23) & 0xffu) - 127;  // max|v| in [2^e, 2^(e+1))
    return e > 13 ? e - 13 : 0;
}
__device__ __forceinline__ float fp16_scale(const unsigned* amax) {
    if (!amax) return 1.f;
    return __uint_as_float((unsigned)(127 - fp16_scale_exp(*amax)) << 23);  // 2^-k
}
__device__ __forceinline__ double fp16_unscale_sq(const unsigned* amax) {
    if (!amax) return 1.0;
    return __longlong_as_double((long long)(1023 + 2 * fp16_scale_exp(*amax)) << 52);  // 2^2k
}

// Linear interpolation (1-t)*a + t*b, the documented texture-filter form.
__device__ __forceinline__ float lerp(float a, float b, float t) { return fmaf(t, b, fmaf(-t, a, a)); }

// Padded copies used by the operators: one zero voxel/pixel on every side, so that every
// texel of a footprint that touches the data lies inside the buffer.
struct PadDims {
    long w, h, d;  // padded extents (nx+2, ny+2, nz+2) or (nu+2, nv+2, P)
};

// Device-side error word bits (bounded loops that gave up).
enum : unsigned { ERR_SIDDON_GUARD = 1u, ERR_TIMEOUT = 2u };

size_t dtype_size(tomo_dtype t);

// Host-side geometry (geometry.cu).
struct HostGeom {
    float fod, fdd, gamma, du, dv, uc, vc, dx, xc, yc, zc;
    float inv_gamma_f;
    double inv_gamma_d;
    float fdk_alpha, fdk_beta, fdd_du;
    int nx, ny, nz, nu, nv, np;
    int p0 = 0;  // acquisition index of view 0
    std::vector<float> alpha, beta;
    std::vector<float4> vi;
    std::vector<int> view_order;  // views whose rays run mostly along x first (view_cols of them)
    int view_cols = 0;
};
void derive_geometry(const tomo_config_ct& c, HostGeom& h);
// Keeps views [begin, begin + count) of the acquisition (tables sliced, np = count, p0 = begin).
void select_views(HostGeom& h, int begin, int count);
void fill_devgeom(const HostGeom& h, const float* d_alpha, const float* d_beta, const float4* d_vi, DevGeom& g,
                  const int* d_order = nullptr);
// Orders the views by ray direction (HostGeom::view_order, view_cols).
void order_views(HostGeom& h);

// Host helpers.
void set_error(const std::string& msg);
tomo_status cuda_fail(cudaError_t e, const char* what);

}  // namespace tomo

#define TOMO_CUDA_TRY(call)                                             \
    do {                                                                \
        cudaError_t _e = (call);                                        \
        if (_e != cudaSuccess) return ::tomo::cuda_fail(_e, #call);     \
    } while (0)

#define TOMO_CHECK_ARG(cond, msg)                  \
    do {                                           \
        if (!(cond)) {                             \
            ::tomo::set_error(msg);                \
            return TOMO_ERR_INVALID;               \
        }                                          \
    } while (0)
