// vi_back.cu -- voxel-driven interpolating (VI) backprojector for sm_100a, plus the
// padding/conversion kernels that feed the operators.
//
// One thread per (x, y) column; each thread owns ZC chunks of 16 consecutive z voxels and
// loops over all views. Per view the detector column coordinate un and the
// magnification factor A are z-invariant (backprojection3D_kernel_16reg.cuh:401-404), so
// the horizontal bilinear weight and column index are computed once per view, and each z
// voxel costs one row lookup (2 x 2 texels) and three lerps. A warp covers 32 adjacent x
// at the same (y, z): its 32 footprints fall on one or two detector rows over ~32
// adjacent columns, i.e. every texel load instruction is a short coalesced row segment.
// Per-view constants ((-beta dx)(FDD/du), (alpha dx)(FDD/du), alpha dx, beta dx) come from a
// float4 table read once per view.
//
// Parity: un, A and v follow the reference's operation order with explicitly rounded
// IEEE operations:
//   TOMO_BACK_VI     backprojection_VIB_kernel_v2_16reg (..._16reg.cuh:350-576): within a
//                    16-slice chunk v advances by repeated addition of A (:410-453).
//   TOMO_BACK_VI_UM  backprojection_VIB_kernel_v1_16reg_UM (..._16reg_UM.cuh:24-151):
//                    v_k = v_0 + k*A.
// The first view uses A = (1.0/gamma)*w in double (:404), the others (1/gamma)*w in float
// (:464). Views accumulate in order 0..P-1 in FP32, the result is acc * dx (:524). The
// sinogram is read from a zero-bordered padded copy, which gives the texture's border
// colour 0 without per-texel bounds checks.
#include "vi_device.cuh"

namespace tomo {

template <int UM, int ZC, typename Ts, typename Tv, bool FDK = false>
__global__ void __launch_bounds__(VI_BX* VI_BY, vi_min_blocks(ZC)) vi_back_kernel(DevGeom g, const Ts* __restrict__ spad,
                                                              Tv* __restrict__ vol, float scale) {
    vi_tile<UM, ZC, Ts, Tv, FDK>(g, spad, vol, scale, blockIdx.x, blockIdx.y, blockIdx.z);
}

// FDK-weighted backprojection (FDK3D_VIB_kernel_v0_16reg), 16 slices per thread.
template <typename Ts, typename Tv>
static cudaError_t launch_fdk_t(const DevGeom& g, const void* spad, void* vol, cudaStream_t st) {
    dim3 block(VI_BX * VI_BY), grid((g.nx + VI_BX - 1) / VI_BX, (g.ny + VI_BY - 1) / VI_BY, (g.nz + 15) / 16);
    vi_back_kernel<0, 1, Ts, Tv, true><<<grid, block, 0, st>>>(g, (const Ts*)spad, (Tv*)vol, 1.0f);
    return cudaGetLastError();
}

template <typename Ts>
static cudaError_t launch_fdk_out(const DevGeom& g, const void* spad, void* vol, tomo_dtype vdt, cudaStream_t st) {
    switch (vdt) {
        case TOMO_F32: return launch_fdk_t<Ts, float>(g, spad, vol, st);
        case TOMO_BF16: return launch_fdk_t<Ts, __nv_bfloat16>(g, spad, vol, st);
        case TOMO_F16: return launch_fdk_t<Ts, __half>(g, spad, vol, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_vi_fdk(const DevGeom& g, const void* spad, tomo_dtype sdt, void* vol, tomo_dtype vdt, cudaStream_t st) {
    switch (sdt) {
        case TOMO_F32: return launch_fdk_out<float>(g, spad, vol, vdt, st);
        case TOMO_BF16: return launch_fdk_out<__nv_bfloat16>(g, spad, vol, vdt, st);
        case TOMO_F16: return launch_fdk_out<__half>(g, spad, vol, vdt, st);
    }
    return cudaErrorInvalidValue;
}

template <int UM, int ZC, typename Ts, typename Tv>
static cudaError_t launch_vi_zc(const DevGeom& g, const void* spad, void* vol, float scale, cudaStream_t st) {
    dim3 block(VI_BX * VI_BY), grid((g.nx + VI_BX - 1) / VI_BX, (g.ny + VI_BY - 1) / VI_BY, (g.nz + 16 * ZC - 1) / (16 * ZC));
    vi_back_kernel<UM, ZC, Ts, Tv><<<grid, block, 0, st>>>(g, (const Ts*)spad, (Tv*)vol, scale);
    return cudaGetLastError();
}

static thread_local int t_vi_zc = 1;  // set by launch_vi_back for the call in progress

template <int UM, typename Ts, typename Tv>
static cudaError_t launch_vi_t(const DevGeom& g, const void* spad, void* vol, float scale, cudaStream_t st) {
    if (t_vi_zc == 1) return launch_vi_zc<UM, 1, Ts, Tv>(g, spad, vol, scale, st);
    if (t_vi_zc == 4) return launch_vi_zc<UM, 4, Ts, Tv>(g, spad, vol, scale, st);
    return launch_vi_zc<UM, 2, Ts, Tv>(g, spad, vol, scale, st);
}

template <int UM, typename Ts>
static cudaError_t launch_vi_out(const DevGeom& g, const void* spad, void* vol, tomo_dtype vdt, float scale,
                                 cudaStream_t st) {
    switch (vdt) {
        case TOMO_F32: return launch_vi_t<UM, Ts, float>(g, spad, vol, scale, st);
        case TOMO_BF16: return launch_vi_t<UM, Ts, __nv_bfloat16>(g, spad, vol, scale, st);
        case TOMO_F16: return launch_vi_t<UM, Ts, __half>(g, spad, vol, scale, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_vi_back(int um, const DevGeom& g, const void* spad, tomo_dtype sdt, void* vol, tomo_dtype vdt,
                           float scale, cudaStream_t st, int zc) {
    t_vi_zc = zc;
    switch (sdt) {
        case TOMO_F32:
            return um ? launch_vi_out<1, float>(g, spad, vol, vdt, scale, st)
                      : launch_vi_out<0, float>(g, spad, vol, vdt, scale, st);
        case TOMO_BF16:
            return um ? launch_vi_out<1, __nv_bfloat16>(g, spad, vol, vdt, scale, st)
                      : launch_vi_out<0, __nv_bfloat16>(g, spad, vol, vdt, scale, st);
        case TOMO_F16:
            return um ? launch_vi_out<1, __half>(g, spad, vol, vdt, scale, st)
                      : launch_vi_out<0, __half>(g, spad, vol, vdt, scale, st);
    }
    return cudaErrorInvalidValue;
}

// Texture form: the sinogram in a 2D layered array (one layer per view).
template <int UM, int ZC, typename Tt, typename Tv>
__global__ void __launch_bounds__(VI_BX* VI_BY) vi_back_tex_kernel(DevGeom g, unsigned long long tex,
                                                                  Tv* __restrict__ vol, float scale) {
    vi_tile_tex<UM, ZC, Tt, Tv>(g, tex, vol, scale, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <int UM, int ZC, typename Tt, typename Tv>
static cudaError_t launch_vi_tex_zc(const DevGeom& g, unsigned long long tex, void* vol, float scale, cudaStream_t st) {
    dim3 block(VI_BX * VI_BY), grid((g.nx + VI_BX - 1) / VI_BX, (g.ny + VI_BY - 1) / VI_BY, (g.nz + 16 * ZC - 1) / (16 * ZC));
    vi_back_tex_kernel<UM, ZC, Tt, Tv><<<grid, block, 0, st>>>(g, tex, (Tv*)vol, scale);
    return cudaGetLastError();
}

template <int UM, typename Tt, typename Tv>
static cudaError_t launch_vi_tex_t(const DevGeom& g, unsigned long long tex, void* vol, float scale, cudaStream_t st,
                                   int zc) {
    if (zc == 1) return launch_vi_tex_zc<UM, 1, Tt, Tv>(g, tex, vol, scale, st);
    if (zc == 4) return launch_vi_tex_zc<UM, 4, Tt, Tv>(g, tex, vol, scale, st);
    return launch_vi_tex_zc<UM, 2, Tt, Tv>(g, tex, vol, scale, st);
}

template <int UM, typename Tt>
static cudaError_t launch_vi_tex_out(const DevGeom& g, unsigned long long tex, void* vol, tomo_dtype vdt, float scale,
                                     cudaStream_t st, int zc) {
    switch (vdt) {
        case TOMO_F32: return launch_vi_tex_t<UM, Tt, float>(g, tex, vol, scale, st, zc);
        case TOMO_BF16: return launch_vi_tex_t<UM, Tt, __nv_bfloat16>(g, tex, vol, scale, st, zc);
        case TOMO_F16: return launch_vi_tex_t<UM, Tt, __half>(g, tex, vol, scale, st, zc);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_vi_back_tex(int um, const DevGeom& g, unsigned long long tex, tomo_dtype tdt, void* vol,
                               tomo_dtype vdt, float scale, cudaStream_t st, int zc) {
    switch (tdt) {
        case TOMO_F32:
            return um ? launch_vi_tex_out<1, float>(g, tex, vol, vdt, scale, st, zc)
                      : launch_vi_tex_out<0, float>(g, tex, vol, vdt, scale, st, zc);
        case TOMO_BF16:
            return um ? launch_vi_tex_out<1, __nv_bfloat16>(g, tex, vol, vdt, scale, st, zc)
                      : launch_vi_tex_out<0, __nv_bfloat16>(g, tex, vol, vdt, scale, st, zc);
        case TOMO_F16:
            return um ? launch_vi_tex_out<1, __half>(g, tex, vol, vdt, scale, st, zc)
                      : launch_vi_tex_out<0, __half>(g, tex, vol, vdt, scale, st, zc);
    }
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------------
// Padding / conversion. The padded buffers are zeroed once when allocated; these kernels
// only rewrite the interior, so the zero border stays intact.
// ---------------------------------------------------------------------------------
template <typename Ti, typename To>
__global__ void pad3_kernel(const Ti* __restrict__ in, To* __restrict__ out, int n0, int n1, int n2, int pad2,
                            const unsigned* amax) {
    const float sc = fp16_scale(amax);
    // in: [i2][i1][i0] dense; out: [i2 + pad2][i1 + 1][i0 + 1] with extents n0+2, n1+2, n2+2*pad2
    const long total = (long)n0 * n1 * n2;
    const long W = n0 + 2, WH = W * (n1 + 2);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long i0 = i % n0, r = i / n0, i1 = r % n1, i2 = r / n1;
        out[(i2 + pad2) * WH + (i1 + 1) * W + (i0 + 1)] = cvt<To>(ldp(in + i) * sc);
    }
}

template <typename Ti, typename To>
__global__ void convert_kernel(const Ti* __restrict__ in, To* __restrict__ out, size_t n, const unsigned* amax) {
    const float sc = fp16_scale(amax);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = cvt<To>(ldp(in + i) * sc);
}

static int grid_for(long n) {
    long b = (n + 255) / 256;
    if (b > 148L * 32) b = 148L * 32;  // a few waves over the 148 SMs, grid-stride beyond
    return (int)(b < 1 ? 1 : b);
}

template <typename Ti>
static cudaError_t pad3_out(const Ti* in, void* out, tomo_dtype odt, int n0, int n1, int n2, int pad2,
                            cudaStream_t st, const unsigned* amax) {
    const int gsz = grid_for((long)n0 * n1 * n2);
    switch (odt) {
        case TOMO_F32: pad3_kernel<Ti, float><<<gsz, 256, 0, st>>>(in, (float*)out, n0, n1, n2, pad2, amax); break;
        case TOMO_BF16:
            pad3_kernel<Ti, __nv_bfloat16><<<gsz, 256, 0, st>>>(in, (__nv_bfloat16*)out, n0, n1, n2, pad2, amax);
            break;
        case TOMO_F16: pad3_kernel<Ti, __half><<<gsz, 256, 0, st>>>(in, (__half*)out, n0, n1, n2, pad2, amax); break;
    }
    return cudaGetLastError();
}

static cudaError_t pad3(const void* in, tomo_dtype idt, void* out, tomo_dtype odt, int n0, int n1, int n2, int pad2,
                        cudaStream_t st, const unsigned* amax = nullptr) {
    switch (idt) {
        case TOMO_F32: return pad3_out((const float*)in, out, odt, n0, n1, n2, pad2, st, amax);
        case TOMO_BF16: return pad3_out((const __nv_bfloat16*)in, out, odt, n0, n1, n2, pad2, st, amax);
        case TOMO_F16: return pad3_out((const __half*)in, out, odt, n0, n1, n2, pad2, st, amax);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_pad_volume(const void* in, tomo_dtype idt, void* out, tomo_dtype odt, int nx, int ny, int nz,
                              cudaStream_t st, const unsigned* amax) {
    return pad3(in, idt, out, odt, nx, ny, nz, 1, st, amax);
}

cudaError_t launch_pad_sinogram(const void* in, tomo_dtype idt, void* out, tomo_dtype odt, int nu, int nv, int np,
                                cudaStream_t st) {
    return pad3(in, idt, out, odt, nu, nv, np, 0, st);
}

template <typename Ti>
static cudaError_t convert_out(const Ti* in, void* out, tomo_dtype odt, size_t n, cudaStream_t st, const unsigned* amax) {
    const int gsz = grid_for((long)n);
    switch (odt) {
        case TOMO_F32: convert_kernel<Ti, float><<<gsz, 256, 0, st>>>(in, (float*)out, n, amax); break;
        case TOMO_BF16: convert_kernel<Ti, __nv_bfloat16><<<gsz, 256, 0, st>>>(in, (__nv_bfloat16*)out, n, amax); break;
        case TOMO_F16: convert_kernel<Ti, __half><<<gsz, 256, 0, st>>>(in, (__half*)out, n, amax); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_convert(const void* in, tomo_dtype idt, void* out, tomo_dtype odt, size_t n, cudaStream_t st,
                           const unsigned* amax) {
    switch (idt) {
        case TOMO_F32: return convert_out((const float*)in, out, odt, n, st, amax);
        case TOMO_BF16: return convert_out((const __nv_bfloat16*)in, out, odt, n, st, amax);
        case TOMO_F16: return convert_out((const __half*)in, out, odt, n, st, amax);
    }
    return cudaErrorInvalidValue;
}

}  // namespace tomo
