// rs_project.cu -- regular-sampling (RS) cone-beam projector for sm_100a.
//
// One thread per detector ray (u, v, phi). A warp covers an 8u x 4v tile of one view so
// that its 32 rays stay spatially coherent while they march: at each step the 32 sample
// points sit within a few voxels of each other and their trilinear footprints share L1
// lines. The volume is read from a zero-bordered padded copy (one voxel on every side),
// so a sample whose footprint touches the data never needs per-texel bounds checks.
//
// Parity: the per-ray prologue (source/detector positions, the y = A1 x + B1 line, the
// FOV intersection, the box and z clipping, the chord length L_r) is written with
// explicitly rounded IEEE operations in the reference's order and precision, so entry
// points and sample counts are bit-identical to the reference kernels compiled on the
// host with exact FP32 texture filtering:
//   TOMO_PROJ_RS     projection_ERB_kernel_v1   (projection_ER_kernel.cuh:57-312)
//   TOMO_PROJ_RS_UM  projection_ERB_kernel_v0_UM (projection_ER_kernel_UM.cuh:26-153)
// The positions march by repeated exact addition (:295-297) and every sample adds
// dx * tex3D(...) with a separate multiply and add (:292). Only the trilinear weights
// use fused multiply-adds (within 1e-6 relative of the exact formula).
#include "tomo_kernels.cuh"

namespace tomo {

// Trilinear interpolation of the padded volume at texture coordinates (tx, ty, tz):
// cudaFilterModeLinear semantics, sample at (t - 0.5), border colour 0.
template <typename Tv>
__device__ __forceinline__ float trilinear_padded(const Tv* __restrict__ vp, int W, int WH, float fnx, float fny,
                                                  float fnz, float tx, float ty, float tz) {
    const float xb = fsub(tx, 0.5f), yb = fsub(ty, 0.5f), zb = fsub(tz, 0.5f);
    if (!(xb > -1.f && yb > -1.f && zb > -1.f && xb < fnx && yb < fny && zb < fnz)) return 0.f;
    const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    const float a = xb - fx, b = yb - fy, c = zb - fz;  // exact: fractional parts
    const int i = (int)fx + 1, j = (int)fy + 1, k = (int)fz + 1;
    const Tv* q = vp + (k * WH + j * W + i);
    const float v000 = ld(q), v100 = ld(q + 1), v010 = ld(q + W), v110 = ld(q + W + 1);
    const float v001 = ld(q + WH), v101 = ld(q + WH + 1), v011 = ld(q + WH + W), v111 = ld(q + WH + W + 1);
    const float c00 = lerp(v000, v100, a), c10 = lerp(v010, v110, a);
    const float c01 = lerp(v001, v101, a), c11 = lerp(v011, v111, a);
    return lerp(lerp(c00, c10, b), lerp(c01, c11, b), c);
}

template <int MODE, typename Tv, typename To, int EPI>
__global__ void __launch_bounds__(256) rs_project_kernel(DevGeom g, const Tv* __restrict__ vpad, OutView<To> out,
                                                         OutView<To> real, double* __restrict__ norm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int v = blockIdx.y * 16 + (warp >> 1) * 4 + (lane >> 3);
    const int p = blockIdx.z;
    const bool active = (u < g.nu) && (v < g.nv);
    float acc = 0.f;
    if (active) {
        RsRay r;
        const bool hit = MODE == 0 ? rs_ray_box(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r)
                                   : rs_ray_um(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r);
        if (hit) {
            const int W = g.nx + 2, WH = (g.nx + 2) * (g.ny + 2);
            const float fnx = (float)g.nx, fny = (float)g.ny, fnz = (float)g.nz;
            float A = r.A, B = r.B, C = r.C;
            const float dx = g.dx;
            for (unsigned n = 0; n < r.n; ++n) {
                const float t =
                    trilinear_padded(vpad, W, WH, fnx, fny, fnz, fadd(A, 0.5f), fadd(B, 0.5f), fadd(C, 0.5f));
                acc = fadd(acc, fmul(dx, t));
                A = fadd(A, r.sx);
                B = fadd(B, r.sy);
                C = fadd(C, r.sz);
            }
        }
    }
    epilogue<EPI>(active, acc, u, v, p, out, real, norm);
}

// Exact transpose: scatter dx * y * w_texel into the (unpadded, FP32) output volume.
template <int MODE, typename Ts>
__global__ void __launch_bounds__(256) rs_adjoint_kernel(DevGeom g, const Ts* __restrict__ sino,
                                                         float* __restrict__ vol) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int v = blockIdx.y * 16 + (warp >> 1) * 4 + (lane >> 3);
    const int p = blockIdx.z;
    if (u >= g.nu || v >= g.nv) return;
    const float y = ld(sino + ((long)p * g.nv + v) * g.nu + u);
    if (y == 0.f) return;
    RsRay r;
    const bool hit = MODE == 0 ? rs_ray_box(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r)
                               : rs_ray_um(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r);
    if (!hit) return;
    const float s = fmul(g.dx, y);
    const float fnx = (float)g.nx, fny = (float)g.ny, fnz = (float)g.nz;
    float A = r.A, B = r.B, C = r.C;
    for (unsigned n = 0; n < r.n; ++n) {
        const float xb = fsub(fadd(A, 0.5f), 0.5f), yb = fsub(fadd(B, 0.5f), 0.5f), zb = fsub(fadd(C, 0.5f), 0.5f);
        if (xb > -1.f && yb > -1.f && zb > -1.f && xb < fnx && yb < fny && zb < fnz) {
            const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
            const float a = xb - fx, b = yb - fy, c = zb - fz;
            const int i = (int)fx, j = (int)fy, k = (int)fz;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int di = q & 1, dj = (q >> 1) & 1, dk = q >> 2;
                const int ii = i + di, jj = j + dj, kk = k + dk;
                if (ii < 0 || jj < 0 || kk < 0 || ii >= g.nx || jj >= g.ny || kk >= g.nz) continue;
                const float w = (di ? a : 1.f - a) * (dj ? b : 1.f - b) * (dk ? c : 1.f - c);
                atomicAdd(vol + ((long)kk * g.ny + jj) * g.nx + ii, s * w);
            }
        }
        A = fadd(A, r.sx);
        B = fadd(B, r.sy);
        C = fadd(C, r.sz);
    }
}

template <int MODE>
__global__ void rs_count_kernel(DevGeom g, unsigned long long* __restrict__ total) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    const int p = blockIdx.z;
    unsigned long long n = 0;
    if (u < g.nu) {
        RsRay r;
        const bool hit = MODE == 0 ? rs_ray_box(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r)
                                   : rs_ray_um(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r);
        if (hit) n = r.n;
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(total, n);
}

// ---------------------------------------------------------------------------------
// Host launchers.
// ---------------------------------------------------------------------------------
template <typename Tv, typename To>
static cudaError_t launch_rs_t(int mode, int epi, const DevGeom& g, const void* vpad, const OutView<void>& out,
                               const OutView<void>& real, double* norm, cudaStream_t st) {
    dim3 block(256), grid((g.nu + 15) / 16, (g.nv + 15) / 16, g.np);
    const OutView<To> o = out.as<To>(), r = real.as<To>();
    const Tv* vp = static_cast<const Tv*>(vpad);
#define TOMO_RS_LAUNCH(M, E) rs_project_kernel<M, Tv, To, E><<<grid, block, 0, st>>>(g, vp, o, r, norm)
    if (mode == 0) {
        if (epi == EPI_STORE) TOMO_RS_LAUNCH(0, EPI_STORE);
        else if (epi == EPI_RESIDUAL) TOMO_RS_LAUNCH(0, EPI_RESIDUAL);
        else TOMO_RS_LAUNCH(0, EPI_NORM);
    } else {
        if (epi == EPI_STORE) TOMO_RS_LAUNCH(1, EPI_STORE);
        else if (epi == EPI_RESIDUAL) TOMO_RS_LAUNCH(1, EPI_RESIDUAL);
        else TOMO_RS_LAUNCH(1, EPI_NORM);
    }
#undef TOMO_RS_LAUNCH
    return cudaGetLastError();
}

cudaError_t launch_rs_project(int mode, int epi, const DevGeom& g, const void* vpad, tomo_dtype vdt,
                              const OutView<void>& out, tomo_dtype odt, const OutView<void>& real, double* norm,
                              cudaStream_t st) {
#define TOMO_RS_OUT(TV)                                                                                    \
    switch (odt) {                                                                                        \
        case TOMO_F32: return launch_rs_t<TV, float>(mode, epi, g, vpad, out, real, norm, st);            \
        case TOMO_BF16: return launch_rs_t<TV, __nv_bfloat16>(mode, epi, g, vpad, out, real, norm, st);   \
        case TOMO_F16: return launch_rs_t<TV, __half>(mode, epi, g, vpad, out, real, norm, st);           \
    }
    switch (vdt) {
        case TOMO_F32: TOMO_RS_OUT(float) break;
        case TOMO_BF16: TOMO_RS_OUT(__nv_bfloat16) break;
        case TOMO_F16: TOMO_RS_OUT(__half) break;
    }
#undef TOMO_RS_OUT
    return cudaErrorInvalidValue;
}

cudaError_t launch_rs_adjoint(int mode, const DevGeom& g, const void* sino, tomo_dtype sdt, float* vol,
                              cudaStream_t st) {
    dim3 block(256), grid((g.nu + 15) / 16, (g.nv + 15) / 16, g.np);
    switch (sdt) {
        case TOMO_F32:
            if (mode == 0) rs_adjoint_kernel<0, float><<<grid, block, 0, st>>>(g, (const float*)sino, vol);
            else rs_adjoint_kernel<1, float><<<grid, block, 0, st>>>(g, (const float*)sino, vol);
            break;
        case TOMO_BF16:
            if (mode == 0) rs_adjoint_kernel<0, __nv_bfloat16><<<grid, block, 0, st>>>(g, (const __nv_bfloat16*)sino, vol);
            else rs_adjoint_kernel<1, __nv_bfloat16><<<grid, block, 0, st>>>(g, (const __nv_bfloat16*)sino, vol);
            break;
        case TOMO_F16:
            if (mode == 0) rs_adjoint_kernel<0, __half><<<grid, block, 0, st>>>(g, (const __half*)sino, vol);
            else rs_adjoint_kernel<1, __half><<<grid, block, 0, st>>>(g, (const __half*)sino, vol);
            break;
    }
    return cudaGetLastError();
}

cudaError_t launch_rs_count(int mode, const DevGeom& g, unsigned long long* total, cudaStream_t st) {
    dim3 block(128), grid((g.nu + 127) / 128, g.nv, g.np);
    if (mode == 0) rs_count_kernel<0><<<grid, block, 0, st>>>(g, total);
    else rs_count_kernel<1><<<grid, block, 0, st>>>(g, total);
    return cudaGetLastError();
}

}  // namespace tomo
