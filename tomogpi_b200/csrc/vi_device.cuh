// vi_device.cuh -- device code of the VI backprojector (one tile of voxel columns),
// shared by vi_back.cu and the batched kernels in batch.cu. See vi_back.cu.
#pragma once

#include <type_traits>

#include "tex_gather.cuh"
#include "tomo_kernels.cuh"

namespace tomo {

constexpr int VI_BX = 32, VI_BY = 8;

// One tile of 32 x 8 columns x (16 ZC) slices (256 threads, x fastest). Shared by the
// single-job kernel and the batched persistent kernel (batch.cu); no block-level syncs.
// FDK: the weighted form of FDK3D_VIB_kernel_v0_16reg (FDK3D_kernel_16reg.cuh:24-349): every
// sample is multiplied by alphaC (FDD/du) / denum^2 / sqrt(betaC + u'^2 + v'^2), with
// denum = x' alpha dx + y' beta dx + FOD (:77-84); all views take A in float (:73) and the
// result is not multiplied by dx.
template <int UM, int ZC, typename Ts, typename Tv, bool FDK = false>
__device__ __forceinline__ void vi_tile(const DevGeom& g, const Ts* __restrict__ spad, Tv* __restrict__ vol, float scale,
                                        int xt, int yt, int zg) {
    const int x = xt * VI_BX + (threadIdx.x & (VI_BX - 1));
    const int y = yt * VI_BY + threadIdx.x / VI_BX;
    const int z0 = zg * (16 * ZC);
    if (x >= g.nx || y >= g.ny) return;
    const float xn = fsub((float)x, g.xc);
    const float yn = fsub((float)y, g.yc);
    const int W = g.nu + 2;
    const long VP = (long)(g.nu + 2) * (g.nv + 2);
    const float fnu = (float)g.nu, fnv = (float)g.nv;
    float zp[ZC];
#pragma unroll
    for (int c = 0; c < ZC; ++c) zp[c] = fsub((float)(z0 + 16 * c), g.zc);
    float acc[ZC][16];
#pragma unroll
    for (int c = 0; c < ZC; ++c)
#pragma unroll
        for (int k = 0; k < 16; ++k) acc[c][k] = 0.f;

    for (int p = 0; p < g.np; ++p) {
        const float4 cv = __ldg(g.vi + p);
        float A = fdiv(1.0f, fadd(fadd(fmul(cv.z, xn), fmul(cv.w, yn)), g.fod));          // :401
        const float up = fmul(fadd(fmul(cv.x, xn), fmul(cv.y, yn)), A);                  // u' (:403)
        const float un = fadd(fadd(up, g.uc), 0.5f);
        A = (p + g.p0 == 0 && !FDK) ? __double2float_rn(dmul(g.inv_gamma_d, (double)A))  // :404
                             : fmul(g.inv_gamma_f, A);                                  // :464
        const float ub = fsub(un, 0.5f);
        if (!(ub > -1.f && ub < fnu)) continue;  // the whole column footprint is border
        const float fu = floorf(ub);
        const float a = ub - fu;
        const Ts* col = spad + p * VP + ((int)fu + 1);
        float fnum = 0.f, upc = 0.f;
        if (FDK) {  // FDK3D_kernel_16reg.cuh:77-80
            const float denum = fadd(fadd(fmul(fmul(xn, __ldg(g.alpha + p)), g.dx), fmul(fmul(yn, __ldg(g.beta + p)), g.dx)),
                                     g.fod);
            fnum = fdiv(fmul(g.fdk_alpha, g.fdd_du), fmul(denum, denum));
            upc = fmul(up, up);
        }
#pragma unroll
        for (int c = 0; c < ZC; ++c) {
            float vp = fmul(A, zp[c]);                                                   // v' (:75)
            float vn = fadd(fadd(vp, g.vc), 0.5f);                                      // :405
            // The chunk's rows grow with k (A > 0). When the first sample is inside the
            // detector and vn + 16 A, an upper bound of the last one (15 rounded additions of
            // values below 8192 err by less than 0.01 < A), is below nv, no sample of the chunk
            // needs the bounds test: the chunk runs without it.
            const bool inside = !FDK && A > 0.25f && fnv <= 8192.f && fsub(vn, 0.5f) > -1.f &&
                                fadd(vn, fmul(16.0f, A)) < fnv;
            auto chunk = [&](auto checked) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const float vk = UM ? fadd(vn, fmul((float)k, A)) : vn;
                const float vb = fsub(vk, 0.5f);
                if (!decltype(checked)::value || (vb > -1.f && vb < fnv)) {
                    const float fv = floorf(vb);
                    const float b = vb - fv;
                    const Ts* q = col + ((int)fv + 1) * W;
                    const float s0 = lerp(ld(q), ld(q + 1), a);
                    const float s1 = lerp(ld(q + W), ld(q + W + 1), a);
                    const float t = lerp(s0, s1, b);
                    if (FDK) {  // :81-84
                        const float w = fdiv(fnum, fsqrt(fadd(g.fdk_beta, fadd(upc, fmul(vp, vp)))));
                        acc[c][k] = fadd(acc[c][k], fmul(w, t));
                    } else {
                        acc[c][k] = fadd(acc[c][k], t);
                    }
                }
                if (!UM) vn = fadd(vn, A);                                              // :410
                if (FDK) vp = fadd(vp, A);
            }
            };
            if (inside)
                chunk(std::false_type{});
            else
                chunk(std::true_type{});
        }
    }
    const long plane = (long)g.nx * g.ny;
#pragma unroll
    for (int c = 0; c < ZC; ++c)
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int z = z0 + 16 * c + k;
            if (z < g.nz)
                vol[z * plane + (long)y * g.nx + x] = cvt<Tv>(FDK ? fmul(acc[c][k], scale) : fmul(fmul(acc[c][k], g.dx), scale));
        }
}

// The same tile reading the sinogram from a 2D layered texture (one layer per view, border
// colour 0, texels in the sinogram's type): one 4-texel gather per (voxel, view) at the
// footprint's centre, weights and lerps in software as above. A footprint outside the
// detector gathers four border zeros and adds exactly 0, so no per-voxel bounds test is
// needed; a column whose footprint misses the detector for a whole view still skips it.
template <int UM, int ZC, typename Tt, typename Tv>
__device__ __forceinline__ void vi_tile_tex(const DevGeom& g, unsigned long long tex, Tv* __restrict__ vol, float scale,
                                            int xt, int yt, int zg) {
    const int x = xt * VI_BX + (threadIdx.x & (VI_BX - 1));
    const int y = yt * VI_BY + threadIdx.x / VI_BX;
    const int z0 = zg * (16 * ZC);
    if (x >= g.nx || y >= g.ny) return;
    const float xn = fsub((float)x, g.xc);
    const float yn = fsub((float)y, g.yc);
    const float fnu = (float)g.nu;
    float zp[ZC];
#pragma unroll
    for (int c = 0; c < ZC; ++c) zp[c] = fsub((float)(z0 + 16 * c), g.zc);
    float acc[ZC][16];
#pragma unroll
    for (int c = 0; c < ZC; ++c)
#pragma unroll
        for (int k = 0; k < 16; ++k) acc[c][k] = 0.f;

    for (int p = 0; p < g.np; ++p) {
        const float4 cv = __ldg(g.vi + p);
        float A = fdiv(1.0f, fadd(fadd(fmul(cv.z, xn), fmul(cv.w, yn)), g.fod));          // :401
        const float un = fadd(fadd(fmul(fadd(fmul(cv.x, xn), fmul(cv.y, yn)), A), g.uc), 0.5f);  // :403
        A = (p + g.p0 == 0) ? __double2float_rn(dmul(g.inv_gamma_d, (double)A))          // :404
                     : fmul(g.inv_gamma_f, A);                                          // :464
        const float ub = fsub(un, 0.5f);
        if (!(ub > -1.f && ub < fnu)) continue;  // the whole column footprint is border
        const float fu = floorf(ub);
        const float a = ub - fu;
        const float gu = fu + 1.0f;
#pragma unroll
        for (int c = 0; c < ZC; ++c) {
            float vn = fadd(fadd(fmul(A, zp[c]), g.vc), 0.5f);                          // :405
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const float vk = UM ? fadd(vn, fmul((float)k, A)) : vn;
                const float vb = fsub(vk, 0.5f);
                const float fv = floorf(vb);
                const float b = vb - fv;
                const float4 t = gather_layer<Tt>(tex, p, gu, fv + 1.0f);
                const float s0 = lerp(t.w, t.z, a);
                const float s1 = lerp(t.x, t.y, a);
                acc[c][k] = fadd(acc[c][k], lerp(s0, s1, b));
                if (!UM) vn = fadd(vn, A);                                              // :410
            }
        }
    }
    const long plane = (long)g.nx * g.ny;
#pragma unroll
    for (int c = 0; c < ZC; ++c)
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int z = z0 + 16 * c + k;
            if (z < g.nz) vol[z * plane + (long)y * g.nx + x] = cvt<Tv>(fmul(fmul(acc[c][k], g.dx), scale));
        }
}

}  // namespace tomo
