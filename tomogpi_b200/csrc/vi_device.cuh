// vi_device.cuh -- device code of the VI backprojector (one tile of voxel columns),
// shared by vi_back.cu and the batched kernels in batch.cu. See vi_back.cu.
#pragma once

#include <type_traits>

#include "tex_gather.cuh"
#include "tomo_kernels.cuh"

namespace tomo {

constexpr int VI_BX = 32, VI_BY = 8;
// Resident blocks per SM the VI kernels are compiled for (a register budget): 16 slices per
// thread fit 5 blocks (48 registers) without spilling; left free, the compiler trades
// residency for registers.
constexpr int vi_min_blocks(int zc) { return zc == 1 ? 5 : zc == 2 ? 2 : 1; }

// Floors of the VI backprojector, as in the RS projector (rs_device.cuh): adding 1.5 * 2^23
// with rounding toward -inf gives floor(v) + 1.5 * 2^23 exactly for |v| < 2^22.
constexpr float VI_FLOOR_K = 12582912.0f;
constexpr int VI_FLOOR_KBITS = 0x4B400000;

// One tile of 32 x 8 columns x (16 ZC) slices (256 threads, x fastest). Shared by the
// single-job kernel and the batched persistent kernel (batch.cu); no block-level syncs.
// The sixteen slices of a chunk are processed in pairs as f32x2 lanes (__fadd2_rn,
// __ffma2_rn: each lane rounds like the scalar operation): the row coordinate, its floor
// and weight, the three lerps and the accumulation of slices k and k + 1 are one packed
// instruction each, while the row coordinate itself still advances by repeated scalar
// addition of A (:410) -- the same values and operation order as one slice at a time.
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
    const float2 MH = make_float2(-0.5f, -0.5f), K = make_float2(VI_FLOOR_K, VI_FLOOR_K);
    const float2 MK = make_float2(-VI_FLOOR_K, -VI_FLOOR_K), M1 = make_float2(-1.0f, -1.0f);
    float zp[ZC];
#pragma unroll
    for (int c = 0; c < ZC; ++c) zp[c] = fsub((float)(z0 + 16 * c), g.zc);
    float2 acc[ZC][8];
#pragma unroll
    for (int c = 0; c < ZC; ++c)
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[c][k] = make_float2(0.f, 0.f);

    for (int p = 0; p < g.np; ++p) {
        const float4 cv = __ldg(g.vi + p);
        float A = frcp(fadd(fadd(fmul(cv.z, xn), fmul(cv.w, yn)), g.fod));                 // :401
        const float up = fmul(fadd(fmul(cv.x, xn), fmul(cv.y, yn)), A);                  // u' (:403)
        const float un = fadd(fadd(up, g.uc), 0.5f);
        A = (p + g.p0 == 0 && !FDK) ? __double2float_rn(dmul(g.inv_gamma_d, (double)A))  // :404
                             : fmul(g.inv_gamma_f, A);                                  // :464
        const float ub = fsub(un, 0.5f);
        if (!(ub > -1.f && ub < fnu)) continue;  // the whole column footprint is border
        const float fu = floorf(ub);
        const float a = ub - fu;
        const float2 aa = make_float2(a, a), na = make_float2(-a, -a);
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
            if (FDK) {
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    const float vb = fsub(vn, 0.5f);
                    if (vb > -1.f && vb < fnv) {
                        const float fv = floorf(vb);
                        const float b = vb - fv;
                        const Ts* q = col + ((int)fv + 1) * W;
                        const float s0 = lerp(ld(q), ld(q + 1), a);
                        const float s1 = lerp(ld(q + W), ld(q + W + 1), a);
                        const float t = lerp(s0, s1, b);
                        const float w = fdiv(fnum, fsqrt(fadd(g.fdk_beta, fadd(upc, fmul(vp, vp)))));  // :81-84
                        float& dst = (k & 1) ? acc[c][k >> 1].y : acc[c][k >> 1].x;
                        dst = fadd(dst, fmul(w, t));
                    }
                    vn = fadd(vn, A);
                    vp = fadd(vp, A);
                }
                continue;
            }
            auto chunk = [&](auto checked) {
#pragma unroll
                for (int k = 0; k < 16; k += 2) {
                    float2 vk;
                    if (UM) {  // v_k = v_0 + k A (_UM.cuh); the products by the scalar, never-fused
                               // multiply (a packed multiply feeding a packed add may be fused)
                        vk = __fadd2_rn(make_float2(vn, vn), make_float2(fmul((float)k, A), fmul((float)(k + 1), A)));
                    } else {   // v += A per slice (:410)
                        vk.x = vn;
                        vn = fadd(vn, A);
                        vk.y = vn;
                        vn = fadd(vn, A);
                    }
                    const float2 vb = __fadd2_rn(vk, MH);
                    const float2 m = __fadd2_rd(vb, K);
                    const float2 f = __fadd2_rn(m, MK);
                    const float2 b = __ffma2_rn(f, M1, vb), nb = __ffma2_rn(vb, M1, f);
                    const bool ok0 = !decltype(checked)::value || (vb.x > -1.f && vb.x < fnv);
                    const bool ok1 = !decltype(checked)::value || (vb.y > -1.f && vb.y < fnv);
                    const Ts* q0 = col + (__float_as_int(m.x) - (VI_FLOOR_KBITS - 1)) * W;  // row floor + 1
                    const Ts* q1 = col + (__float_as_int(m.y) - (VI_FLOOR_KBITS - 1)) * W;
                    const float2 t00 = make_float2(ok0 ? ld(q0) : 0.f, ok1 ? ld(q1) : 0.f);
                    const float2 t10 = make_float2(ok0 ? ld(q0 + 1) : 0.f, ok1 ? ld(q1 + 1) : 0.f);
                    const float2 t01 = make_float2(ok0 ? ld(q0 + W) : 0.f, ok1 ? ld(q1 + W) : 0.f);
                    const float2 t11 = make_float2(ok0 ? ld(q0 + W + 1) : 0.f, ok1 ? ld(q1 + W + 1) : 0.f);
                    const float2 s0 = __ffma2_rn(aa, t10, __ffma2_rn(na, t00, t00));
                    const float2 s1 = __ffma2_rn(aa, t11, __ffma2_rn(na, t01, t01));
                    const float2 t = __ffma2_rn(b, s1, __ffma2_rn(nb, s0, s0));
                    acc[c][k >> 1] = __fadd2_rn(acc[c][k >> 1], t);
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
            const float r = (k & 1) ? acc[c][k >> 1].y : acc[c][k >> 1].x;
            if (z < g.nz)
                vol[z * plane + (long)y * g.nx + x] = cvt<Tv>(FDK ? fmul(r, scale) : fmul(fmul(r, g.dx), scale));
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
        float A = frcp(fadd(fadd(fmul(cv.z, xn), fmul(cv.w, yn)), g.fod));                 // :401
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
