// rs_device.cuh -- device code of the regular-sampling projector (samplers and the
// per-tile ray march), shared by rs_project.cu and the batched kernels in batch.cu.
// See rs_project.cu for the layouts and the parity rules.
#pragma once

#include "tex_gather.cuh"
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

// The eight texels of cell c as FP32, in [dk][dj][di] order.
template <typename Tv>
__device__ __forceinline__ void cell_load(const Tv* __restrict__ cells, long c, float (&t)[8]);
template <>
__device__ __forceinline__ void cell_load<float>(const float* __restrict__ cells, long c, float (&t)[8]) {
    const float4* p = reinterpret_cast<const float4*>(cells) + 2 * c;
    const float4 lo = __ldg(p), hi = __ldg(p + 1);
    t[0] = lo.x; t[1] = lo.y; t[2] = lo.z; t[3] = lo.w; t[4] = hi.x; t[5] = hi.y; t[6] = hi.z; t[7] = hi.w;
}
template <>
__device__ __forceinline__ void cell_load<__nv_bfloat16>(const __nv_bfloat16* __restrict__ cells, long c,
                                                         float (&t)[8]) {
    const uint4 r = __ldg(reinterpret_cast<const uint4*>(cells) + c);
    const unsigned w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        t[2 * q] = __uint_as_float(w[q] << 16);
        t[2 * q + 1] = __uint_as_float(w[q] & 0xffff0000u);
    }
}
template <>
__device__ __forceinline__ void cell_load<__half>(const __half* __restrict__ cells, long c, float (&t)[8]) {
    const uint4 r = __ldg(reinterpret_cast<const uint4*>(cells) + c);
    const unsigned w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[q]));
        t[2 * q] = f.x;
        t[2 * q + 1] = f.y;
    }
}

template <typename Tv>
__device__ __forceinline__ float trilinear_cells(const Tv* __restrict__ cells, int CW, int CWH, float fnx, float fny,
                                                 float fnz, float tx, float ty, float tz) {
    const float xb = fsub(tx, 0.5f), yb = fsub(ty, 0.5f), zb = fsub(tz, 0.5f);
    if (!(xb > -1.f && yb > -1.f && zb > -1.f && xb < fnx && yb < fny && zb < fnz)) return 0.f;
    const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    const float a = xb - fx, b = yb - fy, c = zb - fz;
    const long cell = (long)((int)fz + 1) * CWH + ((int)fy + 1) * CW + ((int)fx + 1);
    float t[8];
    cell_load(cells, cell, t);
    const float c00 = lerp(t[0], t[1], a), c10 = lerp(t[2], t[3], a);
    const float c01 = lerp(t[4], t[5], a), c11 = lerp(t[6], t[7], a);
    return lerp(lerp(c00, c10, b), lerp(c01, c11, b), c);
}

// TEX layout: the texel indices come from our own exact FP32 floor; the texture unit is
// asked for the footprint at the footprint's centre (i + 1, j + 1), half a texel away from
// any boundary, so its fixed-point coordinate rounding cannot pick other texels. Only the
// raw texel values come from the texture; the weights and lerps are ours.
// No bounds tests: slice z sits in layer z + 1 between two zero layers, and x, y outside the
// array read the border colour 0, so a sample whose footprint misses the volume gathers
// eight zeros and returns exactly 0 -- the value the texture's border gives the reference.
// (Clipped rays keep every sample within the box, so the layers used stay in [0, nz + 1].)
// 16-bit textures pack slices floor(zb) and floor(zb) + 1 in one 32-bit texel (layer
// floor(zb) + 2, see rs_vol_tex_create): one gather returns the eight texels.
__device__ __forceinline__ void unpack_pair(unsigned r, float& lo, float& hi, __nv_bfloat16*) {
    lo = __uint_as_float(r << 16);
    hi = __uint_as_float(r & 0xffff0000u);
}
__device__ __forceinline__ void unpack_pair(unsigned r, float& lo, float& hi, __half*) {
    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&r));
    lo = f.x;
    hi = f.y;
}

template <typename Tt>
__device__ __forceinline__ float trilinear_tex(unsigned long long tex, float tx, float ty, float tz) {
    const float xb = fsub(tx, 0.5f), yb = fsub(ty, 0.5f), zb = fsub(tz, 0.5f);
    const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    const float a = xb - fx, b = yb - fy, c = zb - fz;
    const float gx = fx + 1.0f, gy = fy + 1.0f;
    float4 lo, hi;
    if constexpr (sizeof(Tt) == 2) {
        const uint4 r = gather_layer_raw(tex, (int)fz + 2, gx, gy);
        unpack_pair(r.x, lo.x, hi.x, (Tt*)nullptr);
        unpack_pair(r.y, lo.y, hi.y, (Tt*)nullptr);
        unpack_pair(r.z, lo.z, hi.z, (Tt*)nullptr);
        unpack_pair(r.w, lo.w, hi.w, (Tt*)nullptr);
    } else {
        const int layer = (int)fz + 1;  // layer of slice floor(zb)
        lo = gather_layer<Tt>(tex, layer, gx, gy);
        hi = gather_layer<Tt>(tex, layer + 1, gx, gy);
    }
    const float c00 = lerp(lo.w, lo.z, a), c10 = lerp(lo.x, lo.y, a);
    const float c01 = lerp(hi.w, hi.z, a), c11 = lerp(hi.x, hi.y, a);
    return lerp(lerp(c00, c10, b), lerp(c01, c11, b), c);
}

// Row pairs of the HYBRID layout: pair (pi, pj, pk) holds texels (pi-1, pj-1, pk) and
// (pi, pj-1, pk) of one slice, 8 B (FP32) or 4 B (16-bit), so the 2 x 2 footprint of a
// slice is two aligned loads of consecutive rows. Returned as FP32.
template <typename Tv>
__device__ __forceinline__ float2 pair_load(const Tv* __restrict__ pairs, long c);
template <>
__device__ __forceinline__ float2 pair_load<float>(const float* __restrict__ pairs, long c) {
    return __ldg(reinterpret_cast<const float2*>(pairs) + c);
}
template <>
__device__ __forceinline__ float2 pair_load<__nv_bfloat16>(const __nv_bfloat16* __restrict__ pairs, long c) {
    const unsigned r = __ldg(reinterpret_cast<const unsigned*>(pairs) + c);
    return make_float2(__uint_as_float(r << 16), __uint_as_float(r & 0xffff0000u));
}
template <>
__device__ __forceinline__ float2 pair_load<__half>(const __half* __restrict__ pairs, long c) {
    const unsigned r = __ldg(reinterpret_cast<const unsigned*>(pairs) + c);
    return __half22float2(*reinterpret_cast<const __half2*>(&r));
}

// HYBRID layout: the lower slice floor(zb) from the zero-layered volume texture (one gather,
// texture path) and the upper slice from two row pairs in global memory (two 8 B / 4 B
// loads, load/store path), so a sample's texel traffic is split between the two pipes.
// Pairs are indexed (pi, pj, pk), pi in [0, nx], pj in [0, ny + 1], pk in [0, nz] (slice nz
// and texels outside x, y are 0). Same texel values and arithmetic as the other layouts.
// Samples can lie outside the volume (the reference clips to a box and a cylinder sized by
// nx alone, so with ny < nx rays pass beyond the y extent): a footprint outside the stored
// pairs is all zero texels, and those loads are skipped.
// A second array holds column pairs, pair (qi, qj, qk) = texels (qi-1, qj-1, qk) and
// (qi-1, qj, qk), qi in [0, nx + 1], qj in [0, ny], stored with qj fastest. Views whose rays
// run mostly along x (|cos phi| > |sin phi|) read it: their adjacent-u rays are adjacent in
// y, so a warp's column pairs are consecutive in memory, as a warp's row pairs are for the
// other views. Same texel values and arithmetic either way.
template <typename Tv, bool YPAIRS>
__device__ __forceinline__ float trilinear_hybrid(unsigned long long tex, const Tv* __restrict__ pairs, int PW, long PWH,
                                                  int nx, int ny, int nz, float tx, float ty, float tz) {
    const float xb = fsub(tx, 0.5f), yb = fsub(ty, 0.5f), zb = fsub(tz, 0.5f);
    const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    const float a = xb - fx, b = yb - fy, c = zb - fz;
    const int layer = (int)fz + 1;  // texture layer of slice floor(zb); also the cell slice above it
    const float4 lo = gather_layer<Tv>(tex, layer, fx + 1.0f, fy + 1.0f);
    const int ci = (int)fx + 1, cj = (int)fy + 1, ck = layer;
    float2 r0 = make_float2(0.f, 0.f), r1 = r0;
    if ((unsigned)ci <= (unsigned)nx && (unsigned)cj <= (unsigned)ny && (unsigned)ck <= (unsigned)nz) {
        if (YPAIRS) {  // columns ci, ci + 1 of rows cj-1, cj: (r0.x, r1.x) row cj-1, (r0.y, r1.y) row cj
            const long qc = ck * PWH + (long)ci * PW + cj;
            const float2 q0 = pair_load(pairs, qc), q1 = pair_load(pairs, qc + PW);
            r0 = make_float2(q0.x, q1.x);
            r1 = make_float2(q0.y, q1.y);
        } else {
            const long pc = ck * PWH + (long)cj * PW + ci;
            r0 = pair_load(pairs, pc);
            r1 = pair_load(pairs, pc + PW);
        }
    }
    const float c00 = lerp(lo.w, lo.z, a), c10 = lerp(lo.x, lo.y, a);
    const float c01 = lerp(r0.x, r0.y, a), c11 = lerp(r1.x, r1.y, a);
    return lerp(lerp(c00, c10, b), lerp(c01, c11, b), c);
}

// One 16u x 16v tile of view p (256 threads, warps on 8u x 4v sub-tiles): ray set-up,
// trilinear march, epilogue. Shared by the single-job kernel and the batched persistent
// kernel (batch.cu); must be called by all 256 threads of the block (EPI_NORM syncs).
template <int MODE, int LAYOUT, typename Tv, typename To, int EPI, typename Tr = To>
__device__ __forceinline__ void rs_tile(const DevGeom& g, const Tv* __restrict__ vin, unsigned long long tex,
                                        const OutView<To>& out, const OutView<Tr>& real, double* __restrict__ norm,
                                        int p, int ut, int vt) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = ut * 16 + (warp & 1) * 8 + (lane & 7);
    const int v = vt * 16 + (warp >> 1) * 4 + (lane >> 3);
    const bool active = (u < g.nu) && (v < g.nv);
    float acc = 0.f;
    if (active) {
        RsRay r;
        const bool hit = MODE == 0 ? rs_ray_box(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r)
                                   : rs_ray_um(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r);
        if (hit) {
            const bool cellw = LAYOUT == RS_LAYOUT_CELL8 || LAYOUT == RS_LAYOUT_HYBRID;
            const int W = cellw ? g.nx + 1 : g.nx + 2;
            const int WH = LAYOUT == RS_LAYOUT_CELL8    ? (g.nx + 1) * (g.ny + 1)
                           : LAYOUT == RS_LAYOUT_HYBRID ? (g.nx + 1) * (g.ny + 2)
                                                        : (g.nx + 2) * (g.ny + 2);
            const float fnx = (float)g.nx, fny = (float)g.ny, fnz = (float)g.nz;
            float A = r.A, B = r.B, C = r.C;
            const float dx = g.dx;
            auto march = [&](auto sample) {
                for (unsigned n = 0; n < r.n; ++n) {
                    const float tx = fadd(A, 0.5f), ty = fadd(B, 0.5f), tz = fadd(C, 0.5f);
                    acc = fadd(acc, fmul(dx, sample(tx, ty, tz)));
                    A = fadd(A, r.sx);
                    B = fadd(B, r.sy);
                    C = fadd(C, r.sz);
                }
            };
            if (LAYOUT == RS_LAYOUT_HYBRID) {
                // the view's rays run mostly along x: column pairs (second array), else row pairs
                if (fabsf(__ldg(g.alpha + p)) > fabsf(__ldg(g.beta + p))) {
                    const Tv* cols = vin + (size_t)2 * WH * (g.nz + 1);
                    const int QW = g.ny + 1;
                    const long QWH = (long)QW * (g.nx + 2);
                    march([&](float tx, float ty, float tz) {
                        return trilinear_hybrid<Tv, true>(tex, cols, QW, QWH, g.nx, g.ny, g.nz, tx, ty, tz);
                    });
                } else {
                    march([&](float tx, float ty, float tz) {
                        return trilinear_hybrid<Tv, false>(tex, vin, W, WH, g.nx, g.ny, g.nz, tx, ty, tz);
                    });
                }
            } else {
                march([&](float tx, float ty, float tz) {
                    return LAYOUT == RS_LAYOUT_CELL8 ? trilinear_cells(vin, W, WH, fnx, fny, fnz, tx, ty, tz)
                           : LAYOUT == RS_LAYOUT_TEX ? trilinear_tex<Tv>(tex, tx, ty, tz)
                                                     : trilinear_padded(vin, W, WH, fnx, fny, fnz, tx, ty, tz);
                });
            }
        }
    }
    epilogue<EPI, To, Tr>(active, acc, u, v, p, out, real, norm);
}


}  // namespace tomo
