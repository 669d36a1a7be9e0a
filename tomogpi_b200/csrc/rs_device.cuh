// rs_device.cuh -- device code of the regular-sampling projector (samplers and the
// per-tile ray march), shared by rs_project.cu and the batched kernels in batch.cu.
// See rs_project.cu for the layouts and the parity rules.
#pragma once

#include <type_traits>

#include "tex_gather.cuh"
#include "tomo_kernels.cuh"

namespace tomo {

// ---------------------------------------------------------------------------------
// One trilinear sample, sm_100 packed FP32.
//
// The reference samples tex3D at t = P + 0.5 (P the ray position, projection_ER_kernel.cuh
// :292) and the exact-FP32 filter reads the texels around v = t - 0.5 with weights
// v - floor(v). Both roundings are kept (t and v are computed as written); the floors are
// exact: adding 1.5 * 2^23 with rounding toward -inf gives floor(v) + 1.5 * 2^23 exactly for
// |v| < 2^22 (the spacing of floats in [2^23, 2^24) is 1), so the float floor is that sum
// minus the constant and the integer floor is its bit pattern minus the constant's. This
// keeps every floor and conversion off the XU pipe, and the x / y (and duplicated z)
// coordinates run as f32x2 pairs (__fadd2_rn, __ffma2_rn round each lane like the scalar
// operation). Every layout interpolates the same way: first between the two slices (two
// packed lerps over the four texel columns), then along x, then along y, so all layouts
// give bit-identical sums.
// ---------------------------------------------------------------------------------
constexpr float FLOOR_K = 12582912.0f;   // 1.5 * 2^23
constexpr int FLOOR_KBITS = 0x4B400000;  // its bit pattern

struct RsSample {
    float2 v;       // (xb, yb): texel-space position
    float vz;       // zb
    float fz;       // floor(zb)
    float2 f;       // (floor(xb), floor(yb))
    float2 w;       // (xb - floor(xb), yb - floor(yb)), exact
    float2 cc, ncc; // (c, c), (-c, -c), c = zb - floor(zb)
    int ix, iy, iz; // floor + FLOOR_KBITS, as integers
};

__device__ __forceinline__ RsSample rs_sample(float2 AB, float2 CC) {
    const float2 H = make_float2(0.5f, 0.5f), MH = make_float2(-0.5f, -0.5f);
    const float2 K = make_float2(FLOOR_K, FLOOR_K), MK = make_float2(-FLOOR_K, -FLOOR_K);
    const float2 M1 = make_float2(-1.0f, -1.0f);
    RsSample s;
    s.v = __fadd2_rn(__fadd2_rn(AB, H), MH);
    const float2 vzz = __fadd2_rn(__fadd2_rn(CC, H), MH);
    s.vz = vzz.x;
    const float2 m = __fadd2_rd(s.v, K), mz = __fadd2_rd(vzz, K);
    s.f = __fadd2_rn(m, MK);
    const float2 fz = __fadd2_rn(mz, MK);
    s.fz = fz.x;
    s.w = __ffma2_rn(s.f, M1, s.v);
    s.cc = __ffma2_rn(fz, M1, vzz);
    s.ncc = __ffma2_rn(vzz, M1, fz);
    s.ix = __float_as_int(m.x);
    s.iy = __float_as_int(m.y);
    s.iz = __float_as_int(mz.x);
    return s;
}

__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 t, float2 nt) {
    return __ffma2_rn(t, b, __ffma2_rn(nt, a, a));
}

// Trilinear value from the eight texels of a sample's footprint, each slice as a float4 in
// tld4 order: (T[i][j+1], T[i+1][j+1], T[i+1][j], T[i][j]), lo = slice k, up = slice k + 1.
__device__ __forceinline__ float trilerp(float4 lo, float4 up, const RsSample& s) {
    const float2 z1 = lerp2(make_float2(lo.x, lo.y), make_float2(up.x, up.y), s.cc, s.ncc);  // row j+1: i, i+1
    const float2 z0 = lerp2(make_float2(lo.z, lo.w), make_float2(up.z, up.w), s.cc, s.ncc);  // row j: i+1, i
    const float r1 = lerp(z1.x, z1.y, s.w.x);
    const float r0 = lerp(z0.y, z0.x, s.w.x);
    return lerp(r0, r1, s.w.y);
}

__device__ __forceinline__ bool rs_inside(const RsSample& s, float fnx, float fny, float fnz) {
    return s.v.x > -1.f && s.v.y > -1.f && s.vz > -1.f && s.v.x < fnx && s.v.y < fny && s.vz < fnz;
}

// PLAIN layout: zero-bordered padded volume, eight scalar loads; 0 outside the volume.
template <typename Tv>
__device__ __forceinline__ float trilinear_padded(const Tv* __restrict__ vp, int W, int WH, float fnx, float fny,
                                                  float fnz, const RsSample& s) {
    if (!rs_inside(s, fnx, fny, fnz)) return 0.f;
    const int i = s.ix - (FLOOR_KBITS - 1), j = s.iy - (FLOOR_KBITS - 1), k = s.iz - (FLOOR_KBITS - 1);
    const Tv* q = vp + (k * WH + j * W + i);
    const float4 lo = make_float4(ld(q + W), ld(q + W + 1), ld(q + 1), ld(q));
    const float4 up = make_float4(ld(q + WH + W), ld(q + WH + W + 1), ld(q + WH + 1), ld(q + WH));
    return trilerp(lo, up, s);
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

// CELL8 layout: the eight texels of every cell stored together; 0 outside the volume.
template <typename Tv>
__device__ __forceinline__ float trilinear_cells(const Tv* __restrict__ cells, int CW, int CWH, float fnx, float fny,
                                                 float fnz, const RsSample& s) {
    if (!rs_inside(s, fnx, fny, fnz)) return 0.f;
    const long cell = (long)(s.iz - (FLOOR_KBITS - 1)) * CWH + (s.iy - (FLOOR_KBITS - 1)) * CW +
                      (s.ix - (FLOOR_KBITS - 1));
    float t[8];
    cell_load(cells, cell, t);
    return trilerp(make_float4(t[2], t[3], t[1], t[0]), make_float4(t[6], t[7], t[5], t[4]), s);
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
__device__ __forceinline__ float trilinear_tex(unsigned long long tex, const RsSample& s) {
    const float2 g = __fadd2_rn(s.f, make_float2(1.0f, 1.0f));  // footprint centre
    float4 lo, hi;
    if constexpr (sizeof(Tt) == 2) {
        const uint4 r = gather_layer_raw(tex, s.iz - (FLOOR_KBITS - 2), g.x, g.y);
        unpack_pair(r.x, lo.x, hi.x, (Tt*)nullptr);
        unpack_pair(r.y, lo.y, hi.y, (Tt*)nullptr);
        unpack_pair(r.z, lo.z, hi.z, (Tt*)nullptr);
        unpack_pair(r.w, lo.w, hi.w, (Tt*)nullptr);
    } else {
        const int layer = s.iz - (FLOOR_KBITS - 1);  // layer of slice floor(zb)
        lo = gather_layer<Tt>(tex, layer, g.x, g.y);
        hi = gather_layer<Tt>(tex, layer + 1, g.x, g.y);
    }
    return trilerp(lo, hi, s);
}

// Quads of the HYBRID layout: quad (ci, cj, k) holds the four texels of slice k around the
// footprint i = ci - 1, j = cj - 1 in tld4 order, (T[i][j+1], T[i+1][j+1], T[i+1][j], T[i][j])
// (0 outside the volume), 16 B (FP32) or 8 B (16-bit); returned as FP32.
template <typename Tv>
__device__ __forceinline__ float4 quad_load(const Tv* __restrict__ quads, unsigned q);
template <>
__device__ __forceinline__ float4 quad_load<float>(const float* __restrict__ quads, unsigned q) {
    return __ldg(reinterpret_cast<const float4*>(quads) + q);
}
template <>
__device__ __forceinline__ float4 quad_load<__nv_bfloat16>(const __nv_bfloat16* __restrict__ quads, unsigned q) {
    const uint2 r = __ldg(reinterpret_cast<const uint2*>(quads) + q);
    return make_float4(__uint_as_float(r.x << 16), __uint_as_float(r.x & 0xffff0000u), __uint_as_float(r.y << 16),
                       __uint_as_float(r.y & 0xffff0000u));
}
template <>
__device__ __forceinline__ float4 quad_load<__half>(const __half* __restrict__ quads, unsigned q) {
    const uint2 r = __ldg(reinterpret_cast<const uint2*>(quads) + q);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
    return make_float4(a.x, a.y, b.x, b.y);
}

// HYBRID layout: the lower slice floor(zb) from the zero-layered volume texture (one gather,
// texture path) and the upper slice from one quad in global memory (one 16 B / 8 B load,
// load/store path), so a sample's texel traffic is split between the two pipes. Quads are
// indexed (ci, cj, ck), ci in [0, nx], cj in [0, ny], ck in [0, nz] (slice nz is zero), in
// two arrays: row quads (ci fastest), read by views whose rays run mostly along y, and
// column quads (cj fastest), read by views whose rays run mostly along x (|cos phi| >
// |sin phi|): either way a warp's adjacent-u rays read consecutive quads.
// CHECKED: a footprint outside the stored quads reads zero texels and skips the load (rays
// that can leave the volume); otherwise the ray was shown to stay inside (rs_ray_inside) and
// the index is only clamped, as a guard, to the array.
struct QuadIndex {
    int qw, qwh;        // row pitch and slice pitch of the quad array
    unsigned bias;      // the index's offset from the biased integer floors
    unsigned qmax;      // last quad of the array
};

template <typename Tv, bool COLS, bool CHECKED>
__device__ __forceinline__ float trilinear_hybrid(unsigned long long tex, const Tv* __restrict__ quads,
                                                  const QuadIndex& Q, int nx, int ny, int nz, const RsSample& s) {
    const float2 g = __fadd2_rn(s.f, make_float2(1.0f, 1.0f));
    const int layer = s.iz - (FLOOR_KBITS - 1);  // texture layer of slice floor(zb); also the quad slice above it
    const float4 lo = gather_layer<Tv>(tex, layer, g.x, g.y);
    const unsigned q = (unsigned)s.iz * (unsigned)Q.qwh + (COLS ? (unsigned)s.ix * Q.qw + (unsigned)s.iy
                                                                : (unsigned)s.iy * Q.qw + (unsigned)s.ix) - Q.bias;
    float4 up;
    if (CHECKED) {
        const unsigned ci = (unsigned)(s.ix - (FLOOR_KBITS - 1)), cj = (unsigned)(s.iy - (FLOOR_KBITS - 1));
        up = (ci <= (unsigned)nx && cj <= (unsigned)ny && (unsigned)layer <= (unsigned)nz) ? quad_load(quads, q)
                                                                                           : make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
        up = quad_load(quads, min(q, Q.qmax));
    }
    return trilerp(lo, up, s);
}

__host__ __device__ __forceinline__ QuadIndex hybrid_quad_index(int nx, int ny, int nz, bool cols) {
    QuadIndex Q;
    Q.qw = cols ? ny + 1 : nx + 1;
    Q.qwh = (nx + 1) * (ny + 1);
    // q = ck qwh + cj qw + ci with ck = iz - (K - 1) etc.: the constant part, modulo 2^32
    Q.bias = (unsigned)(FLOOR_KBITS - 1) * ((unsigned)Q.qwh + (unsigned)Q.qw + 1u);
    Q.qmax = (unsigned)((long)Q.qwh * (nz + 1) - 1);
    return Q;
}

// MARCH layout (see tomo_kernels.cuh): a sample at floors (i, j, k) needs the faces m and
// m + 1 of the march axis (m = i for x-march, j for y-march) over the footprint (t, k),
// t the other in-plane floor. One of the two faces is even (a texture gather of layer
// layer0 + m / 2 at the footprint centre (t + 1, k + 1)), the other odd (one 16 B quad).
// Consecutive samples of a ray often share the footprint (t, k) (its transverse and z
// floors change on about 40% of the steps at 512^3) and then at least one face: the last
// even and the last odd face are kept with their m, and a face is fetched only when its m
// or the footprint changed, about 1.4 face fetches per sample in place of 2. The values
// are the same texels wherever they come from, so the sums are bit-identical to the other
// layouts'.
struct MarchIndex {
    int qt;             // quads per k row (n_t + 1)
    unsigned qz;        // quads per face ((nz + 1)(n_t + 1))
    unsigned bias;      // the quad index's offset from the biased integer floors
    unsigned qmax;      // last quad of the array
    int layer0;         // texture layer of face 0 minus FLOOR_KBITS / 2 (mod 2^32)
    int na, nt;         // march-axis and transverse sizes
};

__host__ __device__ __forceinline__ MarchIndex march_index(int nx, int ny, int nz, bool xmarch) {
    MarchIndex M;
    M.na = xmarch ? nx : ny;
    M.nt = xmarch ? ny : nx;
    M.qt = M.nt + 1;
    M.qz = (unsigned)(nz + 1) * (unsigned)M.qt;
    // odd face o = m | 1 of a sample at march floor m sits at ((o + 1) / 2) = (m >> 1) + 1
    // (floor division) in the face order; q = ((m >> 1) + 1) qz + (k + 1) qt + (t + 1). With
    // biased floors M = m + K, T = t + K, Z = k + K (K = FLOOR_KBITS, even):
    // q = (M >> 1) qz + Z qt + T - bias
    M.bias = (unsigned)(FLOOR_KBITS / 2 - 1) * M.qz + (unsigned)(FLOOR_KBITS - 1) * (unsigned)M.qt +
             (unsigned)(FLOOR_KBITS - 1);
    M.qmax = (unsigned)(march_quads(M.na, M.nt, nz) - 1);
    M.layer0 = (xmarch ? 0 : march_even_faces(nx)) - FLOOR_KBITS / 2;
    return M;
}

// One MARCH sample. State (kept across the ray's samples): PE / PO the last even / odd
// face (tld4 order over (t, k): T(t, k+1), T(t+1, k+1), T(t+1, k), T(t, k)), pe / po their
// biased m (0 before the first fetch), pkey the footprint (t, k) they were fetched at.
// CHECKED (rays that can leave the volume): no reuse, and faces outside [-1, n_a] x
// [-1, n_t - 1] x [-1, nz - 1] read as zero; otherwise (every floor in [-1, n - 1], so the
// 16-bit footprint key is exact) the quad index is clamped to the array as a guard.
struct MarchState {
    float4 PE = make_float4(0.f, 0.f, 0.f, 0.f), PO = make_float4(0.f, 0.f, 0.f, 0.f);
    int pe = 0, po = 0;
    unsigned pkey = 0;
};

template <bool XMARCH, bool CHECKED>
__device__ __forceinline__ float trilinear_march(unsigned long long tex, const float* __restrict__ quads,
                                                 const MarchIndex& M, int nz, const RsSample& s, MarchState& S) {
    const int im = XMARCH ? s.ix : s.iy;  // biased floor along the march axis (FLOOR_KBITS is even)
    const int it = XMARCH ? s.iy : s.ix;  // biased transverse floor
    const float ft = XMARCH ? s.f.y : s.f.x;
    const unsigned key = __byte_perm((unsigned)it, (unsigned)s.iz, 0x1054);  // low halves: (t, k) of the footprint
    const bool same = !CHECKED && key == S.pkey;
    const int E = (im + 1) & ~1, O = im | 1;  // the even and the odd face of {m, m + 1}
    // a face is fetched when its m or the footprint changed (else it holds the same texels)
    bool needE = !(same && E == S.pe), needO = !(same && O == S.po);
    S.pkey = key;
    S.pe = E;
    S.po = O;
    const unsigned q = (unsigned)(im >> 1) * M.qz + (unsigned)s.iz * (unsigned)M.qt + (unsigned)it - M.bias;
    if (CHECKED) {
        const bool okE = (unsigned)(E - FLOOR_KBITS) <= (unsigned)M.na;
        const bool okO = (unsigned)(O - (FLOOR_KBITS - 1)) <= (unsigned)(M.na + 1) &&
                         (unsigned)(it - (FLOOR_KBITS - 1)) <= (unsigned)M.nt &&
                         (unsigned)(s.iz - (FLOOR_KBITS - 1)) <= (unsigned)nz;
        if (!okE) S.PE = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!okO) S.PO = make_float4(0.f, 0.f, 0.f, 0.f);
        needE = okE;
        needO = okO;
    }
    const float2 c = __fadd2_rn(make_float2(ft, s.fz), make_float2(1.0f, 1.0f));
    if (needE) S.PE = gather_layer<float>(tex, (E >> 1) + M.layer0, c.x, c.y);
    if (needO) S.PO = __ldg(reinterpret_cast<const float4*>(quads) + (CHECKED ? q : min(q, M.qmax)));
    // z lerps of each face's two (t) columns, as trilerp does them
    const float2 zE = lerp2(make_float2(S.PE.w, S.PE.z), make_float2(S.PE.x, S.PE.y), s.cc, s.ncc);
    const float2 zO = lerp2(make_float2(S.PO.w, S.PO.z), make_float2(S.PO.x, S.PO.y), s.cc, s.ncc);
    const bool odd = im & 1;
    const float2 zl = odd ? zO : zE, zh = odd ? zE : zO;  // faces m and m + 1
    if (XMARCH) {  // zl = (z(i, j), z(i, j+1)), zh = (z(i+1, j), z(i+1, j+1))
        const float r0 = lerp(zl.x, zh.x, s.w.x), r1 = lerp(zl.y, zh.y, s.w.x);
        return lerp(r0, r1, s.w.y);
    } else {       // zl = (z(i, j), z(i+1, j)), zh = (z(i, j+1), z(i+1, j+1))
        const float r0 = lerp(zl.x, zl.y, s.w.x), r1 = lerp(zh.x, zh.y, s.w.x);
        return lerp(r0, r1, s.w.y);
    }
}

// True when every sample of the ray provably lies at a texel-space position in (-1, n) on
// each axis, so that every footprint falls inside the quads (ci in [0, nx] ...). The samples
// run from the entry point over n - 1 unit steps; each of the repeated additions (and the
// +0.5 / -0.5 of the texture coordinate) rounds by at most half an ulp of a value below
// `mag`, which bounds the drift from the exact line by (n + 3) mag 2^-23.
__device__ __forceinline__ bool rs_ray_inside(const DevGeom& g, const RsRay& r) {
    if (r.n == 0) return true;
    const float last = (float)(r.n - 1);
    const float mag = (float)max(max(g.nx, g.ny), g.nz) + 2.0f;
    const float e = (last + 4.0f) * mag * 1.1920929e-7f;  // (n + 3) mag 2^-23, rounded up
    const float ex = fmaf(last, r.sx, r.A), ey = fmaf(last, r.sy, r.B), ez = fmaf(last, r.sz, r.C);
    return fminf(r.A, ex) - e > -1.0f && fmaxf(r.A, ex) + e < (float)g.nx && fminf(r.B, ey) - e > -1.0f &&
           fmaxf(r.B, ey) + e < (float)g.ny && fminf(r.C, ez) - e > -1.0f && fmaxf(r.C, ez) + e < (float)g.nz;
}

// One 2^rs_tlog u x 2^(8 - rs_tlog) v tile of view p (256 threads; each warp's rays span
// 2^rs_wlog u x 2^(5 - rs_wlog) v): ray set-up,
// trilinear march, epilogue. Shared by the single-job kernel and the batched persistent
// kernel (batch.cu); must be called by all 256 threads of the block (EPI_NORM syncs).
template <int MODE, int LAYOUT, typename Tv, typename To, int EPI, typename Tr = To>
__device__ __forceinline__ void rs_tile(const DevGeom& g, const Tv* __restrict__ vin, unsigned long long tex,
                                        const OutView<To>& out, const OutView<Tr>& real, double* __restrict__ norm,
                                        int p, int ut, int vt) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wl = g.rs_wlog, wu = 1 << wl;             // a warp: wu x (32 / wu) rays
    const int wpr = 1 << (g.rs_tlog - wl);               // warps per row of the tile
    const int u = (ut << g.rs_tlog) + (warp & (wpr - 1)) * wu + (lane & (wu - 1));
    const int v = vt * rs_tile_v(g) + (warp >> (g.rs_tlog - wl)) * (32 >> wl) + (lane >> wl);
    const bool active = (u < g.nu) && (v < g.nv);
    float acc = 0.f;
    if (active) {
        RsRay r;
        const bool hit = MODE == 0 ? rs_ray_box(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r)
                                   : rs_ray_um(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r);
        if (hit) {
            const float fnx = (float)g.nx, fny = (float)g.ny, fnz = (float)g.nz;
            const float dx = g.dx;
            const float2 SXY = make_float2(r.sx, r.sy), SZZ = make_float2(r.sz, r.sz);
            auto march = [&](auto sample) {
                float2 AB = make_float2(r.A, r.B), CC = make_float2(r.C, r.C);
                for (unsigned n = 0; n < r.n; ++n) {
                    const RsSample s = rs_sample(AB, CC);
                    acc = fadd(acc, fmul(dx, sample(s, n)));  // :292
                    AB = __fadd2_rn(AB, SXY);              // :295-297
                    CC = __fadd2_rn(CC, SZZ);
                }
            };
            if (LAYOUT == RS_LAYOUT_MARCH) {
                // the view's rays run mostly along x: march faces across x, else across y
                const bool xm = fabsf(__ldg(g.alpha + p)) > fabsf(__ldg(g.beta + p));
                const bool inside = rs_ray_inside(g, r);
                const MarchIndex M = march_index(g.nx, g.ny, g.nz, xm);
                const float* quads = reinterpret_cast<const float*>(vin) +
                                     (xm ? 0 : (size_t)4 * march_quads(g.nx, g.ny, g.nz));
                MarchState S;
                if (xm) {
                    if (inside)
                        march([&](const RsSample& s, unsigned) { return trilinear_march<true, false>(tex, quads, M, g.nz, s, S); });
                    else
                        march([&](const RsSample& s, unsigned) { return trilinear_march<true, true>(tex, quads, M, g.nz, s, S); });
                } else {
                    if (inside)
                        march([&](const RsSample& s, unsigned) { return trilinear_march<false, false>(tex, quads, M, g.nz, s, S); });
                    else
                        march([&](const RsSample& s, unsigned) { return trilinear_march<false, true>(tex, quads, M, g.nz, s, S); });
                }
            } else if (LAYOUT == RS_LAYOUT_HYBRID) {
                // the view's rays run mostly along x: column quads (second array), else row quads
                const bool cols = fabsf(__ldg(g.alpha + p)) > fabsf(__ldg(g.beta + p));
                const bool inside = rs_ray_inside(g, r);
                const QuadIndex Q = hybrid_quad_index(g.nx, g.ny, g.nz, cols);
                const Tv* quads = cols ? vin + (size_t)4 * Q.qwh * (g.nz + 1) : vin;
                auto hyb = [&](auto cols_c, auto checked_c) {
                    constexpr bool C = decltype(cols_c)::value, K = decltype(checked_c)::value;
                    march([&](const RsSample& s, unsigned) {
                        return trilinear_hybrid<Tv, C, K>(tex, quads, Q, g.nx, g.ny, g.nz, s);
                    });
                };
                using T_ = std::true_type;
                using F_ = std::false_type;
                if (cols) {
                    if (inside) hyb(T_{}, F_{});
                    else hyb(T_{}, T_{});
                } else {
                    if (inside) hyb(F_{}, F_{});
                    else hyb(F_{}, T_{});
                }
            } else {
                const int W = LAYOUT == RS_LAYOUT_CELL8 ? g.nx + 1 : g.nx + 2;
                const int WH = LAYOUT == RS_LAYOUT_CELL8 ? (g.nx + 1) * (g.ny + 1) : (g.nx + 2) * (g.ny + 2);
                march([&](const RsSample& s, unsigned) {
                    return LAYOUT == RS_LAYOUT_CELL8 ? trilinear_cells(vin, W, WH, fnx, fny, fnz, s)
                           : LAYOUT == RS_LAYOUT_TEX ? trilinear_tex<Tv>(tex, s)
                                                     : trilinear_padded(vin, W, WH, fnx, fny, fnz, s);
                });
            }
        }
    }
    epilogue<EPI, To, Tr>(active, acc, u, v, p, out, real, norm);
}


}  // namespace tomo
