// rs_project.cu -- regular-sampling (RS) cone-beam projector for sm_100a.
//
// One thread per detector ray (u, v, phi). A warp covers an 8u x 4v tile of one view so
// that its 32 rays stay spatially coherent while they march: at each step the 32 sample
// points sit within a few voxels of each other and their trilinear footprints share L1
// lines. The volume is read from a zero-bordered padded copy (one voxel on every side),
// so a sample whose footprint touches the data never needs per-texel bounds checks.
//
// Block order: blockIdx.x is the view, so the blocks resident at any moment are all views
// of one band of detector rows. Those rays only cross the z-slab that the band sees, and
// consecutive views (resident on the same SM) cross nearly the same voxels: the slab stays
// in L2 and the voxels in L1, instead of every view re-streaming the volume from HBM.
//
// Volume layouts (chosen per call, RS_LAYOUT_*):
//   PLAIN  zero-bordered padded copy (nx+2)(ny+2)(nz+2); eight scalar texel loads/sample.
//   CELL8  for every trilinear cell (i..i+1, j..j+1, k..k+1), i in [-1, nx-1] etc., the
//          eight texels stored together: 32 B (FP32) or 16 B (BF16/FP16), aligned, so a
//          sample is two (one) 128-bit loads from a single sector. 8x the volume's bytes.
//   TEX    2D layered array in the storage type (raw 16-bit for BF16/FP16), slice z in
//          layer z + 1 between two zero layers; two 4-texel tld4 gathers per sample.
//   HYBRID TEX for the lower slice of a sample plus, for the upper slice, quads (the slice's
//          four footprint texels in tld4 order, 16 B FP32 / 8 B 16-bit) in global memory, in a
//          row-major and a column-major array: one gather and one 128-bit load per sample.
//   MARCH  (FP32) faces across the march axis of the view (x or y): even faces in a layered
//          texture, odd faces as quads in global memory; a sample reads the faces m and
//          m + 1 around it (one of each kind) and keeps them for the next sample, which
//          fetches only the faces that changed (tomo_kernels.cuh, rs_device.cuh).
//
// Parity: the per-ray prologue (source/detector positions, the y = A1 x + B1 line, the
// FOV intersection, the box and z clipping, the chord length L_r) is written with
// explicitly rounded IEEE operations in the reference's order and precision, so entry
// points and sample counts are bit-identical to the reference kernels compiled on the
// host with exact FP32 texture filtering:
//   TOMO_PROJ_RS     projection_ERB_kernel_v1   (projection_ER_kernel.cuh:57-312)
//   TOMO_PROJ_RS_UM  projection_ERB_kernel_v0_UM (projection_ER_kernel_UM.cuh:26-153)
// The positions march by repeated exact addition (:295-297) and every sample adds
// dx * tex3D(...) with a separate multiply and add (:292). Only the trilinear lerps use
// fused multiply-adds (within 1e-6 relative of the exact formula); see rs_device.cuh.
#include <algorithm>

#include "rs_device.cuh"

// Resident blocks per SM the projection kernels are compiled for (their register budget);
// the MARCH layout's kernels carry their faces across samples and have their own.
#ifndef TOMO_RS_MIN_BLOCKS
#define TOMO_RS_MIN_BLOCKS 4
#endif
#ifndef TOMO_RS_MARCH_MIN_BLOCKS
#define TOMO_RS_MARCH_MIN_BLOCKS 4
#endif

namespace tomo {

// Quads of the HYBRID layout: quad (ci, cj, k) holds the four texels of slice k around the
// footprint i = ci - 1, j = cj - 1 in tld4 order, (T[i][j+1], T[i+1][j+1], T[i+1][j], T[i][j]),
// for ci in [0, nx], cj in [0, ny], k in [0, nz] (slice nz and texels outside x, y: 0).
// Row quads (ci fastest) first, then column quads (cj fastest). A block stages the 33 x 33
// texels of a 32 x 32 quad tile of slice k in shared memory (one coalesced read of the
// slice), then writes the tile's row quads along ci and its column quads along cj, both as
// consecutive 16 B / 8 B stores.
constexpr int QT = 32;  // quads per tile side
template <typename Ti, typename Tc>
__global__ void __launch_bounds__(256) rs_quads_kernel(const Ti* __restrict__ in, Tc* __restrict__ quads, int nx,
                                                       int ny, int nz, const unsigned* amax) {
    __shared__ float tile[QT + 1][QT + 1];  // texels (y0 - 1 + r, x0 - 1 + c); pitch 33: no bank conflicts
    const float sc = fp16_scale(amax);
    const int cx0 = blockIdx.x * QT, cy0 = blockIdx.y * QT, k = blockIdx.z;
    const long plane = (long)nx * ny;
    for (int t = threadIdx.y * QT + threadIdx.x; t < (QT + 1) * (QT + 1); t += QT * 8) {
        const int r = t / (QT + 1), c = t % (QT + 1);
        const int x = cx0 - 1 + c, y = cy0 - 1 + r;
        const bool ok = x >= 0 && y >= 0 && x < nx && y < ny && k < nz;
        tile[r][c] = ok ? ldp(in + (k * plane + (long)y * nx + x)) * sc : 0.f;
    }
    __syncthreads();
    const long QWH = (long)(nx + 1) * (ny + 1), total = QWH * (nz + 1);
    auto put = [&](long q, int r, int c) {  // quad with footprint texels tile[r..r+1][c..c+1], tld4 order
        if constexpr (sizeof(Tc) == 4) {
            reinterpret_cast<float4*>(quads)[q] = make_float4(tile[r + 1][c], tile[r + 1][c + 1], tile[r][c + 1], tile[r][c]);
        } else {
            const Tc v[4] = {cvt<Tc>(tile[r + 1][c]), cvt<Tc>(tile[r + 1][c + 1]), cvt<Tc>(tile[r][c + 1]),
                             cvt<Tc>(tile[r][c])};
            reinterpret_cast<uint2*>(quads)[q] = *reinterpret_cast<const uint2*>(v);
        }
    };
    for (int r = threadIdx.y; r < QT; r += 8) {  // row quads: threads along ci
        const int ci = cx0 + threadIdx.x, cj = cy0 + r;
        if (ci <= nx && cj <= ny) put(k * QWH + (long)cj * (nx + 1) + ci, r, threadIdx.x);
    }
    for (int c = threadIdx.y; c < QT; c += 8) {  // column quads: threads along cj
        const int ci = cx0 + c, cj = cy0 + threadIdx.x;
        if (ci <= nx && cj <= ny) put(total + k * QWH + (long)ci * (ny + 1) + cj, threadIdx.x, c);
    }
}

template <int MODE, int LAYOUT, typename Tv, typename To, int EPI, typename Tr>
__global__ void __launch_bounds__(256, LAYOUT == RS_LAYOUT_MARCH ? TOMO_RS_MARCH_MIN_BLOCKS : TOMO_RS_MIN_BLOCKS)
rs_project_kernel(DevGeom g, const Tv* __restrict__ vin, unsigned long long tex,
                                                         OutView<To> out, OutView<Tr> real, double* __restrict__ norm) {
    if ((LAYOUT == RS_LAYOUT_HYBRID || LAYOUT == RS_LAYOUT_MARCH) && g.view_order) {
        // blockIdx.z runs over the v-tiles of the views whose rays run along x, then over those
        // of the other views: the CTAs resident at a time read one quad array, not both
        const int tv = rs_tiles_v(g);
        const bool other = (int)blockIdx.z >= tv;
        const int i = blockIdx.x, n = other ? g.np - g.view_cols : g.view_cols;
        if (i >= n) {  // uniform over the block: no view here (its norm partial is 0)
            if (EPI == EPI_NORM && threadIdx.x == 0) norm[linear_block()] = 0.0;
            return;
        }
        const int p = __ldg(g.view_order + (other ? g.view_cols + i : i));
        rs_tile<MODE, LAYOUT, Tv, To, EPI, Tr>(g, vin, tex, out, real, norm, p, blockIdx.y, blockIdx.z - (other ? tv : 0));
    } else {
        rs_tile<MODE, LAYOUT, Tv, To, EPI, Tr>(g, vin, tex, out, real, norm, blockIdx.x, blockIdx.y, blockIdx.z);
    }
}

// Cells of the CELL8 layout: cell (ci, cj, ck) holds the texels (ci-1+di, cj-1+dj, ck-1+dk).
template <typename Ti, typename Tc>
__global__ void rs_cells_kernel(const Ti* __restrict__ in, Tc* __restrict__ cells, int nx, int ny, int nz,
                                const unsigned* amax) {
    const float sc = fp16_scale(amax);
    const long CW = nx + 1, CWH = CW * (ny + 1), total = CWH * (nz + 1);
    const long plane = (long)nx * ny;
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < total; c += (long)gridDim.x * blockDim.x) {
        const int ci = (int)(c % CW), cj = (int)((c / CW) % (ny + 1)), ck = (int)(c / CWH);
        Tc v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int i = ci - 1 + (q & 1), j = cj - 1 + ((q >> 1) & 1), k = ck - 1 + (q >> 2);
            const bool ok = i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
            v[q] = cvt<Tc>(ok ? ldp(in + (k * plane + (long)j * nx + i)) * sc : 0.f);
        }
        if (sizeof(Tc) == 4) {
            float4* o = reinterpret_cast<float4*>(cells) + 2 * c;
            const float* f = reinterpret_cast<const float*>(v);
            o[0] = make_float4(f[0], f[1], f[2], f[3]);
            o[1] = make_float4(f[4], f[5], f[6], f[7]);
        } else {
            reinterpret_cast<uint4*>(cells)[c] = *reinterpret_cast<const uint4*>(v);
        }
    }
}

// Exact transpose: scatter dx * y * w_texel into the (unpadded, FP32) output volume.
template <int MODE, typename Ts>
__global__ void __launch_bounds__(256) rs_adjoint_kernel(DevGeom g, const Ts* __restrict__ sino,
                                                         float* __restrict__ vol) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = blockIdx.x;
    const int u = blockIdx.y * 16 + (warp & 1) * 8 + (lane & 7);
    const int v = blockIdx.z * 16 + (warp >> 1) * 4 + (lane >> 3);
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
static dim3 rs_grid(int layout, const DevGeom& g) {
    if ((layout == RS_LAYOUT_HYBRID || layout == RS_LAYOUT_MARCH) && g.view_order)
        return dim3(std::max(g.view_cols, g.np - g.view_cols), rs_tiles_u(g), 2 * rs_tiles_v(g));
    return dim3(g.np, rs_tiles_u(g), rs_tiles_v(g));
}

size_t rs_grid_blocks(int layout, const DevGeom& g) {
    const dim3 d = rs_grid(layout, g);
    return (size_t)d.x * d.y * d.z;
}

template <int LAYOUT, int MODE, int EPI, typename Tv, typename To, typename Tr>
static cudaError_t launch_rs_k(const DevGeom& g, const void* vin, unsigned long long tex, const OutView<void>& out,
                               const OutView<void>& real, double* norm, cudaStream_t st) {
    const dim3 block(256), grid = rs_grid(LAYOUT, g);
    rs_project_kernel<MODE, LAYOUT, Tv, To, EPI, Tr><<<grid, block, 0, st>>>(g, static_cast<const Tv*>(vin), tex,
                                                                              out.as<To>(), real.as<Tr>(), norm);
    return cudaGetLastError();
}

// EPI_STORE: output in odt. EPI_RESIDUAL: FP32 residual, `real` read in rdt. EPI_NORM /
// EPI_PARTIAL: nothing stored.
template <int LAYOUT, int MODE, typename Tv>
static cudaError_t launch_rs_e(int epi, const DevGeom& g, const void* vin, unsigned long long tex,
                               const OutView<void>& out, tomo_dtype odt, const OutView<void>& real, tomo_dtype rdt,
                               double* norm, cudaStream_t st) {
    if (epi == EPI_STORE) {
        switch (odt) {
            case TOMO_F32: return launch_rs_k<LAYOUT, MODE, EPI_STORE, Tv, float, float>(g, vin, tex, out, real, norm, st);
            case TOMO_BF16:
                return launch_rs_k<LAYOUT, MODE, EPI_STORE, Tv, __nv_bfloat16, __nv_bfloat16>(g, vin, tex, out, real, norm, st);
            case TOMO_F16: return launch_rs_k<LAYOUT, MODE, EPI_STORE, Tv, __half, __half>(g, vin, tex, out, real, norm, st);
        }
    } else if (epi == EPI_RESIDUAL) {
        switch (rdt) {
            case TOMO_F32: return launch_rs_k<LAYOUT, MODE, EPI_RESIDUAL, Tv, float, float>(g, vin, tex, out, real, norm, st);
            case TOMO_BF16:
                return launch_rs_k<LAYOUT, MODE, EPI_RESIDUAL, Tv, float, __nv_bfloat16>(g, vin, tex, out, real, norm, st);
            case TOMO_F16: return launch_rs_k<LAYOUT, MODE, EPI_RESIDUAL, Tv, float, __half>(g, vin, tex, out, real, norm, st);
        }
    } else if (epi == EPI_NORM) {
        return launch_rs_k<LAYOUT, MODE, EPI_NORM, Tv, float, float>(g, vin, tex, out, real, norm, st);
    }
    return cudaErrorInvalidValue;
}

template <int LAYOUT>
static cudaError_t launch_rs_layout(int mode, int epi, const DevGeom& g, const void* vin, unsigned long long tex,
                                    tomo_dtype vdt, const OutView<void>& out, tomo_dtype odt, const OutView<void>& real,
                                    double* norm, cudaStream_t st, tomo_dtype rdt) {
#define TOMO_RS_V(TV)                                                                                  \
    return mode == 0 ? launch_rs_e<LAYOUT, 0, TV>(epi, g, vin, tex, out, odt, real, rdt, norm, st)    \
                     : launch_rs_e<LAYOUT, 1, TV>(epi, g, vin, tex, out, odt, real, rdt, norm, st);
    switch (vdt) {
        case TOMO_F32: TOMO_RS_V(float)
        case TOMO_BF16: TOMO_RS_V(__nv_bfloat16)
        case TOMO_F16: TOMO_RS_V(__half)
    }
#undef TOMO_RS_V
    return cudaErrorInvalidValue;
}

cudaError_t launch_rs_project(int layout, int mode, int epi, const DevGeom& g, const void* vin, unsigned long long tex,
                              tomo_dtype vdt, const OutView<void>& out, tomo_dtype odt, const OutView<void>& real,
                              double* norm, cudaStream_t st, tomo_dtype rdt) {
    if (layout == RS_LAYOUT_CELL8)
        return launch_rs_layout<RS_LAYOUT_CELL8>(mode, epi, g, vin, 0, vdt, out, odt, real, norm, st, rdt);
    if (layout == RS_LAYOUT_TEX)  // the texture holds the values; vdt is the texture's type
        return launch_rs_layout<RS_LAYOUT_TEX>(mode, epi, g, nullptr, tex, vdt, out, odt, real, norm, st, rdt);
    if (layout == RS_LAYOUT_HYBRID)  // texture (lower slice) + CELL4 buffer (upper slice), both of type vdt
        return launch_rs_layout<RS_LAYOUT_HYBRID>(mode, epi, g, vin, tex, vdt, out, odt, real, norm, st, rdt);
    if (layout == RS_LAYOUT_MARCH) {  // even-face texture + odd-face quads, FP32 only
        if (vdt != TOMO_F32) return cudaErrorInvalidValue;
        return mode == 0 ? launch_rs_e<RS_LAYOUT_MARCH, 0, float>(epi, g, vin, tex, out, odt, real, rdt, norm, st)
                         : launch_rs_e<RS_LAYOUT_MARCH, 1, float>(epi, g, vin, tex, out, odt, real, rdt, norm, st);
    }
    return launch_rs_layout<RS_LAYOUT_PLAIN>(mode, epi, g, vin, 0, vdt, out, odt, real, norm, st, rdt);
}

cudaError_t launch_rs_project(int mode, int epi, const DevGeom& g, const void* vpad, tomo_dtype vdt,
                              const OutView<void>& out, tomo_dtype odt, const OutView<void>& real, double* norm,
                              cudaStream_t st, tomo_dtype rdt) {
    return launch_rs_layout<RS_LAYOUT_PLAIN>(mode, epi, g, vpad, 0, vdt, out, odt, real, norm, st, rdt);
}

size_t rs_input_elems(int layout, int nx, int ny, int nz) {
    if (layout == RS_LAYOUT_TEX) return 1;  // the values live in a layered cudaArray
    if (layout == RS_LAYOUT_HYBRID)  // row quads, then column quads; + the texture
        return (size_t)8 * (nx + 1) * (ny + 1) * (nz + 1);
    if (layout == RS_LAYOUT_MARCH)  // odd faces: x-march quads, then y-march quads; + the texture
        return (size_t)4 * (march_quads(nx, ny, nz) + march_quads(ny, nx, nz));
    return layout == RS_LAYOUT_CELL8 ? (size_t)8 * (nx + 1) * (ny + 1) * (nz + 1)
                                     : (size_t)(nx + 2) * (ny + 2) * (nz + 2);
}

// A 2D layered array (one layer per z slice) in the storage type -- FP32, or the raw 16
// bits of BF16 / FP16 as unsigned shorts -- with its texture object (point sampling,
// unnormalised coordinates, border colour 0 in x and y) and, for 16-bit textures, a
// surface object through which a kernel fills it from an FP32 volume.
cudaError_t rs_tex_create(int nx, int ny, int nz, tomo_dtype dt, RsTexture* t, bool surface) {
    *t = RsTexture();
    t->dt = dt;
    const bool raw16 = dt != TOMO_F32;
    surface = surface || raw16;
    cudaChannelFormatDesc cd = raw16 ? cudaCreateChannelDesc(16, 0, 0, 0, cudaChannelFormatKindUnsigned)
                                     : cudaCreateChannelDesc<float>();
    cudaError_t e = cudaMalloc3DArray(&t->arr, &cd, make_cudaExtent(nx, ny, nz),
                                      cudaArrayLayered | (surface ? cudaArraySurfaceLoadStore : 0));
    if (e != cudaSuccess) {
        t->arr = nullptr;
        return e;
    }
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = t->arr;
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeBorder;
    td.addressMode[1] = cudaAddressModeBorder;
    td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t to = 0;
    e = cudaCreateTextureObject(&to, &rd, &td, nullptr);
    if (e == cudaSuccess) t->tex = (unsigned long long)to;
    if (e == cudaSuccess && surface) {
        cudaSurfaceObject_t so = 0;
        e = cudaCreateSurfaceObject(&so, &rd);
        if (e == cudaSuccess) t->surf = (unsigned long long)so;
    }
    if (e != cudaSuccess) rs_tex_destroy(t);
    return e;
}

// Zeroes layers `a` and `b` of a layered texture through its surface.
__global__ void rs_tex_zero_layers_kernel(unsigned long long surf, int nx, int ny, int a, int b, int bytes) {
    const long plane = (long)nx * ny;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < 2 * plane; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), layer = i < plane ? a : b;
        if (bytes == 4) surf2DLayeredwrite(0.f, (cudaSurfaceObject_t)surf, x * 4, y, layer);
        else surf2DLayeredwrite((unsigned short)0, (cudaSurfaceObject_t)surf, x * 2, y, layer);
    }
}

cudaError_t rs_vol_tex_create(int nx, int ny, int nz, tomo_dtype dt, RsTexture* t, cudaStream_t st) {
    if (dt != TOMO_F32) {  // packed slice pairs: 32-bit texels, filled whole by the fill kernel
        *t = RsTexture();
        t->dt = dt;
        t->z0 = 2;
        t->zpairs = true;
        cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindUnsigned);
        cudaError_t e = cudaMalloc3DArray(&t->arr, &cd, make_cudaExtent(nx, ny, nz + 3),
                                          cudaArrayLayered | cudaArraySurfaceLoadStore);
        if (e != cudaSuccess) {
            t->arr = nullptr;
            return e;
        }
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = t->arr;
        cudaTextureDesc td{};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        cudaTextureObject_t to = 0;
        cudaSurfaceObject_t so = 0;
        e = cudaCreateTextureObject(&to, &rd, &td, nullptr);
        if (e == cudaSuccess) t->tex = (unsigned long long)to;
        if (e == cudaSuccess) e = cudaCreateSurfaceObject(&so, &rd);
        if (e == cudaSuccess) t->surf = (unsigned long long)so;
        if (e != cudaSuccess) rs_tex_destroy(t);
        return e;
    }
    cudaError_t e = rs_tex_create(nx, ny, nz + 2, dt, t, true);
    if (e != cudaSuccess) return e;
    t->z0 = 1;
    const long n = 2L * nx * ny;
    rs_tex_zero_layers_kernel<<<(int)std::min<long>((n + 255) / 256, 148L * 16), 256, 0, st>>>(
        t->surf, nx, ny, 0, nz + 1, (int)dtype_size(dt));
    e = cudaGetLastError();
    if (e != cudaSuccess) rs_tex_destroy(t);
    return e;
}

// Voxel (x, y, z) of a dense FP32 volume, 0 outside it.
__device__ __forceinline__ float vol_or_zero(const float* __restrict__ in, int x, int y, int z, int nx, int ny, int nz) {
    return (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) ? __ldg(in + ((long)z * ny + y) * nx + x) : 0.f;
}

// Odd faces of the MARCH layout. Threads run z-major (kk slowest, then the face, then t)
// so that the two slices a pass reads stay in L2, and write consecutive quads.
__global__ void rs_march_quads_kernel(const float* __restrict__ in, float4* __restrict__ quads, int nx, int ny, int nz) {
    const long qx = march_quads(nx, ny, nz), total = qx + march_quads(ny, nx, nz);
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < total; c += (long)gridDim.x * blockDim.x) {
        const bool xm = c < qx;
        const long r = xm ? c : c - qx;
        const int na = xm ? nx : ny, nt = xm ? ny : nx, faces = march_odd_faces(na);
        const int tt = (int)(r % (nt + 1));
        const long rest = r / (nt + 1);
        const int o = (int)(rest % faces), kk = (int)(rest / faces);
        const int m = 2 * o - 1, t = tt - 1, k = kk - 1;
        auto T = [&](int tq, int zq) { return xm ? vol_or_zero(in, m, tq, zq, nx, ny, nz) : vol_or_zero(in, tq, m, zq, nx, ny, nz); };
        const long q = ((long)o * (nz + 1) + kk) * (nt + 1) + tt + (xm ? 0 : qx);
        quads[q] = make_float4(T(t, k + 1), T(t + 1, k + 1), T(t + 1, k), T(t, k));
    }
}

// Even faces of the MARCH layout into the layered texture (layer L < Lx: x = 2L over
// (y, z); layer Lx + L: y = 2L over (x, z); 0 past the data). z-major thread order.
__global__ void rs_march_tex_kernel(const float* __restrict__ in, unsigned long long surf, int nx, int ny, int nz,
                                    int width) {
    const int lx = march_even_faces(nx), layers = lx + march_even_faces(ny);
    const long total = (long)width * layers * nz;
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < total; c += (long)gridDim.x * blockDim.x) {
        const int t = (int)(c % width);
        const long rest = c / width;
        const int L = (int)(rest % layers), z = (int)(rest / layers);
        const float v = L < lx ? vol_or_zero(in, 2 * L, t, z, nx, ny, nz) : vol_or_zero(in, t, 2 * (L - lx), z, nx, ny, nz);
        surf2DLayeredwrite(v, (cudaSurfaceObject_t)surf, t * 4, z, L);
    }
}

cudaError_t rs_march_tex_create(int nx, int ny, int nz, RsTexture* t) {
    cudaError_t e = rs_tex_create(std::max(nx, ny), nz, march_even_faces(nx) + march_even_faces(ny), TOMO_F32, t, true);
    if (e == cudaSuccess) t->march = true;
    return e;
}

void rs_tex_destroy(RsTexture* t) {
    if (t->surf) cudaDestroySurfaceObject((cudaSurfaceObject_t)t->surf);
    if (t->tex) cudaDestroyTextureObject((cudaTextureObject_t)t->tex);
    if (t->arr) cudaFreeArray(t->arr);
    *t = RsTexture();
}

// Rounds a volume to the texture's 16-bit type (round to nearest even, as the other
// layouts' conversions) and writes the raw bits into the layered array.
template <typename Ti, typename Tt>
__global__ void rs_tex_convert_kernel(const Ti* __restrict__ in, unsigned long long surf, int nx, int ny, int nz,
                                      int z0, const unsigned* amax) {
    const float sc = fp16_scale(amax);
    const long plane = (long)nx * ny, total = plane * nz;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / plane);
        const Tt h = cvt<Tt>(ldp(in + i) * sc);
        if constexpr (sizeof(Tt) == 4)
            surf2DLayeredwrite(*reinterpret_cast<const float*>(&h), (cudaSurfaceObject_t)surf, x * 4, y, z + z0);
        else
            surf2DLayeredwrite(*reinterpret_cast<const unsigned short*>(&h), (cudaSurfaceObject_t)surf, x * 2, y,
                               z + z0);
    }
}

template <typename Tt>
static cudaError_t tex_convert(const void* vol, tomo_dtype vdt, int nx, int ny, int nz, int z0,
                               unsigned long long surf, cudaStream_t st, const unsigned* amax) {
    const long n = (long)nx * ny * nz;
    const int b = (int)std::min<long>((n + 255) / 256, 148L * 16);
    switch (vdt) {
        case TOMO_F32:
            rs_tex_convert_kernel<float, Tt><<<b, 256, 0, st>>>((const float*)vol, surf, nx, ny, nz, z0, amax);
            break;
        case TOMO_BF16:
            rs_tex_convert_kernel<__nv_bfloat16, Tt><<<b, 256, 0, st>>>((const __nv_bfloat16*)vol, surf, nx, ny, nz, z0,
                                                                        amax);
            break;
        case TOMO_F16:
            rs_tex_convert_kernel<__half, Tt><<<b, 256, 0, st>>>((const __half*)vol, surf, nx, ny, nz, z0, amax);
            break;
    }
    return cudaGetLastError();
}

// The interior of a padded FP32 sinogram into an FP32 layered texture, through its surface.
__global__ void tex_from_padded_kernel(const float* __restrict__ spad, unsigned long long surf, int nu, int nv, int np) {
    const long plane = (long)nu * nv, total = plane * np;
    const long W = nu + 2, WH = W * (nv + 2);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int u = (int)(i % nu), v = (int)((i / nu) % nv), p = (int)(i / plane);
        surf2DLayeredwrite(spad[p * WH + (v + 1) * W + (u + 1)], (cudaSurfaceObject_t)surf, u * (int)sizeof(float), v, p);
    }
}

cudaError_t tex_fill_from_padded(const float* spad, int nu, int nv, int np, const RsTexture& t, cudaStream_t st) {
    if (t.dt != TOMO_F32 || !t.surf) return cudaErrorInvalidValue;
    const long n = (long)nu * nv * np;
    const int b = (int)std::min<long>((n + 255) / 256, 148L * 16);
    tex_from_padded_kernel<<<b, 256, 0, st>>>(spad, t.surf, nu, nv, np);
    return cudaGetLastError();
}


// Packed 16-bit volume texture: layer L in [0, nz + 3) holds slices L - 2 (low 16 bits) and
// L - 1 (high 16 bits), rounded to the texture's type, 0 outside [0, nz).
template <typename Ti, typename Tt>
__global__ void rs_tex_pairs_kernel(const Ti* __restrict__ in, unsigned long long surf, int nx, int ny, int nz,
                                    const unsigned* amax) {
    const float sc = fp16_scale(amax);
    const long plane = (long)nx * ny, total = plane * (nz + 3);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), L = (int)(i / plane);
        const long xy = (long)y * nx + x;
        const int k0 = L - 2, k1 = L - 1;
        const Tt lo = cvt<Tt>(k0 >= 0 && k0 < nz ? ldp(in + (k0 * plane + xy)) * sc : 0.f);
        const Tt hi = cvt<Tt>(k1 >= 0 && k1 < nz ? ldp(in + (k1 * plane + xy)) * sc : 0.f);
        const unsigned bits = (unsigned)*reinterpret_cast<const unsigned short*>(&lo) |
                              ((unsigned)*reinterpret_cast<const unsigned short*>(&hi) << 16);
        surf2DLayeredwrite(bits, (cudaSurfaceObject_t)surf, x * 4, y, L);
    }
}

template <typename Tt>
static cudaError_t tex_pairs(const void* vol, tomo_dtype vdt, int nx, int ny, int nz, unsigned long long surf,
                             cudaStream_t st, const unsigned* amax) {
    const long n = (long)nx * ny * (nz + 3);
    const int b = (int)std::min<long>((n + 255) / 256, 148L * 16);
    switch (vdt) {
        case TOMO_F32: rs_tex_pairs_kernel<float, Tt><<<b, 256, 0, st>>>((const float*)vol, surf, nx, ny, nz, amax); break;
        case TOMO_BF16:
            rs_tex_pairs_kernel<__nv_bfloat16, Tt><<<b, 256, 0, st>>>((const __nv_bfloat16*)vol, surf, nx, ny, nz, amax);
            break;
        case TOMO_F16: rs_tex_pairs_kernel<__half, Tt><<<b, 256, 0, st>>>((const __half*)vol, surf, nx, ny, nz, amax); break;
    }
    return cudaGetLastError();
}

// Fills the texture from a dense device volume: a device-to-device copy when the volume
// has the texture's type, else a conversion kernel (16-bit textures only).
cudaError_t rs_tex_fill(const void* vol, tomo_dtype vdt, int nx, int ny, int nz, const RsTexture& t,
                        cudaStream_t st, const unsigned* amax) {
    if (t.march) {  // the even faces of the MARCH layout, from an FP32 volume
        if (vdt != TOMO_F32 || amax || !t.surf) return cudaErrorInvalidValue;
        const int width = std::max(nx, ny);
        const long n = (long)width * (march_even_faces(nx) + march_even_faces(ny)) * nz;
        const int b = (int)std::min<long>((n + 255) / 256, 148L * 16);
        rs_march_tex_kernel<<<b, 256, 0, st>>>((const float*)vol, t.surf, nx, ny, nz, width);
        return cudaGetLastError();
    }
    if (vdt == t.dt && !amax && t.z0 == 0) {
        const size_t es = dtype_size(t.dt);
        cudaMemcpy3DParms p{};
        p.srcPtr = make_cudaPitchedPtr(const_cast<void*>(vol), (size_t)nx * es, (size_t)nx * es, ny);
        p.dstArray = t.arr;
        p.extent = make_cudaExtent(nx, ny, nz);
        p.kind = cudaMemcpyDeviceToDevice;
        return cudaMemcpy3DAsync(&p, st);
    }
    if (!t.surf) return cudaErrorInvalidValue;  // surface-less FP32 textures take FP32 copies only
    if (t.zpairs)
        return t.dt == TOMO_BF16 ? tex_pairs<__nv_bfloat16>(vol, vdt, nx, ny, nz, t.surf, st, amax)
                                 : tex_pairs<__half>(vol, vdt, nx, ny, nz, t.surf, st, amax);
    switch (t.dt) {
        case TOMO_F32: return tex_convert<float>(vol, vdt, nx, ny, nz, t.z0, t.surf, st, amax);
        case TOMO_BF16: return tex_convert<__nv_bfloat16>(vol, vdt, nx, ny, nz, t.z0, t.surf, st, amax);
        case TOMO_F16: return tex_convert<__half>(vol, vdt, nx, ny, nz, t.z0, t.surf, st, amax);
    }
    return cudaErrorInvalidValue;
}

// Loads the conversion kernels (lazy module loading would load them at their first launch,
// which synchronises the context).
void rs_tex_preload() {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, rs_tex_zero_layers_kernel);
    cudaFuncGetAttributes(&a, rs_march_tex_kernel);
    cudaFuncGetAttributes(&a, rs_march_quads_kernel);
    cudaFuncGetAttributes(&a, rs_tex_pairs_kernel<float, __nv_bfloat16>);
    cudaFuncGetAttributes(&a, rs_tex_pairs_kernel<float, __half>);
    cudaFuncGetAttributes(&a, rs_tex_pairs_kernel<__nv_bfloat16, __nv_bfloat16>);
    cudaFuncGetAttributes(&a, rs_tex_pairs_kernel<__half, __half>);
    cudaFuncGetAttributes(&a, rs_tex_pairs_kernel<__nv_bfloat16, __half>);
    cudaFuncGetAttributes(&a, rs_tex_pairs_kernel<__half, __nv_bfloat16>);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<float, float>);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<__nv_bfloat16, float>);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<__half, float>);
    cudaFuncGetAttributes(&a, tex_from_padded_kernel);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<float, __nv_bfloat16>);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<float, __half>);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<__nv_bfloat16, __half>);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<__half, __nv_bfloat16>);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<__nv_bfloat16, __nv_bfloat16>);
    cudaFuncGetAttributes(&a, rs_tex_convert_kernel<__half, __half>);
}

int rs_tex_max_layers() {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxTexture2DLayeredLayers, dev) != cudaSuccess) return 0;
    return v;
}

template <typename Ti>
static cudaError_t cells_out(const Ti* in, void* out, tomo_dtype odt, int nx, int ny, int nz, cudaStream_t st,
                             const unsigned* amax) {
    long n = (long)(nx + 1) * (ny + 1) * (nz + 1);
    long b = (n + 255) / 256;
    if (b > 148L * 32) b = 148L * 32;
    switch (odt) {
        case TOMO_F32: rs_cells_kernel<Ti, float><<<(int)b, 256, 0, st>>>(in, (float*)out, nx, ny, nz, amax); break;
        case TOMO_BF16:
            rs_cells_kernel<Ti, __nv_bfloat16><<<(int)b, 256, 0, st>>>(in, (__nv_bfloat16*)out, nx, ny, nz, amax);
            break;
        case TOMO_F16: rs_cells_kernel<Ti, __half><<<(int)b, 256, 0, st>>>(in, (__half*)out, nx, ny, nz, amax); break;
    }
    return cudaGetLastError();
}

template <typename Ti>
static cudaError_t quads_out(const Ti* in, void* out, tomo_dtype odt, int nx, int ny, int nz, cudaStream_t st,
                             const unsigned* amax) {
    const dim3 grid((nx + QT) / QT, (ny + QT) / QT, nz + 1), block(QT, 8);  // quads ci in [0, nx], cj in [0, ny]
    switch (odt) {
        case TOMO_F32: rs_quads_kernel<Ti, float><<<grid, block, 0, st>>>(in, (float*)out, nx, ny, nz, amax); break;
        case TOMO_BF16:
            rs_quads_kernel<Ti, __nv_bfloat16><<<grid, block, 0, st>>>(in, (__nv_bfloat16*)out, nx, ny, nz, amax);
            break;
        case TOMO_F16: rs_quads_kernel<Ti, __half><<<grid, block, 0, st>>>(in, (__half*)out, nx, ny, nz, amax); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_rs_prepare(int layout, const void* in, tomo_dtype idt, void* out, tomo_dtype odt, int nx, int ny,
                              int nz, cudaStream_t st, const unsigned* amax) {
    if (layout == RS_LAYOUT_MARCH) {  // the odd faces; the even ones are filled by rs_tex_fill
        if (idt != TOMO_F32 || odt != TOMO_F32 || amax) return cudaErrorInvalidValue;
        const long n = march_quads(nx, ny, nz) + march_quads(ny, nx, nz);
        const int b = (int)std::min<long>((n + 255) / 256, 148L * 16);
        rs_march_quads_kernel<<<b, 256, 0, st>>>((const float*)in, (float4*)out, nx, ny, nz);
        return cudaGetLastError();
    }
    if (layout == RS_LAYOUT_HYBRID) {  // the quads; the texture is filled by rs_tex_fill
        switch (idt) {
            case TOMO_F32: return quads_out((const float*)in, out, odt, nx, ny, nz, st, amax);
            case TOMO_BF16: return quads_out((const __nv_bfloat16*)in, out, odt, nx, ny, nz, st, amax);
            case TOMO_F16: return quads_out((const __half*)in, out, odt, nx, ny, nz, st, amax);
        }
        return cudaErrorInvalidValue;
    }
    if (layout != RS_LAYOUT_CELL8) return launch_pad_volume(in, idt, out, odt, nx, ny, nz, st, amax);
    switch (idt) {
        case TOMO_F32: return cells_out((const float*)in, out, odt, nx, ny, nz, st, amax);
        case TOMO_BF16: return cells_out((const __nv_bfloat16*)in, out, odt, nx, ny, nz, st, amax);
        case TOMO_F16: return cells_out((const __half*)in, out, odt, nx, ny, nz, st, amax);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_rs_adjoint(int mode, const DevGeom& g, const void* sino, tomo_dtype sdt, float* vol,
                              cudaStream_t st) {
    dim3 block(256), grid(g.np, (g.nu + 15) / 16, (g.nv + 15) / 16);
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
