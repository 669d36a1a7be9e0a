// siddon.cu -- Siddon exact-chord cone-beam projector for sm_100a.
//
// One thread per detector ray, warps on 8u x 4v tiles of one view (the rays of a warp
// cross neighbouring voxels in step, so their voxel reads share L1 lines). The set-up
// (cylinder entry/exit lambda_min/max, first voxel, first plane crossings) and the
// traversal follow SiddonProjector_compute_C_mem_CPU::doProjection
// (src/TomoGPI_lib/src/CPP/SiddonProjector_compute_C_mem_CPU.cpp:64-266) with explicitly
// rounded IEEE operations, including its float->double promotions, so every ray visits
// the same voxels with the same chord lengths as the reference's C code.
//   compat = 1 (TOMO_PROJ_SIDDON_REF): the reference as written -- source at +FOD,
//              detector at -(FDD-FOD) (:76-96), voxel index modulo 256 per axis (:228).
//              Indices that land outside the volume read 0 (the C code reads past the
//              array there, which only happens for volumes smaller than 256).
//   compat = 0 (TOMO_PROJ_SIDDON): the RSVI geometry (source at -FOD), no wrap, voxels
//              outside the volume contribute nothing.
// The traversal loop is bounded (4 (Nx+Ny+Nz) + 64 steps); a ray that hits the bound
// sets ERR_SIDDON_GUARD in the device error word instead of looping on.
#include "tomo_kernels.cuh"

namespace tomo {

struct SiddonRay {
    float lambda, lmax, lx, ly, lz, stepx, stepy, stepz;
    int xn, yn, zn, dxn, dyn, dzn;
};

__device__ __forceinline__ void siddon_axis(float smin, float src, float det, int n, float L, float dx, int& idx,
                                            float& lam) {
    if (src <= det) {                                                            // :120
        smin = __double2float_rn(dsub((double)smin, 0.5));
        if (smin < 0.0f) idx = 0;
        else if (smin > (float)(n - 1)) idx = n - 1;
        else idx = (int)floorf(smin);
        if (fabsf(fsub(det, src)) > dx)
            lam = __double2float_rn(ddiv(dmul((double)L, dsub(dmul(dadd((double)(float)idx, 0.5), (double)dx), (double)src)),
                                         (double)fsub(det, src)));              // :130
        else
            lam = L;
    } else {
        smin = __double2float_rn(dadd((double)smin, 0.5));                      // :135
        if (smin < 0.0f) idx = 0;
        else if (smin > (float)(n - 1)) idx = n - 1;
        else idx = (int)ceilf(smin);
        if (fabsf(fsub(det, src)) > dx)
            lam = __double2float_rn(ddiv(dmul((double)L, dsub(dmul(dsub((double)(float)idx, 0.5), (double)dx), (double)src)),
                                         (double)fsub(det, src)));              // :144
        else
            lam = L;
    }
}

template <int COMPAT>
__device__ __forceinline__ bool siddon_setup(const DevGeom& g, int u, int v, float al, float be, SiddonRay& r) {
    const float dx = g.dx;
    const float sgn = COMPAT ? 1.0f : -1.0f;
    const float x_Lr = fmul(g.xc, dx), y_Lr = fmul(g.yc, dx), z_Lr = fmul(g.zc, dx);   // :64-66
    const float sf = fmul(sgn, g.fod);
    const float x_s = fadd(x_Lr, fmul(sf, al));                                  // :76
    const float y_s = fadd(y_Lr, fmul(sf, be));                                  // :77
    const float z_s = z_Lr;                                                      // :78
    const float s = fmul(fsub((float)u, g.uc), g.du);                            // :90
    const float t = fmul(fsub((float)v, g.vc), g.dv);                            // :91
    const float fmo = fsub(g.fdd, g.fod);
    const float x_det = fsub(fsub(x_Lr, fmul(fmul(sgn, al), fmo)), fmul(s, be)); // :94
    const float y_det = fadd(fsub(y_Lr, fmul(fmul(sgn, be), fmo)), fmul(s, al)); // :95
    const float z_det = fadd(z_Lr, t);                                           // :96
    const float f2s2 = fadd(fmul(g.fdd, g.fdd), fmul(s, s));
    const float L = fsqrt(fadd(f2s2, fmul(t, t)));                               // :99
    const float A = fdiv(f2s2, fmul(L, L));                                      // :102
    const float B = fdiv(fmul(-g.fod, g.fdd), L);                                // :103
    const double nxd = (double)(float)g.nx;
    const float C = __double2float_rn(
        dsub((double)fmul(g.fod, g.fod), dmul(dmul(dmul(dmul(0.25, nxd), nxd), (double)dx), (double)dx)));  // :104
    const float delta = fsub(fmul(B, B), fmul(A, C));                            // :105
    if (!(delta > 0.0f)) return false;                                           // :108
    const float sq = fsqrt(delta);
    const float lmin = fdiv(fsub(-B, sq), A);                                    // :110
    r.lmax = fdiv(fadd(-B, sq), A);                                              // :111
    const float xmin = fdiv(fadd(x_s, fdiv(fmul(lmin, fsub(x_det, x_s)), L)), dx);  // :114
    const float ymin = fdiv(fadd(y_s, fdiv(fmul(lmin, fsub(y_det, y_s)), L)), dx);
    const float zmin = fdiv(fadd(z_s, fdiv(fmul(lmin, fsub(z_det, z_s)), L)), dx);
    siddon_axis(xmin, x_s, x_det, g.nx, L, dx, r.xn, r.lx);
    siddon_axis(ymin, y_s, y_det, g.ny, L, dx, r.yn, r.ly);
    siddon_axis(zmin, z_s, z_det, g.nz, L, dx, r.zn, r.lz);
    r.stepx = fmul(fdiv(L, fabsf(fsub(x_det, x_s))), dx);                        // :234
    r.stepy = fmul(fdiv(L, fabsf(fsub(y_det, y_s))), dx);                        // :242
    r.stepz = fmul(fdiv(L, fabsf(fsub(z_det, z_s))), dx);                        // :250
    r.dxn = (x_s <= x_det) ? 1 : -1;
    r.dyn = (y_s <= y_det) ? 1 : -1;
    r.dzn = (z_s <= z_det) ? 1 : -1;
    r.lambda = lmin;
    return true;
}

// Walks the ray; visit(linear index or -1, chord).
template <int COMPAT, typename F>
__device__ __forceinline__ bool siddon_walk(const DevGeom& g, SiddonRay& r, F&& visit) {
    const int guard = 4 * (g.nx + g.ny + g.nz) + 64;
    const long plane = (long)g.nx * g.ny, total = plane * g.nz;
    int it = 0;
    while (r.lambda <= r.lmax) {                                                 // :213
        if (++it > guard) return false;
        float lk = r.lx;
        if (r.ly < lk) lk = r.ly;
        if (r.lz < lk) lk = r.lz;
        const float chord = fsub(lk, r.lambda);                                  // :224
        long idx;
        if (COMPAT) {
            idx = (long)(r.xn & 255) + (long)(r.yn & 255) * g.nx + (long)(r.zn & 255) * plane;  // :228
            if (idx >= total) idx = -1;
        } else {
            idx = ((unsigned)r.xn < (unsigned)g.nx && (unsigned)r.yn < (unsigned)g.ny && (unsigned)r.zn < (unsigned)g.nz)
                      ? (long)r.xn + (long)r.yn * g.nx + (long)r.zn * plane
                      : -1;
        }
        visit(idx, chord);
        r.lambda = lk;
        if (r.lx <= lk) { r.lx = fadd(r.lx, r.stepx); r.xn += r.dxn; }           // :233
        if (r.ly <= lk) { r.ly = fadd(r.ly, r.stepy); r.yn += r.dyn; }           // :241
        if (r.lz <= lk) { r.lz = fadd(r.lz, r.stepz); r.zn += r.dzn; }           // :249
    }
    return true;
}

template <int COMPAT, typename Tv, typename To, int EPI, typename Tr>
__global__ void __launch_bounds__(256) siddon_project_kernel(DevGeom g, const Tv* __restrict__ vol, OutView<To> out,
                                                             OutView<Tr> real, double* __restrict__ norm,
                                                             unsigned* __restrict__ err) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = blockIdx.x;  // views fastest: resident blocks share one row band's slab
    const int u = blockIdx.y * 16 + (warp & 1) * 8 + (lane & 7);
    const int v = blockIdx.z * 16 + (warp >> 1) * 4 + (lane >> 3);
    const bool active = (u < g.nu) && (v < g.nv);
    float acc = 0.f;
    if (active) {
        SiddonRay r;
        if (siddon_setup<COMPAT>(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r)) {
            const bool ok = siddon_walk<COMPAT>(g, r, [&](long idx, float chord) {
                acc = fadd(acc, fmul(chord, idx >= 0 ? ld(vol + idx) : 0.0f));  // :229
            });
            if (!ok) atomicOr(err, ERR_SIDDON_GUARD);
        }
    }
    epilogue<EPI, To, Tr>(active, acc, u, v, p, out, real, norm);
}

template <int COMPAT, typename Ts>
__global__ void __launch_bounds__(256) siddon_adjoint_kernel(DevGeom g, const Ts* __restrict__ sino,
                                                             float* __restrict__ vol, unsigned* __restrict__ err) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = blockIdx.x;  // views fastest: resident blocks share one row band's slab
    const int u = blockIdx.y * 16 + (warp & 1) * 8 + (lane & 7);
    const int v = blockIdx.z * 16 + (warp >> 1) * 4 + (lane >> 3);
    if (u >= g.nu || v >= g.nv) return;
    const float y = ld(sino + ((long)p * g.nv + v) * g.nu + u);
    if (y == 0.f) return;
    SiddonRay r;
    if (!siddon_setup<COMPAT>(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r)) return;
    const bool ok = siddon_walk<COMPAT>(g, r, [&](long idx, float chord) {
        if (idx >= 0) atomicAdd(vol + idx, chord * y);
    });
    if (!ok) atomicOr(err, ERR_SIDDON_GUARD);
}

template <int COMPAT>
__global__ void siddon_count_kernel(DevGeom g, unsigned long long* __restrict__ total, unsigned* __restrict__ err) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    const int p = blockIdx.z;
    unsigned long long n = 0;
    if (u < g.nu) {
        SiddonRay r;
        if (siddon_setup<COMPAT>(g, u, v, __ldg(g.alpha + p), __ldg(g.beta + p), r)) {
            if (!siddon_walk<COMPAT>(g, r, [&](long, float) { ++n; })) atomicOr(err, ERR_SIDDON_GUARD);
        }
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(total, n);
}

template <int C, int EPI, typename Tv, typename To, typename Tr>
static cudaError_t launch_siddon_k(const DevGeom& g, const void* vol, const OutView<void>& out, const OutView<void>& real,
                                   double* norm, unsigned* err, cudaStream_t st) {
    const dim3 block(256), grid(g.np, (g.nu + 15) / 16, (g.nv + 15) / 16);  // siddon_grid_blocks
    siddon_project_kernel<C, Tv, To, EPI, Tr><<<grid, block, 0, st>>>(g, static_cast<const Tv*>(vol), out.as<To>(),
                                                                        real.as<Tr>(), norm, err);
    return cudaGetLastError();
}

template <int C, typename Tv>
static cudaError_t launch_siddon_e(int epi, const DevGeom& g, const void* vol, const OutView<void>& out, tomo_dtype odt,
                                   const OutView<void>& real, tomo_dtype rdt, double* norm, unsigned* err,
                                   cudaStream_t st) {
    if (epi == EPI_STORE) {
        switch (odt) {
            case TOMO_F32: return launch_siddon_k<C, EPI_STORE, Tv, float, float>(g, vol, out, real, norm, err, st);
            case TOMO_BF16:
                return launch_siddon_k<C, EPI_STORE, Tv, __nv_bfloat16, __nv_bfloat16>(g, vol, out, real, norm, err, st);
            case TOMO_F16: return launch_siddon_k<C, EPI_STORE, Tv, __half, __half>(g, vol, out, real, norm, err, st);
        }
    } else if (epi == EPI_RESIDUAL) {
        switch (rdt) {
            case TOMO_F32: return launch_siddon_k<C, EPI_RESIDUAL, Tv, float, float>(g, vol, out, real, norm, err, st);
            case TOMO_BF16:
                return launch_siddon_k<C, EPI_RESIDUAL, Tv, float, __nv_bfloat16>(g, vol, out, real, norm, err, st);
            case TOMO_F16: return launch_siddon_k<C, EPI_RESIDUAL, Tv, float, __half>(g, vol, out, real, norm, err, st);
        }
    } else if (epi == EPI_NORM) {
        return launch_siddon_k<C, EPI_NORM, Tv, float, float>(g, vol, out, real, norm, err, st);
    }
    return cudaErrorInvalidValue;
}

size_t siddon_grid_blocks(const DevGeom& g) { return (size_t)g.np * ((g.nu + 15) / 16) * ((g.nv + 15) / 16); }

cudaError_t launch_siddon_project(int compat, int epi, const DevGeom& g, const void* vol, tomo_dtype vdt,
                                  const OutView<void>& out, tomo_dtype odt, const OutView<void>& real,
                                  double* norm, unsigned* err, cudaStream_t st, tomo_dtype rdt) {
#define TOMO_SD_V(TV)                                                                                   \
    return compat ? launch_siddon_e<1, TV>(epi, g, vol, out, odt, real, rdt, norm, err, st)            \
                  : launch_siddon_e<0, TV>(epi, g, vol, out, odt, real, rdt, norm, err, st);
    switch (vdt) {
        case TOMO_F32: TOMO_SD_V(float)
        case TOMO_BF16: TOMO_SD_V(__nv_bfloat16)
        case TOMO_F16: TOMO_SD_V(__half)
    }
#undef TOMO_SD_V
    return cudaErrorInvalidValue;
}

cudaError_t launch_siddon_adjoint(int compat, const DevGeom& g, const void* sino, tomo_dtype sdt, float* vol,
                                  unsigned* err, cudaStream_t st) {
    dim3 block(256), grid(g.np, (g.nu + 15) / 16, (g.nv + 15) / 16);
#define TOMO_SA(TS)                                                                                     \
    if (compat) siddon_adjoint_kernel<1, TS><<<grid, block, 0, st>>>(g, (const TS*)sino, vol, err);     \
    else siddon_adjoint_kernel<0, TS><<<grid, block, 0, st>>>(g, (const TS*)sino, vol, err);
    switch (sdt) {
        case TOMO_F32: TOMO_SA(float) break;
        case TOMO_BF16: TOMO_SA(__nv_bfloat16) break;
        case TOMO_F16: TOMO_SA(__half) break;
    }
#undef TOMO_SA
    return cudaGetLastError();
}

cudaError_t launch_siddon_count(int compat, const DevGeom& g, unsigned long long* total, unsigned* err,
                                cudaStream_t st) {
    dim3 block(128), grid((g.nu + 127) / 128, g.nv, g.np);
    if (compat) siddon_count_kernel<1><<<grid, block, 0, st>>>(g, total, err);
    else siddon_count_kernel<0><<<grid, block, 0, st>>>(g, total, err);
    return cudaGetLastError();
}

}  // namespace tomo
