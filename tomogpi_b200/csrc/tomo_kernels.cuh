// tomo_kernels.cuh -- device building blocks shared by the operator kernels and the
// host launcher declarations.
#pragma once

#include "tomo_common.cuh"

namespace tomo {

// Output descriptor of a sinogram-shaped result: element (p, v, u) lives at
// ptr[offset + p*view_pitch + v*row_pitch + u]. Lets the projector write either the
// plain [phi][v][u] array or straight into a zero-bordered padded buffer.
template <typename T>
struct OutView {
    T* ptr;
    long offset, row_pitch, view_pitch;
    template <typename U>
    __host__ __device__ OutView<U> as() const {
        return OutView<U>{(U*)ptr, offset, row_pitch, view_pitch};
    }
    __host__ __device__ long at(int p, int v, int u) const { return offset + p * view_pitch + v * row_pitch + u; }
};

enum { EPI_STORE = 0, EPI_RESIDUAL = 1, EPI_NORM = 2, EPI_PARTIAL = 3 };

// RS projector tiles: one 256-thread block covers 2^rs_tlog u x 2^(8 - rs_tlog) v rays of
// one view (DevGeom::rs_tlog, 4..7); its warps cover 2^rs_wlog u x 2^(5 - rs_wlog) v rays
// each (DevGeom::rs_wlog, 3..5, at most rs_tlog).
constexpr int RS_WLOG_DEFAULT = 3;
constexpr int RS_TLOG_DEFAULT = 5;
__host__ __device__ __forceinline__ int rs_tile_u(const DevGeom& g) { return 1 << g.rs_tlog; }
__host__ __device__ __forceinline__ int rs_tile_v(const DevGeom& g) { return 256 >> g.rs_tlog; }
__host__ __device__ __forceinline__ int rs_tiles_u(const DevGeom& g) { return (g.nu + rs_tile_u(g) - 1) >> g.rs_tlog; }
__host__ __device__ __forceinline__ int rs_tiles_v(const DevGeom& g) { return (g.nv + rs_tile_v(g) - 1) / rs_tile_v(g); }
// The launch shape a tuning asks for (0 = the defaults: warps of 8 u x 4 v, blocks of 32 u x 8 v).
inline bool rs_shape_valid(const tomo_tuning& t) {
    const int wu = t.rs_warp_u ? t.rs_warp_u : 1 << RS_WLOG_DEFAULT;
    const int tu = t.rs_tile_u ? t.rs_tile_u : 1 << RS_TLOG_DEFAULT;
    return (wu == 8 || wu == 16 || wu == 32) && (tu == 16 || tu == 32 || tu == 64 || tu == 128) && wu <= tu;
}
inline void rs_shape_of(const tomo_tuning& t, DevGeom& g) {
    const int wu = t.rs_warp_u ? t.rs_warp_u : 1 << RS_WLOG_DEFAULT;
    const int tu = t.rs_tile_u ? t.rs_tile_u : 1 << RS_TLOG_DEFAULT;
    g.rs_wlog = wu == 32 ? 5 : wu == 16 ? 4 : 3;
    g.rs_tlog = tu == 128 ? 7 : tu == 64 ? 6 : tu == 32 ? 5 : 4;
}

// Volume layouts read by the RS projector (see rs_project.cu).
enum { RS_LAYOUT_PLAIN = 0, RS_LAYOUT_CELL8 = 1, RS_LAYOUT_TEX = 2, RS_LAYOUT_HYBRID = 3, RS_LAYOUT_MARCH = 4 };

// MARCH layout (FP32): the volume cut into faces across the axis a view's rays mostly run
// along (x for the views with |alpha| > |beta|, else y), face m holding the texels of
// x = m (resp. y = m), m in [-1, n_a], as a 2D image over (t, z), t the other in-plane axis.
// Faces of even m are layers of one layered texture (the x-march faces first, then the
// y-march faces; width max(nx, ny), height nz; texels past the data are 0); faces of odd m
// are quads in global memory (the 2 x 2 footprint at (t, k) in tld4 order, t in [-1, n_t-1]
// fastest, k in [-1, nz-1], then m), x-march faces first.
__host__ __device__ __forceinline__ int march_even_faces(int n) { return n / 2 + 1; }      // m = 0, 2, ..., <= n
__host__ __device__ __forceinline__ int march_odd_faces(int n) { return (n + 1) / 2 + 1; }  // m = -1, 1, ..., <= n
__host__ __device__ __forceinline__ long march_quads(int na, int nt, int nz) {
    return (long)march_odd_faces(na) * (nz + 1) * (nt + 1);
}

// Projector epilogue:
//   EPI_STORE    out = acc
//   EPI_RESIDUAL out = real - acc          (Sinogram3D_CPU::diffSinogram, Sinogram3D_CPU.cu:311-336);
//                the residual is FP32 whatever the storage of `real`
//   EPI_NORM     norm[linear block index] = the block's sum of double(acc*acc), nothing
//                stored; launch_sum_partials then adds the partials in a fixed order
//                (Sinogram3D_CPU::getSinogramL2Norm, Sinogram3D_CPU.cu:358-374): no atomics
//                on one address, and the same total on every run
//   EPI_PARTIAL  *norm  = that block sum (deterministic per-item partials)
__device__ __forceinline__ double block_sum(double s);
__device__ __forceinline__ long linear_block() {
    return blockIdx.x + (long)gridDim.x * (blockIdx.y + (long)gridDim.y * blockIdx.z);
}

template <int EPI, typename To, typename Tr>
__device__ __forceinline__ void epilogue(bool active, float acc, int u, int v, int p, const OutView<To>& out,
                                         const OutView<Tr>& real, double* norm) {
    if (EPI == EPI_STORE) {
        if (active) out.ptr[out.at(p, v, u)] = cvt<To>(acc);
    } else if (EPI == EPI_RESIDUAL) {
        if (active) out.ptr[out.at(p, v, u)] = cvt<To>(fsub(ldp(real.ptr + real.at(p, v, u)), acc));
    } else if (EPI == EPI_PARTIAL) {
        // the block's sum of double(acc*acc) stored (not added) at *norm: one slot per work
        // item, summed later in a fixed order, so the total does not depend on scheduling
        const double s = block_sum(active ? (double)fmul(acc, acc) : 0.0);
        if (threadIdx.x == 0) *norm = s;
    } else {  // EPI_NORM: the block's partial at its linear index
        const double s = block_sum(active ? (double)fmul(acc, acc) : 0.0);
        if (threadIdx.x == 0 && threadIdx.y == 0) norm[linear_block()] = s;
    }
}

// Sum of the three 1-D {-1, 2, -1} convolutions at (x, y, z), zero padded, accumulated per
// axis as the reference's separable kernels do (tmp = 0; tmp += s[-1]*k2; tmp += s[0]*k1;
// tmp += s[+1]*k0, Convolution3D_sep_shared_kernel.cuh:81-90), then h + v + p.
__device__ __forceinline__ float lap_at(const float* __restrict__ in, int x, int y, int z, int nx, int ny, int nz) {
    const long plane = (long)nx * ny;
    const long i = z * plane + (long)y * nx + x;
    const float c = in[i];
    const float xm = x > 0 ? in[i - 1] : 0.f, xp = x < nx - 1 ? in[i + 1] : 0.f;
    const float ym = y > 0 ? in[i - nx] : 0.f, yp = y < ny - 1 ? in[i + nx] : 0.f;
    const float zm = z > 0 ? in[i - plane] : 0.f, zp = z < nz - 1 ? in[i + plane] : 0.f;
    const float c2 = fmul(c, 2.0f);
    const float h = fadd(fadd(fmul(xm, -1.0f), c2), fmul(xp, -1.0f));
    const float v = fadd(fadd(fmul(ym, -1.0f), c2), fmul(yp, -1.0f));
    const float p = fadd(fadd(fmul(zm, -1.0f), c2), fmul(zp, -1.0f));
    return fadd(fadd(h, v), p);
}

// Deterministic block sum (all threads of the block call it; thread 0 gets the total).
__device__ __forceinline__ double block_sum(double s) {
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = t & 31, warp = t >> 5, nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (lane == 0) red[warp] = s;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------------
// Regular-sampling ray set-up.
// ---------------------------------------------------------------------------------
struct RsRay {
    float A, B, C;     // entry point, voxel coordinates
    float sx, sy, sz;  // unit step (ctheta, stheta, salpha)
    unsigned n;        // L_r, number of samples
};

// (unsigned)(unsigned long long)len as the reference truncates it; a chord inside the
// volume is at most its diagonal, so the bound below never binds for a finite ray and
// only keeps a non-finite length from turning into a multi-billion-step loop.
__device__ __forceinline__ unsigned rs_clamp_samples(const DevGeom& g, float len) {
    const unsigned n = (unsigned)__float2ull_rz(len);
    const unsigned cap = 2u * (unsigned)(g.nx + g.ny + g.nz) + 8u;
    return n < cap ? n : cap;
}

// projection_ERB_kernel_v1 prologue (projection_ER_kernel.cuh:69-288), FOV_CYLINDER 0.
__device__ __forceinline__ bool rs_ray_box(const DevGeom& g, int u, int v, float al, float be, RsRay& r) {
    const float x_s = fmul(-g.fod, al);                                          // :69
    const float y_s = fmul(-g.fod, be);                                          // :70
    const float uu = fsub((float)u, g.uc);
    const float fmo = fsub(g.fdd, g.fod);
    float A = fsub(fmul(al, fmo), fmul(fmul(uu, be), g.du));                     // :71
    float B = fadd(fmul(be, fmo), fmul(fmul(uu, g.du), al));                     // :72
    float C = fmul(fsub((float)v, g.vc), g.dv);                                  // :73
    const float ax = fsub(A, x_s), by = fsub(B, y_s);
    float E = fdiv(1.0f, fsqrt(fadd(fadd(fmul(ax, ax), fmul(by, by)), fmul(C, C))));  // :76
    r.sz = fmul(C, E);                                                           // :77
    r.sx = fmul(ax, E);                                                          // :79
    r.sy = fmul(by, E);                                                          // :80
    const float A1 = fdiv(by, ax);                                               // :92
    const float B1 = fdiv(fsub(B, fmul(A1, A)), g.dx);                           // :93
    const float C1 = fdiv(C, ax);                                                // :94
    const float D1 = fdiv(fsub(C, fmul(C1, A)), g.dx);                           // :95
    const float Nf = (float)g.nx;
    const float nn = fmul(fdiv(fmul(2.0f, Nf), 2.0f), Nf);                       // :102, float part
    const float F = __double2float_rn(
        dsub(dmul(ddiv((double)nn, 2.0), (double)fadd(fmul(A1, A1), 1.0f)), (double)fmul(B1, B1)));
    if (!(F >= 0.0f)) return false;                                              // :107
    E = fsqrt(F);
    const float den = fadd(1.0f, fmul(A1, A1));
    const float nab = fmul(-A1, B1);
    const float x_p1 = fdiv(fadd(nab, E), den);
    const float y_p1 = fadd(fmul(A1, x_p1), B1);
    const float z_p1 = fadd(fmul(C1, x_p1), D1);
    const float x_p2 = fdiv(fsub(nab, E), den);
    const float y_p2 = fadd(fmul(A1, x_p2), B1);
    const float z_p2 = fadd(fmul(C1, x_p2), D1);
    const float d1x = fsub(x_p1, x_s), d1y = fsub(y_p1, y_s);
    const float d2x = fsub(x_p2, x_s), d2y = fsub(y_p2, y_s);
    const float dist1 = fadd(fadd(fmul(d1x, d1x), fmul(d1y, d1y)), fmul(z_p1, z_p1));  // :117
    const float dist2 = fadd(fadd(fmul(d2x, d2x), fmul(d2y, d2y)), fmul(z_p2, z_p2));  // :118
    float x_f, y_f, z_f;
    if (dist1 <= dist2) {                                                        // :156
        A = fadd(x_p1, g.xc); B = fadd(y_p1, g.yc); C = fadd(z_p1, g.zc);
        x_f = fadd(x_p2, g.xc); y_f = fadd(y_p2, g.yc); z_f = fadd(z_p2, g.zc);
    } else {
        A = fadd(x_p2, g.xc); B = fadd(y_p2, g.yc); C = fadd(z_p2, g.zc);
        x_f = fadd(x_p1, g.xc); y_f = fadd(y_p1, g.yc); z_f = fadd(z_p1, g.zc);
    }
    const float xmax = (float)(g.nx - 1), ymax = (float)(g.ny - 1), zmax = (float)(g.nz - 1);
    if (A < 0.0f) {                                                              // :182
        A = 0.0f;
        B = fadd(fmul(A1, fsub(A, g.xc)), B1); C = fadd(fmul(C1, fsub(A, g.xc)), D1);
        B = fadd(B, g.yc); C = fadd(C, g.zc);
    }
    if (B < 0.0f) {                                                              // :190
        B = 0.0f;
        A = fdiv(fsub(fsub(B, g.yc), B1), A1); C = fadd(fmul(C1, A), D1);
        A = fadd(A, g.xc); C = fadd(C, g.zc);
    }
    if (A > xmax) {                                                              // :199
        A = xmax;
        B = fadd(fmul(A1, fsub(A, g.xc)), B1); C = fadd(fmul(C1, fsub(A, g.xc)), D1);
        B = fadd(B, g.yc); C = fadd(C, g.zc);
    }
    if (B > ymax) {                                                              // :207
        B = ymax;
        A = fdiv(fsub(fsub(B, g.yc), B1), A1); C = fadd(fmul(C1, A), D1);
        A = fadd(A, g.xc); C = fadd(C, g.zc);
    }
    if (x_f < 0.0f) {                                                            // :217
        x_f = 0.0f;
        y_f = fadd(fmul(A1, fsub(x_f, g.xc)), B1); z_f = fadd(fmul(C1, fsub(x_f, g.xc)), D1);
        y_f = fadd(y_f, g.yc); z_f = fadd(z_f, g.zc);
    }
    if (y_f < 0.0f) {                                                            // :226
        y_f = 0.0f;
        x_f = fdiv(fsub(fsub(y_f, g.yc), B1), A1); z_f = fadd(fmul(C1, x_f), D1);
        x_f = fadd(x_f, g.xc); z_f = fadd(z_f, g.zc);
    }
    if (x_f > xmax) {                                                            // :235
        x_f = xmax;
        y_f = fadd(fmul(A1, fsub(x_f, g.xc)), B1); z_f = fadd(fmul(C1, fsub(x_f, g.xc)), D1);
        y_f = fadd(y_f, g.yc); z_f = fadd(z_f, g.zc);
    }
    if (y_f > ymax) {                                                            // :244
        y_f = ymax;
        x_f = fdiv(fsub(fsub(y_f, g.yc), B1), A1); z_f = fadd(fmul(C1, x_f), D1);
        x_f = fadd(x_f, g.xc); z_f = fadd(z_f, g.zc);
    }
    if (!((C <= zmax) && (C >= 0.0f))) return false;                            // :259
    if (z_f > zmax) {                                                            // :263
        z_f = fsub(zmax, g.zc);
        x_f = fdiv(fsub(z_f, D1), C1); y_f = fadd(fmul(A1, x_f), B1);
        x_f = fadd(x_f, g.xc); y_f = fadd(y_f, g.yc); z_f = fadd(z_f, g.zc);
    } else if (z_f < 0.0f) {                                                     // :273
        z_f = -g.zc;
        x_f = fdiv(fsub(z_f, D1), C1); y_f = fadd(fmul(A1, x_f), B1);
        x_f = fadd(x_f, g.xc); y_f = fadd(y_f, g.yc); z_f = fadd(z_f, g.zc);
    }
    const float ex = fsub(A, x_f), ey = fsub(B, y_f), ez = fsub(C, z_f);
    const float len = fsqrt(fadd(fadd(fmul(ex, ex), fmul(ey, ey)), fmul(ez, ez)));  // :285
    r.n = rs_clamp_samples(g, len);
    r.A = A; r.B = B; r.C = C;  // :288 with zn_start = 0
    return true;
}

// projection_ERB_kernel_v0_UM prologue (projection_ER_kernel_UM.cuh:39-123).
__device__ __forceinline__ bool rs_ray_um(const DevGeom& g, int u, int v, float al, float be, RsRay& r) {
    const float x_s = fmul(-g.fod, al);                                          // :39
    const float y_s = fmul(-g.fod, be);                                          // :40
    const float uu = fsub((float)u, g.uc), vv = fsub((float)v, g.vc);
    const float fmo = fsub(g.fdd, g.fod);
    float A = fsub(fmul(al, fmo), fmul(fmul(uu, be), g.du));                     // :41
    float B = fadd(fmul(be, fmo), fmul(fmul(uu, g.du), al));                     // :42
    float C = fmul(vv, g.dv);                                                    // :43
    const float ax = fsub(A, x_s), by = fsub(B, y_s);
    float D = __double2float_rn(ddiv(1.0, (double)fsqrt(fadd(fadd(fmul(ax, ax), fmul(by, by)), fmul(C, C)))));  // :47
    r.sz = fmul(C, D);                                                           // :49
    r.sx = fmul(ax, D);                                                          // :50
    r.sy = fmul(by, D);                                                          // :51
    const float bdx = fmul(-be, g.dx), adx = fmul(al, g.dx), fdu = fdiv(g.fdd, g.du);
    D = fdiv(1.0f, fadd(fmul(bdx, uu), fmul(adx, fdu)));                         // :53
    const float A1 = fmul(fsub(fmul(adx, uu), fmul(bdx, fdu)), D);               // :54
    const float B1 = fmul(fmul(uu, g.fod), D);                                   // :55
    const float gv = fmul(g.gamma, vv);
    const float C1 = fmul(gv, fadd(adx, fmul(fmul(A1, be), g.dx)));              // :56
    const float D1 = fmul(gv, fadd(fmul(fmul(be, g.dx), B1), g.fod));            // :57
    const double Nd = (double)(float)g.nx;
    const float F = __double2float_rn(
        dsub(dmul(ddiv(dmul(ddiv(Nd, 2.0), Nd), 2.0), (double)fadd(fmul(A1, A1), 1.0f)), (double)fmul(B1, B1)));  // :59
    if (!(F >= 0.0f)) return false;                                              // :62
    const float E = fsqrt(F);
    const float den = fadd(1.0f, fmul(A1, A1));
    const float nab = fmul(-A1, B1);
    const float x_p1 = fdiv(fadd(nab, E), den);
    const float y_p1 = fadd(fmul(A1, x_p1), B1);
    const float z_p1 = fadd(fmul(C1, x_p1), D1);
    const float x_p2 = fdiv(fsub(nab, E), den);
    const float y_p2 = fadd(fmul(A1, x_p2), B1);
    const float z_p2 = fadd(fmul(C1, x_p2), D1);
    const float d1x = fsub(x_p1, x_s), d1y = fsub(y_p1, y_s);
    const float d2x = fsub(x_p2, x_s), d2y = fsub(y_p2, y_s);
    const float dist1 = fadd(fadd(fmul(d1x, d1x), fmul(d1y, d1y)), fmul(z_p1, z_p1));
    const float dist2 = fadd(fadd(fmul(d2x, d2x), fmul(d2y, d2y)), fmul(z_p2, z_p2));
    float x_f, y_f, z_f;
    if (dist1 <= dist2) {
        A = fadd(x_p1, g.xc); B = fadd(y_p1, g.yc); C = fadd(z_p1, g.zc);
        x_f = fadd(x_p2, g.xc); y_f = fadd(y_p2, g.yc); z_f = fadd(z_p2, g.zc);
    } else {
        A = fadd(x_p2, g.xc); B = fadd(y_p2, g.yc); C = fadd(z_p2, g.zc);
        x_f = fadd(x_p1, g.xc); y_f = fadd(y_p1, g.yc); z_f = fadd(z_p1, g.zc);
    }
    if (!(C < (float)g.nz && C >= 0.0f)) return false;                          // :100
    const float zmax = (float)(g.nz - 1);
    if (z_f > zmax) {                                                            // :102
        z_f = fsub(zmax, g.zc);
        x_f = fdiv(fsub(z_f, D1), C1); y_f = fadd(fmul(A1, x_f), B1);
        x_f = fadd(x_f, g.xc); y_f = fadd(y_f, g.yc); z_f = fadd(z_f, g.zc);
    } else if (z_f < 0.0f) {                                                     // :112
        z_f = -g.zc;
        x_f = fdiv(fsub(z_f, D1), C1); y_f = fadd(fmul(A1, x_f), B1);
        x_f = fadd(x_f, g.xc); y_f = fadd(y_f, g.yc); z_f = fadd(z_f, g.zc);
    }
    const float ex = fsub(A, x_f), ey = fsub(B, y_f), ez = fsub(C, z_f);
    const float len = fsqrt(fadd(fadd(fmul(ex, ex), fmul(ey, ey)), fmul(ez, ez)));  // :123
    r.n = rs_clamp_samples(g, len);
    r.A = A; r.B = B; r.C = C;
    return true;
}

// ---------------------------------------------------------------------------------
// Host launchers (defined in the .cu files).
// ---------------------------------------------------------------------------------
// (EPI_STORE writes odt; EPI_RESIDUAL writes FP32 and reads `real` in rdt.)
cudaError_t launch_rs_project(int mode, int epi, const DevGeom& g, const void* vpad, tomo_dtype vdt,
                              const OutView<void>& out, tomo_dtype odt, const OutView<void>& real, double* norm,
                              cudaStream_t st, tomo_dtype rdt = TOMO_F32);
// Layout-selecting form; the form above reads the PLAIN padded layout.
cudaError_t launch_rs_project(int layout, int mode, int epi, const DevGeom& g, const void* vin, unsigned long long tex,
                              tomo_dtype vdt, const OutView<void>& out, tomo_dtype odt, const OutView<void>& real,
                              double* norm, cudaStream_t st, tomo_dtype rdt = TOMO_F32);
// TEX layout resources: a layered array of the texels in the storage type (FP32, or the
// raw bits of BF16 / FP16), its texture object and (16-bit) a surface object for filling.
struct RsTexture {
    cudaArray_t arr = nullptr;
    unsigned long long tex = 0, surf = 0;
    tomo_dtype dt = TOMO_F32;
    int z0 = 0;  // layer of the first data slice: 1 for FP32 volume textures (zero layers around)
    bool zpairs = false;  // 16-bit volume texture: each 32-bit texel packs slices (L-2, L-1)
    bool march = false;   // the even faces of the MARCH layout (rs_march_tex_create)
};
// surface: also make a surface object (always for 16-bit textures, which are filled by
// conversion kernels).
cudaError_t rs_tex_create(int nx, int ny, int nz, tomo_dtype dt, RsTexture* t, bool surface = false);
// Volume texture of the RS projector, with a surface; every fill goes through a kernel.
// FP32: nz data layers between two zero layers (layer z + 1 holds slice z); 16-bit: nz + 3
// layers of 32-bit texels, layer L packing slices L - 2 (low half) and L - 1 (high half),
// zero outside the volume, so one gather returns the eight texels of a sample. Either way a
// sample's layers are valid for any z and off-volume footprints gather exact zeros, so the
// sampler needs no bounds tests. The zero layers are written on `st`: use the texture on
// `st` (or after it).
cudaError_t rs_vol_tex_create(int nx, int ny, int nz, tomo_dtype dt, RsTexture* t, cudaStream_t st);
// The even-face texture of the MARCH layout (FP32, with a surface; filled by rs_tex_fill).
cudaError_t rs_march_tex_create(int nx, int ny, int nz, RsTexture* t);
void rs_tex_destroy(RsTexture* t);
// amax (optional, 16-bit textures filled by conversion): FP16 range guard scale source.
cudaError_t rs_tex_fill(const void* vol, tomo_dtype vdt, int nx, int ny, int nz, const RsTexture& t, cudaStream_t st,
                        const unsigned* amax = nullptr);
void rs_tex_preload();
int rs_tex_max_layers();
// Elements of the RS input buffer for a layout, and the kernel that fills it from a volume.
size_t rs_input_elems(int layout, int nx, int ny, int nz);
cudaError_t launch_rs_prepare(int layout, const void* in, tomo_dtype idt, void* out, tomo_dtype odt, int nx, int ny,
                              int nz, cudaStream_t st, const unsigned* amax = nullptr);
cudaError_t launch_rs_adjoint(int mode, const DevGeom& g, const void* sino, tomo_dtype sdt, float* vol,
                              cudaStream_t st);
cudaError_t launch_rs_count(int mode, const DevGeom& g, unsigned long long* total, cudaStream_t st);
// Blocks of a projection launch (the EPI_NORM partials it writes).
size_t rs_grid_blocks(int layout, const DevGeom& g);
size_t siddon_grid_blocks(const DevGeom& g);
// *out = the sum of the n partials in a fixed order (one block), overwriting *out.
cudaError_t launch_sum_partials(const double* partials, size_t n, double* out, cudaStream_t st);

cudaError_t launch_siddon_project(int compat, int epi, const DevGeom& g, const void* vol, tomo_dtype vdt,
                                  const OutView<void>& out, tomo_dtype odt, const OutView<void>& real,
                                  double* norm, unsigned* err, cudaStream_t st, tomo_dtype rdt = TOMO_F32);
cudaError_t launch_siddon_adjoint(int compat, const DevGeom& g, const void* sino, tomo_dtype sdt, float* vol,
                                  unsigned* err, cudaStream_t st);
cudaError_t launch_siddon_count(int compat, const DevGeom& g, unsigned long long* total, unsigned* err,
                                cudaStream_t st);

// VI backprojection from a padded sinogram (nu+2 x nv+2 per view, zero border).
// scale multiplies the result after the reference's "* dx" (1 for --op=back, -2 inside
// the gradient loop, Iter3D_Algo_Gradient.cu:111).
cudaError_t launch_vi_back(int um, const DevGeom& g, const void* spad, tomo_dtype sdt, void* vol, tomo_dtype vdt,
                           float scale, cudaStream_t st, int zc = 1);
// Spatial taps of the ramp filter (fdk.cu); returns half, taps has 2 half entries.
int ramp_taps(int nu, int oversampling, double cutoff, double du, std::vector<float>& taps);
// FDK-weighted VI backprojection (FDK3D_VIB_kernel_v0_16reg) of a padded sinogram.
cudaError_t launch_vi_fdk(const DevGeom& g, const void* spad, tomo_dtype sdt, void* vol, tomo_dtype vdt, cudaStream_t st);
// Ramp filter of every detector row: out[p][v][i] = sum_l taps[l] in[p][v][i - (l - half)],
// in = 0 outside [0, nu), l in [0, 2 half); FP32 out.
cudaError_t launch_ramp_filter(const void* in, tomo_dtype idt, float* out, const float* taps, int half, int nu, int nv,
                               int np, cudaStream_t st);
// The same from a 2D layered texture of the sinogram (one layer per view, texels of type
// tdt: FP32 or raw 16-bit), e.g. an RsTexture made with (nu, nv, np) as its dimensions.
cudaError_t launch_vi_back_tex(int um, const DevGeom& g, unsigned long long tex, tomo_dtype tdt, void* vol,
                               tomo_dtype vdt, float scale, cudaStream_t st, int zc = 1);
// VI backprojection through detector windows staged in shared memory by TMA (vi_tma.cu), of
// an FP32 sinogram in the plain [P][nv][nu] layout: needs nu a multiple of 4 and a 16-byte
// aligned buffer (vi_tma_supported); bounded waits report ERR_TIMEOUT in *err.
bool vi_tma_supported(const DevGeom& g, const void* sino);
// stall (tests of the bounded waits only): the producer issues nothing, every consumer wait
// runs out after its one-second bound and ERR_TIMEOUT is set.
cudaError_t launch_vi_back_tma(int um, const DevGeom& g, const float* sino, void* vol, tomo_dtype vdt, float scale,
                               unsigned* err, cudaStream_t st, int stall = 0);
// Copies the interior of a zero-bordered padded FP32 sinogram ((nu+2) x (nv+2) per view)
// into an FP32 layered texture of (nu, nv, np) made with a surface.
cudaError_t tex_fill_from_padded(const float* spad, int nu, int nv, int np, const RsTexture& t, cudaStream_t st);

// Padding / conversion kernels. amax (optional): values are multiplied by the FP16 range
// guard's 2^-k before the conversion (fp16_scale).
cudaError_t launch_pad_volume(const void* in, tomo_dtype idt, void* out, tomo_dtype odt, int nx, int ny, int nz,
                              cudaStream_t st, const unsigned* amax = nullptr);
cudaError_t launch_pad_sinogram(const void* in, tomo_dtype idt, void* out, tomo_dtype odt, int nu, int nv, int np,
                                cudaStream_t st);
cudaError_t launch_convert(const void* in, tomo_dtype idt, void* out, tomo_dtype odt, size_t n, cudaStream_t st,
                           const unsigned* amax = nullptr);

// Regulariser / element-wise / reduction kernels (gd.cu).
cudaError_t launch_laplacian(const float* in, float* out, int nx, int ny, int nz, cudaStream_t st);
cudaError_t launch_sq_norm(const void* x, tomo_dtype dt, size_t n, double* out, cudaStream_t st);

}  // namespace tomo
