// gd.cu -- the element-wise, stencil and reduction kernels of the simple gradient loop
// (Iter3D::doSimpleGradient, src/TomoGPI_lib/src/CPP/Iter3D_Algo_Gradient.cu:25-223) and
// the phantom rasteriser.
//
// The regulariser gradient is the generalised-Gaussian criterion
// (GeneralizedGaussianRegularizer_CPU.cu:158-225, GeneralizedGaussianRegularizer_GPU.cu:
// 161-225): L = sum of the three 1-D {-1, 2, -1} convolutions with zero padding,
// dJ += beta*lambda * L(grad) with grad = L f for beta = 2 and grad = sign(f) |f|^(beta-1)
// otherwise (the reference applies the power to the volume, not to its Laplacian), and for
// the optimal step normdJProjReg = beta * sum |L dJ|^beta (2 ||L dJ||^2 for beta = 2). The
// stencil evaluates each axis as the reference's separable kernels do (tmp = 0;
// tmp += s[-1]*k2; tmp += s[0]*k1; tmp += s[+1]*k0, then h + v + p), in exactly rounded
// FP32. Passes are fused where a pass would only re-read what the previous one wrote:
//   laplacian_kernel        grad = L f
//   gg_abspow_kernel        grad = sign(f) |f|^(beta-1)            (beta != 2)
//   laplacian_axpy_kernel   dJ   = dJ + w * L(grad)
//   laplacian_norm_kernel   nrm[0] += ||dJ||^2, nrm[2] += sum |L dJ|^beta (nothing stored)
// and for the weighted gradient (Iter3D::doWeightedGradient, Iter3D_Algo_Gradient.cu:
// 227-373) sino_weight_kernel multiplies the residual by the weight sinogram (:289).
// and for the Huber regulariser (HuberRegularizer_CPU.cu:206-253), grad = L f being stored:
//   huber_axpy_kernel       dJ   = dJ + lambda * L(psi'(grad))
//   huber_t_kernel          t    = L(psi''(grad) * dJ)
//   huber_l1_kernel         nrm[4] += sum |L(t) * dJ|
// All norms accumulate in FP64 (as Image3D_CPU::getImageL2Norm and
// Sinogram3D_CPU::getSinogramL2Norm do).
#include <algorithm>

#include "tomo_kernels.cuh"
#include "tomo_solver.cuh"

namespace tomo {

__device__ __forceinline__ void block_reduce_add(double s, double* out) {
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = t & 31, warp = t >> 5, nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (warp == 0) {
        s = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0 && s != 0.0) atomicAdd(out, s);
    }
    __syncthreads();
}

// The block's sum stored at part[linear block] when part is given (summed later in a fixed
// order by launch_sum_partials, so the total is the same on every run), else added to *out.
__device__ __forceinline__ void block_reduce_to(double s, double* out, double* part) {
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = t & 31, warp = t >> 5, nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (warp == 0) {
        s = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) {
            if (part) part[linear_block()] = s;
            else if (s != 0.0) atomicAdd(out, s);
        }
    }
    __syncthreads();
}

// Largest of the block's values (FP32 bits of non-negative floats), one atomicMax per block.
__device__ __forceinline__ void block_reduce_max(unsigned m, unsigned* out) {
    __shared__ unsigned red[32];
    m = __reduce_max_sync(0xffffffffu, m);
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = t & 31, warp = t >> 5, nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (lane == 0) red[warp] = m;
    __syncthreads();
    if (warp == 0) {
        m = __reduce_max_sync(0xffffffffu, lane < nw ? red[lane] : 0u);
        if (lane == 0 && m) atomicMax(out, m);
    }
    __syncthreads();
}

// Block (32, 8): x fastest for coalescing; z from the grid.
__global__ void laplacian_kernel(const float* __restrict__ in, float* __restrict__ out, int nx, int ny, int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    out[z * (long)nx * ny + (long)y * nx + x] = lap_at(in, x, y, z, nx, ny, nz);
}

__global__ void laplacian_axpy_kernel(const float* __restrict__ in, float* __restrict__ dj, float w, int nx, int ny,
                                      int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const long i = z * (long)nx * ny + (long)y * nx + x;
    dj[i] = fadd(dj[i], fmul(w, lap_at(in, x, y, z, nx, ny, nz)));   // Image3D_CPU::addImage
}

// |x|^p in FP64 as Image3D_CPU::getImageLpNorm / getImageAbsPow take it (Image3D_CPU.cu:409, :564).
__device__ __forceinline__ double abs_pow(double x, double p) { return p == 2.0 ? x * x : pow(fabs(x), p); }

// The reductions run their blocks over z (grid-stride, reduce_grid), so that each block
// sums many voxels before its one atomic per sum.
__global__ void laplacian_norm_kernel(const float* __restrict__ dj, double* __restrict__ nrm, int nx, int ny, int nz,
                                      int want_lap, double beta, unsigned* amax, double* part) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    double s0 = 0.0, s2 = 0.0;
    unsigned m = 0;
    if (x < nx && y < ny) {
        for (int z = blockIdx.z; z < nz; z += gridDim.z) {
            const float df = dj[z * (long)nx * ny + (long)y * nx + x];
            m = max(m, __float_as_uint(fabsf(df)));
            const double d = (double)df;
            s0 += d * d;
            if (want_lap) s2 += abs_pow((double)lap_at(dj, x, y, z, nx, ny, nz), beta);
        }
    }
    const long nb = (long)gridDim.x * gridDim.y * gridDim.z;
    block_reduce_to(s0, nrm + 0, part);
    if (want_lap) block_reduce_to(s2, nrm + 2, part ? part + nb : nullptr);
    if (amax) block_reduce_max(m, amax);
}

// grad = sign(f) * (float)|f|^p with p = beta - 1: Image3D::getImageSign, getImageAbsPow and
// multImage in the order GeneralizedGaussianRegularizer_CPU.cu:191-197 calls them (sign of
// +x, -x, 0 as +1, -1, 0: Image3D_GPU_kernel.cuh:10; the power in FP64 rounded to FP32, as
// Image3D_CPU.cu:564 writes it; the FP32 pow of Image3D_GPU_kernel.cuh:699 differs from it
// by FP32 rounding only).
__global__ void gg_abspow_kernel(const float* __restrict__ f, float* __restrict__ out, size_t n, double p) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float x = f[i];
        const float sg = x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f);
        out[i] = fmul(__double2float_rn(pow(fabs((double)x), p)), sg);
    }
}

// sum |x|^p in FP64 (Image3D_CPU::getImageLpNorm, Image3D_CPU.cu:396-412)
__global__ void lp_norm_kernel(const float* __restrict__ x, size_t n, double p, double* __restrict__ out) {
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s += abs_pow((double)x[i], p);
    block_reduce_add(s, out);
}

// r = r * w over a residual view (Sinogram3D::multSinogram, Sinogram3D_GPU_kernel.cuh:118-127),
// w a plain [p][v][u] FP32 sinogram. Block (32, 8): u fastest; v from y, the view from z.
__global__ void sino_weight_kernel(OutView<float> r, const float* __restrict__ w, int nu, int nv) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y * blockDim.y + threadIdx.y, p = blockIdx.z;
    if (u >= nu || v >= nv) return;
    const long i = r.at(p, v, u);
    r.ptr[i] = fmul(r.ptr[i], w[((long)p * nv + v) * nu + u]);
}

// ---- Huber regulariser (HuberRegularizer_CPU.cu:206-253) ----
// psi'(g): -2 thr for g <= -thr, 2 g for |g| < thr, 2 thr for g >= thr (NaN passes through);
// psi''(g): 0 for |g| > thr, 1 for |g| <= thr (:24-96). Comparisons in double against the
// double threshold, as the reference compares its float value with it.
__device__ __forceinline__ float huber_d1(float v, double thr) {
    const double d = (double)v;
    if (d <= -1.0 * thr) return __double2float_rn(-2.0 * thr);
    if (fabs(d) < thr) return __double2float_rn(2.0 * d);
    if (d >= thr) return __double2float_rn(2.0 * thr);
    return v;
}
__device__ __forceinline__ float huber_d2(float v, double thr) {
    const double a = fabs((double)v);
    if (a > thr) return 0.f;
    if (a <= thr) return 1.f;
    return v;
}

// The {-1, 2, -1} stencil of lap_at over values produced by `load(linear index)`; outside
// the volume the input is 0 (the convolution's zero padding applies to the loaded volume).
template <class F>
__device__ __forceinline__ float lap_of(F load, int x, int y, int z, int nx, int ny, int nz) {
    const long plane = (long)nx * ny;
    const long i = z * plane + (long)y * nx + x;
    const float c = load(i);
    const float xm = x > 0 ? load(i - 1) : 0.f, xp = x < nx - 1 ? load(i + 1) : 0.f;
    const float ym = y > 0 ? load(i - nx) : 0.f, yp = y < ny - 1 ? load(i + nx) : 0.f;
    const float zm = z > 0 ? load(i - plane) : 0.f, zp = z < nz - 1 ? load(i + plane) : 0.f;
    const float c2 = fmul(c, 2.0f);
    const float h = fadd(fadd(fmul(xm, -1.0f), c2), fmul(xp, -1.0f));
    const float v = fadd(fadd(fmul(ym, -1.0f), c2), fmul(yp, -1.0f));
    const float p = fadd(fadd(fmul(zm, -1.0f), c2), fmul(zp, -1.0f));
    return fadd(fadd(h, v), p);
}

// dJ = dJ + w * L(psi'(grad))   (:218-228; w = the float lambda)
__global__ void huber_axpy_kernel(const float* __restrict__ grad, float* __restrict__ dj, float w, double thr, int nx,
                                  int ny, int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const long i = z * (long)nx * ny + (long)y * nx + x;
    const float l = lap_of([&](long k) { return huber_d1(grad[k], thr); }, x, y, z, nx, ny, nz);
    dj[i] = fadd(dj[i], fmul(w, l));
}

// t = L(psi''(grad) * dJ)   (:233-236)
__global__ void huber_t_kernel(const float* __restrict__ grad, const float* __restrict__ dj, float* __restrict__ t,
                               double thr, int nx, int ny, int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    t[z * (long)nx * ny + (long)y * nx + x] =
        lap_of([&](long k) { return fmul(huber_d2(grad[k], thr), dj[k]); }, x, y, z, nx, ny, nz);
}

// *out += sum |L(t) * dJ| in FP64   (:237-239, Image3D_CPU::getImageL1Norm)
__global__ void huber_l1_kernel(const float* __restrict__ t, const float* __restrict__ dj, double* __restrict__ out,
                                int nx, int ny, int nz, double* part) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    double s = 0.0;
    if (x < nx && y < ny) {
        for (int z = blockIdx.z; z < nz; z += gridDim.z) {
            const long i = z * (long)nx * ny + (long)y * nx + x;
            s += fabs((double)fmul(lap_at(t, x, y, z, nx, ny, nz), dj[i]));
        }
    }
    block_reduce_to(s, out, part);
}

// Image3D_CPU::getImageHuberNorm (Image3D_CPU.cu:415-440): sum of g^2 inside the threshold,
// 2 thr |g| - thr^2 outside, in double.
__global__ void huber_jreg_kernel(const float* __restrict__ g, size_t n, double thr, double* __restrict__ out) {
    double s = 0.0;
    const double t2 = thr * thr;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = (double)g[i];
        if (fabs(v) < thr) s += v * v;
        else if (fabs(v) >= thr) s += 2.0 * thr * fabs(v) - t2;
        else s += v;
    }
    block_reduce_add(s, out);
}

template <typename T>
__global__ void sq_norm_kernel(const T* __restrict__ x, size_t n, double* __restrict__ out) {
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double d = (double)ldp(x + i);
        s += d * d;
    }
    block_reduce_add(s, out);
}

// Sum of a projection's per-block norm partials in a fixed order: thread t adds partials
// t, t + 1024, ... in turn, then a fixed tree over the 1024 thread sums.
__global__ void __launch_bounds__(1024) sum_partials_kernel(const double* __restrict__ p, size_t n,
                                                            double* __restrict__ out) {
    __shared__ double red[1024];
    double s = 0.0;
    for (size_t i = threadIdx.x; i < n; i += 1024) s += p[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// Step size (Iter3D_Algo_Gradient.cu:133-158). state: [0] alpha, [1] alpha_min.
// nrm: [0] ||dJ||^2, [1] ||H dJ||^2, [2] sum |L dJ|^beta, [4] the Huber normdJProjReg.
// reg: 0 none, 1 GG (normdJProjReg = beta sum |L dJ|^beta), 2 Huber (normdJProjReg = nrm[4]).
__global__ void gd_alpha_kernel(const double* __restrict__ nrm, double* __restrict__ state, double* __restrict__ log,
                                int it, int optimal_step_nb, double lambda, int reg, double beta, const unsigned* amax) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double alpha;
    if (it < optimal_step_nb) {
        const double normdJProjReg = reg == 1 ? beta * nrm[2] : (reg == 2 ? nrm[4] : 0.0);  // GG..._CPU.cu:210-218
        const double normdJ = nrm[0];                                              // :145
        const double hdj = nrm[1] * fp16_unscale_sq(amax);                          // FP16-stored dJ was scaled
        const double normdJProj = 2.0 * hdj + lambda * normdJProjReg;              // :146
        alpha = -1.0 * normdJ / normdJProj;                                        // :150
        state[1] = fmax(alpha, state[1]);                                          // :151
    } else {
        alpha = state[1];                                                          // :156
    }
    state[0] = alpha;
    if (log) log[it - 1] = alpha;
}

// f = f + (float)alpha * dJ, optional positivity (Projector::updateVolume, Projector.cu:110-124).
__global__ void gd_update_kernel(float* __restrict__ f, const float* __restrict__ dj, const double* __restrict__ state,
                                 size_t n, int positivity) {
    const float a = __double2float_rn(state[0]);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v = fadd(f[i], fmul(a, dj[i]));
        if (positivity && v < 0.f) v = 0.f;
        f[i] = v;
    }
}

// normdJProjReg = beta sum |L dJ|^beta (GeneralizedGaussianRegularizer_CPU.cu:210-218)
__global__ void gg_finish_kernel(const double* __restrict__ nrm, double beta, double* __restrict__ out) {
    if (threadIdx.x == 0) out[1] = beta * nrm[2];
}

__global__ void fill_double_kernel(double* p, int n, double v) {
    const int i = threadIdx.x;
    if (i < n) p[i] = v;
}

// phantom3d.m:72-116: value = sum of A over the ellipsoids containing the voxel centre,
// coordinates on [-1, 1] per axis, rotated by the host-computed Euler matrix.
struct PhantomEll {
    double A, asq, bsq, csq, x0, y0, z0, m[9];
};

__global__ void phantom_kernel(const PhantomEll* __restrict__ ell, int count, int nx, int ny, int nz,
                               float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const double hx = (nx - 1) / 2.0, hy = (ny - 1) / 2.0, hz = (nz - 1) / 2.0;
    const double cx = ddiv(dsub((double)x, hx), hx), cy = ddiv(dsub((double)y, hy), hy), cz = ddiv(dsub((double)z, hz), hz);
    float acc = 0.f;
    for (int e = 0; e < count; ++e) {
        const PhantomEll E = ell[e];
        const double xp = dadd(dadd(dmul(E.m[0], cx), dmul(E.m[1], cy)), dmul(E.m[2], cz));
        const double yp = dadd(dadd(dmul(E.m[3], cx), dmul(E.m[4], cy)), dmul(E.m[5], cz));
        const double zp = dadd(dadd(dmul(E.m[6], cx), dmul(E.m[7], cy)), dmul(E.m[8], cz));
        const double ex = dsub(xp, E.x0), ey = dsub(yp, E.y0), ez = dsub(zp, E.z0);
        const double q = dadd(dadd(ddiv(dmul(ex, ex), E.asq), ddiv(dmul(ey, ey), E.bsq)), ddiv(dmul(ez, ez), E.csq));
        if (q <= 1.0) acc = fadd(acc, (float)E.A);
    }
    out[z * (long)nx * ny + (long)y * nx + x] = acc;
}

// ---------------------------------------------------------------------------------
static dim3 vol_grid(int nx, int ny, int nz) { return dim3((nx + 31) / 32, (ny + 7) / 8, nz); }
// Reductions: about 148 x 8 blocks of 32 x 8 threads, each looping over z.
static dim3 reduce_grid(int nx, int ny, int nz) {
    const int gx = (nx + 31) / 32, gy = (ny + 7) / 8;
    const int gz = std::max(1, std::min(nz, (148 * 8 + gx * gy - 1) / (gx * gy)));
    return dim3(gx, gy, gz);
}

cudaError_t launch_laplacian(const float* in, float* out, int nx, int ny, int nz, cudaStream_t st) {
    laplacian_kernel<<<vol_grid(nx, ny, nz), dim3(32, 8), 0, st>>>(in, out, nx, ny, nz);
    return cudaGetLastError();
}

cudaError_t launch_laplacian_axpy(const float* in, float* dj, float w, int nx, int ny, int nz, cudaStream_t st) {
    laplacian_axpy_kernel<<<vol_grid(nx, ny, nz), dim3(32, 8), 0, st>>>(in, dj, w, nx, ny, nz);
    return cudaGetLastError();
}

size_t reduce_blocks(int nx, int ny, int nz) {
    const dim3 d = reduce_grid(nx, ny, nz);
    return (size_t)d.x * d.y * d.z;
}

cudaError_t launch_laplacian_norm(const float* dj, double* nrm, int nx, int ny, int nz, int want_lap, cudaStream_t st,
                                  unsigned* amax, double beta, double* part) {
    laplacian_norm_kernel<<<reduce_grid(nx, ny, nz), dim3(32, 8), 0, st>>>(dj, nrm, nx, ny, nz, want_lap, beta, amax,
                                                                         part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !part) return e;
    const size_t nb = reduce_blocks(nx, ny, nz);
    if ((e = launch_sum_partials(part, nb, nrm + 0, st)) != cudaSuccess || !want_lap) return e;
    return launch_sum_partials(part + nb, nb, nrm + 2, st);
}

static int flat_blocks(size_t n, long cap) {
    long b = (long)((n + 255) / 256);
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

cudaError_t launch_gg_abspow(const float* f, float* out, size_t n, double p, cudaStream_t st) {
    gg_abspow_kernel<<<flat_blocks(n, 148L * 16), 256, 0, st>>>(f, out, n, p);
    return cudaGetLastError();
}

cudaError_t launch_lp_norm(const float* x, size_t n, double p, double* out, cudaStream_t st) {
    lp_norm_kernel<<<flat_blocks(n, 148L * 8), 256, 0, st>>>(x, n, p, out);
    return cudaGetLastError();
}

// r = real - r over a residual view holding a projection (EPI_RESIDUAL's arithmetic,
// Sinogram3D_CPU::diffSinogram, in a separate pass); real plain [p][v][u] in its dtype.
template <typename Tr>
__global__ void sino_residual_kernel(OutView<float> r, const Tr* __restrict__ real, int nu, int nv) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y * blockDim.y + threadIdx.y, p = blockIdx.z;
    if (u >= nu || v >= nv) return;
    const long i = r.at(p, v, u);
    r.ptr[i] = fsub(ldp(real + ((long)p * nv + v) * nu + u), r.ptr[i]);
}

cudaError_t launch_sino_residual(OutView<float> r, const void* real, tomo_dtype rdt, int nu, int nv, int np,
                                 cudaStream_t st) {
    const dim3 grid((nu + 31) / 32, (nv + 7) / 8, np), block(32, 8);
    switch (rdt) {
        case TOMO_F32: sino_residual_kernel<float><<<grid, block, 0, st>>>(r, (const float*)real, nu, nv); break;
        case TOMO_BF16:
            sino_residual_kernel<__nv_bfloat16><<<grid, block, 0, st>>>(r, (const __nv_bfloat16*)real, nu, nv);
            break;
        case TOMO_F16: sino_residual_kernel<__half><<<grid, block, 0, st>>>(r, (const __half*)real, nu, nv); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_sino_weight(OutView<float> r, const float* w, int nu, int nv, int np, cudaStream_t st) {
    sino_weight_kernel<<<dim3((nu + 31) / 32, (nv + 7) / 8, np), dim3(32, 8), 0, st>>>(r, w, nu, nv);
    return cudaGetLastError();
}

cudaError_t launch_huber_axpy(const float* grad, float* dj, float w, double thr, int nx, int ny, int nz,
                              cudaStream_t st) {
    huber_axpy_kernel<<<vol_grid(nx, ny, nz), dim3(32, 8), 0, st>>>(grad, dj, w, thr, nx, ny, nz);
    return cudaGetLastError();
}

cudaError_t launch_huber_norm(const float* grad, const float* dj, float* t, double thr, double* out, int nx, int ny,
                              int nz, cudaStream_t st, double* part) {
    huber_t_kernel<<<vol_grid(nx, ny, nz), dim3(32, 8), 0, st>>>(grad, dj, t, thr, nx, ny, nz);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    huber_l1_kernel<<<reduce_grid(nx, ny, nz), dim3(32, 8), 0, st>>>(t, dj, out, nx, ny, nz, part);
    e = cudaGetLastError();
    if (e != cudaSuccess || !part) return e;
    return launch_sum_partials(part, reduce_blocks(nx, ny, nz), out, st);
}

cudaError_t launch_huber_jreg(const float* g, size_t n, double thr, double* out, cudaStream_t st) {
    long b = (long)((n + 255) / 256);
    if (b > 148L * 8) b = 148L * 8;
    huber_jreg_kernel<<<(int)(b < 1 ? 1 : b), 256, 0, st>>>(g, n, thr, out);
    return cudaGetLastError();
}

cudaError_t launch_sq_norm(const void* x, tomo_dtype dt, size_t n, double* out, cudaStream_t st) {
    long b = (long)((n + 255) / 256);
    if (b > 148L * 8) b = 148L * 8;
    if (b < 1) b = 1;
    switch (dt) {
        case TOMO_F32: sq_norm_kernel<float><<<(int)b, 256, 0, st>>>((const float*)x, n, out); break;
        case TOMO_BF16: sq_norm_kernel<__nv_bfloat16><<<(int)b, 256, 0, st>>>((const __nv_bfloat16*)x, n, out); break;
        case TOMO_F16: sq_norm_kernel<__half><<<(int)b, 256, 0, st>>>((const __half*)x, n, out); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_gd_alpha(const double* nrm, double* state, double* log, int it, int optimal_step_nb, double lambda,
                            int reg, cudaStream_t st, const unsigned* amax, double beta) {
    gd_alpha_kernel<<<1, 32, 0, st>>>(nrm, state, log, it, optimal_step_nb, lambda, reg, beta, amax);
    return cudaGetLastError();
}

cudaError_t launch_gd_update(float* f, const float* dj, const double* state, size_t n, int positivity,
                             cudaStream_t st) {
    long b = (long)((n + 255) / 256);
    if (b > 148L * 16) b = 148L * 16;
    gd_update_kernel<<<(int)(b < 1 ? 1 : b), 256, 0, st>>>(f, dj, state, n, positivity);
    return cudaGetLastError();
}

cudaError_t launch_sum_partials(const double* partials, size_t n, double* out, cudaStream_t st) {
    sum_partials_kernel<<<1, 1024, 0, st>>>(partials, n, out);
    return cudaGetLastError();
}

cudaError_t launch_gg_finish(const double* nrm, double* out, cudaStream_t st, double beta) {
    gg_finish_kernel<<<1, 32, 0, st>>>(nrm, beta, out);
    return cudaGetLastError();
}

cudaError_t launch_fill_double(double* p, int n, double v, cudaStream_t st) {
    fill_double_kernel<<<1, 32, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

cudaError_t launch_phantom(const double* ell_host, int count, int nx, int ny, int nz, float* out, void** scratch,
                           cudaStream_t st) {
    // Host: Euler rotation matrices as in phantom3d.m:94-109.
    PhantomEll* h = new PhantomEll[count > 0 ? count : 1];
    for (int e = 0; e < count; ++e) {
        const double* E = ell_host + 10 * e;
        const double ph = E[7] * M_PI / 180.0, th = E[8] * M_PI / 180.0, ps = E[9] * M_PI / 180.0;
        const double cphi = cos(ph), sphi = sin(ph), cth = cos(th), sth = sin(th), cpsi = cos(ps), spsi = sin(ps);
        const double m[9] = {cpsi * cphi - cth * sphi * spsi, cpsi * sphi + cth * cphi * spsi, spsi * sth,
                             -spsi * cphi - cth * sphi * cpsi, -spsi * sphi + cth * cphi * cpsi, cpsi * sth,
                             sth * sphi, -sth * cphi, cth};
        h[e].A = E[0];
        h[e].asq = E[1] * E[1];
        h[e].bsq = E[2] * E[2];
        h[e].csq = E[3] * E[3];
        h[e].x0 = E[4];
        h[e].y0 = E[5];
        h[e].z0 = E[6];
        for (int k = 0; k < 9; ++k) h[e].m[k] = m[k];
    }
    const size_t bytes = sizeof(PhantomEll) * (count > 0 ? count : 1);
    cudaError_t e = cudaMalloc(scratch, bytes);
    if (e != cudaSuccess) {
        delete[] h;
        return e;
    }
    e = cudaMemcpyAsync(*scratch, h, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    delete[] h;
    if (e != cudaSuccess) return e;
    phantom_kernel<<<vol_grid(nx, ny, nz), dim3(32, 8), 0, st>>>((const PhantomEll*)*scratch, count, nx, ny, nz, out);
    return cudaGetLastError();
}

}  // namespace tomo
