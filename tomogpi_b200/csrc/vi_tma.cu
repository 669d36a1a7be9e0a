// vi_tma.cu -- VI backprojector with each view's detector window staged in shared memory by
// the Tensor Memory Accelerator (TMA), single GPU.
//
// The block is the VI tile of vi_device.cuh (32 x 8 voxel columns, 16 slices per thread:
// eight consumer warps) plus one producer warp. For every view the producer bounds the
// detector window the tile's 4096 voxels can touch -- the projections of the tile's corner
// columns at its first and last slice; u and v are monotone in x, y and z over the tile, so
// the corners give the extremes -- and copies that box of the FP32 sinogram [P][nv][nu] into
// one of three shared-memory stages with one cp.async.bulk.tensor (into this CTA only; the tensor
// map covers this GPU's own buffer). Texels off the detector come back as zeros (the TMA's
// out-of-bounds fill), which is the texture border of the reference (a sample there adds 0,
// as skipping it does). mbarriers hand the stages over: `full` (the copy's bytes landed),
// `empty` (the 256 consumers are done with it). Consumers run the same arithmetic as
// vi_tile (backprojection3D_kernel_16reg.cuh:401-453: un, A, v by repeated addition, the
// three lerps, FP32 sums in view order) with the four texels of a sample read from shared
// memory; a thread whose footprint leaves the staged box for a view (a box too small for the
// tile at that view) reads that view's texels from global memory instead. Same texels, same
// operations, bit-identical to vi_tile.
//
// Every wait is bounded (one second by the global timer): a wait that gives up sets
// ERR_TIMEOUT in the context's error word and the block stops; the producer first waits
// (bounded) for the copies it issued.
#include <cuda.h>

#include <climits>
#include <mutex>

#include "vi_device.cuh"

namespace tomo {

// Box rows of 80 floats: a row pitch of 16 banks modulo 32, so a warp's footprints on two
// adjacent rows fall on different banks.
constexpr int VT_BOX_U = 80, VT_BOX_V = 40, VT_STAGES = 3;
constexpr int VT_CONSUMERS = VI_BX * VI_BY;  // 256
constexpr unsigned VT_BYTES = VT_BOX_U * VT_BOX_V * 4;
constexpr unsigned long long VT_WAIT_NS = 1000000000ull;  // bound of every wait: one second

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the phase of parity `parity` to complete; false once a second has passed (the
// clock is read every 256 polls; a poll may itself suspend the thread for a short while).
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity) {
    unsigned long long t0 = 0;
    for (unsigned i = 0;; ++i) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(b)), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255u) == 0) {
            const unsigned long long t = global_ns();
            if (i == 0) t0 = t;
            else if (t - t0 > VT_WAIT_NS) return false;
        }
    }
}
__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_addr(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
        : "memory");
}

// The detector box of view p for the tile (x0..x1, y0..y1, z0..z1): origin (u0, v0) with u0 a
// multiple of 4 (the copy's row starts on 16 bytes); false when the window exceeds the box.
__device__ __forceinline__ bool vt_window(const DevGeom& g, int p, int x0, int x1, int y0, int y1, int z0, int z1,
                                          int& u0, int& v0) {
    const float4 cv = __ldg(g.vi + p);
    float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
    const float zl = (float)z0 - g.zc, zh = (float)z1 - g.zc;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float xn = (float)((c & 1) ? x1 : x0) - g.xc, yn = (float)((c & 2) ? y1 : y0) - g.yc;
        const float w = cv.z * xn + cv.w * yn + g.fod;
        if (!(w > 0.f)) return false;
        const float a0 = 1.0f / w;
        const float ub = (cv.x * xn + cv.y * yn) * a0 + g.uc;  // un - 0.5
        const float A = a0 * g.inv_gamma_f;
        umin = fminf(umin, ub);
        umax = fmaxf(umax, ub);
        vmin = fminf(vmin, fminf(A * zl, A * zh) + g.vc);
        vmax = fmaxf(vmax, fmaxf(A * zl, A * zh) + g.vc);
    }
    // texels floor(.) and floor(.) + 1, one more on each side for the rounding of the bound
    const float ulo = floorf(umin) - 1.f, uhi = floorf(umax) + 2.f, vlo = floorf(vmin) - 1.f, vhi = floorf(vmax) + 2.f;
    if (!(ulo > -1.0e6f && uhi < 1.0e6f && vlo > -1.0e6f && vhi < 1.0e6f)) return false;
    u0 = (int)ulo;
    u0 -= ((u0 % 4) + 4) % 4;  // round down to a multiple of 4
    v0 = (int)vlo;
    return (int)uhi - u0 < VT_BOX_U && (int)vhi - v0 < VT_BOX_V;
}

template <int UM, typename Tv>
__global__ void __launch_bounds__(VT_CONSUMERS + 32, 4)
    vi_back_tma_kernel(DevGeom g, const __grid_constant__ CUtensorMap map, const float* __restrict__ sino,
                       Tv* __restrict__ vol, float scale, unsigned* err, int stall) {
    __shared__ __align__(128) float win[VT_STAGES][VT_BOX_V * VT_BOX_U];
    __shared__ __align__(8) unsigned long long full[VT_STAGES], empty[VT_STAGES];
    __shared__ int2 org[VT_STAGES];  // window origin of the stage; x = INT_MIN: not staged
    __shared__ int abort_flag;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * VI_BX, y0 = blockIdx.y * VI_BY, z0 = blockIdx.z * 16;
    if (tid == 0) {
        for (int s = 0; s < VT_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], VT_CONSUMERS);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (tid >= VT_CONSUMERS) {  // producer warp: one lane issues the copies
        if (tid == VT_CONSUMERS && !stall) {  // stall (tests only): no copy, so every wait runs out
            const int x1 = min(x0 + VI_BX, g.nx) - 1, y1 = min(y0 + VI_BY, g.ny) - 1, z1 = min(z0 + 16, g.nz) - 1;
            int issued = 0;
            for (int p = 0; p < g.np; ++p) {
                const int s = p % VT_STAGES, k = p / VT_STAGES;
                if (k > 0 && !mbar_wait(&empty[s], (k - 1) & 1)) {
                    atomicOr(err, ERR_TIMEOUT);
                    abort_flag = 1;
                    break;
                }
                int u0 = 0, v0 = 0;
                if (vt_window(g, p, x0, x1, y0, y1, z0, z1, u0, v0)) {
                    org[s] = make_int2(u0, v0);
                    mbar_arrive_tx(&full[s], VT_BYTES);
                    tma_load_3d(win[s], &map, u0, v0, p, &full[s]);
                } else {
                    org[s] = make_int2(INT_MIN, 0);
                    mbar_arrive(&full[s]);
                }
                issued = p + 1;
            }
            // the copies in flight land before the block may exit
            for (int p = max(0, issued - VT_STAGES); p < issued; ++p)
                if (!mbar_wait(&full[p % VT_STAGES], (p / VT_STAGES) & 1)) atomicOr(err, ERR_TIMEOUT);
        }
        return;
    }

    // a warp covers 8 x by 4 y columns (not 32 x 1): its footprints span about a third of the
    // detector columns a 32-wide row of voxels does, so its shared-memory reads need fewer
    // wavefronts
    const int lane = tid & 31, warp = tid >> 5;
    const int x = x0 + (warp & 3) * 8 + (lane & 7), y = y0 + (warp >> 2) * 4 + (lane >> 3);
    const bool live = x < g.nx && y < g.ny;
    const float xn = fsub((float)min(x, g.nx - 1), g.xc);
    const float yn = fsub((float)min(y, g.ny - 1), g.yc);
    const float fnu = (float)g.nu, fnv = (float)g.nv;
    const float2 MH = make_float2(-0.5f, -0.5f), K = make_float2(VI_FLOOR_K, VI_FLOOR_K);
    const float2 MK = make_float2(-VI_FLOOR_K, -VI_FLOOR_K), M1 = make_float2(-1.0f, -1.0f);
    const float zp = fsub((float)z0, g.zc);
    float2 acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = make_float2(0.f, 0.f);
    const long VP = (long)g.nu * g.nv;

    for (int p = 0; p < g.np; ++p) {
        const int s = p % VT_STAGES;
        if (!mbar_wait(&full[s], (p / VT_STAGES) & 1)) {
            atomicOr(err, ERR_TIMEOUT);
            break;
        }
        if (abort_flag) break;
        const int2 o = org[s];
        const float4 cv = __ldg(g.vi + p);
        float A = frcp(fadd(fadd(fmul(cv.z, xn), fmul(cv.w, yn)), g.fod));                 // :401
        const float up = fmul(fadd(fmul(cv.x, xn), fmul(cv.y, yn)), A);                  // u' (:403)
        const float un = fadd(fadd(up, g.uc), 0.5f);
        A = (p + g.p0 == 0) ? __double2float_rn(dmul(g.inv_gamma_d, (double)A))         // :404
                            : fmul(g.inv_gamma_f, A);                                   // :464
        const float ub = fsub(un, 0.5f);
        if (ub > -1.f && ub < fnu) {  // else the whole column footprint is border (adds zeros)
            const float fu = floorf(ub);
            const float a = ub - fu;
            const float2 aa = make_float2(a, a), na = make_float2(-a, -a);
            const int iu = (int)fu;
            float vn = fadd(fadd(fmul(A, zp), g.vc), 0.5f);                              // :405
            // rows floor(v - 0.5) of the first slice and an upper bound of the last one's (the
            // rows grow with k; 15 rounded additions of values below 8192 err by less than
            // 0.01 < A, as in vi_tile)
            const bool bounded = A > 0.25f && fnv <= 8192.f;
            const int vfirst = (int)floorf(fsub(vn, 0.5f));
            const int vlast = (int)floorf(fsub(fadd(vn, fmul(16.0f, A)), 0.5f));
            const bool staged = o.x != INT_MIN && bounded && iu - o.x >= 0 && iu + 1 - o.x < VT_BOX_U &&
                                vfirst - o.y >= 0 && vlast + 1 - o.y < VT_BOX_V;
            // the 16 slices in pairs; fetch(mx, my) returns the texel pairs (t00, t10, t01, t11)
            // of the two slices whose row floors + FLOOR_K have the bit patterns mx, my
            auto run = [&](auto fetch) {
#pragma unroll
                for (int k = 0; k < 16; k += 2) {
                    float2 vk;
                    if (UM) {
                        vk = __fadd2_rn(make_float2(vn, vn), make_float2(fmul((float)k, A), fmul((float)(k + 1), A)));
                    } else {
                        vk.x = vn;
                        vn = fadd(vn, A);
                        vk.y = vn;
                        vn = fadd(vn, A);
                    }
                    const float2 vb = __fadd2_rn(vk, MH);
                    const float2 m = __fadd2_rd(vb, K);
                    const float2 f = __fadd2_rn(m, MK);
                    const float2 b = __ffma2_rn(f, M1, vb), nb = __ffma2_rn(vb, M1, f);
                    float2 t00, t10, t01, t11;
                    fetch((unsigned)__float_as_int(m.x), (unsigned)__float_as_int(m.y), t00, t10, t01, t11);
                    const float2 s0 = __ffma2_rn(aa, t10, __ffma2_rn(na, t00, t00));
                    const float2 s1 = __ffma2_rn(aa, t11, __ffma2_rn(na, t01, t01));
                    const float2 t = __ffma2_rn(b, s1, __ffma2_rn(nb, s0, s0));
                    acc[k >> 1] = __fadd2_rn(acc[k >> 1], t);
                }
            };
            if (staged) {
                // shared-memory word of (row floor(v), column iu): rb + bits(floor + K) * box row,
                // modulo 2^32 (the bias and the window origin folded into rb)
                const unsigned rb = (unsigned)(s * (VT_BOX_V * VT_BOX_U) + (iu - o.x)) -
                                    (unsigned)(VI_FLOOR_KBITS + o.y) * (unsigned)VT_BOX_U;
                const float* wf = &win[0][0];
                run([&](unsigned mx, unsigned my, float2& t00, float2& t10, float2& t01, float2& t11) {
                    const unsigned i0 = rb + mx * (unsigned)VT_BOX_U, i1 = rb + my * (unsigned)VT_BOX_U;
                    t00 = make_float2(wf[i0], wf[i1]);
                    t10 = make_float2(wf[i0 + 1], wf[i1 + 1]);
                    t01 = make_float2(wf[i0 + VT_BOX_U], wf[i1 + VT_BOX_U]);
                    t11 = make_float2(wf[i0 + VT_BOX_U + 1], wf[i1 + VT_BOX_U + 1]);
                });
            } else {  // from global memory, zero off the detector
                const float* sg = sino + p * VP + iu;  // column iu of view p
                const bool c0 = iu >= 0, c1 = iu + 1 < g.nu;
                run([&](unsigned mx, unsigned my, float2& t00, float2& t10, float2& t01, float2& t11) {
                    const int r0 = (int)mx - VI_FLOOR_KBITS, r1 = (int)my - VI_FLOOR_KBITS;
                    const bool a0r = r0 >= 0 && r0 < g.nv, a1r = r0 + 1 >= 0 && r0 + 1 < g.nv;
                    const bool b0r = r1 >= 0 && r1 < g.nv, b1r = r1 + 1 >= 0 && r1 + 1 < g.nv;
                    const float* q0 = sg + (long)r0 * g.nu;
                    const float* q1 = sg + (long)r1 * g.nu;
                    t00 = make_float2(c0 && a0r ? __ldg(q0) : 0.f, c0 && b0r ? __ldg(q1) : 0.f);
                    t10 = make_float2(c1 && a0r ? __ldg(q0 + 1) : 0.f, c1 && b0r ? __ldg(q1 + 1) : 0.f);
                    t01 = make_float2(c0 && a1r ? __ldg(q0 + g.nu) : 0.f, c0 && b1r ? __ldg(q1 + g.nu) : 0.f);
                    t11 = make_float2(c1 && a1r ? __ldg(q0 + g.nu + 1) : 0.f, c1 && b1r ? __ldg(q1 + g.nu + 1) : 0.f);
                });
            }
        }
        mbar_arrive(&empty[s]);
    }
    if (!live) return;
    const long plane = (long)g.nx * g.ny;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int z = z0 + k;
        const float r = (k & 1) ? acc[k >> 1].y : acc[k >> 1].x;
        if (z < g.nz) vol[z * plane + (long)y * g.nx + x] = cvt<Tv>(fmul(fmul(r, g.dx), scale));
    }
}

// ---------------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------------
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
        cudaGetLastError();
    });
    return fn;
}

template <int UM, typename Tv>
cudaError_t launch_tma_t(const DevGeom& g, const CUtensorMap& map, const float* sino, void* vol, float scale,
                         unsigned* err, cudaStream_t st, int stall) {
    dim3 block(VT_CONSUMERS + 32), grid((g.nx + VI_BX - 1) / VI_BX, (g.ny + VI_BY - 1) / VI_BY, (g.nz + 15) / 16);
    vi_back_tma_kernel<UM, Tv><<<grid, block, 0, st>>>(g, map, sino, (Tv*)vol, scale, err, stall);
    return cudaGetLastError();
}

}  // namespace

bool vi_tma_supported(const DevGeom& g, const void* sino) {
    return encode_fn() != nullptr && g.nu % 4 == 0 && ((uintptr_t)sino & 15) == 0 && g.nu >= 4 && g.nv >= 1;
}

// VI backprojection of an FP32 sinogram [P][nv][nu] (plain layout, nu a multiple of 4,
// 16-byte aligned) through TMA-staged windows; 16 slices per thread.
cudaError_t launch_vi_back_tma(int um, const DevGeom& g, const float* sino, void* vol, tomo_dtype vdt, float scale,
                               unsigned* err, cudaStream_t st, int stall) {
    if (!vi_tma_supported(g, sino)) return cudaErrorNotSupported;
    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t)g.nu, (cuuint64_t)g.nv, (cuuint64_t)g.np};
    const cuuint64_t strides[2] = {(cuuint64_t)g.nu * 4, (cuuint64_t)g.nu * g.nv * 4};
    const cuuint32_t box[3] = {VT_BOX_U, VT_BOX_V, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(sino), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    switch (vdt) {
        case TOMO_F32: return um ? launch_tma_t<1, float>(g, map, sino, vol, scale, err, st, stall)
                                 : launch_tma_t<0, float>(g, map, sino, vol, scale, err, st, stall);
        case TOMO_BF16: return um ? launch_tma_t<1, __nv_bfloat16>(g, map, sino, vol, scale, err, st, stall)
                                  : launch_tma_t<0, __nv_bfloat16>(g, map, sino, vol, scale, err, st, stall);
        case TOMO_F16: return um ? launch_tma_t<1, __half>(g, map, sino, vol, scale, err, st, stall)
                                 : launch_tma_t<0, __half>(g, map, sino, vol, scale, err, st, stall);
    }
    return cudaErrorInvalidValue;
}

}  // namespace tomo
