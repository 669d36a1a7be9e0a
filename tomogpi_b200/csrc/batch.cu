// batch.cu -- many reconstructions of uneven size advanced together: every phase of a
// gradient iteration is ONE launch over all live jobs.
//
// Projection and backprojection run as persistent kernels (one wave of CTAs, sized by the
// occupancy calculator) that pop work items from a device queue, one launch per group of
// jobs sharing an RS input layout (projection) or a z-chunking (backprojection), so each
// launch is specialised and keeps its register budget small:
//   projection      item = (job, view, u-tile, v-tile)   -- a 16 x 16 ray tile of one view
//   backprojection  item = (job, x-tile, y-tile, z-group) -- 32 x 8 columns x 16*ZC slices
// Items are ordered longest-first (estimated cost) so that the dynamic queue balances
// jobs of different sizes. The element-wise and stencil phases (RS input preparation,
// Laplacians, norms, update) are one ordinary launch each with one CTA per (job, z-slice).
//
// Determinism: every norm is accumulated as per-item partial sums stored by item index and
// reduced in a fixed order per job, and every item computes only its own job's outputs;
// so a job's iterates are bit-identical whether it runs alone or in any mix of jobs.
//
// Each job carries its own iteration counter on the device; a job whose counter passed its
// iteration count is skipped by every phase. So one iteration of the whole batch is a fixed
// sequence of launches, captured once as a CUDA graph and replayed.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <mutex>
#include <numeric>
#include <vector>

#include "rs_device.cuh"
#include "tomo_solver.cuh"
#include "vi_device.cuh"

namespace tomo {

struct BatchJob {  // device descriptor of one job
    DevGeom g;
    int layout;               // RS input layout of this job
    int zc;                   // VI slices per thread / 16 (1 or 2)
    void* rs_in;              // PLAIN / CELL8 buffer (storage dtype)
    unsigned long long tex;   // TEX layout texture object
    float* resid;             // padded residual sinogram (FP32 whatever the storage)
    const void* real;         // real sinogram (storage dtype, or FP32 when real_f32; dense)
    int real_f32;
    float* vol;               // FP32 iterate (owned by the caller)
    float* dJ;
    float* grad;
    double* part_proj;        // [P * UT * VT] partials of ||H dJ||^2
    double* part_lap;         // [2 * nz] partials of ||dJ||^2 and ||L dJ||^2
    int* iter;                // next iteration (1-based)
    unsigned* amax;           // FP16 storage: FP32 bits of max|dJ| (range guard), else null
    double* state;            // [0] alpha, [1] alpha_min, [2] 1 if the job stepped this iteration
    double* alpha_log;        // [iters]
    int iters, opt_nb, positivity, reg_on;
    float w;
    double lambda;
    int ut, vt;               // RS tiles per view in u and v
};

__device__ __forceinline__ bool job_active(const BatchJob& J) { return *J.iter <= J.iters; }
__device__ __forceinline__ bool job_opt(const BatchJob& J) { return *J.iter <= J.iters && *J.iter < J.opt_nb; }

// CTA share: a launch's CTAs with blockIdx.x >= max(1, share * gridDim.x / 1000) stop
// taking items, so that batches running side by side on other streams get those SM slots.
// The host may change `share` (per mille) while a launch runs; thread 0 reads it one item
// ahead, so the read's latency hides behind the item's work.
__device__ __forceinline__ int share_now(const int* share) { return *(volatile const int*)share; }

// A work queue without an item list: the items of a group are those of job[0], then of
// job[1], ...; start[i] is the first queue index of the i-th job (start[n] = the total).
// An item's job is found by binary search (jobs are few) and its tile decoded from the
// job-local index, so the host's queue set-up is linear in the number of jobs.
struct JobRanges {
    const int* job;
    const long long* start;
    int n;
};

// The i with start[i] <= idx < start[i + 1]; (job index, job-local item index).
__device__ __forceinline__ void locate(const JobRanges& r, long long idx, int& j, long long& local) {
    int lo = 0, hi = r.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(r.start + mid) <= idx) lo = mid;
        else hi = mid - 1;
    }
    j = __ldg(r.job + lo);
    local = idx - __ldg(r.start + lo);
}

// Pops the next item for the whole CTA: false when the queue is empty or the CTA is beyond
// its share; else the item's job and job-local index. `s` is thread 0's copy of the share.
__device__ __forceinline__ bool pop_item(int* head, const int* share, int& s, const JobRanges& r, int n_items, int& j,
                                         long long& local) {
    __shared__ int s_idx, s_job;
    __shared__ long long s_local;
    __syncthreads();
    if (threadIdx.x == 0) {
        const int lim = max(1, (int)(((long long)s * gridDim.x) / 1000));
        s_idx = (int)blockIdx.x < lim ? atomicAdd(head, 1) : INT_MAX;
        s = share_now(share);
        if (s_idx < n_items) locate(r, s_idx, s_job, s_local);
    }
    __syncthreads();
    j = s_job;
    local = s_local;
    return s_idx < n_items;
}

// The (job, job-local index) of this CTA in a one-CTA-per-item launch.
__device__ __forceinline__ void cta_item(const JobRanges& r, int& j, long long& local) {
    __shared__ int s_job;
    __shared__ long long s_local;
    if (threadIdx.x == 0) locate(r, blockIdx.x, s_job, s_local);
    __syncthreads();
    j = s_job;
    local = s_local;
}

// ---------------------------------------------------------------------------------
// Persistent projection: EPI_RESIDUAL (resid = real - H f) or EPI_PARTIAL (||H dJ||^2).
// ---------------------------------------------------------------------------------
template <int MODE, int LAYOUT, typename Ts, int EPI>
__global__ void __launch_bounds__(256, 5) batch_rs_kernel(const BatchJob* __restrict__ jobs,
                                                          JobRanges r, int n_items, int* head, const int* share) {
    int s = threadIdx.x == 0 ? share_now(share) : 1000;
    int j;
    long long local;
    while (pop_item(head, share, s, r, n_items, j, local)) {
        const BatchJob& J = jobs[j];
        if (!(EPI == EPI_PARTIAL ? job_opt(J) : job_active(J))) continue;
        // view fastest, then u-tile, then v-tile (the single-job grid order): the CTAs
        // resident at one moment work on one band of detector rows over all views, i.e.
        // one z-slab of the volume, which stays in L2
        const int p = (int)(local % J.g.np);
        const long long t = local / J.g.np;
        const int ut = (int)(t % J.ut), vt = (int)(t / J.ut);
        const long W = J.g.nu + 2;
        const OutView<float> resid{J.resid, W + 1, W, W * (J.g.nv + 2)};
        double* slot = J.part_proj + ((long)p * J.ut + ut) * J.vt + vt;
        if (EPI == EPI_RESIDUAL && J.real_f32) {  // the measured sinogram kept in FP32
            const OutView<float> real{(float*)J.real, 0, (long)J.g.nu, (long)J.g.nu * J.g.nv};
            rs_tile<MODE, LAYOUT, Ts, float, EPI, float>(J.g, (const Ts*)J.rs_in, J.tex, resid, real, slot, p, ut, vt);
        } else {
            const OutView<Ts> real{(Ts*)J.real, 0, (long)J.g.nu, (long)J.g.nu * J.g.nv};
            rs_tile<MODE, LAYOUT, Ts, float, EPI, Ts>(J.g, (const Ts*)J.rs_in, J.tex, resid, real, slot, p, ut, vt);
        }
    }
}

// Largest of a 256-thread block's values (FP32 bits of non-negative floats), in thread 0.
__device__ __forceinline__ unsigned block_max_u32(unsigned m) {
    __shared__ unsigned red[8];
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) m = __reduce_max_sync(0xffffffffu, threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0u);
    __syncthreads();
    return m;
}

// Persistent VI backprojection of the FP32 residual into dJ (scale -2).
template <int UM, int ZC>
__global__ void __launch_bounds__(VI_BX* VI_BY, vi_min_blocks(ZC)) batch_vi_kernel(const BatchJob* __restrict__ jobs,
                                                               JobRanges r, int n_items, int* head, const int* share) {
    int s = threadIdx.x == 0 ? share_now(share) : 1000;
    int j;
    long long local;
    while (pop_item(head, share, s, r, n_items, j, local)) {
        const BatchJob& J = jobs[j];
        if (!job_active(J)) continue;
        // x-tile fastest, then y-tile, then z-group (the single-job grid order): resident
        // CTAs read the residual rows of one z band
        const int xt = (J.g.nx + VI_BX - 1) / VI_BX, yt = (J.g.ny + VI_BY - 1) / VI_BY;
        const long long t = local / xt;
        vi_tile<UM, ZC, float, float>(J.g, J.resid, J.dJ, -2.0f, (int)(local % xt), (int)(t % yt), (int)(t / yt));
    }
}

// ---------------------------------------------------------------------------------
// Per-slice phases: one CTA per (job, slice).
// ---------------------------------------------------------------------------------
// RS input of the job from vol (src 0) or dJ (src 1); one CTA per (job, input slice).
template <typename Ts>
__global__ void batch_prep_kernel(const BatchJob* __restrict__ jobs, JobRanges r, int src) {
    int jj;
    long long slice;
    cta_item(r, jj, slice);
    const int2 it = make_int2(jj, (int)slice);
    const BatchJob& J = jobs[it.x];
    if (!(src ? job_opt(J) : job_active(J))) return;
    if (J.layout == RS_LAYOUT_TEX) return;  // textures are filled by a copy or a conversion kernel
    const float* in = src ? J.dJ : J.vol;
    const float sc = src ? fp16_scale(J.amax) : 1.f;  // FP16 range guard of dJ
    const int nx = J.g.nx, ny = J.g.ny, nz = J.g.nz;
    const long plane = (long)nx * ny;
    if (J.layout == RS_LAYOUT_CELL8) {
        const int ck = it.y;  // cell slice 0..nz
        const long CW = nx + 1, CWH = CW * (ny + 1);
        for (long c2 = threadIdx.x; c2 < CWH; c2 += blockDim.x) {
            const int ci = (int)(c2 % CW), cj = (int)(c2 / CW);
            Ts v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int i = ci - 1 + (q & 1), j = cj - 1 + ((q >> 1) & 1), k = ck - 1 + (q >> 2);
                const bool ok = i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
                v[q] = cvt<Ts>(ok ? in[k * plane + (long)j * nx + i] * sc : 0.f);
            }
            const long c = ck * CWH + c2;
            if (sizeof(Ts) == 4) {
                float4* o = reinterpret_cast<float4*>(J.rs_in) + 2 * c;
                const float* f = reinterpret_cast<const float*>(v);
                o[0] = make_float4(f[0], f[1], f[2], f[3]);
                o[1] = make_float4(f[4], f[5], f[6], f[7]);
            } else {
                reinterpret_cast<uint4*>(J.rs_in)[c] = *reinterpret_cast<const uint4*>(v);
            }
        }
    } else {
        const int k = it.y;  // interior slice 0..nz-1 of the padded layout
        if (k >= nz) return;
        const long W = nx + 2, WH = W * (ny + 2);
        Ts* o = (Ts*)J.rs_in;
        for (long r = threadIdx.x; r < plane; r += blockDim.x) {
            const long i = r % nx, j = r / nx;
            o[(k + 1) * WH + (j + 1) * W + (i + 1)] = cvt<Ts>(in[k * plane + r] * sc);
        }
    }
}

// grad = L vol (op 0);  dJ = dJ + w L(grad) (op 1);  partials of ||dJ||^2, ||L dJ||^2 (op 2);
// vol = vol + alpha dJ (op 3).
__global__ void batch_slice_kernel(const BatchJob* __restrict__ jobs, JobRanges r, int op) {
    int jj;
    long long slice;
    cta_item(r, jj, slice);
    const int2 it = make_int2(jj, (int)slice);
    const BatchJob& J = jobs[it.x];
    const int nx = J.g.nx, ny = J.g.ny, nz = J.g.nz, z = it.y;
    if (z >= nz) return;
    const long plane = (long)nx * ny, base = z * plane;
    if (op == 0 || op == 1) {
        if (!job_active(J) || !J.reg_on) return;
        for (long r = threadIdx.x; r < plane; r += blockDim.x) {
            const int x = (int)(r % nx), y = (int)(r / nx);
            if (op == 0) J.grad[base + r] = lap_at(J.vol, x, y, z, nx, ny, nz);
            else J.dJ[base + r] = fadd(J.dJ[base + r], fmul(J.w, lap_at(J.grad, x, y, z, nx, ny, nz)));
        }
    } else if (op == 2) {
        if (!job_opt(J)) return;
        double s0 = 0.0, s2 = 0.0;
        unsigned m = 0;
        for (long r = threadIdx.x; r < plane; r += blockDim.x) {
            const float df = J.dJ[base + r];
            m = max(m, __float_as_uint(fabsf(df)));
            const double d = (double)df;
            s0 += d * d;
            if (J.reg_on) {
                const double l = (double)lap_at(J.dJ, (int)(r % nx), (int)(r / nx), z, nx, ny, nz);
                s2 += l * l;
            }
        }
        s0 = block_sum(s0);
        s2 = block_sum(s2);
        if (J.amax) m = block_max_u32(m);  // max is order-free: deterministic across mixes
        if (threadIdx.x == 0) {
            J.part_lap[z] = s0;
            J.part_lap[nz + z] = s2;
            if (J.amax && m) atomicMax(J.amax, m);
        }
    } else {
        if (J.state[2] == 0.0) return;
        const float a = __double2float_rn(J.state[0]);
        for (long r = threadIdx.x; r < plane; r += blockDim.x) {
            float v = fadd(J.vol[base + r], fmul(a, J.dJ[base + r]));
            if (J.positivity && v < 0.f) v = 0.f;
            J.vol[base + r] = v;
        }
    }
}

// One CTA per job: fixed-order reduction of the partials, step size, iteration counter.
__global__ void batch_alpha_kernel(const BatchJob* __restrict__ jobs) {
    const BatchJob& J = jobs[blockIdx.x];
    const int it = *J.iter;
    const bool active = it <= J.iters;
    const bool opt = active && it < J.opt_nb;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (opt) {
        const long np = (long)J.g.np * J.ut * J.vt;
        for (long i = threadIdx.x; i < np; i += blockDim.x) s1 += J.part_proj[i];
        for (int z = threadIdx.x; z < J.g.nz; z += blockDim.x) {
            s0 += J.part_lap[z];
            s2 += J.part_lap[J.g.nz + z];
        }
    }
    s0 = block_sum(s0);
    s1 = block_sum(s1);
    s2 = block_sum(s2);
    if (threadIdx.x != 0) return;
    if (!active) {
        J.state[2] = 0.0;
        return;
    }
    double alpha;
    if (opt) {
        s1 *= fp16_unscale_sq(J.amax);                                  // FP16-stored dJ was scaled
        if (J.amax) *J.amax = 0u;                                        // next iteration's max|dJ|
        const double normdJProjReg = J.reg_on ? 2.0 * s2 : 0.0;        // GG..._CPU.cu:216
        const double normdJProj = 2.0 * s1 + J.lambda * normdJProjReg;  // Iter3D_Algo_Gradient.cu:146
        alpha = -1.0 * s0 / normdJProj;                                  // :150
        J.state[1] = fmax(alpha, J.state[1]);                            // :151
    } else {
        alpha = J.state[1];                                              // :156
    }
    J.state[0] = alpha;
    J.state[2] = 1.0;
    J.alpha_log[it - 1] = alpha;
    *J.iter = it + 1;
}

// Loads every kernel a batch launches. With lazy module loading (the CUDA 12 default) the
// first launch of a kernel loads it, and loading synchronises the context: a batch whose
// first iteration starts while another batch's kernels run would wait for all of them.
template <int MODE, typename Ts>
static void preload_rs() {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, batch_rs_kernel<MODE, RS_LAYOUT_PLAIN, Ts, EPI_RESIDUAL>);
    cudaFuncGetAttributes(&a, batch_rs_kernel<MODE, RS_LAYOUT_CELL8, Ts, EPI_RESIDUAL>);
    cudaFuncGetAttributes(&a, batch_rs_kernel<MODE, RS_LAYOUT_TEX, Ts, EPI_RESIDUAL>);
    cudaFuncGetAttributes(&a, batch_rs_kernel<MODE, RS_LAYOUT_PLAIN, Ts, EPI_PARTIAL>);
    cudaFuncGetAttributes(&a, batch_rs_kernel<MODE, RS_LAYOUT_CELL8, Ts, EPI_PARTIAL>);
    cudaFuncGetAttributes(&a, batch_rs_kernel<MODE, RS_LAYOUT_TEX, Ts, EPI_PARTIAL>);
    cudaFuncGetAttributes(&a, batch_prep_kernel<Ts>);
}

static void preload_batch_kernels() {
    cudaFuncAttributes a;
    preload_rs<0, float>();
    preload_rs<1, float>();
    preload_rs<0, __nv_bfloat16>();
    preload_rs<1, __nv_bfloat16>();
    preload_rs<0, __half>();
    preload_rs<1, __half>();
    cudaFuncGetAttributes(&a, batch_vi_kernel<0, 1>);
    cudaFuncGetAttributes(&a, batch_vi_kernel<0, 2>);
    cudaFuncGetAttributes(&a, batch_vi_kernel<1, 1>);
    cudaFuncGetAttributes(&a, batch_vi_kernel<1, 2>);
    cudaFuncGetAttributes(&a, batch_slice_kernel);
    cudaFuncGetAttributes(&a, batch_alpha_kernel);
    rs_tex_preload();
    cudaGetLastError();
}

template <typename K>
static int persistent_grid(K kernel, int threads, int device) {
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (per_sm < 1) per_sm = 1;
    return per_sm * (sms > 0 ? sms : 148);
}

}  // namespace tomo

using namespace tomo;

struct HostBatchJob {
    bool used = false;
    tomo_config_ct cfg{};
    HostGeom hg;
    tomo_tuning tuning{};
    BatchJob d{};                 // descriptor as uploaded
    float* d_alpha = nullptr;
    float* d_beta = nullptr;
    float4* d_vi = nullptr;
    RsTexture tex;                // TEX layout resources (storage type)
    size_t bytes = 0;
    std::vector<void*> allocs;    // everything allocated for this job
};

struct tomo_batch {
    int device = 0;
    tomo_gradient_params prm{};
    std::vector<HostBatchJob> jobs;
    bool dirty = true;
    // device-side tables
    BatchJob* d_jobs = nullptr;
    // work queues as job ranges, 7 groups: RS by layout [PLAIN, CELL8, TEX], VI by chunking
    // [zc 1, zc 2], RS input slices (nz + 1 per job), volume slices (nz per job)
    int* d_job_ids = nullptr;
    long long* d_starts = nullptr;
    JobRanges ranges[7] = {};
    long long counts[7] = {0, 0, 0, 0, 0, 0, 0};
    int n_jobs_dev = 0;
    std::vector<int> dev_to_slot;
    int* d_heads = nullptr;  // [0..2] residual projection per layout, [3..5] norm projection, [6..7] VI,
                             // [8] CTA share of the persistent launches (per mille)
    cudaMemPool_t pool = nullptr;       // job buffers and tables: stream-ordered, so that adding or
                                        // retiring a job never waits for other streams' work
    cudaStream_t ctl_stream = nullptr;  // share updates, which must not queue behind own_stream
    int* h_share = nullptr;             // pinned source of the share copies
    // Texture arrays of removed jobs, kept for the next job of the same size: freeing a CUDA
    // array synchronises the whole device, which would stall the host (and every other
    // batch's next launch) behind the longest kernel in flight. tomo_batch_trim frees them.
    struct Parked {
        RsTexture t;
        int nx, ny, nz;
        size_t bytes;
    };
    std::vector<Parked> parked;
    int grid_rs = 0, grid_vi = 0;
    // graph
    bool use_graph = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t own_stream = nullptr;
    long long launches = 0;
    long long graph_launches = 0;
    // A job-set change re-captures the iteration and updates the executable graph in place
    // (cudaGraphExecUpdate); executable graphs that could not be updated are destroyed only
    // at trim or destroy time, never while other streams run.
    bool recapture = false;
    std::vector<cudaGraphExec_t> old_execs;
    double host_ms[4] = {0, 0, 0, 0};  // rebuild, capture, instantiate/update, launch
};

namespace {

tomo_dtype storage_of(const tomo_batch* b) { return b->prm.storage; }

int batch_layout(const tomo_tuning& t, tomo_dtype st, int nz) {
    int l = t.rs_layout;
    if (l == RS_LAYOUT_HYBRID || l == RS_LAYOUT_MARCH) l = RS_LAYOUT_TEX;  // the batch's queue groups PLAIN, CELL8, TEX
    (void)st;
    if (l == RS_LAYOUT_TEX && nz + 3 > rs_tex_max_layers()) l = RS_LAYOUT_CELL8;  // data + up to three layers
    return l;
}

size_t job_bytes(const tomo_config_ct& c, const tomo_gradient_params& p, const tomo_tuning& t) {
    const size_t nx = c.x_volume_pixel_nb, ny = c.y_volume_pixel_nb, nz = c.z_volume_pixel_nb;
    const size_t nu = c.u_detector_pixel_nb, nv = c.v_detector_pixel_nb, np = c.projection_nb;
    const size_t es = dtype_size(p.storage);
    const int layout = batch_layout(t, p.storage, (int)nz);
    size_t b = 0;
    b += 2 * nx * ny * nz * sizeof(float);                                        // dJ, grad
    // TEX: FP32 slices between two zero layers, or 16-bit slice pairs (4 B) in nz + 3 layers
    b += layout == RS_LAYOUT_TEX ? nx * ny * (es == 4 ? (nz + 2) * 4 : (nz + 3) * 4)
                                 : rs_input_elems(layout, nx, ny, nz) * es;
    b += (nu + 2) * (nv + 2) * np * sizeof(float);                               // padded FP32 residual
    DevGeom sg{};
    sg.nu = (int)nu;
    sg.nv = (int)nv;
    rs_shape_of(t, sg);
    b += np * rs_tiles_u(sg) * rs_tiles_v(sg) * sizeof(double);                 // projection partials
    b += 2 * nz * sizeof(double) + np * (2 * sizeof(float) + sizeof(float4)) + 64 * sizeof(double) +
         (size_t)std::max(1, p.gradient_iteration_nb) * sizeof(double);
    return b;
}

void free_job(tomo_batch* b, HostBatchJob& j) {
    for (void* p : j.allocs) cudaFreeAsync(p, b->own_stream);
    j.allocs.clear();
    if (j.tex.arr)
        b->parked.push_back({j.tex, j.hg.nx, j.hg.ny, j.hg.nz,
                             (size_t)j.hg.nx * j.hg.ny * (j.tex.zpairs ? j.hg.nz + 3 : j.hg.nz + 2) * 4});
    j.tex = RsTexture();
    j.d.tex = 0;
    j.used = false;
}

// A parked texture of this size and type, or a new one.
cudaError_t take_texture(tomo_batch* b, int nx, int ny, int nz, tomo_dtype dt, RsTexture* t) {
    for (size_t i = 0; i < b->parked.size(); ++i) {
        const auto& q = b->parked[i];
        if (q.nx == nx && q.ny == ny && q.nz == nz && q.t.dt == dt) {
            *t = q.t;
            b->parked.erase(b->parked.begin() + i);
            return cudaSuccess;
        }
    }
    return rs_vol_tex_create(nx, ny, nz, dt, t, b->own_stream);
}

void trim_textures(tomo_batch* b) {
    for (auto& q : b->parked) rs_tex_destroy(&q.t);
    b->parked.clear();
}

void drop_graph(tomo_batch* b) {
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
}

void drop_old_execs(tomo_batch* b) {
    for (cudaGraphExec_t e : b->old_execs) cudaGraphExecDestroy(e);
    b->old_execs.clear();
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Rebuild the device descriptor table and the work-item lists for the live jobs.
void free_tables(tomo_batch* b) {
    void* t[3] = {b->d_jobs, b->d_job_ids, b->d_starts};
    for (void* p : t)
        if (p) cudaFreeAsync(p, b->own_stream);
}

// Stream-ordered allocation from the batch's pool, and an upload, both on own_stream.
template <typename T>
cudaError_t upload(tomo_batch* b, T** dst, const std::vector<T>& v) {
    cudaError_t e = cudaMallocFromPoolAsync((void**)dst, sizeof(T) * std::max<size_t>(1, v.size()), b->pool, b->own_stream);
    if (e == cudaSuccess && !v.empty())
        e = cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, b->own_stream);
    return e;
}

tomo_status rebuild(tomo_batch* b) {
    b->recapture = true;  // the graph's kernel parameters (tables, item counts) change
    free_tables(b);
    b->d_jobs = nullptr;
    b->d_job_ids = nullptr;
    b->d_starts = nullptr;
    std::vector<BatchJob> descs;
    b->dev_to_slot.clear();
    for (size_t s = 0; s < b->jobs.size(); ++s)
        if (b->jobs[s].used) {
            descs.push_back(b->jobs[s].d);
            b->dev_to_slot.push_back((int)s);
        }
    const int J = (int)descs.size();
    // Longest first: jobs in decreasing order of their per-item cost (stable); each job's
    // items are contiguous, in the single-job grid order (decoded in the kernels).
    std::vector<int> rs_order(J), vi_order(J);
    std::iota(rs_order.begin(), rs_order.end(), 0);
    std::iota(vi_order.begin(), vi_order.end(), 0);
    auto ray_cost = [&](int j) { return (double)(descs[j].g.nx + descs[j].g.ny + descs[j].g.nz); };  // ~ chord
    auto col_cost = [&](int j) { return (double)descs[j].g.np * 16 * descs[j].zc; };
    std::stable_sort(rs_order.begin(), rs_order.end(), [&](int a, int c) { return ray_cost(a) > ray_cost(c); });
    std::stable_sort(vi_order.begin(), vi_order.end(), [&](int a, int c) { return col_cost(a) > col_cost(c); });
    // groups: RS by layout (3), VI by chunking (2), RS input slices, volume slices
    std::vector<int> ids[7];
    std::vector<long long> starts[7];
    auto add = [&](int grp, int j, long long items) {
        if (starts[grp].empty()) starts[grp].push_back(0);
        ids[grp].push_back(j);
        starts[grp].push_back(starts[grp].back() + items);
    };
    for (int j : rs_order) {
        const BatchJob& d = descs[j];
        add(d.layout, j, (long long)d.g.np * d.ut * d.vt);
    }
    for (int j : vi_order) {
        const BatchJob& d = descs[j];
        const long long xt = (d.g.nx + VI_BX - 1) / VI_BX, yt = (d.g.ny + VI_BY - 1) / VI_BY;
        const long long zg = (d.g.nz + 16 * d.zc - 1) / (16 * d.zc);
        add(3 + d.zc - 1, j, xt * yt * zg);
    }
    for (int j = 0; j < J; ++j) {
        add(5, j, descs[j].g.nz + 1);
        add(6, j, descs[j].g.nz);
    }
    std::vector<int> all_ids;
    std::vector<long long> all_starts;
    size_t id_off[7], st_off[7];
    for (int g = 0; g < 7; ++g) {
        id_off[g] = all_ids.size();
        st_off[g] = all_starts.size();
        all_ids.insert(all_ids.end(), ids[g].begin(), ids[g].end());
        all_starts.insert(all_starts.end(), starts[g].begin(), starts[g].end());
        b->counts[g] = starts[g].empty() ? 0 : starts[g].back();
        TOMO_CHECK_ARG(b->counts[g] < (long long)INT_MAX - 148L * 64, "tomo_batch: too many work items in one launch");
    }
    b->n_jobs_dev = J;
    b->dirty = false;
    if (J == 0) return TOMO_OK;
    TOMO_CUDA_TRY(upload(b, &b->d_jobs, descs));
    TOMO_CUDA_TRY(upload(b, &b->d_job_ids, all_ids));
    TOMO_CUDA_TRY(upload(b, &b->d_starts, all_starts));
    for (int g = 0; g < 7; ++g) b->ranges[g] = JobRanges{b->d_job_ids + id_off[g], b->d_starts + st_off[g], (int)ids[g].size()};
    // the host vectors die on return: the pageable copies must have consumed them
    TOMO_CUDA_TRY(cudaStreamSynchronize(b->own_stream));
    return TOMO_OK;
}

template <int MODE, int LAYOUT, typename Ts, int EPI>
cudaError_t launch_batch_rs_group(tomo_batch* b, cudaStream_t st) {
    const int n = (int)b->counts[LAYOUT];
    if (n == 0) return cudaSuccess;
    int* head = b->d_heads + (EPI == EPI_PARTIAL ? 3 : 0) + LAYOUT;
    auto k = batch_rs_kernel<MODE, LAYOUT, Ts, EPI>;
    static int grid = 0;
    if (!grid) grid = persistent_grid(k, 256, b->device);
    k<<<std::min(grid, n), 256, 0, st>>>(b->d_jobs, b->ranges[LAYOUT], n, head, b->d_heads + 8);
    b->launches += 1;
    return cudaGetLastError();
}

template <int MODE, typename Ts, int EPI>
cudaError_t launch_batch_rs(tomo_batch* b, cudaStream_t st) {
    cudaError_t e = launch_batch_rs_group<MODE, RS_LAYOUT_PLAIN, Ts, EPI>(b, st);
    if (e == cudaSuccess) e = launch_batch_rs_group<MODE, RS_LAYOUT_CELL8, Ts, EPI>(b, st);
    if (e == cudaSuccess) e = launch_batch_rs_group<MODE, RS_LAYOUT_TEX, Ts, EPI>(b, st);
    return e;
}

template <int UM, int ZC>
cudaError_t launch_batch_vi_group(tomo_batch* b, cudaStream_t st) {
    const int n = (int)b->counts[3 + ZC - 1];
    if (n == 0) return cudaSuccess;
    auto k = batch_vi_kernel<UM, ZC>;
    static int grid = 0;
    if (!grid) grid = persistent_grid(k, VI_BX * VI_BY, b->device);
    k<<<std::min(grid, n), VI_BX * VI_BY, 0, st>>>(b->d_jobs, b->ranges[3 + ZC - 1], n, b->d_heads + 5 + ZC,
                                                   b->d_heads + 8);
    b->launches += 1;
    return cudaGetLastError();
}

template <int UM>
cudaError_t launch_batch_vi(tomo_batch* b, cudaStream_t st) {
    cudaError_t e = launch_batch_vi_group<UM, 1>(b, st);
    if (e == cudaSuccess) e = launch_batch_vi_group<UM, 2>(b, st);
    return e;
}

template <typename Ts>
tomo_status enqueue_iteration_t(tomo_batch* b, cudaStream_t st) {
    const tomo_gradient_params& P = b->prm;
    const int um_back = P.backprojector == TOMO_BACK_VI_UM;
    const int um_proj = P.projector == TOMO_PROJ_RS_UM;
    const bool reg = P.regularization_parameter != 0.0;
    TOMO_CUDA_TRY(cudaMemsetAsync(b->d_heads, 0, 8 * sizeof(int), st));  // [8], the share, is kept
    // 1. RS input from the iterate; texture jobs copy into their arrays
    for (int j = 0; j < b->n_jobs_dev; ++j) {
        HostBatchJob& hj = b->jobs[b->dev_to_slot[j]];
        if (hj.d.layout == RS_LAYOUT_TEX)
            TOMO_CUDA_TRY(rs_tex_fill(hj.d.vol, TOMO_F32, hj.hg.nx, hj.hg.ny, hj.hg.nz, hj.tex, st));
    }
    batch_prep_kernel<Ts><<<(int)b->counts[5], 256, 0, st>>>(b->d_jobs, b->ranges[5], 0);
    // 2. residual projection (persistent)
    TOMO_CUDA_TRY((um_proj ? launch_batch_rs<1, Ts, EPI_RESIDUAL>(b, st) : launch_batch_rs<0, Ts, EPI_RESIDUAL>(b, st)));
    // 3. backprojection into dJ (persistent)
    TOMO_CUDA_TRY((um_back ? launch_batch_vi<1>(b, st) : launch_batch_vi<0>(b, st)));
    // 4. regulariser
    if (reg) {
        batch_slice_kernel<<<(int)b->counts[6], 256, 0, st>>>(b->d_jobs, b->ranges[6], 0);
        batch_slice_kernel<<<(int)b->counts[6], 256, 0, st>>>(b->d_jobs, b->ranges[6], 1);
    }
    // 5. norms for the optimal step
    batch_slice_kernel<<<(int)b->counts[6], 256, 0, st>>>(b->d_jobs, b->ranges[6], 2);
    for (int j = 0; j < b->n_jobs_dev; ++j) {
        HostBatchJob& hj = b->jobs[b->dev_to_slot[j]];
        if (hj.d.layout == RS_LAYOUT_TEX)
            TOMO_CUDA_TRY(rs_tex_fill(hj.d.dJ, TOMO_F32, hj.hg.nx, hj.hg.ny, hj.hg.nz, hj.tex, st, hj.d.amax));
    }
    batch_prep_kernel<Ts><<<(int)b->counts[5], 256, 0, st>>>(b->d_jobs, b->ranges[5], 1);
    TOMO_CUDA_TRY((um_proj ? launch_batch_rs<1, Ts, EPI_PARTIAL>(b, st) : launch_batch_rs<0, Ts, EPI_PARTIAL>(b, st)));
    // 6. step size and counters, 7. update
    batch_alpha_kernel<<<b->n_jobs_dev, 256, 0, st>>>(b->d_jobs);
    batch_slice_kernel<<<(int)b->counts[6], 256, 0, st>>>(b->d_jobs, b->ranges[6], 3);
    TOMO_CUDA_TRY(cudaGetLastError());
    b->launches += (reg ? 6 : 4);  // prep x2, alpha, update (+ 2 Laplacians); persistent launches counted above
    return TOMO_OK;
}

tomo_status enqueue_iteration(tomo_batch* b, cudaStream_t st) {
    switch (storage_of(b)) {
        case TOMO_F32: return enqueue_iteration_t<float>(b, st);
        case TOMO_BF16: return enqueue_iteration_t<__nv_bfloat16>(b, st);
        case TOMO_F16: return enqueue_iteration_t<__half>(b, st);
    }
    return TOMO_ERR_INVALID;
}

}  // namespace

extern "C" {

tomo_status tomo_batch_create(int device, const tomo_gradient_params* params, tomo_batch** out) {
    TOMO_CHECK_ARG(params && out, "tomo_batch_create: null argument");
    *out = nullptr;
    TOMO_CHECK_ARG(params->storage == TOMO_F32 || params->storage == TOMO_BF16 || params->storage == TOMO_F16,
                   "tomo_batch_create: unknown storage dtype");
    TOMO_CHECK_ARG(params->projector == TOMO_PROJ_RS || params->projector == TOMO_PROJ_RS_UM,
                   "tomo_batch_create: the batched loop projects with RS");
    TOMO_CHECK_ARG(params->backprojector == TOMO_BACK_VI || params->backprojector == TOMO_BACK_VI_UM,
                   "tomo_batch_create: the batched loop backprojects with VI");
    TOMO_CHECK_ARG(params->gradient_iteration_nb >= 1, "tomo_batch_create: at least one iteration");
    TOMO_CUDA_TRY(cudaSetDevice(device));
    tomo_batch* b = new tomo_batch();
    b->device = device;
    b->prm = *params;
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    const int full = 1000;
    if (cudaMalloc(&b->d_heads, 16 * sizeof(int)) != cudaSuccess ||
        cudaMemcpy(b->d_heads + 8, &full, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->ctl_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaHostAlloc(&b->h_share, sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
        cudaMemPoolCreate(&b->pool, &pp) != cudaSuccess) {
        const cudaError_t e = cudaGetLastError();
        cudaFree(b->d_heads);
        if (b->own_stream) cudaStreamDestroy(b->own_stream);
        if (b->ctl_stream) cudaStreamDestroy(b->ctl_stream);
        if (b->h_share) cudaFreeHost(b->h_share);
        delete b;
        return cuda_fail(e, "tomo_batch_create");
    }
    preload_batch_kernels();
    *out = b;
    return TOMO_OK;
}

tomo_status tomo_batch_destroy(tomo_batch* b) {
    if (!b) return TOMO_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->own_stream);
    drop_graph(b);
    drop_old_execs(b);
    for (auto& j : b->jobs)
        if (j.used) free_job(b, j);
    free_tables(b);
    cudaStreamSynchronize(b->own_stream);
    cudaStreamSynchronize(b->ctl_stream);
    trim_textures(b);
    cudaFree(b->d_heads);
    cudaStreamDestroy(b->own_stream);
    cudaStreamDestroy(b->ctl_stream);
    cudaFreeHost(b->h_share);
    cudaMemPoolDestroy(b->pool);
    cudaGetLastError();
    delete b;
    return TOMO_OK;
}

tomo_status tomo_batch_footprint(const tomo_config_ct* cfg, const tomo_gradient_params* params, const tomo_tuning* tuning,
                                 size_t* bytes) {
    TOMO_CHECK_ARG(cfg && params && bytes, "tomo_batch_footprint: null argument");
    tomo_tuning t{};
    t.rs_layout = RS_LAYOUT_TEX;
    if (tuning) t = *tuning;
    *bytes = job_bytes(*cfg, *params, t);
    return TOMO_OK;
}

tomo_status tomo_batch_add(tomo_batch* b, const tomo_config_ct* cfg, const tomo_tuning* tuning, float* volume,
                           const void* real_sinogram, int32_t* job) {
    TOMO_CHECK_ARG(b && cfg && volume && real_sinogram && job, "tomo_batch_add: null argument");
    TOMO_CHECK_ARG(!tuning || rs_shape_valid(*tuning), "tomo_batch_add: invalid RS launch shape in the tuning");
    TOMO_CHECK_ARG(cfg->projection_nb > 0 && cfg->u_detector_pixel_nb > 0 && cfg->v_detector_pixel_nb > 0 &&
                       cfg->x_volume_pixel_nb > 0 && cfg->y_volume_pixel_nb > 0 && cfg->z_volume_pixel_nb > 0 &&
                       cfg->den_start_angle != 0 && cfg->den_stop_angle != 0 && cfg->x_volume_size > 0 &&
                       cfg->u_detector_size > 0 && cfg->v_detector_size > 0 && cfg->fod > 0 && cfg->fdd > 0,
                   "tomo_batch_add: invalid geometry");
    TOMO_CUDA_TRY(cudaSetDevice(b->device));
    size_t slot = 0;
    while (slot < b->jobs.size() && b->jobs[slot].used) ++slot;
    if (slot == b->jobs.size()) b->jobs.emplace_back();
    HostBatchJob& hj = b->jobs[slot];
    hj = HostBatchJob();
    hj.used = true;
    hj.cfg = *cfg;
    hj.tuning.rs_layout = RS_LAYOUT_TEX;
    hj.tuning.vi_zc = 1;
    if (tuning) hj.tuning = *tuning;
    derive_geometry(*cfg, hj.hg);
    const HostGeom& h = hj.hg;
    const tomo_dtype sd = b->prm.storage;
    const size_t es = dtype_size(sd), nvox = (size_t)h.nx * h.ny * h.nz;
    BatchJob& d = hj.d;
    d = BatchJob();
    d.layout = batch_layout(hj.tuning, sd, h.nz);
    d.zc = hj.tuning.vi_zc == 1 ? 1 : 2;  // the batched VI kernel instantiates 1 and 2
    rs_shape_of(hj.tuning, d.g);  // the launch shape (fill_devgeom below keeps it)
    d.ut = (h.nu + (1 << d.g.rs_tlog) - 1) >> d.g.rs_tlog;
    d.vt = (h.nv + (256 >> d.g.rs_tlog) - 1) / (256 >> d.g.rs_tlog);
    cudaStream_t st = b->own_stream;
    auto alloc = [&](void** p, size_t bytes, bool zero) -> bool {
        if (cudaMallocFromPoolAsync(p, bytes, b->pool, st) != cudaSuccess) return false;
        hj.allocs.push_back(*p);
        return !zero || cudaMemsetAsync(*p, 0, bytes, st) == cudaSuccess;
    };
    bool ok = alloc((void**)&hj.d_alpha, sizeof(float) * h.np, false) && alloc((void**)&hj.d_beta, sizeof(float) * h.np, false) &&
              alloc((void**)&hj.d_vi, sizeof(float4) * h.np, false) && alloc((void**)&d.dJ, nvox * sizeof(float), false) &&
              alloc((void**)&d.grad, nvox * sizeof(float), false) &&
              alloc((void**)&d.resid, (size_t)(h.nu + 2) * (h.nv + 2) * h.np * sizeof(float), true) &&
              alloc((void**)&d.part_proj, (size_t)h.np * d.ut * d.vt * sizeof(double), true) &&
              alloc((void**)&d.part_lap, 2 * (size_t)h.nz * sizeof(double), true) &&
              alloc((void**)&d.iter, sizeof(int) * 4, true) && alloc((void**)&d.state, sizeof(double) * 4, false) &&
              alloc((void**)&d.alpha_log, sizeof(double) * b->prm.gradient_iteration_nb, true);
    if (ok && d.layout != RS_LAYOUT_TEX) ok = alloc(&d.rs_in, rs_input_elems(d.layout, h.nx, h.ny, h.nz) * es, true);
    if (ok && d.layout == RS_LAYOUT_TEX) {
        ok = take_texture(b, h.nx, h.ny, h.nz, sd, &hj.tex) == cudaSuccess;
        d.tex = hj.tex.tex;
    }
    if (ok) {
        const int one = 1;
        const double st0[4] = {0.0, -0.0347711, 0.0, 0.0};  // alpha, alpha_min (Iter3D_Algo_Gradient.cu:61-62)
        const auto h2d = cudaMemcpyHostToDevice;
        ok = cudaMemcpyAsync(hj.d_alpha, h.alpha.data(), sizeof(float) * h.np, h2d, st) == cudaSuccess &&
             cudaMemcpyAsync(hj.d_beta, h.beta.data(), sizeof(float) * h.np, h2d, st) == cudaSuccess &&
             cudaMemcpyAsync(hj.d_vi, h.vi.data(), sizeof(float4) * h.np, h2d, st) == cudaSuccess &&
             cudaMemcpyAsync(d.iter, &one, sizeof(int), h2d, st) == cudaSuccess &&
             cudaMemcpyAsync(d.state, st0, sizeof(st0), h2d, st) == cudaSuccess;
    }
    // the sources above are host locals: wait for the copies (this stream only)
    ok = cudaStreamSynchronize(st) == cudaSuccess && ok;
    if (!ok) {
        cudaGetLastError();
        free_job(b, hj);
        set_error("tomo_batch_add: device allocation failed");
        return TOMO_ERR_NO_MEMORY;
    }
    fill_devgeom(h, hj.d_alpha, hj.d_beta, hj.d_vi, d.g);
    rs_shape_of(hj.tuning, d.g);
    d.amax = sd == TOMO_F16 ? reinterpret_cast<unsigned*>(d.iter + 1) : nullptr;
    d.real = real_sinogram;
    d.real_f32 = b->prm.real_sinogram_f32 != 0;
    d.vol = volume;
    d.iters = b->prm.gradient_iteration_nb;
    d.opt_nb = b->prm.optimal_step_iteration_nb;
    d.positivity = b->prm.positivity;
    d.reg_on = b->prm.regularization_parameter != 0.0;
    d.w = (float)(2.0 * (double)(float)b->prm.regularization_parameter);  // beta * lambda, GG..._CPU.cu:205
    d.lambda = b->prm.regularization_parameter;
    hj.bytes = job_bytes(*cfg, b->prm, hj.tuning);
    b->dirty = true;
    *job = (int32_t)slot;
    return TOMO_OK;
}

tomo_status tomo_batch_remove(tomo_batch* b, int32_t job) {
    TOMO_CHECK_ARG(b && job >= 0 && (size_t)job < b->jobs.size() && b->jobs[job].used, "tomo_batch_remove: no such job");
    TOMO_CUDA_TRY(cudaSetDevice(b->device));
    // only this batch's stream: other batches (other streams) keep running meanwhile
    TOMO_CUDA_TRY(cudaStreamSynchronize(b->own_stream));
    free_job(b, b->jobs[job]);  // stream-ordered; the memory stays reserved in the pool
    b->dirty = true;
    return TOMO_OK;
}

tomo_status tomo_batch_set_graph(tomo_batch* b, int enable) {
    TOMO_CHECK_ARG(b, "tomo_batch_set_graph: null argument");
    b->use_graph = enable != 0;
    drop_graph(b);
    return TOMO_OK;
}

tomo_status tomo_batch_set_share(tomo_batch* b, double fraction) {
    TOMO_CHECK_ARG(b && fraction > 0.0 && fraction <= 1.0, "tomo_batch_set_share: fraction in (0, 1]");
    TOMO_CUDA_TRY(cudaSetDevice(b->device));
    TOMO_CUDA_TRY(cudaStreamSynchronize(b->ctl_stream));  // the previous copy has read h_share
    *b->h_share = std::max(1, std::min(1000, (int)std::lround(fraction * 1000.0)));
    TOMO_CUDA_TRY(cudaMemcpyAsync(b->d_heads + 8, b->h_share, sizeof(int), cudaMemcpyHostToDevice, b->ctl_stream));
    return TOMO_OK;
}

tomo_status tomo_batch_set_priority(tomo_batch* b, int32_t priority) {
    TOMO_CHECK_ARG(b, "tomo_batch_set_priority: null argument");
    TOMO_CUDA_TRY(cudaSetDevice(b->device));
    int lo = 0, hi = 0;  // cudaDeviceGetStreamPriorityRange: (least, greatest), greatest < least
    TOMO_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    const int pr = std::max(hi, std::min(lo, (int)priority));
    cudaStream_t ns = nullptr;
    TOMO_CUDA_TRY(cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, pr));
    cudaError_t e = cudaStreamSynchronize(b->own_stream);
    if (e != cudaSuccess) {
        cudaStreamDestroy(ns);
        return cuda_fail(e, "tomo_batch_set_priority");
    }
    drop_graph(b);  // a replay would run on the new stream anyway; recapture for clarity
    cudaStreamDestroy(b->own_stream);
    b->own_stream = ns;
    return TOMO_OK;
}

tomo_status tomo_batch_iterate(tomo_batch* b, int32_t count, void* stream) {
    TOMO_CHECK_ARG(b && count >= 0, "tomo_batch_iterate: bad argument");
    TOMO_CUDA_TRY(cudaSetDevice(b->device));
    cudaGetLastError();
    tomo_status s;
    auto t0 = std::chrono::steady_clock::now();
    if (b->dirty && (s = rebuild(b)) != TOMO_OK) return s;
    b->host_ms[0] += ms_since(t0);
    if (b->n_jobs_dev == 0 || count == 0) return TOMO_OK;
    // Graph capture needs a non-legacy stream: work on the batch's own stream, ordered after
    // the caller's stream and before whatever the caller enqueues next.
    cudaStream_t caller = (cudaStream_t)stream, st = b->own_stream;
    cudaEvent_t ev;
    TOMO_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    TOMO_CUDA_TRY(cudaEventRecord(ev, caller));
    TOMO_CUDA_TRY(cudaStreamWaitEvent(st, ev, 0));
    if (b->use_graph) {
        if (!b->graph_exec || b->recapture) {
            t0 = std::chrono::steady_clock::now();
            TOMO_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            const long long before = b->launches;
            s = enqueue_iteration(b, st);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(st, &g);
            b->graph_launches = b->launches - before;  // kernels per replayed iteration
            b->launches = before;
            if (s != TOMO_OK) {
                if (g) cudaGraphDestroy(g);
                cudaEventDestroy(ev);
                return s;
            }
            if (e != cudaSuccess) {
                cudaEventDestroy(ev);
                return cuda_fail(e, "cudaStreamEndCapture");
            }
            b->host_ms[1] += ms_since(t0);
            t0 = std::chrono::steady_clock::now();
            bool updated = false;
            if (b->graph_exec) {
                cudaGraphExecUpdateResultInfo info{};
                updated = cudaGraphExecUpdate(b->graph_exec, g, &info) == cudaSuccess;
                if (!updated) {
                    cudaGetLastError();  // a topology change: instantiate anew, retire the old one
                    b->old_execs.push_back(b->graph_exec);
                    b->graph_exec = nullptr;
                }
            }
            if (b->graph) cudaGraphDestroy(b->graph);
            b->graph = g;
            if (!updated) TOMO_CUDA_TRY(cudaGraphInstantiate(&b->graph_exec, g, 0));
            b->recapture = false;
            b->host_ms[2] += ms_since(t0);
        }
        t0 = std::chrono::steady_clock::now();
        for (int i = 0; i < count; ++i) {
            TOMO_CUDA_TRY(cudaGraphLaunch(b->graph_exec, st));
            b->launches += b->graph_launches;
        }
        b->host_ms[3] += ms_since(t0);
    } else {
        for (int i = 0; i < count; ++i)
            if ((s = enqueue_iteration(b, st)) != TOMO_OK) {
                cudaEventDestroy(ev);
                return s;
            }
    }
    TOMO_CUDA_TRY(cudaEventRecord(ev, st));
    TOMO_CUDA_TRY(cudaStreamWaitEvent(caller, ev, 0));
    cudaEventDestroy(ev);
    return TOMO_OK;
}

tomo_status tomo_batch_job_status(tomo_batch* b, int32_t job, int32_t* iterations_done, double* alpha_min, void* stream) {
    TOMO_CHECK_ARG(b && iterations_done && job >= 0 && (size_t)job < b->jobs.size() && b->jobs[job].used,
                   "tomo_batch_job_status: no such job");
    TOMO_CUDA_TRY(cudaSetDevice(b->device));
    TOMO_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    TOMO_CUDA_TRY(cudaStreamSynchronize(b->own_stream));
    int it = 0;
    double st[2] = {0, 0};
    TOMO_CUDA_TRY(cudaMemcpyAsync(&it, b->jobs[job].d.iter, sizeof(int), cudaMemcpyDeviceToHost, b->own_stream));
    TOMO_CUDA_TRY(cudaMemcpyAsync(st, b->jobs[job].d.state, sizeof(st), cudaMemcpyDeviceToHost, b->own_stream));
    TOMO_CUDA_TRY(cudaStreamSynchronize(b->own_stream));
    *iterations_done = it - 1;
    if (alpha_min) *alpha_min = st[1];
    return TOMO_OK;
}

tomo_status tomo_batch_job_alphas(tomo_batch* b, int32_t job, double* alpha, int32_t n, int32_t* written, void* stream) {
    TOMO_CHECK_ARG(b && alpha && written && job >= 0 && (size_t)job < b->jobs.size() && b->jobs[job].used,
                   "tomo_batch_job_alphas: no such job");
    int32_t done = 0;
    tomo_status s = tomo_batch_job_status(b, job, &done, nullptr, stream);
    if (s != TOMO_OK) return s;
    const int m = std::max(0, std::min(n, done));
    if (m) {
        TOMO_CUDA_TRY(cudaMemcpyAsync(alpha, b->jobs[job].d.alpha_log, m * sizeof(double), cudaMemcpyDeviceToHost,
                                      b->own_stream));
        TOMO_CUDA_TRY(cudaStreamSynchronize(b->own_stream));
    }
    *written = m;
    return TOMO_OK;
}

tomo_status tomo_batch_trim(tomo_batch* b, size_t* parked_bytes) {
    TOMO_CHECK_ARG(b, "tomo_batch_trim: null argument");
    TOMO_CUDA_TRY(cudaSetDevice(b->device));
    size_t by = 0;
    for (auto& q : b->parked) by += q.bytes;
    if (parked_bytes) {  // query only
        *parked_bytes = by;
        return TOMO_OK;
    }
    TOMO_CUDA_TRY(cudaStreamSynchronize(b->own_stream));
    trim_textures(b);
    drop_old_execs(b);
    TOMO_CUDA_TRY(cudaMemPoolTrimTo(b->pool, 0));
    return TOMO_OK;
}

tomo_status tomo_batch_host_times(tomo_batch* b, double* ms) {
    TOMO_CHECK_ARG(b && ms, "tomo_batch_host_times: null argument");
    for (int i = 0; i < 4; ++i) ms[i] = b->host_ms[i];
    return TOMO_OK;
}

tomo_status tomo_batch_stats(tomo_batch* b, int32_t* live_jobs, int64_t* work_items, size_t* bytes,
                             int64_t* kernel_launches) {
    TOMO_CHECK_ARG(b, "tomo_batch_stats: null argument");
    int live = 0;
    size_t by = 0;
    for (auto& j : b->jobs)
        if (j.used) {
            ++live;
            by += j.bytes;
        }
    if (live_jobs) *live_jobs = live;
    if (bytes) *bytes = by;
    if (work_items) *work_items = (int64_t)(b->counts[0] + b->counts[1] + b->counts[2] + b->counts[3] + b->counts[4]);
    if (kernel_launches) *kernel_launches = b->launches;
    return TOMO_OK;
}

}  // extern "C"
