// noalloc.cu -- tomo_project_noalloc: the RS projection for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc at all: code inside a host framework whose memory
// pool or arena must own every device allocation, or real-time code that must not allocate
// once it runs. tomo_project (and tomo_context_create before it) allocate the padded copy
// of the volume and the per-view geometry tables on first use; this entry point instead
// keeps both in fixed-size arrays that live in this file as static __device__ storage.
// Every GPU that loads the library holds these arrays (32 MiB plus 96 KiB) until the
// process exits. The call allocates nothing: no cudaMalloc, no cudaFree, no allocating
// library routine.
//
// Limits: (nx+2)*(ny+2)*(nz+2) <= TOMO_NOALLOC_MAX_PADDED_VOXELS (8 Mi voxels, i.e. 32 MiB of
// FP32 -- up to 201^3) and P <= TOMO_NOALLOC_MAX_VIEWS (4096); larger sizes are rejected
// with TOMO_ERR_INVALID before any work is queued.
//
// Sharing: all calls on a device use the same arrays, which keep the previous call's
// contents; each call clears the whole padded region it uses before filling it. Two calls
// whose work overlaps on the GPU (different streams, or different host threads) race on
// the arrays and corrupt each other's result: serialise them.
//
// Set-up: the first call on a device looks up the arrays' device addresses with
// cudaGetSymbolAddress (in host code the array names are host-side stand-ins, not device
// addresses) and caches them; that first call makes this blocking runtime query.
//
// The view tables are copied from host memory the call owns (pageable): each copy has
// taken its data by the time cudaMemcpyAsync returns. The caller's current device is
// restored before the call returns. Like the library's other entry points, a call first
// clears a pending non-sticky CUDA error of the calling thread, so that the launch checks
// report errors of this call only.
#include <mutex>

#include "tomo_kernels.cuh"

#define TOMO_NOALLOC_MAX_PADDED_VOXELS (8u * 1024u * 1024u)
#define TOMO_NOALLOC_MAX_VIEWS 4096
#define TOMO_NOALLOC_MAX_DEVICES 64

namespace tomo {
namespace {

static __device__ __align__(256) float g_noalloc_padded[TOMO_NOALLOC_MAX_PADDED_VOXELS];
static __device__ __align__(256) float g_noalloc_alpha[TOMO_NOALLOC_MAX_VIEWS];
static __device__ __align__(256) float g_noalloc_beta[TOMO_NOALLOC_MAX_VIEWS];
static __device__ __align__(256) float4 g_noalloc_vi[TOMO_NOALLOC_MAX_VIEWS];

struct NoallocAddrs {
    float* padded = nullptr;
    float* alpha = nullptr;
    float* beta = nullptr;
    float4* vi = nullptr;
};

std::mutex g_setup_mu;
NoallocAddrs g_addrs[TOMO_NOALLOC_MAX_DEVICES];
bool g_ready[TOMO_NOALLOC_MAX_DEVICES] = {};

// Once per device, with that device current.
tomo_status noalloc_setup(int device, NoallocAddrs* out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_ready[device]) {
        NoallocAddrs a;
        TOMO_CUDA_TRY(cudaGetSymbolAddress((void**)&a.padded, g_noalloc_padded));
        TOMO_CUDA_TRY(cudaGetSymbolAddress((void**)&a.alpha, g_noalloc_alpha));
        TOMO_CUDA_TRY(cudaGetSymbolAddress((void**)&a.beta, g_noalloc_beta));
        TOMO_CUDA_TRY(cudaGetSymbolAddress((void**)&a.vi, g_noalloc_vi));
        g_addrs[device] = a;
        g_ready[device] = true;
    }
    *out = g_addrs[device];
    return TOMO_OK;
}

// The geometry set-up of the reference's host classes (same arithmetic as the context's),
// into caller-provided fixed arrays instead of heap containers.
void noalloc_geometry(const tomo_config_ct& c, DevGeom& g, float* alpha, float* beta, float4* vi) {
    const double start = c.num_start_angle / c.den_start_angle;
    const double stop = c.num_stop_angle / c.den_stop_angle;
    const unsigned long np = (unsigned long)c.projection_nb;
    const double step = M_PI * (double)(stop - start) / np;
    g.np = c.projection_nb;
    g.nu = c.u_detector_pixel_nb;
    g.nv = c.v_detector_pixel_nb;
    g.du = c.u_detector_size / (float)(unsigned long)g.nu;
    g.dv = c.v_detector_size / (float)(unsigned long)g.nv;
    g.uc = (float)((unsigned long)g.nu / 2.0 - 0.5);
    g.vc = (float)((unsigned long)g.nv / 2.0 - 0.5);
    g.nx = c.x_volume_pixel_nb;
    g.ny = c.y_volume_pixel_nb;
    g.nz = c.z_volume_pixel_nb;
    g.dx = c.x_volume_size / (float)(unsigned long)g.nx;
    g.xc = (float)((unsigned long)g.nx / 2.0 - 0.5);
    g.yc = (float)((unsigned long)g.ny / 2.0 - 0.5);
    g.zc = (float)((unsigned long)g.nz / 2.0 - 0.5);
    g.fod = (float)c.fod;
    g.fdd = (float)c.fdd;
    g.gamma = g.dv / (g.fdd * g.dx);
    g.inv_gamma_f = 1.0f / g.gamma;
    g.inv_gamma_d = 1.0 / (double)g.gamma;
    g.rs_wlog = RS_WLOG_DEFAULT;
    g.rs_tlog = RS_TLOG_DEFAULT;
    const float fdu = g.fdd / g.du;
    for (int p = 0; p < g.np; ++p) {
        const double phi = (p + start) * step;
        alpha[p] = (float)cos(phi);
        beta[p] = (float)sin(phi);
        vi[p] = make_float4((-beta[p] * g.dx) * fdu, (alpha[p] * g.dx) * fdu, alpha[p] * g.dx, beta[p] * g.dx);
    }
}

}  // namespace
}  // namespace tomo

using namespace tomo;

namespace {

// Restores the calling thread's current device when the call returns.
struct DeviceRestore {
    int prev = -1;
    ~DeviceRestore() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

tomo_status project_noalloc(const tomo_config_ct* cfg, int device, tomo_projector kind, const float* volume,
                            float* sinogram, cudaStream_t st, double padded) {
    NoallocAddrs a;
    tomo_status s = noalloc_setup(device, &a);
    if (s != TOMO_OK) return s;
    DevGeom g{};
    float alpha[TOMO_NOALLOC_MAX_VIEWS], beta[TOMO_NOALLOC_MAX_VIEWS];
    static thread_local float4 vi[TOMO_NOALLOC_MAX_VIEWS];
    noalloc_geometry(*cfg, g, alpha, beta, vi);
    const size_t np = (size_t)g.np;
    TOMO_CUDA_TRY(cudaMemcpyAsync(a.alpha, alpha, np * sizeof(float), cudaMemcpyHostToDevice, st));
    TOMO_CUDA_TRY(cudaMemcpyAsync(a.beta, beta, np * sizeof(float), cudaMemcpyHostToDevice, st));
    TOMO_CUDA_TRY(cudaMemcpyAsync(a.vi, vi, np * sizeof(float4), cudaMemcpyHostToDevice, st));
    g.alpha = a.alpha;
    g.beta = a.beta;
    g.vi = a.vi;
    // The array keeps the previous call's contents: clear the region this call uses so the
    // zero border of the padded volume holds, then copy the interior.
    TOMO_CUDA_TRY(cudaMemsetAsync(a.padded, 0, (size_t)padded * sizeof(float), st));
    cudaError_t e = launch_pad_volume(volume, TOMO_F32, a.padded, TOMO_F32, g.nx, g.ny, g.nz, st);
    if (e != cudaSuccess) return cuda_fail(e, "tomo_project_noalloc: pad");
    const OutView<void> out{sinogram, 0, (long)g.nu, (long)g.nu * g.nv};
    e = launch_rs_project(kind == TOMO_PROJ_RS ? 0 : 1, EPI_STORE, g, a.padded, TOMO_F32, out, TOMO_F32,
                          OutView<void>{nullptr, 0, 0, 0}, nullptr, st);
    if (e != cudaSuccess) return cuda_fail(e, "tomo_project_noalloc: rs_project_kernel");
    return TOMO_OK;
}

}  // namespace

extern "C" tomo_status tomo_project_noalloc(const tomo_config_ct* cfg, int device, tomo_projector kind,
                                           const float* volume, float* sinogram, void* stream) {
    TOMO_CHECK_ARG(cfg && volume && sinogram, "tomo_project_noalloc: null argument");
    TOMO_CHECK_ARG(kind == TOMO_PROJ_RS || kind == TOMO_PROJ_RS_UM,
                   "tomo_project_noalloc: only the RS projectors (TOMO_PROJ_RS, TOMO_PROJ_RS_UM)");
    TOMO_CHECK_ARG(device >= 0 && device < TOMO_NOALLOC_MAX_DEVICES, "tomo_project_noalloc: bad device index");
    TOMO_CHECK_ARG(cfg->projection_nb > 0 && cfg->u_detector_pixel_nb > 0 && cfg->v_detector_pixel_nb > 0 &&
                       cfg->x_volume_pixel_nb > 0 && cfg->y_volume_pixel_nb > 0 && cfg->z_volume_pixel_nb > 0,
                   "tomo_project_noalloc: sizes must be positive");
    TOMO_CHECK_ARG(cfg->den_start_angle != 0 && cfg->den_stop_angle != 0 && cfg->x_volume_size > 0 &&
                       cfg->u_detector_size > 0 && cfg->v_detector_size > 0 && cfg->fdd > 0 && cfg->fod > 0,
                   "tomo_project_noalloc: sizes and distances must be positive");
    TOMO_CHECK_ARG(cfg->projection_nb <= TOMO_NOALLOC_MAX_VIEWS,
                   "tomo_project_noalloc: more than 4096 views (the static table size)");
    const double padded = (double)(cfg->x_volume_pixel_nb + 2) * (cfg->y_volume_pixel_nb + 2) *
                          (cfg->z_volume_pixel_nb + 2);
    TOMO_CHECK_ARG(padded <= (double)TOMO_NOALLOC_MAX_PADDED_VOXELS,
                   "tomo_project_noalloc: (nx+2)*(ny+2)*(nz+2) exceeds the 8 Mi-voxel static scratch (32 MiB)");
    DeviceRestore restore;
    TOMO_CUDA_TRY(cudaGetDevice(&restore.prev));
    if (restore.prev != device) TOMO_CUDA_TRY(cudaSetDevice(device));
    cudaGetLastError();  // drop a stale non-sticky error so the launch checks report their own
    cudaStream_t st = (cudaStream_t)stream;
    if (st) {
        int sdev = -1;
        TOMO_CUDA_TRY(cudaStreamGetDevice(st, &sdev));
        TOMO_CHECK_ARG(sdev == device, "tomo_project_noalloc: the stream belongs to another device");
    }
    return project_noalloc(cfg, device, kind, volume, sinogram, st, padded);
}
