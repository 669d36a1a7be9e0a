// capi.cu -- the C-ABI of libtomogpi_b200.so: contexts (geometry set-up and device
// tables), operator dispatch, host-buffer forms, and the device-resident gradient solver.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "tomo_kernels.cuh"
#include "tomo_solver.cuh"

namespace tomo {

static thread_local std::string g_last_error = "no error";

void set_error(const std::string& msg) { g_last_error = msg; }

tomo_status cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? TOMO_ERR_NO_MEMORY : TOMO_ERR_CUDA;
}

size_t dtype_size(tomo_dtype t) { return t == TOMO_F32 ? 4 : 2; }

static bool valid_dtype(int t) { return t == TOMO_F32 || t == TOMO_BF16 || t == TOMO_F16; }

}  // namespace tomo

using namespace tomo;

struct tomo_context {
    int device = 0;
    tomo_config_ct cfg{};
    HostGeom hg;
    DevGeom g{};
    float* d_alpha = nullptr;
    float* d_beta = nullptr;
    float4* d_vi = nullptr;
    int* d_order = nullptr;
    unsigned* d_err = nullptr;
    int test_stall = 0;  // tomo_context_test_stall
    unsigned long long* d_count = nullptr;
    void* vpad[3] = {nullptr, nullptr, nullptr};  // padded volume per storage dtype
    void* spad[3] = {nullptr, nullptr, nullptr};  // padded sinogram per storage dtype
    float* adj_scratch = nullptr;                  // FP32 volume for adjoints into 16-bit outputs
    float* h_vol = nullptr;                        // device buffers of the host-buffer forms
    float* h_sino = nullptr;
    cudaStream_t host_stream = nullptr;
    std::mutex mu;
    tomo_tuning tuning{};
    int rs_in_layout[3] = {-1, -1, -1};  // layout the cached RS input buffer was sized for
    RsTexture tex;                       // TEX layout: layered array of the volume's type
    RsTexture vtex;                      // VI texture layout: layered array of the sinogram
    float* d_ramp = nullptr;             // ramp-filter taps for (ramp_over, ramp_cut)
    int ramp_half = 0, ramp_over = 0;
    double ramp_cut = -1.0;

    size_t nvox() const { return (size_t)hg.nx * hg.ny * hg.nz; }
    size_t nsino() const { return (size_t)hg.nu * hg.nv * hg.np; }
    size_t nvox_pad() const { return (size_t)(hg.nx + 2) * (hg.ny + 2) * (hg.nz + 2); }
    size_t nsino_pad() const { return (size_t)(hg.nu + 2) * (hg.nv + 2) * hg.np; }
};

struct tomo_solver {
    tomo_context* ctx = nullptr;
    int rs_layout = 0;
    int device = 0;  // kept so that destroy never touches the context
    tomo_gradient_params prm{};
    void* vpad = nullptr;    // padded projector input (storage dtype)
    void* vplain = nullptr;  // unpadded storage copy for the Siddon projector (16-bit storage only)
    void* spad = nullptr;    // padded residual sinogram (FP32 whatever the storage)
    float* dJ = nullptr;
    float* grad = nullptr;
    double* nrm = nullptr;    // [0] ||dJ||^2, [1] ||H dJ||^2, [2] ||L dJ||^2, [3] FP16 max|dJ|, [4] Huber
    double* partials = nullptr;  // per-block partials of ||H dJ||^2 (one per block of the projection)
    size_t npartials = 0;
    int reg_kind = 0;         // 0 generalised Gaussian, 1 Huber
    double huber_thr = 0.0;
    double gg_beta = 2.0;     // generalised-Gaussian shape parameter beta
    float* weights = nullptr;  // the solver's copy of the weighted gradient's weight sinogram (FP32)
    bool weighted = false;
    float* htmp = nullptr;    // Huber scratch volume (allocated when the Huber regulariser is chosen)
    double* state = nullptr;  // [0] alpha, [1] alpha_min
    double* alpha_log = nullptr;
    int log_cap = 0;
    int next_it = 1;
    RsTexture tex;   // TEX layout resources of this solver (storage type)
    RsTexture vtex;  // VI texture layout: the FP32 residual, one layer per view
    bool vi_tma = false;  // VI through TMA-staged windows: the residual is kept plain, not padded
    // host-buffer form
    float* d_vol = nullptr;
    void* d_real = nullptr;
    cudaStream_t copy_st = nullptr;  // the real sinogram's host copy, beside the first projection
    cudaEvent_t ev_vol = nullptr, ev_real = nullptr;
    bool real_pending = false;       // d_real is still being copied: ev_real marks its arrival
    // statistics
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_proj, ev_back;
    size_t ev_proj_used = 0, ev_back_used = 0;
    long long launches = 0;
};

namespace {
// An event pair from the solver's pool (created on first use, reused after a reset).
std::pair<cudaEvent_t, cudaEvent_t>* next_events(std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& pool, size_t& used) {
    if (used == pool.size()) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess) return nullptr;
        if (cudaEventCreate(&b) != cudaSuccess) {
            cudaEventDestroy(a);
            return nullptr;
        }
        pool.emplace_back(a, b);
    }
    return &pool[used++];
}
}  // namespace

namespace {

tomo_status ensure(void** p, size_t bytes, bool zero) {
    if (*p) return TOMO_OK;
    TOMO_CUDA_TRY(cudaMalloc(p, bytes));
    if (zero) TOMO_CUDA_TRY(cudaMemset(*p, 0, bytes));
    return TOMO_OK;
}

tomo_status set_device(const tomo_context* ctx) {
    TOMO_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaGetLastError();  // drop a stale non-sticky error so launch checks report their own
    return TOMO_OK;
}

tomo_status check_launch(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return cuda_fail(e, what);
    return TOMO_OK;
}

OutView<void> plain_view(void* p, const HostGeom& h) {
    return OutView<void>{p, 0, (long)h.nu, (long)h.nu * h.nv};
}

OutView<void> padded_view(void* p, const HostGeom& h) {
    const long W = h.nu + 2;
    return OutView<void>{p, W + 1, W, W * (h.nv + 2)};
}

// The VI backprojectors read a layered texture of the sinogram (one layer per view) unless
// that layout is off or the view count exceeds the layer limit.
bool vi_texture(const tomo_context* ctx) {
    return ctx->tuning.vi_layout == 1 && ctx->hg.np <= rs_tex_max_layers();
}

// The RS layout actually used: the texture layouts need an array layer per z slice (plus
// up to three), so depths beyond the device's layer limit use the cell layout instead; for
// 16-bit storage the texture packs slice pairs and HYBRID (slower there) is TEX; HYBRID
// indexes its quads with 32-bit integers, so larger volumes use TEX. MARCH (FP32 only)
// needs a layer per even face of x and of y and 32-bit quad indices, else it is HYBRID.
int effective_layout(int requested, tomo_dtype vdt, int nx, int ny, int nz) {
    if (requested == RS_LAYOUT_MARCH) {
        const double quads = (double)march_quads(nx, ny, nz) + (double)march_quads(ny, nx, nz);
        if (vdt == TOMO_F32 && march_even_faces(nx) + march_even_faces(ny) <= rs_tex_max_layers() &&
            quads < 4294967295.0)
            return RS_LAYOUT_MARCH;
        requested = RS_LAYOUT_HYBRID;
    }
    if (requested != RS_LAYOUT_TEX && requested != RS_LAYOUT_HYBRID) return requested;
    if (nz + 3 > rs_tex_max_layers()) return RS_LAYOUT_CELL8;
    if (requested == RS_LAYOUT_HYBRID &&
        (vdt != TOMO_F32 || (double)(nx + 1) * (ny + 1) * (nz + 1) >= 4294967295.0))
        return RS_LAYOUT_TEX;
    return requested;
}

// Projection of a device volume into an output view (shared by tomo_project and the solver).
tomo_status project_into(tomo_context* ctx, tomo_projector kind, const void* vol, tomo_dtype vdt, void* vpad,
                         const OutView<void>& out, tomo_dtype odt, int epi, const OutView<void>& real,
                         double* norm, cudaStream_t st) {
    const DevGeom& g = ctx->g;
    if (kind == TOMO_PROJ_RS || kind == TOMO_PROJ_RS_UM) {
        const int layout = effective_layout(ctx->tuning.rs_layout, vdt, g.nx, g.ny, g.nz);
        if (layout == RS_LAYOUT_TEX || layout == RS_LAYOUT_HYBRID || layout == RS_LAYOUT_MARCH) {
            const bool march = layout == RS_LAYOUT_MARCH;
            if (!ctx->tex.tex || ctx->tex.dt != vdt || ctx->tex.march != march) {  // the volume's type and layout
                if (ctx->tex.tex) {
                    TOMO_CUDA_TRY(cudaStreamSynchronize(st));
                    rs_tex_destroy(&ctx->tex);
                }
                cudaError_t e = march ? rs_march_tex_create(g.nx, g.ny, g.nz, &ctx->tex)
                                      : rs_vol_tex_create(g.nx, g.ny, g.nz, vdt, &ctx->tex, st);
                if (e != cudaSuccess) return cuda_fail(e, "rs texture");
            }
            if (check_launch(rs_tex_fill(vol, vdt, g.nx, g.ny, g.nz, ctx->tex, st), "rs texture fill") != TOMO_OK)
                return TOMO_ERR_CUDA;
        }
        if (layout != RS_LAYOUT_TEX &&  // HYBRID: the texture above plus its cell buffer
            check_launch(launch_rs_prepare(layout, vol, vdt, vpad, vdt, g.nx, g.ny, g.nz, st), "rs input") != TOMO_OK)
            return TOMO_ERR_CUDA;
        return check_launch(launch_rs_project(layout, kind == TOMO_PROJ_RS ? 0 : 1, epi, g, vpad, ctx->tex.tex, vdt, out,
                                              odt, real, norm, st),
                            "rs_project_kernel");
    }
    return check_launch(launch_siddon_project(kind == TOMO_PROJ_SIDDON_REF ? 1 : 0, epi, g, vol, vdt, out, odt, real,
                                              norm, ctx->d_err, st),
                        "siddon_project_kernel");
}

}  // namespace

extern "C" {

const char* tomo_last_error(void) { return g_last_error.c_str(); }

const char* tomo_version(void) { return "tomogpi_b200 0.1 (sm_100a)"; }

tomo_status tomo_context_create(const tomo_config_ct* cfg, int device, tomo_context** out) {
    TOMO_CHECK_ARG(cfg, "tomo_context_create: null argument");
    return tomo_context_create_views(cfg, device, 0, cfg->projection_nb, out);
}

tomo_status tomo_context_create_views(const tomo_config_ct* cfg, int device, int32_t view_begin, int32_t view_count,
                                      tomo_context** out) {
    TOMO_CHECK_ARG(cfg && out, "tomo_context_create: null argument");
    *out = nullptr;
    TOMO_CHECK_ARG(cfg->projection_nb > 0 && cfg->u_detector_pixel_nb > 0 && cfg->v_detector_pixel_nb > 0 &&
                       cfg->x_volume_pixel_nb > 0 && cfg->y_volume_pixel_nb > 0 && cfg->z_volume_pixel_nb > 0,
                   "tomo_context_create: sizes must be positive");
    TOMO_CHECK_ARG(cfg->den_start_angle != 0 && cfg->den_stop_angle != 0, "tomo_context_create: zero angle denominator");
    TOMO_CHECK_ARG(cfg->x_volume_size > 0 && cfg->u_detector_size > 0 && cfg->v_detector_size > 0 && cfg->fdd > 0 &&
                       cfg->fod > 0,
                   "tomo_context_create: sizes and distances must be positive");
    const double padded = (double)(cfg->x_volume_pixel_nb + 2) * (cfg->y_volume_pixel_nb + 2) *
                          (cfg->z_volume_pixel_nb + 2);
    TOMO_CHECK_ARG(padded < 2147483647.0, "tomo_context_create: volume too large for 32-bit voxel indexing");
    TOMO_CHECK_ARG(view_begin >= 0 && view_count >= 1 && (long)view_begin + view_count <= cfg->projection_nb,
                   "tomo_context_create_views: the view range must lie within the acquisition");
    int ndev = 0;
    TOMO_CUDA_TRY(cudaGetDeviceCount(&ndev));
    TOMO_CHECK_ARG(device >= 0 && device < ndev, "tomo_context_create: no such CUDA device");
    tomo_context* ctx = new tomo_context();
    ctx->device = device;
    // Measured on B200 (512^3, 512 views). RS: texture gathers 218 ms (FP32) / 156 ms (BF16),
    // 2x2x2 cells 269 / 155 ms, padded scalar loads 367 ms; at 1024^3 BF16 the texture wins
    // 2.49 s to 5.25 s (the cells' 8x footprint overflows L2). VI: 16 slices per thread 80 ms,
    // 32 slices 95 ms (64 registers halve residency), 64 slices 180 ms; the texture form of
    // the sinogram 111 ms.
    ctx->tuning.rs_layout = RS_LAYOUT_TEX;
    ctx->tuning.vi_zc = 1;
    ctx->tuning.vi_layout = 0;
    ctx->cfg = *cfg;
    derive_geometry(*cfg, ctx->hg);
    if (view_begin != 0 || view_count != cfg->projection_nb) select_views(ctx->hg, view_begin, view_count);
    const HostGeom& h = ctx->hg;
    auto fail = [&](tomo_status s) {
        tomo_context_destroy(ctx);
        return s;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "cudaSetDevice"));
    cudaError_t e = cudaMalloc(&ctx->d_alpha, sizeof(float) * h.np);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_beta, sizeof(float) * h.np);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_vi, sizeof(float4) * h.np);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_order, sizeof(int) * h.np);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_err, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_count, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemcpy(ctx->d_alpha, h.alpha.data(), sizeof(float) * h.np, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ctx->d_beta, h.beta.data(), sizeof(float) * h.np, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ctx->d_vi, h.vi.data(), sizeof(float4) * h.np, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(ctx->d_order, h.view_order.data(), sizeof(int) * h.np, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(ctx->d_err, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->host_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(e, "tomo_context_create"));
    fill_devgeom(h, ctx->d_alpha, ctx->d_beta, ctx->d_vi, ctx->g, ctx->d_order);
    *out = ctx;
    return TOMO_OK;
}

tomo_status tomo_context_destroy(tomo_context* ctx) {
    if (!ctx) return TOMO_OK;
    cudaSetDevice(ctx->device);
    if (ctx->host_stream) cudaStreamSynchronize(ctx->host_stream);
    cudaGetLastError();
    cudaFree(ctx->d_alpha);
    cudaFree(ctx->d_beta);
    cudaFree(ctx->d_vi);
    cudaFree(ctx->d_order);
    cudaFree(ctx->d_err);
    cudaFree(ctx->d_count);
    for (int i = 0; i < 3; ++i) {
        cudaFree(ctx->vpad[i]);
        cudaFree(ctx->spad[i]);
    }
    cudaFree(ctx->adj_scratch);
    rs_tex_destroy(&ctx->tex);
    rs_tex_destroy(&ctx->vtex);
    cudaFree(ctx->d_ramp);
    cudaFree(ctx->h_vol);
    cudaFree(ctx->h_sino);
    if (ctx->host_stream) cudaStreamDestroy(ctx->host_stream);
    delete ctx;
    return TOMO_OK;
}

tomo_status tomo_context_geometry(const tomo_context* ctx, float* scalars, float* alpha, float* beta) {
    TOMO_CHECK_ARG(ctx && scalars, "tomo_context_geometry: null argument");
    const HostGeom& h = ctx->hg;
    const float s[11] = {h.fod, h.fdd, h.gamma, h.du, h.dv, h.uc, h.vc, h.dx, h.xc, h.yc, h.zc};
    std::memcpy(scalars, s, sizeof(s));
    if (alpha) std::memcpy(alpha, h.alpha.data(), sizeof(float) * h.np);
    if (beta) std::memcpy(beta, h.beta.data(), sizeof(float) * h.np);
    return TOMO_OK;
}

tomo_status tomo_context_get_tuning(const tomo_context* ctx, tomo_tuning* out) {
    TOMO_CHECK_ARG(ctx && out, "tomo_context_get_tuning: null argument");
    *out = ctx->tuning;
    return TOMO_OK;
}

tomo_status tomo_context_rs_layout(const tomo_context* ctx, tomo_dtype dtype, int32_t* layout) {
    TOMO_CHECK_ARG(ctx && layout && valid_dtype(dtype), "tomo_context_rs_layout: bad argument");
    *layout = effective_layout(ctx->tuning.rs_layout, dtype, ctx->hg.nx, ctx->hg.ny, ctx->hg.nz);
    return TOMO_OK;
}

tomo_status tomo_context_set_tuning(tomo_context* ctx, const tomo_tuning* in) {
    TOMO_CHECK_ARG(ctx && in, "tomo_context_set_tuning: null argument");
    TOMO_CHECK_ARG(in->rs_layout >= RS_LAYOUT_PLAIN && in->rs_layout <= RS_LAYOUT_MARCH,
                   "tomo_context_set_tuning: rs_layout must be 0 (padded), 1 (cells), 2 (texture), 3 (hybrid) or 4 (march)");
    TOMO_CHECK_ARG(in->vi_zc == 0 || in->vi_zc == 1 || in->vi_zc == 2 || in->vi_zc == 4,
                   "tomo_context_set_tuning: vi_zc must be 1, 2 or 4");
    TOMO_CHECK_ARG(in->vi_layout >= 0 && in->vi_layout <= 2, "tomo_context_set_tuning: vi_layout must be 0, 1 or 2");
    TOMO_CHECK_ARG(rs_shape_valid(*in), "tomo_context_set_tuning: rs_warp_u must be 8, 16 or 32 and rs_tile_u 16, 32, "
                   "64 or 128, rs_warp_u <= rs_tile_u");
    ctx->tuning = *in;
    if (ctx->tuning.vi_zc == 0) ctx->tuning.vi_zc = 1;
    rs_shape_of(ctx->tuning, ctx->g);
    return TOMO_OK;
}

tomo_status tomo_project(tomo_context* ctx, tomo_projector kind, const void* volume, tomo_dtype volume_dtype,
                         void* sinogram, tomo_dtype sinogram_dtype, void* stream) {
    TOMO_CHECK_ARG(ctx && volume && sinogram, "tomo_project: null argument");
    TOMO_CHECK_ARG(kind >= TOMO_PROJ_RS && kind <= TOMO_PROJ_SIDDON, "tomo_project: unknown projector");
    TOMO_CHECK_ARG(valid_dtype(volume_dtype) && valid_dtype(sinogram_dtype), "tomo_project: unknown dtype");
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    void* vpad = nullptr;
    if (kind == TOMO_PROJ_RS || kind == TOMO_PROJ_RS_UM) {
        const int layout = effective_layout(ctx->tuning.rs_layout, volume_dtype, ctx->hg.nx, ctx->hg.ny, ctx->hg.nz);
        if (ctx->rs_in_layout[volume_dtype] != layout) {  // resize for a new layout
            cudaFree(ctx->vpad[volume_dtype]);
            ctx->vpad[volume_dtype] = nullptr;
        }
        s = ensure(&ctx->vpad[volume_dtype], rs_input_elems(layout, ctx->hg.nx, ctx->hg.ny, ctx->hg.nz) *
                                                 dtype_size(volume_dtype), true);
        if (s != TOMO_OK) return s;
        ctx->rs_in_layout[volume_dtype] = layout;
        vpad = ctx->vpad[volume_dtype];
    }
    return project_into(ctx, kind, volume, volume_dtype, vpad, plain_view(sinogram, ctx->hg), sinogram_dtype,
                        EPI_STORE, plain_view(nullptr, ctx->hg), nullptr, st);
}

tomo_status tomo_backproject(tomo_context* ctx, tomo_backprojector kind, const void* sinogram,
                             tomo_dtype sinogram_dtype, void* volume, tomo_dtype volume_dtype, void* stream) {
    TOMO_CHECK_ARG(ctx && volume && sinogram, "tomo_backproject: null argument");
    TOMO_CHECK_ARG(kind >= TOMO_BACK_VI && kind <= TOMO_BACK_FDK, "tomo_backproject: unknown backprojector");
    TOMO_CHECK_ARG(valid_dtype(volume_dtype) && valid_dtype(sinogram_dtype), "tomo_backproject: unknown dtype");
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const DevGeom& g = ctx->g;
    if ((kind == TOMO_BACK_VI || kind == TOMO_BACK_VI_UM) && vi_texture(ctx)) {
        if (!ctx->vtex.tex || ctx->vtex.dt != sinogram_dtype) {  // the texture holds the sinogram's type
            if (ctx->vtex.tex) {
                TOMO_CUDA_TRY(cudaStreamSynchronize(st));
                rs_tex_destroy(&ctx->vtex);
            }
            cudaError_t e = rs_tex_create(g.nu, g.nv, g.np, sinogram_dtype, &ctx->vtex);
            if (e != cudaSuccess) return cuda_fail(e, "vi texture");
        }
        if ((s = check_launch(rs_tex_fill(sinogram, sinogram_dtype, g.nu, g.nv, g.np, ctx->vtex, st), "vi texture fill")) !=
            TOMO_OK)
            return s;
        return check_launch(launch_vi_back_tex(kind == TOMO_BACK_VI_UM ? 1 : 0, g, ctx->vtex.tex, sinogram_dtype, volume,
                                               volume_dtype, 1.0f, st, ctx->tuning.vi_zc),
                            "vi_back_tex_kernel");
    }
    if ((kind == TOMO_BACK_VI || kind == TOMO_BACK_VI_UM) && ctx->tuning.vi_layout == 2 &&
        sinogram_dtype == TOMO_F32 && vi_tma_supported(g, sinogram))  // the caller's sinogram, no padded copy
        return check_launch(launch_vi_back_tma(kind == TOMO_BACK_VI_UM ? 1 : 0, g, (const float*)sinogram, volume,
                                               volume_dtype, 1.0f, ctx->d_err, st, ctx->test_stall),
                            "vi_back_tma_kernel");
    if (kind == TOMO_BACK_FDK) {
        s = ensure(&ctx->spad[sinogram_dtype], ctx->nsino_pad() * dtype_size(sinogram_dtype), true);
        if (s != TOMO_OK) return s;
        void* sp = ctx->spad[sinogram_dtype];
        if ((s = check_launch(launch_pad_sinogram(sinogram, sinogram_dtype, sp, sinogram_dtype, g.nu, g.nv, g.np, st),
                              "pad sinogram")) != TOMO_OK)
            return s;
        return check_launch(launch_vi_fdk(g, sp, sinogram_dtype, volume, volume_dtype, st), "vi_back_kernel (FDK)");
    }
    if (kind == TOMO_BACK_VI || kind == TOMO_BACK_VI_UM) {
        s = ensure(&ctx->spad[sinogram_dtype], ctx->nsino_pad() * dtype_size(sinogram_dtype), true);
        if (s != TOMO_OK) return s;
        void* sp = ctx->spad[sinogram_dtype];
        if ((s = check_launch(launch_pad_sinogram(sinogram, sinogram_dtype, sp, sinogram_dtype, g.nu, g.nv, g.np, st),
                              "pad sinogram")) != TOMO_OK)
            return s;
        return check_launch(launch_vi_back(kind == TOMO_BACK_VI_UM ? 1 : 0, g, sp, sinogram_dtype, volume, volume_dtype,
                                           1.0f, st, ctx->tuning.vi_zc),
                            "vi_back_kernel");
    }
    // Matched transposes: FP32 scatter, converted if the output is 16-bit.
    float* acc = (float*)volume;
    if (volume_dtype != TOMO_F32) {
        s = ensure((void**)&ctx->adj_scratch, ctx->nvox() * sizeof(float), false);
        if (s != TOMO_OK) return s;
        acc = ctx->adj_scratch;
    }
    TOMO_CUDA_TRY(cudaMemsetAsync(acc, 0, ctx->nvox() * sizeof(float), st));
    cudaError_t e;
    if (kind == TOMO_BACK_RS_ADJOINT || kind == TOMO_BACK_RS_UM_ADJOINT)
        e = launch_rs_adjoint(kind == TOMO_BACK_RS_ADJOINT ? 0 : 1, g, sinogram, sinogram_dtype, acc, st);
    else
        e = launch_siddon_adjoint(0, g, sinogram, sinogram_dtype, acc, ctx->d_err, st);
    if ((s = check_launch(e, "adjoint kernel")) != TOMO_OK) return s;
    if (volume_dtype != TOMO_F32)
        return check_launch(launch_convert(acc, TOMO_F32, volume, volume_dtype, ctx->nvox(), st), "convert");
    return TOMO_OK;
}

tomo_status tomo_ramp_filter(tomo_context* ctx, const void* sinogram, tomo_dtype sinogram_dtype, float* out,
                             int32_t oversampling, double cutoff, void* stream) {
    TOMO_CHECK_ARG(ctx && sinogram && out && valid_dtype(sinogram_dtype), "tomo_ramp_filter: bad argument");
    TOMO_CHECK_ARG(oversampling >= 2 && oversampling % 2 == 0 && cutoff > 0.0 && cutoff <= 1.0,
                   "tomo_ramp_filter: oversampling must be even and >= 2, cutoff in (0, 1]");
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const HostGeom& h = ctx->hg;
    if (!ctx->d_ramp || ctx->ramp_over != oversampling || ctx->ramp_cut != cutoff) {
        std::vector<float> taps;
        const int half = ramp_taps(h.nu, oversampling, cutoff, (double)h.du, taps);
        TOMO_CUDA_TRY(cudaStreamSynchronize(st));  // a previous filter may still read the old taps
        cudaFree(ctx->d_ramp);
        ctx->d_ramp = nullptr;
        TOMO_CUDA_TRY(cudaMalloc(&ctx->d_ramp, sizeof(float) * taps.size()));
        TOMO_CUDA_TRY(cudaMemcpy(ctx->d_ramp, taps.data(), sizeof(float) * taps.size(), cudaMemcpyHostToDevice));
        ctx->ramp_half = half;
        ctx->ramp_over = oversampling;
        ctx->ramp_cut = cutoff;
    }
    return check_launch(launch_ramp_filter(sinogram, sinogram_dtype, out, ctx->d_ramp, ctx->ramp_half, h.nu, h.nv, h.np, st),
                        "ramp_filter_kernel");
}

tomo_status tomo_ramp_filter_host(tomo_context* ctx, const float* sinogram, float* out, int32_t oversampling,
                                  double cutoff) {
    TOMO_CHECK_ARG(ctx && sinogram && out, "tomo_ramp_filter_host: null argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    if ((s = ensure(&ctx->spad[TOMO_F32], ctx->nsino_pad() * sizeof(float), true)) != TOMO_OK) return s;
    if ((s = ensure((void**)&ctx->h_sino, ctx->nsino() * sizeof(float), false)) != TOMO_OK) return s;
    cudaStream_t st = ctx->host_stream;
    float* filt = (float*)ctx->spad[TOMO_F32];  // scratch of at least nsino floats
    TOMO_CUDA_TRY(cudaMemcpyAsync(ctx->h_sino, sinogram, ctx->nsino() * sizeof(float), cudaMemcpyHostToDevice, st));
    if ((s = tomo_ramp_filter(ctx, ctx->h_sino, TOMO_F32, filt, oversampling, cutoff, st)) != TOMO_OK) return s;
    TOMO_CUDA_TRY(cudaMemcpyAsync(out, filt, ctx->nsino() * sizeof(float), cudaMemcpyDeviceToHost, st));
    TOMO_CUDA_TRY(cudaStreamSynchronize(st));
    return TOMO_OK;
}

tomo_status tomo_project_host(tomo_context* ctx, tomo_projector kind, const float* volume, float* sinogram) {
    TOMO_CHECK_ARG(ctx && volume && sinogram, "tomo_project_host: null argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    if ((s = ensure((void**)&ctx->h_vol, ctx->nvox() * sizeof(float), false)) != TOMO_OK) return s;
    if ((s = ensure((void**)&ctx->h_sino, ctx->nsino() * sizeof(float), false)) != TOMO_OK) return s;
    cudaStream_t st = ctx->host_stream;
    TOMO_CUDA_TRY(cudaMemcpyAsync(ctx->h_vol, volume, ctx->nvox() * sizeof(float), cudaMemcpyHostToDevice, st));
    if ((s = tomo_project(ctx, kind, ctx->h_vol, TOMO_F32, ctx->h_sino, TOMO_F32, st)) != TOMO_OK) return s;
    TOMO_CUDA_TRY(cudaMemcpyAsync(sinogram, ctx->h_sino, ctx->nsino() * sizeof(float), cudaMemcpyDeviceToHost, st));
    TOMO_CUDA_TRY(cudaStreamSynchronize(st));
    return TOMO_OK;
}

tomo_status tomo_backproject_host(tomo_context* ctx, tomo_backprojector kind, const float* sinogram, float* volume) {
    TOMO_CHECK_ARG(ctx && volume && sinogram, "tomo_backproject_host: null argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    if ((s = ensure((void**)&ctx->h_vol, ctx->nvox() * sizeof(float), false)) != TOMO_OK) return s;
    if ((s = ensure((void**)&ctx->h_sino, ctx->nsino() * sizeof(float), false)) != TOMO_OK) return s;
    cudaStream_t st = ctx->host_stream;
    TOMO_CUDA_TRY(cudaMemcpyAsync(ctx->h_sino, sinogram, ctx->nsino() * sizeof(float), cudaMemcpyHostToDevice, st));
    if ((s = tomo_backproject(ctx, kind, ctx->h_sino, TOMO_F32, ctx->h_vol, TOMO_F32, st)) != TOMO_OK) return s;
    TOMO_CUDA_TRY(cudaMemcpyAsync(volume, ctx->h_vol, ctx->nvox() * sizeof(float), cudaMemcpyDeviceToHost, st));
    TOMO_CUDA_TRY(cudaStreamSynchronize(st));
    return TOMO_OK;
}

tomo_status tomo_count_samples(tomo_context* ctx, tomo_projector kind, unsigned long long* out, void* stream) {
    TOMO_CHECK_ARG(ctx && out, "tomo_count_samples: null argument");
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    TOMO_CUDA_TRY(cudaMemsetAsync(ctx->d_count, 0, sizeof(unsigned long long), st));
    cudaError_t e;
    if (kind == TOMO_PROJ_RS || kind == TOMO_PROJ_RS_UM)
        e = launch_rs_count(kind == TOMO_PROJ_RS ? 0 : 1, ctx->g, ctx->d_count, st);
    else
        e = launch_siddon_count(kind == TOMO_PROJ_SIDDON_REF ? 1 : 0, ctx->g, ctx->d_count, ctx->d_err, st);
    if ((s = check_launch(e, "count kernel")) != TOMO_OK) return s;
    TOMO_CUDA_TRY(cudaMemcpyAsync(out, ctx->d_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    TOMO_CUDA_TRY(cudaStreamSynchronize(st));
    return TOMO_OK;
}

tomo_status tomo_context_errors(tomo_context* ctx, unsigned* bits, int clear) {
    TOMO_CHECK_ARG(ctx && bits, "tomo_context_errors: null argument");
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    TOMO_CUDA_TRY(cudaMemcpy(bits, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (clear) TOMO_CUDA_TRY(cudaMemset(ctx->d_err, 0, sizeof(unsigned)));
    return TOMO_OK;
}

tomo_status tomo_context_test_stall(tomo_context* ctx, int enable) {
    TOMO_CHECK_ARG(ctx, "tomo_context_test_stall: null argument");
    ctx->test_stall = enable != 0;
    return TOMO_OK;
}

// ------------------------------------------------------------------------------------
// Gradient solver.
// ------------------------------------------------------------------------------------
tomo_status tomo_solver_create(tomo_context* ctx, const tomo_gradient_params* prm, tomo_solver** out) {
    TOMO_CHECK_ARG(ctx && prm && out, "tomo_solver_create: null argument");
    *out = nullptr;
    TOMO_CHECK_ARG(valid_dtype(prm->storage), "tomo_solver_create: unknown storage dtype");
    TOMO_CHECK_ARG(prm->projector >= TOMO_PROJ_RS && prm->projector <= TOMO_PROJ_SIDDON,
                   "tomo_solver_create: unknown projector");
    TOMO_CHECK_ARG(prm->backprojector == TOMO_BACK_VI || prm->backprojector == TOMO_BACK_VI_UM,
                   "tomo_solver_create: the gradient loop backprojects with VI");
    TOMO_CHECK_ARG(prm->gradient_iteration_nb >= 0, "tomo_solver_create: negative iteration count");
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    tomo_solver* sv = new tomo_solver();
    sv->ctx = ctx;
    sv->device = ctx->device;
    sv->rs_layout = effective_layout(ctx->tuning.rs_layout, prm->storage, ctx->hg.nx, ctx->hg.ny, ctx->hg.nz);
    sv->prm = *prm;
    sv->log_cap = prm->gradient_iteration_nb > 0 ? prm->gradient_iteration_nb : 1;
    const size_t es = dtype_size(prm->storage);
    auto alloc = [&](void** p, size_t bytes, bool zero) -> bool {
        if (cudaMalloc(p, bytes) != cudaSuccess) return false;
        if (zero && cudaMemset(*p, 0, bytes) != cudaSuccess) return false;
        return true;
    };
    bool ok = alloc(&sv->vpad, rs_input_elems(sv->rs_layout, ctx->hg.nx, ctx->hg.ny, ctx->hg.nz) * es, true) && alloc(&sv->spad, ctx->nsino_pad() * sizeof(float), true) &&
              alloc((void**)&sv->dJ, ctx->nvox() * sizeof(float), false) &&
              alloc((void**)&sv->grad, ctx->nvox() * sizeof(float), false) &&
              alloc((void**)&sv->nrm, 8 * sizeof(double), true) && alloc((void**)&sv->state, 4 * sizeof(double), true) &&
              alloc((void**)&sv->alpha_log, sv->log_cap * sizeof(double), true);
    if (ok && prm->storage != TOMO_F32 && (prm->projector == TOMO_PROJ_SIDDON || prm->projector == TOMO_PROJ_SIDDON_REF))
        ok = alloc(&sv->vplain, ctx->nvox() * es, false);
    if (ok) {  // the norm projection's per-block partials (the launch shape is fixed by now)
        const bool sid = prm->projector == TOMO_PROJ_SIDDON || prm->projector == TOMO_PROJ_SIDDON_REF;
        sv->npartials = sid ? siddon_grid_blocks(ctx->g) : rs_grid_blocks(sv->rs_layout, ctx->g);
        // the volume norms use the same buffer (two sums of reduce_blocks partials each)
        sv->npartials = std::max(sv->npartials, 2 * reduce_blocks(ctx->hg.nx, ctx->hg.ny, ctx->hg.nz));
        ok = alloc((void**)&sv->partials, sv->npartials * sizeof(double), false);
    }
    if (ok && (sv->rs_layout == RS_LAYOUT_TEX || sv->rs_layout == RS_LAYOUT_HYBRID))
        ok = rs_vol_tex_create(ctx->hg.nx, ctx->hg.ny, ctx->hg.nz, prm->storage, &sv->tex, 0) == cudaSuccess &&
             cudaStreamSynchronize(0) == cudaSuccess;  // creation only: the zero layers are written
    if (ok && sv->rs_layout == RS_LAYOUT_MARCH)
        ok = rs_march_tex_create(ctx->hg.nx, ctx->hg.ny, ctx->hg.nz, &sv->tex) == cudaSuccess;
    if (ok && vi_texture(ctx))
        ok = rs_tex_create(ctx->hg.nu, ctx->hg.nv, ctx->hg.np, TOMO_F32, &sv->vtex, true) == cudaSuccess;
    if (ok) sv->vi_tma = ctx->tuning.vi_layout == 2 && vi_tma_supported(ctx->g, sv->spad);
    if (!ok) {
        cudaGetLastError();
        tomo_solver_destroy(sv);
        set_error("tomo_solver_create: device allocation failed");
        return TOMO_ERR_NO_MEMORY;
    }
    const double init[2] = {0.0, -0.0347711};  // alpha, alpha_min (Iter3D_Algo_Gradient.cu:61-62)
    if (cudaMemcpy(sv->state, init, sizeof(init), cudaMemcpyHostToDevice) != cudaSuccess) {
        tomo_solver_destroy(sv);
        return cuda_fail(cudaGetLastError(), "tomo_solver_create");
    }
    *out = sv;
    return TOMO_OK;
}

tomo_status tomo_solver_destroy(tomo_solver* sv) {
    if (!sv) return TOMO_OK;
    cudaSetDevice(sv->device);
    cudaFree(sv->vpad);
    cudaFree(sv->vplain);
    cudaFree(sv->spad);
    cudaFree(sv->dJ);
    cudaFree(sv->grad);
    cudaFree(sv->htmp);
    cudaFree(sv->nrm);
    cudaFree(sv->partials);
    cudaFree(sv->state);
    cudaFree(sv->alpha_log);
    cudaFree(sv->d_vol);
    cudaFree(sv->d_real);
    if (sv->copy_st) cudaStreamDestroy(sv->copy_st);
    if (sv->ev_vol) cudaEventDestroy(sv->ev_vol);
    if (sv->ev_real) cudaEventDestroy(sv->ev_real);
    cudaFree(sv->weights);
    rs_tex_destroy(&sv->tex);
    rs_tex_destroy(&sv->vtex);
    for (auto& e : sv->ev_proj) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    for (auto& e : sv->ev_back) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    cudaGetLastError();
    delete sv;
    return TOMO_OK;
}

tomo_status tomo_solver_set_regularizer(tomo_solver* sv, int32_t kind, double huber_threshold) {
    TOMO_CHECK_ARG(sv, "tomo_solver_set_regularizer: null solver");
    TOMO_CHECK_ARG(kind == TOMO_REG_GG || kind == TOMO_REG_HUBER, "tomo_solver_set_regularizer: unknown regulariser");
    TOMO_CHECK_ARG(kind != TOMO_REG_HUBER || (std::isfinite(huber_threshold) && huber_threshold >= 0.0),
                   "tomo_solver_set_regularizer: the Huber threshold must be finite and non-negative");
    if (kind == TOMO_REG_HUBER && !sv->htmp) {
        TOMO_CUDA_TRY(cudaSetDevice(sv->device));
        if (cudaMalloc((void**)&sv->htmp, sv->ctx->nvox() * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            sv->htmp = nullptr;
            set_error("tomo_solver_set_regularizer: device allocation failed");
            return TOMO_ERR_NO_MEMORY;
        }
    }
    sv->reg_kind = kind;
    sv->huber_thr = huber_threshold;
    return TOMO_OK;
}

tomo_status tomo_solver_set_gg_beta(tomo_solver* sv, double beta) {
    TOMO_CHECK_ARG(sv, "tomo_solver_set_gg_beta: null solver");
    TOMO_CHECK_ARG(std::isfinite(beta) && beta >= 1.0, "tomo_solver_set_gg_beta: beta must be finite and at least 1");
    sv->gg_beta = beta;
    return TOMO_OK;
}

tomo_status tomo_solver_set_weights(tomo_solver* sv, const float* weights, int32_t host, void* stream) {
    TOMO_CHECK_ARG(sv, "tomo_solver_set_weights: null solver");
    TOMO_CHECK_ARG(sv->next_it == 1, "tomo_solver_set_weights: the weights are set before the first iteration");
    tomo_status s = set_device(sv->ctx);
    if (s != TOMO_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    if (weights) {  // Iter3D_Algo_Gradient.cu:243-248: the loop holds its own weight sinogram
        const size_t bytes = sv->ctx->nsino() * sizeof(float);
        if ((s = ensure((void**)&sv->weights, bytes, false)) != TOMO_OK) return s;
        if (host) {
            TOMO_CUDA_TRY(cudaMemcpy(sv->weights, weights, bytes, cudaMemcpyHostToDevice));
        } else {
            TOMO_CUDA_TRY(cudaMemcpyAsync(sv->weights, weights, bytes, cudaMemcpyDeviceToDevice, st));
        }
    }
    // alpha_min starts at -999999999999 in the weighted loop (:257), at -0.0347711 in the simple one (:62)
    if ((s = check_launch(launch_fill_double(sv->state + 1, 1, weights ? -999999999999.0 : -0.0347711, st),
                          "tomo_solver_set_weights")) != TOMO_OK)
        return s;
    sv->weighted = weights != nullptr;
    return TOMO_OK;
}

static tomo_status solver_run(tomo_solver* sv, float* volume, const void* real_sinogram, int32_t first, int32_t count,
                              int phases, void* stream) {
    TOMO_CHECK_ARG(sv && volume && real_sinogram, "tomo_solver_iterate: null argument");
    TOMO_CHECK_ARG(first >= 1 && count >= 0 && first + count - 1 <= sv->log_cap,
                   "tomo_solver_iterate: iteration range outside [1, gradient_iteration_nb]");
    tomo_context* ctx = sv->ctx;
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const DevGeom& g = ctx->g;
    const HostGeom& h = ctx->hg;
    const tomo_gradient_params& P = sv->prm;
    const tomo_dtype sd = P.storage;
    const tomo_dtype rd = P.real_sinogram_f32 ? TOMO_F32 : sd;  // the real sinogram's type
    const bool reg = P.regularization_parameter != 0.0;
    const bool huber = sv->reg_kind == 1;
    const double beta = sv->gg_beta;
    // dJ->addVolume(djReg, beta*lambda) with the regulariser's float lambda (GG..._CPU.cu:205).
    const float w = (float)(beta * (double)(float)P.regularization_parameter);
    const OutView<void> resid = sv->vi_tma ? plain_view(sv->spad, h) : padded_view(sv->spad, h);
    const OutView<void> realv = plain_view(const_cast<void*>(real_sinogram), h);
    const bool siddon = P.projector == TOMO_PROJ_SIDDON || P.projector == TOMO_PROJ_SIDDON_REF;
    const size_t nparts = siddon ? siddon_grid_blocks(g) : rs_grid_blocks(sv->rs_layout, g);
    TOMO_CHECK_ARG(nparts <= sv->npartials,
                   "tomo_solver_iterate: the context's launch shape changed after the solver was created");
    // FP16 storage: max|dJ| (nrm[3] as FP32 bits) scales dJ into FP16's range before it is
    // stored for the projection of the step size (fp16_scale); other types need no guard.
    unsigned* amax = sd == TOMO_F16 ? reinterpret_cast<unsigned*>(sv->nrm + 3) : nullptr;
    // Optional CUDA-event timing of the operator launches on `st`.
    auto tic = [&](bool proj) -> std::pair<cudaEvent_t, cudaEvent_t>* {
        if (!sv->timing) return nullptr;
        auto* e = proj ? next_events(sv->ev_proj, sv->ev_proj_used) : next_events(sv->ev_back, sv->ev_back_used);
        if (e) cudaEventRecord(e->first, st);
        return e;
    };
    auto toc = [&](std::pair<cudaEvent_t, cudaEvent_t>* e) {
        if (e) cudaEventRecord(e->second, st);
    };
    // RS input from an FP32 volume in the storage type: the texture (TEX, HYBRID) and/or the
    // padded / cell buffer (PLAIN, CELL8, HYBRID).
    auto rs_input = [&](const float* src, const unsigned* am) -> tomo_status {
        tomo_status r;
        if (sv->tex.tex &&
            (r = check_launch(rs_tex_fill(src, TOMO_F32, g.nx, g.ny, g.nz, sv->tex, st, am), "rs texture fill")) != TOMO_OK)
            return r;
        if (sv->rs_layout != RS_LAYOUT_TEX)
            return check_launch(launch_rs_prepare(sv->rs_layout, src, TOMO_F32, sv->vpad, sd, g.nx, g.ny, g.nz, st, am),
                                "rs input");
        return TOMO_OK;
    };
    for (int it = first; it < first + count; ++it) {
        if (phases & TOMO_PHASE_GRADIENT) {  // residual, backprojection: dJ = -2 H^T (g - H f)
            // ghat = H f, r = g - ghat (Iter3D_Algo_Gradient.cu:80-85), written into the padded residual.
            const void* pin = volume;
            tomo_dtype pdt = TOMO_F32;
            if (siddon && sd != TOMO_F32) {
                if ((s = check_launch(launch_convert(volume, TOMO_F32, sv->vplain, sd, ctx->nvox(), st), "convert")) != TOMO_OK)
                    return s;
                pin = sv->vplain;
                pdt = sd;
            }
            if (!siddon) pdt = sd;  // the pad kernel converts the FP32 iterate to the storage type
            if (!siddon && sv->real_pending) {
                // the real sinogram is still on its way (host-buffer form): project into the
                // residual buffer, then form r = g - Hf once it has arrived (the same arithmetic)
                sv->real_pending = false;
                if ((s = rs_input(volume, nullptr)) != TOMO_OK) return s;
                auto* e = tic(true);
                if ((s = check_launch(launch_rs_project(sv->rs_layout, P.projector == TOMO_PROJ_RS ? 0 : 1, EPI_STORE, g,
                                                        sv->vpad, sv->tex.tex, sd, resid, TOMO_F32, realv, nullptr, st),
                                      "rs projection")) != TOMO_OK)
                    return s;
                toc(e);
                TOMO_CUDA_TRY(cudaStreamWaitEvent(st, sv->ev_real, 0));
                if ((s = check_launch(launch_sino_residual(resid.as<float>(), real_sinogram, rd, g.nu, g.nv, g.np, st),
                                      "residual")) != TOMO_OK)
                    return s;
                sv->launches += 3;
            } else if (!siddon) {
                if ((s = rs_input(volume, nullptr)) != TOMO_OK) return s;
                auto* e = tic(true);
                if ((s = check_launch(launch_rs_project(sv->rs_layout, P.projector == TOMO_PROJ_RS ? 0 : 1, EPI_RESIDUAL, g,
                                                        sv->vpad, sv->tex.tex, sd,
                                                        resid, TOMO_F32, realv, nullptr, st, rd),
                                      "rs residual")) != TOMO_OK)
                    return s;
                toc(e);
                sv->launches += 2;
            } else {
                auto* e = tic(true);
                if ((s = check_launch(launch_siddon_project(P.projector == TOMO_PROJ_SIDDON_REF ? 1 : 0, EPI_RESIDUAL, g, pin,
                                                            pdt, resid, TOMO_F32, realv, nullptr, ctx->d_err, st, rd),
                                      "siddon residual")) != TOMO_OK)
                    return s;
                toc(e);
                sv->launches += (pin != volume) ? 2 : 1;
            }
            // the weighted gradient: r = r * w (Iter3D_Algo_Gradient.cu:289)
            if (sv->weighted) {
                if ((s = check_launch(launch_sino_weight(resid.as<float>(), sv->weights, g.nu, g.nv, g.np, st),
                                      "weights")) != TOMO_OK)
                    return s;
                sv->launches += 1;
            }
            // dJ = -2 H^T r (:106, :111)
            {
                const int um = P.backprojector == TOMO_BACK_VI_UM ? 1 : 0;
                if (sv->vtex.tex &&
                    (s = check_launch(tex_fill_from_padded((const float*)sv->spad, g.nu, g.nv, g.np, sv->vtex, st),
                                      "vi texture fill")) != TOMO_OK)
                    return s;
                auto* e = tic(false);
                if ((s = check_launch(sv->vtex.tex ? launch_vi_back_tex(um, g, sv->vtex.tex, TOMO_F32, sv->dJ, TOMO_F32, -2.0f,
                                                                        st, ctx->tuning.vi_zc)
                                      : sv->vi_tma ? launch_vi_back_tma(um, g, (const float*)sv->spad, sv->dJ, TOMO_F32, -2.0f,
                                                                        ctx->d_err, st)
                                                   : launch_vi_back(um, g, sv->spad, TOMO_F32, sv->dJ, TOMO_F32, -2.0f, st,
                                                                    ctx->tuning.vi_zc),
                                      "vi back")) != TOMO_OK)
                    return s;
                toc(e);
                sv->launches += 1;
            }
        }
        if (phases & TOMO_PHASE_NORMS) {  // regulariser on dJ, norms for the step size
            // GG: dJ += beta*lambda * L(L f) for beta = 2, beta*lambda * L(sign(f) |f|^(beta-1))
            // otherwise (GG..._CPU.cu:170-205); Huber: dJ += lambda * L(psi'(L f))
            // (HuberRegularizer_CPU.cu:211-228)
            if (reg) {
                if ((s = check_launch(!huber && beta != 2.0
                                          ? launch_gg_abspow(volume, sv->grad, ctx->nvox(), beta - 1.0, st)
                                          : launch_laplacian(volume, sv->grad, g.nx, g.ny, g.nz, st),
                                      "regulariser gradient")) != TOMO_OK)
                    return s;
                if ((s = check_launch(huber ? launch_huber_axpy(sv->grad, sv->dJ, (float)P.regularization_parameter,
                                                                sv->huber_thr, g.nx, g.ny, g.nz, st)
                                            : launch_laplacian_axpy(sv->grad, sv->dJ, w, g.nx, g.ny, g.nz, st),
                                      "regulariser axpy")) != TOMO_OK)
                    return s;
                sv->launches += 2;
            }
            const bool opt = it < P.optimal_step_iteration_nb;
            if (opt) {
                TOMO_CUDA_TRY(cudaMemsetAsync(sv->nrm, 0, 5 * sizeof(double), st));
                if ((s = check_launch(launch_laplacian_norm(sv->dJ, sv->nrm, g.nx, g.ny, g.nz, reg && !huber ? 1 : 0, st,
                                                            amax, beta, sv->partials),
                                      "norms")) !=
                    TOMO_OK)
                    return s;
                sv->launches += 1;
                if (reg && huber) {  // normdJProjReg = sum |L(L(psi''(L f) dJ)) dJ| (:230-242)
                    if ((s = check_launch(launch_huber_norm(sv->grad, sv->dJ, sv->htmp, sv->huber_thr, sv->nrm + 4, g.nx,
                                                            g.ny, g.nz, st, sv->partials),
                                          "huber norm")) != TOMO_OK)
                        return s;
                    sv->launches += 2;
                }
                // ||H dJ||^2 (:142, :146)
                if (!siddon) {
                    if ((s = rs_input(sv->dJ, amax)) != TOMO_OK) return s;
                    auto* e = tic(true);
                    if ((s = check_launch(launch_rs_project(sv->rs_layout, P.projector == TOMO_PROJ_RS ? 0 : 1, EPI_NORM, g,
                                                            sv->vpad, sv->tex.tex, sd,
                                                            resid, sd, realv, sv->partials, st),
                                          "rs norm")) != TOMO_OK)
                        return s;
                    toc(e);
                    sv->launches += 2;
                } else {
                    const void* din = sv->dJ;
                    tomo_dtype ddt = TOMO_F32;
                    if (sd != TOMO_F32) {
                        if ((s = check_launch(launch_convert(sv->dJ, TOMO_F32, sv->vplain, sd, ctx->nvox(), st, amax),
                                              "convert")) !=
                            TOMO_OK)
                            return s;
                        din = sv->vplain;
                        ddt = sd;
                    }
                    auto* e = tic(true);
                    if ((s = check_launch(launch_siddon_project(P.projector == TOMO_PROJ_SIDDON_REF ? 1 : 0, EPI_NORM, g, din,
                                                                ddt, resid, sd, realv, sv->partials, ctx->d_err, st),
                                          "siddon norm")) != TOMO_OK)
                        return s;
                    toc(e);
                    sv->launches += (din != sv->dJ) ? 2 : 1;
                }
                // nrm[1] = the projection's per-block partials added in a fixed order
                if ((s = check_launch(launch_sum_partials(sv->partials, nparts, sv->nrm + 1, st),
                                      "norm partials")) != TOMO_OK)
                    return s;
                sv->launches += 1;
            }
        }
        if (phases & TOMO_PHASE_UPDATE) {  // step size, f += alpha dJ
            if ((s = check_launch(launch_gd_alpha(sv->nrm, sv->state, sv->alpha_log, it, P.optimal_step_iteration_nb,
                                                  P.regularization_parameter, reg ? (huber ? 2 : 1) : 0, st, amax, beta),
                                  "alpha")) != TOMO_OK)
                return s;
            if ((s = check_launch(launch_gd_update(volume, sv->dJ, sv->state, ctx->nvox(), P.positivity, st), "update")) !=
                TOMO_OK)
                return s;
            sv->launches += 2;
        }
    }
    if (phases & TOMO_PHASE_UPDATE) sv->next_it = first + count;
    return TOMO_OK;
}

tomo_status tomo_solver_iterate(tomo_solver* sv, float* volume, const void* real_sinogram, int32_t first, int32_t count,
                                void* stream) {
    return solver_run(sv, volume, real_sinogram, first, count,
                      TOMO_PHASE_GRADIENT | TOMO_PHASE_NORMS | TOMO_PHASE_UPDATE, stream);
}

tomo_status tomo_solver_phase(tomo_solver* sv, float* volume, const void* real_sinogram, int32_t iteration,
                              int32_t phases, void* stream) {
    TOMO_CHECK_ARG(sv, "tomo_solver_phase: null solver");
    TOMO_CHECK_ARG(phases > 0 && (phases & ~(TOMO_PHASE_GRADIENT | TOMO_PHASE_NORMS | TOMO_PHASE_UPDATE)) == 0,
                   "tomo_solver_phase: unknown phase bits");
    return solver_run(sv, volume, real_sinogram ? real_sinogram : (const void*)volume, iteration, 1, phases, stream);
}

tomo_status tomo_solver_buffers(tomo_solver* sv, float** dJ, double** norms) {
    TOMO_CHECK_ARG(sv && dJ && norms, "tomo_solver_buffers: null argument");
    *dJ = sv->dJ;
    *norms = sv->nrm;
    return TOMO_OK;
}

tomo_status tomo_solver_iterate_host(tomo_solver* sv, float* volume, const void* real_sinogram, int32_t first,
                                     int32_t count, void* stream) {
    TOMO_CHECK_ARG(sv && volume && real_sinogram, "tomo_solver_iterate_host: null argument");
    tomo_context* ctx = sv->ctx;
    tomo_status s = set_device(ctx);
    if (s != TOMO_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t rb = ctx->nsino() * dtype_size(sv->prm.real_sinogram_f32 ? TOMO_F32 : sv->prm.storage);
    if ((s = ensure((void**)&sv->d_vol, ctx->nvox() * sizeof(float), false)) != TOMO_OK) return s;
    if ((s = ensure(&sv->d_real, rb, false)) != TOMO_OK) return s;
    TOMO_CUDA_TRY(cudaMemcpyAsync(sv->d_vol, volume, ctx->nvox() * sizeof(float), cudaMemcpyHostToDevice, st));
    const bool siddon = sv->prm.projector == TOMO_PROJ_SIDDON || sv->prm.projector == TOMO_PROJ_SIDDON_REF;
    if (!siddon && count > 0) {
        // the real sinogram is first read at the end of the first projection: copy it on a
        // second stream after the iterate's copy, while that projection runs
        if (!sv->copy_st) {
            TOMO_CUDA_TRY(cudaStreamCreateWithFlags(&sv->copy_st, cudaStreamNonBlocking));
            TOMO_CUDA_TRY(cudaEventCreateWithFlags(&sv->ev_vol, cudaEventDisableTiming));
            TOMO_CUDA_TRY(cudaEventCreateWithFlags(&sv->ev_real, cudaEventDisableTiming));
        }
        TOMO_CUDA_TRY(cudaEventRecord(sv->ev_vol, st));
        TOMO_CUDA_TRY(cudaStreamWaitEvent(sv->copy_st, sv->ev_vol, 0));
        TOMO_CUDA_TRY(cudaMemcpyAsync(sv->d_real, real_sinogram, rb, cudaMemcpyHostToDevice, sv->copy_st));
        TOMO_CUDA_TRY(cudaEventRecord(sv->ev_real, sv->copy_st));
        sv->real_pending = true;
    } else {
        TOMO_CUDA_TRY(cudaMemcpyAsync(sv->d_real, real_sinogram, rb, cudaMemcpyHostToDevice, st));
    }
    s = tomo_solver_iterate(sv, sv->d_vol, sv->d_real, first, count, stream);
    if (sv->real_pending) {  // not consumed (an error before the first projection): order st after the copy
        sv->real_pending = false;
        cudaStreamWaitEvent(st, sv->ev_real, 0);
    }
    if (s != TOMO_OK) return s;
    TOMO_CUDA_TRY(cudaMemcpyAsync(volume, sv->d_vol, ctx->nvox() * sizeof(float), cudaMemcpyDeviceToHost, st));
    TOMO_CUDA_TRY(cudaStreamSynchronize(st));
    return TOMO_OK;
}

tomo_status tomo_solver_set_timing(tomo_solver* sv, int enable) {
    TOMO_CHECK_ARG(sv, "tomo_solver_set_timing: null argument");
    sv->timing = enable != 0;
    return TOMO_OK;
}

tomo_status tomo_solver_get_stats(tomo_solver* sv, tomo_solver_stats* out, int reset, void* stream) {
    TOMO_CHECK_ARG(sv && out, "tomo_solver_get_stats: null argument");
    tomo_status s = set_device(sv->ctx);
    if (s != TOMO_OK) return s;
    TOMO_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    auto sum = [](std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& pool, size_t used, double& ms) -> cudaError_t {
        ms = 0.0;
        for (size_t i = 0; i < used; ++i) {
            float t = 0.f;
            cudaError_t e = cudaEventElapsedTime(&t, pool[i].first, pool[i].second);
            if (e != cudaSuccess) return e;
            ms += t;
        }
        return cudaSuccess;
    };
    TOMO_CUDA_TRY(sum(sv->ev_proj, sv->ev_proj_used, out->proj_ms));
    TOMO_CUDA_TRY(sum(sv->ev_back, sv->ev_back_used, out->back_ms));
    out->proj_launches = (int32_t)sv->ev_proj_used;
    out->back_launches = (int32_t)sv->ev_back_used;
    out->kernel_launches = sv->launches;
    if (reset) {
        sv->ev_proj_used = sv->ev_back_used = 0;
        sv->launches = 0;
    }
    return TOMO_OK;
}

tomo_status tomo_solver_alphas(tomo_solver* sv, double* alpha, int32_t n, int32_t* written, void* stream) {
    TOMO_CHECK_ARG(sv && alpha && written, "tomo_solver_alphas: null argument");
    tomo_status s = set_device(sv->ctx);
    if (s != TOMO_OK) return s;
    const int m = std::min(n, std::min(sv->log_cap, sv->next_it - 1));
    if (m > 0) {
        TOMO_CUDA_TRY(cudaMemcpyAsync(alpha, sv->alpha_log, m * sizeof(double), cudaMemcpyDeviceToHost,
                                      (cudaStream_t)stream));
    }
    TOMO_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    *written = m > 0 ? m : 0;
    return TOMO_OK;
}

tomo_status tomo_solver_get_state(tomo_solver* sv, double* alpha_min, int32_t* next_iteration, void* stream) {
    TOMO_CHECK_ARG(sv && alpha_min && next_iteration, "tomo_solver_get_state: null argument");
    tomo_status s = set_device(sv->ctx);
    if (s != TOMO_OK) return s;
    double st[2];
    TOMO_CUDA_TRY(cudaMemcpyAsync(st, sv->state, sizeof(st), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    TOMO_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    *alpha_min = st[1];
    *next_iteration = sv->next_it;
    return TOMO_OK;
}

tomo_status tomo_solver_set_state(tomo_solver* sv, double alpha_min, int32_t next_iteration, void* stream) {
    TOMO_CHECK_ARG(sv, "tomo_solver_set_state: null argument");
    TOMO_CHECK_ARG(next_iteration >= 1, "tomo_solver_set_state: iteration index starts at 1");
    tomo_status s = set_device(sv->ctx);
    if (s != TOMO_OK) return s;
    const double st[2] = {0.0, alpha_min};
    TOMO_CUDA_TRY(cudaMemcpyAsync(sv->state, st, sizeof(st), cudaMemcpyHostToDevice, (cudaStream_t)stream));
    TOMO_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    sv->next_it = next_iteration;
    return TOMO_OK;
}

// ------------------------------------------------------------------------------------
tomo_status tomo_laplacian(const float* in, float* out, int32_t nx, int32_t ny, int32_t nz, void* stream) {
    TOMO_CHECK_ARG(in && out && nx > 0 && ny > 0 && nz > 0, "tomo_laplacian: bad argument");
    TOMO_CHECK_ARG(in != out, "tomo_laplacian: in and out must not alias");
    return check_launch(launch_laplacian(in, out, nx, ny, nz, (cudaStream_t)stream), "laplacian");
}

tomo_status tomo_sq_norm(const void* x, tomo_dtype dtype, size_t n, double* out, void* stream) {
    TOMO_CHECK_ARG(x && out && valid_dtype(dtype), "tomo_sq_norm: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    TOMO_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double), st));
    if (n == 0) return TOMO_OK;
    return check_launch(launch_sq_norm(x, dtype, n, out, st), "sq_norm");
}

tomo_status tomo_gg_regularization_beta(const float* volume, float* dJ, int32_t nx, int32_t ny, int32_t nz,
                                        double lambda, double beta, int32_t total_iteration,
                                        int32_t optimal_step_iteration_nb, double* out, void* stream) {
    TOMO_CHECK_ARG(volume && dJ && out && nx > 0 && ny > 0 && nz > 0, "tomo_gg_regularization: bad argument");
    TOMO_CHECK_ARG(volume != dJ, "tomo_gg_regularization: volume and dJ must not alias");
    TOMO_CHECK_ARG(std::isfinite(beta) && beta >= 1.0, "tomo_gg_regularization: beta must be finite and at least 1");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)nx * ny * nz;
    const size_t grad_bytes = (n * sizeof(float) + 255) / 256 * 256;
    void* scratch = nullptr;
    TOMO_CUDA_TRY(cudaMallocAsync(&scratch, grad_bytes + 4 * sizeof(double), st));
    float* grad = (float*)scratch;
    double* nrm = (double*)((char*)scratch + grad_bytes);
    const float w = (float)(beta * (double)(float)lambda);  // beta * lambda, lambda passed as float (Mex.cu:513)
    tomo_status s = TOMO_OK;
    do {
        // grad = L f; jReg = sum |grad|^beta (:165-182); for beta != 2 grad = sign(f) |f|^(beta-1)
        // (:190-198); dJ += beta*lambda L(grad) (:200-205)
        if ((s = check_launch(launch_laplacian(volume, grad, nx, ny, nz, st), "laplacian")) != TOMO_OK) break;
        if ((s = check_launch(cudaMemsetAsync(out, 0, sizeof(double), st), "memset")) != TOMO_OK) break;
        if ((s = check_launch(launch_lp_norm(grad, n, beta, out, st), "jreg")) != TOMO_OK) break;
        if (beta != 2.0 && (s = check_launch(launch_gg_abspow(volume, grad, n, beta - 1.0, st), "abs pow")) != TOMO_OK)
            break;
        if ((s = check_launch(launch_laplacian_axpy(grad, dJ, w, nx, ny, nz, st), "laplacian axpy")) != TOMO_OK) break;
        if (total_iteration < optimal_step_iteration_nb) {  // :207-218
            if ((s = check_launch(cudaMemsetAsync(nrm, 0, 4 * sizeof(double), st), "memset")) != TOMO_OK) break;
            if ((s = check_launch(launch_laplacian_norm(dJ, nrm, nx, ny, nz, 1, st, nullptr, beta), "norms")) != TOMO_OK)
                break;
            if ((s = check_launch(launch_gg_finish(nrm, out, st, beta), "gg finish")) != TOMO_OK) break;
        }
    } while (false);
    const cudaError_t fe = cudaFreeAsync(scratch, st);
    if (s == TOMO_OK && fe != cudaSuccess) return check_launch(fe, "free");
    return s;
}

tomo_status tomo_gg_regularization(const float* volume, float* dJ, int32_t nx, int32_t ny, int32_t nz, double lambda,
                                   int32_t total_iteration, int32_t optimal_step_iteration_nb, double* out,
                                   void* stream) {
    return tomo_gg_regularization_beta(volume, dJ, nx, ny, nz, lambda, 2.0, total_iteration, optimal_step_iteration_nb,
                                       out, stream);
}

tomo_status tomo_huber_regularization(const float* volume, float* dJ, int32_t nx, int32_t ny, int32_t nz, double lambda,
                                      double huber_threshold, int32_t total_iteration,
                                      int32_t optimal_step_iteration_nb, double* out, void* stream) {
    TOMO_CHECK_ARG(volume && dJ && out && nx > 0 && ny > 0 && nz > 0, "tomo_huber_regularization: bad argument");
    TOMO_CHECK_ARG(volume != dJ, "tomo_huber_regularization: volume and dJ must not alias");
    TOMO_CHECK_ARG(std::isfinite(huber_threshold) && huber_threshold >= 0.0,
                   "tomo_huber_regularization: the threshold must be finite and non-negative");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)nx * ny * nz;
    const size_t vb = (n * sizeof(float) + 255) / 256 * 256;
    void* scratch = nullptr;
    TOMO_CUDA_TRY(cudaMallocAsync(&scratch, 2 * vb, st));
    float* grad = (float*)scratch;
    float* t = (float*)((char*)scratch + vb);
    tomo_status s = TOMO_OK;
    do {
        // grad = L f; out[0] = jReg = Huber norm of grad (:214-217); dJ += lambda L(psi'(grad)) (:218-228)
        if ((s = check_launch(launch_laplacian(volume, grad, nx, ny, nz, st), "laplacian")) != TOMO_OK) break;
        if ((s = check_launch(cudaMemsetAsync(out, 0, sizeof(double), st), "memset")) != TOMO_OK) break;
        if ((s = check_launch(launch_huber_jreg(grad, n, huber_threshold, out, st), "huber norm")) != TOMO_OK) break;
        if ((s = check_launch(launch_huber_axpy(grad, dJ, (float)lambda, huber_threshold, nx, ny, nz, st), "axpy")) !=
            TOMO_OK)
            break;
        if (total_iteration < optimal_step_iteration_nb) {  // :230-242
            if ((s = check_launch(cudaMemsetAsync(out + 1, 0, sizeof(double), st), "memset")) != TOMO_OK) break;
            if ((s = check_launch(launch_huber_norm(grad, dJ, t, huber_threshold, out + 1, nx, ny, nz, st),
                                  "huber step norm")) != TOMO_OK)
                break;
        }
    } while (false);
    const cudaError_t fe = cudaFreeAsync(scratch, st);
    if (s == TOMO_OK && fe != cudaSuccess) return check_launch(fe, "free");
    return s;
}

// Host-buffer forms of the Laplacian and the regulariser criteria (the reference's
// --op=laplacien and --op=reg_GG, Iter3D_main.cu:215-272): copies in, the device entry, copies out.
tomo_status tomo_laplacian_host(int device, const float* in, float* out, int32_t nx, int32_t ny, int32_t nz) {
    TOMO_CHECK_ARG(in && out && nx > 0 && ny > 0 && nz > 0, "tomo_laplacian_host: bad argument");
    TOMO_CUDA_TRY(cudaSetDevice(device));
    const size_t bytes = (size_t)nx * ny * nz * sizeof(float);
    float *d_in = nullptr, *d_out = nullptr;
    tomo_status s = TOMO_OK;
    if (cudaMalloc(&d_in, bytes) != cudaSuccess || cudaMalloc(&d_out, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("tomo_laplacian_host: device allocation failed");
        s = TOMO_ERR_NO_MEMORY;
    }
    if (s == TOMO_OK) s = check_launch(cudaMemcpy(d_in, in, bytes, cudaMemcpyHostToDevice), "copy in");
    if (s == TOMO_OK) s = tomo_laplacian(d_in, d_out, nx, ny, nz, nullptr);
    if (s == TOMO_OK) s = check_launch(cudaMemcpy(out, d_out, bytes, cudaMemcpyDeviceToHost), "copy out");
    cudaFree(d_in);
    cudaFree(d_out);
    return s;
}

tomo_status tomo_regularization_host(int device, int32_t kind, const float* volume, float* dJ, int32_t nx, int32_t ny,
                                     int32_t nz, double lambda, double huber_threshold, double gg_beta,
                                     int32_t total_iteration, int32_t optimal_step_iteration_nb, double* out) {
    TOMO_CHECK_ARG(volume && dJ && out && nx > 0 && ny > 0 && nz > 0, "tomo_regularization_host: bad argument");
    TOMO_CHECK_ARG(kind == TOMO_REG_GG || kind == TOMO_REG_HUBER, "tomo_regularization_host: unknown regulariser");
    TOMO_CHECK_ARG(kind != TOMO_REG_GG || (std::isfinite(gg_beta) && gg_beta >= 1.0),
                   "tomo_regularization_host: beta must be finite and at least 1");
    TOMO_CHECK_ARG(kind != TOMO_REG_HUBER || (std::isfinite(huber_threshold) && huber_threshold >= 0.0),
                   "tomo_regularization_host: the Huber threshold must be finite and non-negative");
    TOMO_CUDA_TRY(cudaSetDevice(device));
    const size_t bytes = (size_t)nx * ny * nz * sizeof(float);
    float *d_vol = nullptr, *d_dj = nullptr;
    double* d_out = nullptr;
    tomo_status s = TOMO_OK;
    if (cudaMalloc(&d_vol, bytes) != cudaSuccess || cudaMalloc(&d_dj, bytes) != cudaSuccess ||
        cudaMalloc(&d_out, 2 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        set_error("tomo_regularization_host: device allocation failed");
        s = TOMO_ERR_NO_MEMORY;
    }
    if (s == TOMO_OK) s = check_launch(cudaMemcpy(d_vol, volume, bytes, cudaMemcpyHostToDevice), "copy in");
    if (s == TOMO_OK) s = check_launch(cudaMemcpy(d_dj, dJ, bytes, cudaMemcpyHostToDevice), "copy in");
    if (s == TOMO_OK) s = check_launch(cudaMemcpy(d_out, out, 2 * sizeof(double), cudaMemcpyHostToDevice), "copy in");
    if (s == TOMO_OK)
        s = kind == TOMO_REG_HUBER ? tomo_huber_regularization(d_vol, d_dj, nx, ny, nz, lambda, huber_threshold,
                                                                total_iteration, optimal_step_iteration_nb, d_out,
                                                                nullptr)
                                   : tomo_gg_regularization_beta(d_vol, d_dj, nx, ny, nz, lambda, gg_beta,
                                                                 total_iteration, optimal_step_iteration_nb, d_out,
                                                                 nullptr);
    if (s == TOMO_OK) s = check_launch(cudaMemcpy(dJ, d_dj, bytes, cudaMemcpyDeviceToHost), "copy out");
    if (s == TOMO_OK) s = check_launch(cudaMemcpy(out, d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost), "copy out");
    cudaFree(d_vol);
    cudaFree(d_dj);
    cudaFree(d_out);
    return s;
}

tomo_status tomo_convert(const void* in, tomo_dtype in_dtype, void* out, tomo_dtype out_dtype, size_t n, void* stream) {
    TOMO_CHECK_ARG(in && out && valid_dtype(in_dtype) && valid_dtype(out_dtype), "tomo_convert: bad argument");
    if (n == 0) return TOMO_OK;
    return check_launch(launch_convert(in, in_dtype, out, out_dtype, n, (cudaStream_t)stream), "convert");
}

tomo_status tomo_phantom(const double* ellipsoids, int32_t count, int32_t nx, int32_t ny, int32_t nz, float* volume,
                         void* stream) {
    TOMO_CHECK_ARG(volume && nx > 0 && ny > 0 && nz > 0 && count >= 0 && (count == 0 || ellipsoids),
                   "tomo_phantom: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    void* scratch = nullptr;
    cudaError_t e = launch_phantom(ellipsoids, count, nx, ny, nz, volume, &scratch, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(scratch);
    return check_launch(e, "phantom");
}

}  // extern "C"
