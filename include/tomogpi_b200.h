/*
 * tomogpi_b200.h -- C-ABI of the B200-native cone-beam projector/backprojector library.
 *
 * Drop-in for the operator layer of TomoGPI_lib (paths below are inside the TomoGPI
 * project). Every function returns a tomo_status; plain pointers and sizes only, no C++
 * or framework types. Device pointers are CUDA global-memory addresses on the context's
 * device; "_host" entry points take host memory and do the copies themselves. Streams
 * are cudaStream_t passed as void* (NULL = the legacy default stream).
 *
 * Layouts (as in the reference, Sinogram3D.cu:138-184, Volume.cu:248-272):
 *   volume   [z][y][x], x fastest, Nx*Ny*Nz elements
 *   sinogram [phi][v][u], u fastest, Nu*Nv*P elements
 */
#ifndef TOMOGPI_B200_H_
#define TOMOGPI_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TOMO_OK = 0,
    TOMO_ERR_INVALID = 1,     /* bad argument (null pointer, bad size, bad enum)        */
    TOMO_ERR_CUDA = 2,        /* a CUDA runtime call failed; see tomo_last_error()       */
    TOMO_ERR_NO_MEMORY = 3,   /* device allocation failed or admission refused           */
    TOMO_ERR_UNSUPPORTED = 4, /* combination not available (e.g. pair/storage)           */
    TOMO_ERR_TIMEOUT = 5,     /* a bounded device wait ran out; the kernel returned      */
    TOMO_ERR_NUMERIC = 6,     /* a non-finite value was detected in a reduction          */
    TOMO_ERR_IO = 7           /* a file could not be opened or was too short             */
} tomo_status;

/* Storage types for volumes and sinograms. Arithmetic is FP32 in every case. */
typedef enum { TOMO_F32 = 0, TOMO_BF16 = 1, TOMO_F16 = 2 } tomo_dtype;

/* Projectors (the reference's --pair=RSVI / SiddonVI projection halves). */
typedef enum {
    /* RegularSamplingProjector_compute_CUDA_mem_CPU: projection_ERB_kernel_v1
       (src/TomoGPI_lib/src/CUDA/Projector/projection_ER_kernel.cuh:57-312), box FOV. */
    TOMO_PROJ_RS = 0,
    /* RegularSamplingProjector_compute_CUDA_mem_GPU: projection_ERB_kernel_v0_UM
       (src/TomoGPI_lib/src/CUDA/Projector/projection_ER_kernel_UM.cuh:26-153). */
    TOMO_PROJ_RS_UM = 1,
    /* SiddonProjector_compute_C_mem_CPU as written
       (src/TomoGPI_lib/src/CPP/SiddonProjector_compute_C_mem_CPU.cpp:21-276): mirrored
       source/detector and voxel indices modulo 256 per axis. */
    TOMO_PROJ_SIDDON_REF = 2,
    /* The same Siddon traversal in the RSVI geometry, no index wrap. */
    TOMO_PROJ_SIDDON = 3
} tomo_projector;

/* Backprojectors. */
typedef enum {
    /* VIBackProjector_compute_CUDA_mem_CPU: backprojection_VIB_kernel_v2_16reg
       (src/TomoGPI_lib/src/CUDA/BackProjector/backprojection3D_kernel_16reg.cuh:350-576). */
    TOMO_BACK_VI = 0,
    /* VIBackProjector_compute_CUDA_mem_GPU: backprojection_VIB_kernel_v1_16reg_UM
       (src/TomoGPI_lib/src/CUDA/BackProjector/backprojection3D_kernel_16reg_UM.cuh:24-151). */
    TOMO_BACK_VI_UM = 1,
    /* Exact transpose of TOMO_PROJ_RS (no counterpart in the reference; used for the
       matched-pair adjoint test). */
    TOMO_BACK_RS_ADJOINT = 2,
    /* Exact transpose of TOMO_PROJ_SIDDON. */
    TOMO_BACK_SIDDON_ADJOINT = 3,
    /* Exact transpose of TOMO_PROJ_RS_UM. */
    TOMO_BACK_RS_UM_ADJOINT = 4,
    /* VIBackProjector with setFdk(1) (--op=back_fdk, Iter3D_main.cu:296-316):
       FDK3D_VIB_kernel_v0_16reg (src/TomoGPI_lib/src/CUDA/BackProjector/FDK3D_kernel_16reg.cuh:24-349),
       the VI backprojection with the FDK distance weights and no dx factor. The sinogram is
       expected ramp-filtered (tomo_ramp_filter). */
    TOMO_BACK_FDK = 5
} tomo_backprojector;

/* configCT: the fields ConfigCT::createUniformAcquisition / createDetector / createVolume
   read (src/TomoGPI_lib/src/CPP/Config/ConfigCT.cpp:43-54,110-147), same types. */
typedef struct {
    double fod, fdd;                               /* FOD, FDD                            */
    double num_start_angle, den_start_angle;       /* start angle, in units of pi (num/den) */
    double num_stop_angle, den_stop_angle;         /* stop angle, in units of pi           */
    int32_t projection_nb;                         /* P                                    */
    float u_detector_size, v_detector_size;        /* horizontal/verticalDetectorSize      */
    int32_t u_detector_pixel_nb, v_detector_pixel_nb;
    float x_volume_size, y_volume_size, z_volume_size;
    int32_t x_volume_pixel_nb, y_volume_pixel_nb, z_volume_pixel_nb;
} tomo_config_ct;

typedef struct tomo_context tomo_context;

/* Last error text of the calling thread (never NULL). */
const char* tomo_last_error(void);
/* Library version string. */
const char* tomo_version(void);

/* Geometry set-up as the reference's host classes do it: Projector/BackProjector ctors
   (src/TomoGPI_lib/src/CPP/Projector.cu:16-38, BackProjector.cu:16-37) plus the values
   copyConstantGPU uploads (RegularSamplingProjector_compute_CUDA_mem_CPU.cu:906-951).
   The tables live in device memory owned by the context, so calls are re-entrant per
   context (the reference uses process-global __constant__ symbols). */
tomo_status tomo_context_create(const tomo_config_ct* cfg, int device, tomo_context** out);
/* A context over views [view_begin, view_begin + view_count) of the acquisition `cfg`
   describes: the per-view tables are those of the whole acquisition, sliced, so each view's
   geometry is bit-identical to the full context's; sinograms passed to it hold only these
   views. Splits one reconstruction across GPUs by views (the reference splits its
   projector by detector rows and its backprojector by z slabs,
   RegularSamplingProjector_compute_CUDA_mem_CPU.cu:243-278,
   VIBackProjector_compute_CUDA_mem_CPU.cu:214-245; by views every rank keeps the whole
   volume and one sum of gradients per iteration is the only exchange). */
tomo_status tomo_context_create_views(const tomo_config_ct* cfg, int device, int32_t view_begin, int32_t view_count,
                                      tomo_context** out);
tomo_status tomo_context_destroy(tomo_context* ctx);
/* scalars[11] = fod, fdd, gamma, du, dv, uc, vc, dx, xc, yc, zc (float32 as uploaded);
   alpha/beta: P floats each (may be NULL). */
tomo_status tomo_context_geometry(const tomo_context* ctx, float* scalars, float* alpha, float* beta);

/* Launch/layout choices of a context (the project's autotuner writes them; the defaults
   are the measured best for B200). rs_layout: volume layout read by the RS projectors,
   0 = zero-bordered padded copy (1x), 1 = 2x2x2 texel cells (8x the volume's bytes, one
   aligned 32 B / 16 B vector load per sample), 2 = 2D layered texture in the storage type
   (FP32, or the raw bits of BF16 / FP16), one layer per z slice, read with 4-texel gathers
   (depths beyond the device's layer limit use 1), 3 = the texture for the lower slice of
   each sample plus, for the upper slice, the slice's four footprint texels stored together
   (FP32 only; 8x the volume's bytes besides the texture), 4 = faces across the axis the
   view's rays mostly run along, even faces in a layered texture and odd faces as stored
   2 x 2 footprints, each sample reusing the faces it shares with the previous sample of its
   ray (FP32 only, 5x the volume's bytes; otherwise 3). Batches use 2 for 3 and 4.
   rs_warp_u: the RS projectors'
   launch shape: rays of one warp along u (8, 16 or 32, the rest of its 32 along v; 0 = 8)
   and of one 256-thread block along u (16, 32, 64 or 128, at least rs_warp_u; 0 = 32).
   vi_layout: sinogram read by the VI
   backprojectors, 0 = zero-bordered padded copy (four scalar loads per voxel and view),
   1 = 2D layered texture, one layer per view, one 4-texel gather per voxel and view (view
   counts beyond the layer limit use 0), 2 = FP32 sinogram windows staged in shared memory
   by TMA, one per (voxel tile, view), read by the bilinear samples (FP32 sinograms with nu
   a multiple of 4; otherwise 0). Set before creating solvers on the context. */
typedef struct {
    int32_t rs_layout;
    int32_t vi_zc;       /* VI: 16-slice chunks per thread (1, 2 or 4; 0 = default 1) */
    int32_t vi_layout;
    int32_t rs_warp_u;   /* RS: rays of a warp along u (8, 16 or 32; 0 = default 8)        */
    int32_t rs_tile_u;   /* RS: rays of a block along u (16, 32, 64, 128; 0 = default 32) */
    int32_t reserved[3];
} tomo_tuning;
tomo_status tomo_context_get_tuning(const tomo_context* ctx, tomo_tuning* out);
tomo_status tomo_context_set_tuning(tomo_context* ctx, const tomo_tuning* in);
/* The RS input layout a projection of a volume of this type actually uses (the tuning's
   choice, or the cells where the texture's layer limit rules it out). */
tomo_status tomo_context_rs_layout(const tomo_context* ctx, tomo_dtype dtype, int32_t* layout);

/* Projector<V,S,T>::doProjection(S* estimatedSinogram, V* volume)
   (src/TomoGPI_lib/inc/Projector.cuh:118): sinogram := H volume (overwrite).
   Device pointers. */
tomo_status tomo_project(tomo_context* ctx, tomo_projector kind, const void* volume, tomo_dtype volume_dtype,
                         void* sinogram, tomo_dtype sinogram_dtype, void* stream);

/* BackProjector<V,S,T>::doBackProjection(V* estimatedVolume, S* sinogram)
   (src/TomoGPI_lib/inc/BackProjector.cuh:144): volume := H^T sinogram (overwrite).
   Device pointers. */
tomo_status tomo_backproject(tomo_context* ctx, tomo_backprojector kind, const void* sinogram,
                             tomo_dtype sinogram_dtype, void* volume, tomo_dtype volume_dtype, void* stream);

/* The mem_CPU classes' form (RegularSamplingProjector_compute_CUDA_mem_CPU::doProjection,
   ...mem_CPU.cu:27-341; VIBackProjector_compute_CUDA_mem_CPU::doBackProjection,
   ...mem_CPU.cu:20-411): host buffers in and out (FP32), copies included, synchronous. */
tomo_status tomo_project_host(tomo_context* ctx, tomo_projector kind, const float* volume, float* sinogram);
tomo_status tomo_backproject_host(tomo_context* ctx, tomo_backprojector kind, const float* sinogram, float* volume);

/* Ramp filter of filtered backprojection (Matlab/Tomo8/ramp_filter_TOMO8.m: ramp over
   oversampling x nu frequencies, Hann window of cutoff x that length, convolution of every
   detector row, / (2 du)); the reference calls it with oversampling 16 and cutoff 1.0.
   `out` is an FP32 device sinogram; the taps are cached in the context per (oversampling,
   cutoff). */
tomo_status tomo_ramp_filter(tomo_context* ctx, const void* sinogram, tomo_dtype sinogram_dtype, float* out,
                             int32_t oversampling, double cutoff, void* stream);
/* The same on host FP32 buffers (out may be the input). */
tomo_status tomo_ramp_filter_host(tomo_context* ctx, const float* sinogram, float* out, int32_t oversampling,
                                  double cutoff);

/* RS projection for callers that cannot allocate device memory: a host framework whose
   memory pool owns every device allocation, or real-time code that must not allocate once
   it runs. No counterpart in the reference. Takes the configCT directly (no context) and
   FP32 device pointers; the padded volume and the view tables live in static __device__
   arrays of this library (32 MiB + 96 KiB on every GPU that loads it, held until exit), and
   the call allocates nothing. Limits: (nx+2)*(ny+2)*(nz+2) <= 8 Mi voxels (up to 201^3) and
   P <= 4096, else TOMO_ERR_INVALID. kind: TOMO_PROJ_RS or TOMO_PROJ_RS_UM. All calls on a
   device share the arrays, which keep the last call's contents (each call clears what it
   uses): calls that overlap on the GPU race, so serialise them. The first call on a device
   looks up the arrays' device addresses (a synchronous runtime query). `stream` must belong
   to `device`; the caller's current device is restored on return, and a pending non-sticky
   CUDA error of the calling thread is cleared on entry. Asynchronous on `stream`. */
tomo_status tomo_project_noalloc(const tomo_config_ct* cfg, int device, tomo_projector kind, const float* volume,
                                 float* sinogram, void* stream);

/* Number of samples one projection call visits (RS: sum of L_r over rays; Siddon: voxel
   visits). Device computation; used for the roofline's algorithmic-byte count. */
tomo_status tomo_count_samples(tomo_context* ctx, tomo_projector kind, unsigned long long* out, void* stream);

/* Device error word of the context (bit 0: a Siddon traversal hit its step bound, bit 1:
   a bounded wait gave up). Synchronous; clear != 0 resets it. */
tomo_status tomo_context_errors(tomo_context* ctx, unsigned* bits, int clear);
/* For tests of the bounded waits only (no counterpart in the reference): with enable != 0,
   the TMA-staged VI backprojection of this context (vi_layout 2) issues no copies, so every
   wait of its consumers runs out after its one-second bound; the call completes with the
   volume undefined and bit 1 (a bounded wait gave up) set in the error word, and the
   context stays usable. Never enabled otherwise. */
tomo_status tomo_context_test_stall(tomo_context* ctx, int enable);

/* ---- gradient descent (Iter3D::doSimpleGradient, src/TomoGPI_lib/src/CPP/Iter3D_Algo_Gradient.cu:25-223,
        and Iter3D::doWeightedGradient, :227-373; generalised-Gaussian regulariser
        GeneralizedGaussianRegularizer_CPU.cu:158-225, or Huber) ---- */
typedef struct {
    tomo_projector projector;        /* TOMO_PROJ_RS for --pair=RSVI                       */
    tomo_backprojector backprojector;/* TOMO_BACK_VI                                       */
    tomo_dtype storage;              /* operator input/output storage; FP32 master iterate */
    int32_t gradient_iteration_nb;   /* configIteration gradientIterationNb                */
    int32_t optimal_step_iteration_nb;/* configIteration optimalStepIterationNb            */
    double regularization_parameter; /* lambda                                             */
    int32_t positivity;              /* clamp the iterate at 0 after each update           */
    int32_t real_sinogram_f32;       /* nonzero: the real (measured) sinogram is FP32 whatever
                                        `storage` (the residual is FP32 anyway); 0: it is in
                                        `storage`. A measured sinogram rounded to BF16 carries
                                        a 2^-9 relative error per ray sum into the result. */
} tomo_gradient_params;

typedef struct tomo_solver tomo_solver;

/* A solver belongs to the context it was created on: destroy it before that context
   (tomo_solver_destroy itself never dereferences the context).
   A solver owns the device work buffers of one reconstruction (residual sinogram,
   gradient volume, regulariser scratch, FP64 norm accumulators, operator shadows). */
tomo_status tomo_solver_create(tomo_context* ctx, const tomo_gradient_params* params, tomo_solver** out);
/* Regulariser of the gradient loop (configIteration penaltyFunction, Iter3D.cu:58-69):
   TOMO_REG_GG, the generalised Gaussian (the default; beta = 2 unless tomo_solver_set_gg_beta:
   GeneralizedGaussianRegularizer_CPU.cu:158-226), or TOMO_REG_HUBER with configIteration's
   huberThreshold (HuberRegularizer_CPU.cu:206-253: dJ += lambda L(psi'(L f)), and for the
   optimal step normdJProjReg = sum |L(L(psi''(L f) dJ)) dJ|). Huber allocates one more
   volume of scratch. Applies from the next iteration. */
enum { TOMO_REG_GG = 0, TOMO_REG_HUBER = 1 };
tomo_status tomo_solver_set_regularizer(tomo_solver* s, int32_t kind, double huber_threshold);
/* Shape parameter of the generalised-Gaussian regulariser (configIteration beta, default 2;
   R_GG(beta), Iter3D.cu:72), finite and >= 1. For beta != 2 the loop adds
   beta*lambda * L(sign(f) |f|^(beta-1)) to dJ and takes normdJProjReg = beta * sum |L dJ|^beta
   (GeneralizedGaussianRegularizer_GPU.cu:161-225, the same steps as
   GeneralizedGaussianRegularizer_CPU.cu:158-226). Applies from the next iteration. */
tomo_status tomo_solver_set_gg_beta(tomo_solver* s, double beta);
/* The weighted gradient (Iter3D::doWeightedGradient, Iter3D_Algo_Gradient.cu:227-373):
   with weights != NULL every iteration multiplies the residual g - H f by the weight
   sinogram before the backprojection (:289) and alpha_min starts at -999999999999 (:257);
   everything else is the simple gradient. weights: FP32 in the layout of the solver's real
   sinogram (its context's views), HOST memory when host != 0 (copied before the call
   returns), else device memory (copied in order on `stream`); the solver keeps its own copy
   (one more FP32 sinogram). NULL returns to the simple gradient. Only before the first
   iteration (TOMO_ERR_INVALID otherwise). */
tomo_status tomo_solver_set_weights(tomo_solver* s, const float* weights, int32_t host, void* stream);

/* One iteration in phases, for a reconstruction whose views are split over several
   solvers (one per GPU, each on a tomo_context_create_views context):
     TOMO_PHASE_GRADIENT  residual and backprojection of this solver's views:
                          dJ = -2 H_k^T (g_k - H_k f)   (a partial sum over views)
     TOMO_PHASE_NORMS     regulariser on dJ, ||dJ||^2 and ||L dJ||^2 into norms[0], [2]
                          (Huber: norms[4]), and this solver's views' ||H_k dJ||^2 into
                          norms[1]   (only while iteration < optimal_step_iteration_nb)
     TOMO_PHASE_UPDATE    step size from norms, f += alpha dJ, positivity
   Between GRADIENT and NORMS the caller sums dJ over the solvers (an all-reduce of the
   tomo_solver_buffers dJ volume); between NORMS and UPDATE it sums norms[1] only (the
   other norms are of the summed dJ and already equal on every solver). Phases may be
   combined (all three = tomo_solver_iterate of one iteration). real_sinogram is read by
   GRADIENT only. */
enum { TOMO_PHASE_GRADIENT = 1, TOMO_PHASE_NORMS = 2, TOMO_PHASE_UPDATE = 4 };
tomo_status tomo_solver_phase(tomo_solver* s, float* volume, const void* real_sinogram, int32_t iteration,
                              int32_t phases, void* stream);
/* Device pointers of the solver's gradient volume (FP32, nx*ny*nz) and norms (8 doubles). */
tomo_status tomo_solver_buffers(tomo_solver* s, float** dJ, double** norms);
tomo_status tomo_solver_destroy(tomo_solver* s);
/* Runs iterations [first, first+count) of the simple gradient on device memory:
   volume (FP32, in/out, the master iterate) and real_sinogram (in the solver's storage
   dtype, or FP32 with real_sinogram_f32). Fully asynchronous on `stream` (no host synchronisation inside), so a call can
   be captured in a CUDA graph. */
tomo_status tomo_solver_iterate(tomo_solver* s, float* volume, const void* real_sinogram, int32_t first,
                                int32_t count, void* stream);
/* Per-iteration step sizes alpha of the iterations run so far (host copy; synchronises
   the stream). n = capacity; returns the count written in *written. */
tomo_status tomo_solver_alphas(tomo_solver* s, double* alpha, int32_t n, int32_t* written, void* stream);
/* The solver's state for checkpoint/resume: alpha_min and the iteration counter. */
tomo_status tomo_solver_get_state(tomo_solver* s, double* alpha_min, int32_t* next_iteration, void* stream);
tomo_status tomo_solver_set_state(tomo_solver* s, double alpha_min, int32_t next_iteration, void* stream);

/* Host-buffer form of tomo_solver_iterate (the mem_CPU Iter3D form): copies the FP32
   iterate and the real sinogram (storage dtype, or FP32) from host memory, runs the iterations,
   copies the iterate back and synchronises. Pinned host memory makes the copies async. With
   an RS projector the sinogram is copied on a second stream of the solver while the first
   projection runs (that iteration's residual is then formed in a pass of its own; the
   iterate is the same as tomo_solver_iterate's). */
tomo_status tomo_solver_iterate_host(tomo_solver* s, float* volume, const void* real_sinogram, int32_t first,
                                     int32_t count, void* stream);

/* Device timing of the operator launches inside tomo_solver_iterate: with timing on,
   CUDA events are recorded on the launching stream around every projector and
   backprojector launch. Stats synchronise the stream and report the summed durations and
   the number of launches of each, plus the count of all library kernels launched. */
typedef struct {
    double proj_ms;          /* sum of projector launch durations            */
    int32_t proj_launches;
    double back_ms;          /* sum of backprojector launch durations        */
    int32_t back_launches;
    int64_t kernel_launches; /* every kernel the solver launched             */
} tomo_solver_stats;
tomo_status tomo_solver_set_timing(tomo_solver* s, int enable);
tomo_status tomo_solver_get_stats(tomo_solver* s, tomo_solver_stats* out, int reset, void* stream);

/* ---- many reconstructions at once ----
   A batch advances every live job by whole gradient iterations; each phase of an
   iteration is one launch over all jobs (projection and backprojection as persistent
   kernels over a device work queue of (job, view, tile) / (job, column tile, slab) items,
   longest first). Each job keeps its own iteration counter, so jobs added later run
   behind the others and finished jobs are skipped; one iteration of the batch is captured
   as a CUDA graph (rebuilt when the job set changes) and replayed. Norms are per-item
   partials reduced in a fixed order, so a job's result does not depend on the other jobs.
   The parameters (storage, lambda, iteration counts, positivity) are shared by the jobs;
   the projector must be RS or RS_UM and the backprojector VI or VI_UM. Batched jobs run
   the simple gradient with the generalised Gaussian of beta = 2 (the Huber potential,
   other shapes and the weighted gradient are solver options). */
typedef struct tomo_batch tomo_batch;
tomo_status tomo_batch_create(int device, const tomo_gradient_params* params, tomo_batch** out);
tomo_status tomo_batch_destroy(tomo_batch* b);
/* Device bytes tomo_batch_add allocates for a job (excluding the caller's iterate and real
   sinogram): the admission price of the job. tuning may be NULL (defaults). */
tomo_status tomo_batch_footprint(const tomo_config_ct* cfg, const tomo_gradient_params* params,
                                 const tomo_tuning* tuning, size_t* bytes);
/* Adds a job: `volume` is its FP32 iterate (device, updated in place), `real_sinogram` its
   measured sinogram (device, the batch's storage dtype, or FP32 with real_sinogram_f32). Both stay owned by the caller and
   must outlive the job. tuning may be NULL. Returns the job id. */
tomo_status tomo_batch_add(tomo_batch* b, const tomo_config_ct* cfg, const tomo_tuning* tuning, float* volume,
                           const void* real_sinogram, int32_t* job);
/* Removes a job (waits for the batch's own work first). Job buffers come from a
   stream-ordered pool of the batch (released at the batch's own synchronisations). */
tomo_status tomo_batch_remove(tomo_batch* b, int32_t job);
/* enable != 0: capture one iteration as a CUDA graph and replay it (default on). */
tomo_status tomo_batch_set_graph(tomo_batch* b, int enable);
/* Fraction in (0, 1] of the persistent projection/backprojection CTAs that take work items
   (default 1). Takes effect within one work item, also in a launch already running, so
   batches on other streams (e.g. size-class lanes of a server) can split the SMs. */
tomo_status tomo_batch_set_share(tomo_batch* b, double fraction);
/* CUDA stream priority of the batch's work (lower = more urgent, clamped to the device's
   range); waits for the batch's own work first. */
tomo_status tomo_batch_set_priority(tomo_batch* b, int32_t priority);
/* Runs `count` iterations of every live job, ordered after the work already on `stream`. */
tomo_status tomo_batch_iterate(tomo_batch* b, int32_t count, void* stream);
/* Iterations a job has completed and its alpha_min (synchronises). */
tomo_status tomo_batch_job_status(tomo_batch* b, int32_t job, int32_t* iterations_done, double* alpha_min,
                                  void* stream);
tomo_status tomo_batch_job_alphas(tomo_batch* b, int32_t job, double* alpha, int32_t n, int32_t* written,
                                  void* stream);
/* Texture arrays of removed jobs stay parked in the batch for the next job of the same size
   and type (freeing a CUDA array synchronises the device). parked_bytes != NULL: report the
   parked textures' bytes and free nothing; NULL: free them and the pool's unused memory. */
tomo_status tomo_batch_trim(tomo_batch* b, size_t* parked_bytes);
/* Host milliseconds spent so far in tomo_batch_iterate: ms[0] rebuilding the work queues,
   ms[1] capturing an iteration, ms[2] updating / instantiating the executable graph,
   ms[3] launching it. */
tomo_status tomo_batch_host_times(tomo_batch* b, double* ms);
/* Live jobs, work items per iteration, device bytes held for them, kernels launched so far. */
tomo_status tomo_batch_stats(tomo_batch* b, int32_t* live_jobs, int64_t* work_items, size_t* bytes,
                             int64_t* kernel_launches);

/* ---- element-wise pieces of the loop (Image3D/Sinogram3D ops), device pointers, FP32 ---- */
/* out = sum of the three {-1,2,-1} 1-D convolutions of in, zero padded
   (Convolution3D_CPU::doSeparableConvolution3D with the GG kernels). */
tomo_status tomo_laplacian(const float* in, float* out, int32_t nx, int32_t ny, int32_t nz, void* stream);
/* Generalised-Gaussian beta = 2 regularisation criterion
   (GeneralizedGaussianRegularizer_CPU::getLaplacianRegularizationCriterion,
   GeneralizedGaussianRegularizer_CPU.cu:158-226; the MEX command
   ApplyLaplacianRegularization_to_dJ, Mex.cu:505-531): with L the {-1,2,-1} Laplacian,
   out[0] = jReg = ||L volume||^2, dJ += 2*lambda * L(L volume) (lambda rounded to float as
   the reference passes it), and, when total_iteration < optimal_step_iteration_nb,
   out[1] = normdJProjReg = 2 ||L dJ||^2 (out[1] untouched otherwise). FP32 device volumes,
   `out` a device pointer to two doubles; stream-ordered scratch of one volume. */
tomo_status tomo_gg_regularization(const float* volume, float* dJ, int32_t nx, int32_t ny, int32_t nz, double lambda,
                                   int32_t total_iteration, int32_t optimal_step_iteration_nb, double* out,
                                   void* stream);
/* The same criterion for any shape parameter beta >= 1 (configIteration beta;
   GeneralizedGaussianRegularizer_CPU.cu:158-226 and GeneralizedGaussianRegularizer_GPU.cu:
   161-225, which take the same steps): out[0] = jReg = sum |L volume|^beta; for beta != 2
   g = sign(volume) |volume|^(beta-1) (the power of the volume itself, as the reference
   computes it), else g = L volume; dJ += beta*lambda * L(g); and, when total_iteration <
   optimal_step_iteration_nb, out[1] = normdJProjReg = beta * sum |L dJ|^beta. beta = 2 is
   tomo_gg_regularization. */
tomo_status tomo_gg_regularization_beta(const float* volume, float* dJ, int32_t nx, int32_t ny, int32_t nz,
                                        double lambda, double beta, int32_t total_iteration,
                                        int32_t optimal_step_iteration_nb, double* out, void* stream);
/* Huber regularisation criterion (HuberRegularizer_CPU::getLaplacianRegularizationCriterion,
   HuberRegularizer_CPU.cu:206-253; the MEX command ApplyLaplacianRegularization_to_dJ under
   penaltyFunction Huber): with g = L volume, out[0] = jReg = Huber norm of g
   (Image3D_CPU::getImageHuberNorm), dJ += lambda * L(psi'(g)) (lambda rounded to float), and,
   when total_iteration < optimal_step_iteration_nb, out[1] = normdJProjReg =
   sum |L(L(psi''(g) dJ)) dJ| (out[1] untouched otherwise). FP32 device volumes, `out` a device
   pointer to two doubles; stream-ordered scratch of two volumes. */
tomo_status tomo_huber_regularization(const float* volume, float* dJ, int32_t nx, int32_t ny, int32_t nz, double lambda,
                                      double huber_threshold, int32_t total_iteration,
                                      int32_t optimal_step_iteration_nb, double* out, void* stream);
/* Host-buffer forms (copies inside, synchronous, on `device`): the Laplacian of the
   reference's --op=laplacien, and one regulariser criterion call (kind TOMO_REG_GG with
   gg_beta, or TOMO_REG_HUBER with huber_threshold) of --op=reg_GG /
   ApplyLaplacianRegularization_to_dJ (Iter3D_main.cu:215-272).
   `out` is HOST memory for two doubles (jReg, normdJProjReg; the second kept when
   total_iteration >= optimal_step_iteration_nb). */
tomo_status tomo_laplacian_host(int device, const float* in, float* out, int32_t nx, int32_t ny, int32_t nz);
tomo_status tomo_regularization_host(int device, int32_t kind, const float* volume, float* dJ, int32_t nx, int32_t ny,
                                     int32_t nz, double lambda, double huber_threshold, double gg_beta,
                                     int32_t total_iteration, int32_t optimal_step_iteration_nb, double* out);
/* *out = sum (double)x*(double)x  (Image3D_CPU::getImageL2Norm); FP64 accumulation.
   `out` is a device pointer to one double. */
tomo_status tomo_sq_norm(const void* x, tomo_dtype dtype, size_t n, double* out, void* stream);
/* Convert between storage types (round to nearest even). */
tomo_status tomo_convert(const void* in, tomo_dtype in_dtype, void* out, tomo_dtype out_dtype, size_t n,
                         void* stream);

/* ---- real-data ingest (host only, no device) ---- */
/* The detector-file fields of the reference's configTiff (ConfigTiff.cpp:13-26). */
typedef struct {
    int32_t total_projection_nb;   /* totalProjectionNb: files on disk                      */
    int32_t used_projection_nb;    /* usedProjectionNb: every (total/used)-th file is read  */
    int32_t u_initial_nb;          /* uDetectorPixelInitialNb: columns of a file            */
    int32_t v_initial_nb;          /* vDetectorPixelInitialNb: rows of a file               */
    int32_t u_final_nb;            /* uDetectorPixelFinalNb: columns kept                   */
    int32_t v_final_nb;            /* vDetectorPixelFinalNb: rows kept                      */
    int32_t u_center_final;        /* uDetectorCenterFinal: centre column of the window     */
    int32_t v_center_final;        /* vDetectorCenterFinal: centre row of the window        */
    int32_t u_calibration_nb;      /* uCalibrationImagePixelNb                              */
    int32_t v_calibration_nb;      /* vCalibrationImagePixelNb                              */
    int32_t calibration_energy_nb; /* CalibrationEnergyNb: the white field is the last 1/E
                                      of the calibration image's rows                      */
    int32_t digits;                /* 5: <name>_%05d.tif (--op=tiff5), 4: _%04d (--op=tiff4) */
} tomo_tiff_config;

/* White level of a calibration file (ImageCalibration::getWhiteMeanValue,
   ImageTiff.cu:81-94): four 16-bit header words, nx*ny 16-bit pixels row-major; the mean
   over rows [(E-1)*ny/E, ny) divided as sum / (nx*ny/E) in FP64. */
tomo_status tomo_tiff_white_mean(const char* calibration_file, int32_t nx, int32_t ny, int32_t energy_nb,
                                 double* mean);
/* Normalised negative-log sinogram (ConfigTiff::createNormalizedMeanNegativeLogSinogram_5dig
   / _4dig, ConfigTiff.hpp:287-420): reads <tif_dir>/<tiff_name>_<p+1>.tif for p = total,
   total - rate, ... (used files, rate = total/used), crops the u_final x v_final window
   around the centre and writes -log(pixel / white) to `sinogram` (HOST FP32, used x v_final
   x u_final, view-major in the order read). */
tomo_status tomo_tiff_negative_log_sinogram(const tomo_tiff_config* config, const char* tif_dir,
                                            const char* tiff_name, const char* calibration_file,
                                            float* sinogram);

/* ---- synthetic inputs ---- */
/* Sum of ellipsoids on the [-1,1]^3 grid (phantom3d.m semantics, 10 doubles per row:
   A, a, b, c, x0, y0, z0, phi, theta, psi in degrees). `ellipsoids` is HOST memory,
   `volume` device memory (FP32, overwritten). */
tomo_status tomo_phantom(const double* ellipsoids, int32_t count, int32_t nx, int32_t ny, int32_t nz,
                         float* volume, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TOMOGPI_B200_H_ */
