// tomo_solver.cuh -- launcher declarations of the gradient-loop kernels (gd.cu).
#pragma once

#include "tomo_kernels.cuh"

namespace tomo {

cudaError_t launch_laplacian_axpy(const float* in, float* dj, float w, int nx, int ny, int nz, cudaStream_t st);
// nrm[0] += ||dJ||^2 and, with want_lap, nrm[2] += sum |L dJ|^beta.
// amax (optional): also the FP32 bits of max|dJ| (atomicMax), for the FP16 range guard.
// part (optional, reduce_blocks(...) x 2 doubles): per-block partials summed in a fixed order
// into nrm[0] and nrm[2] (the same totals on every run); without it, atomics add the blocks.
cudaError_t launch_laplacian_norm(const float* dj, double* nrm, int nx, int ny, int nz, int want_lap, cudaStream_t st,
                                  unsigned* amax = nullptr, double beta = 2.0, double* part = nullptr);
// Blocks of the volume reductions (laplacian_norm, huber_l1).
size_t reduce_blocks(int nx, int ny, int nz);
// amax (optional): nrm[1] is the squared norm of the projection of 2^-k dJ (FP16 range guard).
cudaError_t launch_gd_alpha(const double* nrm, double* state, double* log, int it, int optimal_step_nb, double lambda,
                            int reg, cudaStream_t st, const unsigned* amax = nullptr, double beta = 2.0);
// out = sign(f) * |f|^p (the generalised-Gaussian gradient input for beta = p + 1 != 2).
cudaError_t launch_gg_abspow(const float* f, float* out, size_t n, double p, cudaStream_t st);
// *out += sum |x|^p in FP64.
cudaError_t launch_lp_norm(const float* x, size_t n, double p, double* out, cudaStream_t st);
// r *= w element-wise: r a residual view, w a plain [p][v][u] FP32 sinogram.
cudaError_t launch_sino_weight(OutView<float> r, const float* w, int nu, int nv, int np, cudaStream_t st);
// r = real - r element-wise: r a residual view holding a projection, real a plain [p][v][u]
// sinogram of type rdt.
cudaError_t launch_sino_residual(OutView<float> r, const void* real, tomo_dtype rdt, int nu, int nv, int np,
                                 cudaStream_t st);
cudaError_t launch_gd_update(float* f, const float* dj, const double* state, size_t n, int positivity,
                             cudaStream_t st);
cudaError_t launch_fill_double(double* p, int n, double v, cudaStream_t st);
cudaError_t launch_gg_finish(const double* nrm, double* out, cudaStream_t st, double beta = 2.0);
cudaError_t launch_huber_jreg(const float* g, size_t n, double thr, double* out, cudaStream_t st);
cudaError_t launch_huber_axpy(const float* grad, float* dj, float w, double thr, int nx, int ny, int nz,
                              cudaStream_t st);
cudaError_t launch_huber_norm(const float* grad, const float* dj, float* t, double thr, double* out, int nx, int ny,
                              int nz, cudaStream_t st, double* part = nullptr);
cudaError_t launch_phantom(const double* ell_host, int count, int nx, int ny, int nz, float* out, void** scratch,
                           cudaStream_t st);

}  // namespace tomo
