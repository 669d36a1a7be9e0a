// C entry points over the reference's own regularisation criteria, compiled on the host for
// the oracle: GeneralizedGaussianRegularizer_CPU<float>::getLaplacianRegularizationCriterion
// (GeneralizedGaussianRegularizer_CPU.cu:158-226) and
// HuberRegularizer_CPU<float>::getLaplacianRegularizationCriterion (HuberRegularizer_CPU.cu:
// 206-253), built with COMPUTE_J so that jReg is computed. The GG shape beta is the
// regulariser's constructor argument (configIteration beta). dJ is updated in place; out[0] =
// jReg, out[1] = normdJProjReg (written only while total < optimal). Test infrastructure only.
#include <cstring>
#include "GeneralizedGaussianRegularizer_CPU.cuh"
#include "HuberRegularizer_CPU.cuh"

namespace {
template <class R>
void run(R& reg, const float* vol, float* dj, int nx, int ny, int nz, float lambda, int total, int opt, double* out) {
    Volume_CPU<float> v((float)nx, (float)ny, (float)nz, nx, ny, nz), d((float)nx, (float)ny, (float)nz, nx, ny, nz);
    const size_t n = (size_t)nx * ny * nz;
    std::memcpy(v.getVolumeData(), vol, n * sizeof(float));
    std::memcpy(d.getVolumeData(), dj, n * sizeof(float));
    reg.getLaplacianRegularizationCriterion(&v, &d, out, out + 1, lambda, (unsigned)total, (unsigned)opt);
    std::memcpy(dj, d.getVolumeData(), n * sizeof(float));
}
}  // namespace

extern "C" {
void ref_gg_criterion(const float* vol, float* dj, int nx, int ny, int nz, float lambda, double beta, int total,
                      int opt, double* out) {
    GeneralizedGaussianRegularizer_CPU<float> reg(beta);
    run(reg, vol, dj, nx, ny, nz, lambda, total, opt, out);
}
void ref_huber_criterion(const float* vol, float* dj, int nx, int ny, int nz, float lambda, double thr, int total,
                         int opt, double* out) {
    HuberRegularizer_CPU<float> reg(thr);
    run(reg, vol, dj, nx, ny, nz, lambda, total, opt, out);
}
}
