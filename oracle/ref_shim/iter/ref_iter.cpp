// C entry point over the reference's own Iter3D::doSimpleGradient (Iter3D_Algo_Gradient.cu:
// 25-223) and Iter3D::doWeightedGradient (:227-373) compiled on the host, with the
// reference's RS / VI kernel sources and GG (shape beta) / Huber regularisers under it. With
// weights != NULL the weighted loop runs; the sinogram it loads from
// <sinogramDirectory>/weightedSinogram.s (:243-248) is `weights`. Writes the iterate in
// place. Test infrastructure only.
#include <cstring>
#include "Iter3D.cuh"

const float* shim_weight_sinogram = nullptr;

extern "C" void ref_gradient(const ref_config_ct* c, float* vol, const float* real_sino, int iterations,
                             double lambda, int optimal, int positivity, int huber, double huber_threshold,
                             double beta, const float* weights) {
    RefIter3D it(*c, iterations, optimal, lambda, positivity, huber ? HUBER : GG, huber_threshold, beta);
    const size_t nv = (size_t)c->x_volume_pixel_nb * c->y_volume_pixel_nb * c->z_volume_pixel_nb;
    const size_t ns = (size_t)c->u_detector_pixel_nb * c->v_detector_pixel_nb * c->projection_nb;
    Volume_CPU<float> v(c->x_volume_size, c->y_volume_size, c->z_volume_size, c->x_volume_pixel_nb,
                        c->y_volume_pixel_nb, c->z_volume_pixel_nb);
    Sinogram3D_CPU<float> g(c->u_detector_pixel_nb, c->v_detector_pixel_nb, c->projection_nb);
    std::memcpy(v.getVolumeData(), vol, nv * sizeof(float));
    std::memcpy(g.getDataSinogram(), real_sino, ns * sizeof(float));
    shim_weight_sinogram = weights;
    if (weights)
        it.doWeightedGradient(&v, &g, nullptr);
    else
        it.doSimpleGradient(&v, &g, nullptr);
    shim_weight_sinogram = nullptr;
    std::memcpy(vol, v.getVolumeData(), nv * sizeof(float));
}
