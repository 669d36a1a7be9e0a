// C entry point over the reference's own Iter3D::doSimpleGradient (Iter3D_Algo_Gradient.cu:
// 25-223) compiled on the host, with the reference's RS / VI kernel sources and GG / Huber
// regularisers under it. Writes the iterate in place. Test infrastructure only.
#include <cstring>
#include "Iter3D.cuh"

extern "C" void ref_simple_gradient(const ref_config_ct* c, float* vol, const float* real_sino, int iterations,
                                    double lambda, int optimal, int positivity, int huber, double huber_threshold) {
    RefIter3D it(*c, iterations, optimal, lambda, positivity, huber ? HUBER : GG, huber_threshold);
    const size_t nv = (size_t)c->x_volume_pixel_nb * c->y_volume_pixel_nb * c->z_volume_pixel_nb;
    const size_t ns = (size_t)c->u_detector_pixel_nb * c->v_detector_pixel_nb * c->projection_nb;
    Volume_CPU<float> v(c->x_volume_size, c->y_volume_size, c->z_volume_size, c->x_volume_pixel_nb,
                        c->y_volume_pixel_nb, c->z_volume_pixel_nb);
    Sinogram3D_CPU<float> g(c->u_detector_pixel_nb, c->v_detector_pixel_nb, c->projection_nb);
    std::memcpy(v.getVolumeData(), vol, nv * sizeof(float));
    std::memcpy(g.getDataSinogram(), real_sino, ns * sizeof(float));
    it.doSimpleGradient(&v, &g, nullptr);
    std::memcpy(vol, v.getVolumeData(), nv * sizeof(float));
}
