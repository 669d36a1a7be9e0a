// ref_rs_um.cpp -- TEST INFRASTRUCTURE ONLY: runs the reference's own
// projection_ERB_kernel_v0_UM source (projection_ER_kernel_UM.cuh, included from the
// TomoGPI source tree at build time) on the host, one call per detector ray.
#include "cuda_host_shim.h"
#include "projection_ER_kernel_UM.cuh"

extern "C" void ref_rs_um_project(const ref_config_ct* c, const float* vol, float* sino) {
    shim_copy_constants(c);
    volume_tex = shim_tex3d{vol, c->x_volume_pixel_nb, c->y_volume_pixel_nb, c->z_volume_pixel_nb};
    blockDim = shim_dim3{1, 1, 1};
    gridDim = shim_dim3{(unsigned)c->u_detector_pixel_nb, (unsigned)c->v_detector_pixel_nb,
                        (unsigned)c->projection_nb};
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int p = 0; p < c->projection_nb; p++)
        for (int v = 0; v < c->v_detector_pixel_nb; v++)
            for (int u = 0; u < c->u_detector_pixel_nb; u++) {
                threadIdx = shim_dim3{0, 0, 0};
                blockIdx = shim_dim3{(unsigned)u, (unsigned)v, (unsigned)p};
                projection_ERB_kernel_v0_UM<float>(sino);
            }
}
