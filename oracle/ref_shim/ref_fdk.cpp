// ref_fdk.cpp -- TEST INFRASTRUCTURE ONLY: runs the reference's own
// FDK3D_VIB_kernel_v0_16reg source (FDK3D_kernel_16reg.cuh, included from the TomoGPI
// source tree at build time) on the host, one call per (x, y) column and 16-slice chunk,
// with the whole sinogram as the layered texture (vn_start = 0).
#include "cuda_host_shim.h"
#include "FDK3D_kernel_16reg.cuh"

extern "C" void ref_fdk_backproject(const ref_config_ct* c, const float* sino, float* vol) {
    shim_copy_constants(c);
    sinogram_tex0 = shim_tex2d_layered{sino, c->u_detector_pixel_nb, c->v_detector_pixel_nb, c->projection_nb};
    const long nx = c->x_volume_pixel_nb, ny = c->y_volume_pixel_nb, nz = c->z_volume_pixel_nb;
    blockDim = shim_dim3{1, 1, 1};
    gridDim = shim_dim3{(unsigned)nx, (unsigned)ny, 1};
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (long zc = 0; zc < nz / 16; zc++)
        for (long y = 0; y < ny; y++)
            for (long x = 0; x < nx; x++) {
                threadIdx = shim_dim3{0, 0, 0};
                blockIdx = shim_dim3{(unsigned)x, (unsigned)y, 0};
                FDK3D_VIB_kernel_v0_16reg<float>(vol + zc * 16 * nx * ny, 0, (int)(zc * 16), c->projection_nb, 0);
            }
}
