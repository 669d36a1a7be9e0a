// shim_common.cpp -- TEST INFRASTRUCTURE ONLY: storage for the host-side stand-ins of
// the reference's __constant__ symbols and textures, and the geometry set-up that the
// reference's host classes perform before a launch.
#include "cuda_host_shim.h"

#include <cstring>

thread_local shim_dim3 threadIdx;
thread_local shim_dim3 blockIdx;
shim_dim3 blockDim;
shim_dim3 gridDim;

float alphaIOcylinderC_GPU[MAX_PROJECTION];
float betaIOcylinderC_GPU[MAX_PROJECTION];
float gammaIOcylinderC_GPU;
float xVolumeCenterPixel_GPU, yVolumeCenterPixel_GPU, zVolumeCenterPixel_GPU;
float xVolumePixelSize_GPU;
unsigned long int xVolumePixelNb_GPU, yVolumePixelNb_GPU, zVolumePixelNb_GPU;
float focusDetectorDistance_GPU, focusObjectDistance_GPU;
float uDetectorCenterPixel_GPU, vDetectorCenterPixel_GPU;
float uDetectorPixelSize_GPU, vDetectorPixelSize_GPU;
unsigned long int uDetectorPixelNb_GPU, vDetectorPixelNb_GPU, projectionNb_GPU;
float alphaC_GPU, betaC_GPU;

shim_tex3d volume_tex;
shim_tex2d_layered sinogram_tex0;

void shim_copy_constants(const ref_config_ct* c) {
    // UniformAcquisition: phi_p = (p + start) * pi * (stop - start) / P, in double.
    const double start = c->num_start_angle / c->den_start_angle;
    const double stop = c->num_stop_angle / c->den_stop_angle;
    const unsigned long np = (unsigned long)c->projection_nb;
    const double step = M_PI * (double)(stop - start) / np;
    for (unsigned long p = 0; p < np && p < MAX_PROJECTION; p++) {
        const double phi = ((int)p + start) * step;
        alphaIOcylinderC_GPU[p] = cos(phi);
        betaIOcylinderC_GPU[p] = sin(phi);
    }
    // Detector: pitch = size / count (float), centre = count/2 - 0.5 (double -> float).
    const float usize = c->u_detector_size, vsize = c->v_detector_size;
    const unsigned long nu = c->u_detector_pixel_nb, nv = c->v_detector_pixel_nb;
    uDetectorPixelSize_GPU = usize / nu;
    vDetectorPixelSize_GPU = vsize / nv;
    uDetectorCenterPixel_GPU = nu / 2.0 - 0.5;
    vDetectorCenterPixel_GPU = nv / 2.0 - 0.5;
    uDetectorPixelNb_GPU = nu;
    vDetectorPixelNb_GPU = nv;
    projectionNb_GPU = np;
    // Volume: voxel size = size / count, z voxel size := x voxel size.
    const float xsize = c->x_volume_size;
    const unsigned long nx = c->x_volume_pixel_nb, ny = c->y_volume_pixel_nb, nz = c->z_volume_pixel_nb;
    xVolumePixelSize_GPU = xsize / nx;
    xVolumeCenterPixel_GPU = nx / 2.0 - 0.5;
    yVolumeCenterPixel_GPU = ny / 2.0 - 0.5;
    zVolumeCenterPixel_GPU = nz / 2.0 - 0.5;
    xVolumePixelNb_GPU = nx;
    yVolumePixelNb_GPU = ny;
    zVolumePixelNb_GPU = nz;
    // Acquisition distances are stored double and copied to the device as float.
    const float fdd = c->fdd, fod = c->fod;
    focusDetectorDistance_GPU = fdd;
    focusObjectDistance_GPU = fod;
    const float zVolumePixelSize = xVolumePixelSize_GPU;
    gammaIOcylinderC_GPU = vDetectorPixelSize_GPU / (fdd * zVolumePixelSize);
    // BackProjector ctor (BackProjector.cu:34-35): double distances, float detector pitch,
    // stored as float members and copied as float.
    alphaC_GPU = (float)((M_PI * c->fod * c->fdd) / (double)np);
    betaC_GPU = (float)((c->fdd / (double)uDetectorPixelSize_GPU) * (c->fdd / (double)uDetectorPixelSize_GPU));
}
