// cuda_host_shim.h -- TEST INFRASTRUCTURE ONLY.
//
// Lets the reference's own CUDA kernel sources (read in place from the TomoGPI source
// tree at build time; nothing of them is copied here) compile as host C++:
//   * __global__/__device__/__host__/__constant__ vanish,
//   * threadIdx/blockIdx are per-thread host globals set by the grid loop in
//     ref_kernels_*.cpp, blockDim/gridDim are host globals,
//   * the __constant__ geometry symbols of GPUConstant.cuh become host globals,
//   * tex3D / tex2DLayered become exact FP32 software filtering with border colour 0
//     and unnormalised coordinates (the CUDA filtering formula without its 8-bit
//     weight quantisation).
#pragma once
#include <math.h>
#include <cmath>
#include <cstdint>

#define __global__
#define __device__
#define __host__
#define __constant__
#define FOV_CYLINDER 0
#define MAX_PROJECTION 2400

struct shim_dim3 {
    unsigned int x, y, z;
};
extern thread_local shim_dim3 threadIdx;
extern thread_local shim_dim3 blockIdx;
extern shim_dim3 blockDim;
extern shim_dim3 gridDim;

// GPUConstant.cuh symbols used by the projector / backprojector kernels.
extern float alphaIOcylinderC_GPU[MAX_PROJECTION];
extern float betaIOcylinderC_GPU[MAX_PROJECTION];
extern float gammaIOcylinderC_GPU;
extern float xVolumeCenterPixel_GPU, yVolumeCenterPixel_GPU, zVolumeCenterPixel_GPU;
extern float xVolumePixelSize_GPU;
extern unsigned long int xVolumePixelNb_GPU, yVolumePixelNb_GPU, zVolumePixelNb_GPU;
extern float focusDetectorDistance_GPU, focusObjectDistance_GPU;
extern float uDetectorCenterPixel_GPU, vDetectorCenterPixel_GPU;
extern float uDetectorPixelSize_GPU, vDetectorPixelSize_GPU;
extern unsigned long int uDetectorPixelNb_GPU, vDetectorPixelNb_GPU, projectionNb_GPU;
extern float alphaC_GPU, betaC_GPU;

struct shim_tex3d {
    const float* d;
    long nx, ny, nz;
};
struct shim_tex2d_layered {
    const float* d;
    long nu, nv, nl;
};
extern shim_tex3d volume_tex;
extern shim_tex2d_layered sinogram_tex0;

static inline float shim_lerp(float a, float b, float t) { return (1.0f - t) * a + t * b; }

static inline float tex3D(const shim_tex3d& t, float x, float y, float z) {
    const float xb = x - 0.5f, yb = y - 0.5f, zb = z - 0.5f;
    if (!(xb > -1.0f && yb > -1.0f && zb > -1.0f && xb < (float)t.nx && yb < (float)t.ny && zb < (float)t.nz))
        return 0.0f;
    const float fx = std::floor(xb), fy = std::floor(yb), fz = std::floor(zb);
    const float a = xb - fx, b = yb - fy, c = zb - fz;
    const long i = (long)fx, j = (long)fy, k = (long)fz;
    auto at = [&](long ii, long jj, long kk) -> float {
        if (ii < 0 || jj < 0 || kk < 0 || ii >= t.nx || jj >= t.ny || kk >= t.nz) return 0.0f;
        return t.d[(kk * t.ny + jj) * t.nx + ii];
    };
    const float c00 = shim_lerp(at(i, j, k), at(i + 1, j, k), a);
    const float c10 = shim_lerp(at(i, j + 1, k), at(i + 1, j + 1, k), a);
    const float c01 = shim_lerp(at(i, j, k + 1), at(i + 1, j, k + 1), a);
    const float c11 = shim_lerp(at(i, j + 1, k + 1), at(i + 1, j + 1, k + 1), a);
    return shim_lerp(shim_lerp(c00, c10, b), shim_lerp(c01, c11, b), c);
}

static inline float tex2DLayered(const shim_tex2d_layered& t, float x, float y, int layer) {
    const float xb = x - 0.5f, yb = y - 0.5f;
    if (layer < 0 || layer >= t.nl) return 0.0f;
    if (!(xb > -1.0f && yb > -1.0f && xb < (float)t.nu && yb < (float)t.nv)) return 0.0f;
    const float fx = std::floor(xb), fy = std::floor(yb);
    const float a = xb - fx, b = yb - fy;
    const long i = (long)fx, j = (long)fy;
    const float* s = t.d + (long)layer * t.nu * t.nv;
    auto at = [&](long ii, long jj) -> float {
        if (ii < 0 || jj < 0 || ii >= t.nu || jj >= t.nv) return 0.0f;
        return s[jj * t.nu + ii];
    };
    return shim_lerp(shim_lerp(at(i, j), at(i + 1, j), a), shim_lerp(at(i, j + 1), at(i + 1, j + 1), a), b);
}

// Geometry set-up as the reference host code performs it (ConfigCT.cpp:112-121,
// Acquisition.cpp:90-97, Detector.cpp:9-15, Volume.cu:17-26, Projector.cu:16-38,
// RegularSamplingProjector_compute_CUDA_mem_CPU.cu:906-951).
extern "C" {
typedef struct {
    double fod, fdd;
    double num_start_angle, den_start_angle, num_stop_angle, den_stop_angle;
    int32_t projection_nb;
    float u_detector_size, v_detector_size;
    int32_t u_detector_pixel_nb, v_detector_pixel_nb;
    float x_volume_size, y_volume_size, z_volume_size;
    int32_t x_volume_pixel_nb, y_volume_pixel_nb, z_volume_pixel_nb;
} ref_config_ct;
}

void shim_copy_constants(const ref_config_ct* c);
