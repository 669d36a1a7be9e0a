// ref_siddon.cpp -- TEST INFRASTRUCTURE ONLY: compiles the reference's
// SiddonProjector_compute_C_mem_CPU.cpp unmodified (included from the TomoGPI source tree
// at build time, against the Projector_CPU.cuh shim in this directory) and runs its
// doProjection, single-threaded as written.
#include "cuda_host_shim.h"
#include "SiddonProjector_compute_C_mem_CPU.cpp"

template class SiddonProjector_compute_C_mem_CPU<float>;

extern "C" void ref_siddon_project(const ref_config_ct* c, const float* vol, float* sino) {
    shim_copy_constants(c);
    Acquisition acq;
    acq.fdd = c->fdd;
    acq.fod = c->fod;
    acq.np = (unsigned long)c->projection_nb;
    Detector det;
    det.uc = uDetectorCenterPixel_GPU;
    det.vc = vDetectorCenterPixel_GPU;
    det.du = uDetectorPixelSize_GPU;
    det.dv = vDetectorPixelSize_GPU;
    det.nu = (unsigned long)c->u_detector_pixel_nb;
    det.nv = (unsigned long)c->v_detector_pixel_nb;
    Volume_CPU<float> v;
    v.data = const_cast<float*>(vol);
    v.xc = xVolumeCenterPixel_GPU;
    v.yc = yVolumeCenterPixel_GPU;
    v.zc = zVolumeCenterPixel_GPU;
    v.dx = xVolumePixelSize_GPU;
    v.nx = xVolumePixelNb_GPU;
    v.ny = yVolumePixelNb_GPU;
    v.nz = zVolumePixelNb_GPU;
    Sinogram3D_CPU<float> s;
    s.data = sino;
    SiddonProjector_compute_C_mem_CPU<float> proj(&acq, &det, &v);
    proj.alpha = alphaIOcylinderC_GPU;
    proj.beta = betaIOcylinderC_GPU;
    std::streambuf* old = std::cout.rdbuf(nullptr);  // silence its progress line
    proj.doProjection(&s, &v);
    std::cout.rdbuf(old);
}
