// geometry.cu -- host-side geometry set-up, exactly as the reference's host classes do it
// (ConfigCT::createUniformAcquisition ConfigCT.cpp:112-121, UniformAcquisition
// Acquisition.cpp:90-97, Detector Detector.cpp:9-15, Volume Volume.cu:17-26, the
// Projector/BackProjector constructors Projector.cu:16-38 / BackProjector.cu:16-37, and the
// float values copyConstantGPU uploads, RegularSamplingProjector_compute_CUDA_mem_CPU.cu:906-951).
#include <cmath>

#include "tomo_kernels.cuh"

namespace tomo {


void derive_geometry(const tomo_config_ct& c, HostGeom& h) {
    // UniformAcquisition (Acquisition.cpp:90-97) with the step of ConfigCT.cpp:119.
    const double start = c.num_start_angle / c.den_start_angle;
    const double stop = c.num_stop_angle / c.den_stop_angle;
    const unsigned long np = (unsigned long)c.projection_nb;
    const double step = M_PI * (double)(stop - start) / np;
    h.np = c.projection_nb;
    h.p0 = 0;
    h.alpha.resize(h.np);
    h.beta.resize(h.np);
    for (int p = 0; p < h.np; ++p) {
        const double phi = (p + start) * step;
        h.alpha[p] = (float)cos(phi);  // Projector.cu:33
        h.beta[p] = (float)sin(phi);   // Projector.cu:34
    }
    // Detector (Detector.cpp:9-15).
    h.nu = c.u_detector_pixel_nb;
    h.nv = c.v_detector_pixel_nb;
    h.du = c.u_detector_size / (float)(unsigned long)h.nu;
    h.dv = c.v_detector_size / (float)(unsigned long)h.nv;
    h.uc = (float)((unsigned long)h.nu / 2.0 - 0.5);
    h.vc = (float)((unsigned long)h.nv / 2.0 - 0.5);
    // Volume (Volume.cu:17-26); zVolumePixelSize := xVolumePixelSize.
    h.nx = c.x_volume_pixel_nb;
    h.ny = c.y_volume_pixel_nb;
    h.nz = c.z_volume_pixel_nb;
    h.dx = c.x_volume_size / (float)(unsigned long)h.nx;
    h.xc = (float)((unsigned long)h.nx / 2.0 - 0.5);
    h.yc = (float)((unsigned long)h.ny / 2.0 - 0.5);
    h.zc = (float)((unsigned long)h.nz / 2.0 - 0.5);
    // Acquisition distances are double in the reference and uploaded as float.
    h.fod = (float)c.fod;
    h.fdd = (float)c.fdd;
    h.gamma = h.dv / (h.fdd * h.dx);  // Projector.cu:27
    h.inv_gamma_f = 1.0f / h.gamma;
    h.inv_gamma_d = 1.0 / (double)h.gamma;
    const float fdu = h.fdd / h.du;
    // FDK weights (BackProjector.cu:34-35): alphaC = pi FOD FDD / P and betaC = (FDD / du)^2,
    // in double from the double distances, stored as float.
    h.fdk_alpha = (float)((M_PI * c.fod * c.fdd) / (double)np);
    h.fdk_beta = (float)((c.fdd / (double)h.du) * (c.fdd / (double)h.du));
    h.fdd_du = fdu;
    h.vi.resize(h.np);
    for (int p = 0; p < h.np; ++p) {
        const float a = h.alpha[p], b = h.beta[p];
        h.vi[p] = make_float4((-b * h.dx) * fdu, (a * h.dx) * fdu, a * h.dx, b * h.dx);
    }
    order_views(h);
}

void order_views(HostGeom& h) {
    h.view_order.clear();
    for (int p = 0; p < h.np; ++p)
        if (std::fabs(h.alpha[p]) > std::fabs(h.beta[p])) h.view_order.push_back(p);
    h.view_cols = (int)h.view_order.size();
    for (int p = 0; p < h.np; ++p)
        if (!(std::fabs(h.alpha[p]) > std::fabs(h.beta[p]))) h.view_order.push_back(p);
}


void select_views(HostGeom& h, int begin, int count) {
    h.alpha = std::vector<float>(h.alpha.begin() + begin, h.alpha.begin() + begin + count);
    h.beta = std::vector<float>(h.beta.begin() + begin, h.beta.begin() + begin + count);
    h.vi = std::vector<float4>(h.vi.begin() + begin, h.vi.begin() + begin + count);
    h.np = count;
    h.p0 += begin;
    order_views(h);
}


void fill_devgeom(const HostGeom& h, const float* d_alpha, const float* d_beta, const float4* d_vi, DevGeom& g,
                  const int* d_order) {
    g.fod = h.fod; g.fdd = h.fdd; g.gamma = h.gamma; g.du = h.du; g.dv = h.dv; g.uc = h.uc; g.vc = h.vc;
    g.dx = h.dx; g.xc = h.xc; g.yc = h.yc; g.zc = h.zc;
    g.inv_gamma_f = h.inv_gamma_f; g.inv_gamma_d = h.inv_gamma_d;
    g.fdk_alpha = h.fdk_alpha; g.fdk_beta = h.fdk_beta; g.fdd_du = h.fdd_du;
    g.nx = h.nx; g.ny = h.ny; g.nz = h.nz; g.nu = h.nu; g.nv = h.nv; g.np = h.np; g.p0 = h.p0;
    g.alpha = d_alpha; g.beta = d_beta; g.vi = d_vi;
    g.rs_wlog = RS_WLOG_DEFAULT;
    g.rs_tlog = RS_TLOG_DEFAULT;
    g.view_order = d_order;
    g.view_cols = h.view_cols;
}

}  // namespace tomo
