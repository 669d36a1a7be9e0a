// Stand-in for the reference's Iter3D.cuh when its gradient loops
// (Iter3D_Algo_Gradient.cu) are compiled on the host for the oracle: an Iter3D class
// template with the members the loops call, a projector and a backprojector that run the
// reference's own kernel sources built for the host (ref_rs_box_project,
// ref_vi_backproject of the oracle's reference build), the reference's GG and Huber
// regularisers, and a host sinogram. doSimpleGradient and doWeightedGradient are
// instantiated. Test infrastructure only.
#pragma once
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <iostream>
#include <string>
#include <vector>

#include "GeneralizedGaussianRegularizer_CPU.cuh"
#include "HuberRegularizer_CPU.cuh"
using namespace std;

// ---- CUDA runtime names the loops mention (events for a timing print only) ----
typedef int cudaError_t;
typedef void* cudaEvent_t;
inline cudaError_t cudaEventCreate(cudaEvent_t*) { return 0; }
inline cudaError_t cudaEventRecord(cudaEvent_t, void*) { return 0; }
inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return 0; }
inline cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t, cudaEvent_t) { *ms = 0.f; return 0; }
#define checkCudaErrors(x) (void)(x)

typedef enum { HUBER, GG } kind_reg;  // Iter3D.cuh:58

// The loops append a timing line to ./timings.log; the host build writes nothing.
struct shim_null_ofstream {
    void open(const char*, std::ios_base::openmode = std::ios_base::out) {}
    void open(const std::string&, std::ios_base::openmode = std::ios_base::out) {}
    void close() {}
    template <class X> shim_null_ofstream& operator<<(const X&) { return *this; }
};
#define ofstream shim_null_ofstream

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
void ref_rs_box_project(const ref_config_ct* c, const float* vol, float* sino);
void ref_vi_backproject(const ref_config_ct* c, const float* sino, float* vol);
}

// The weight sinogram of the weighted loop, set by the entry point (ref_iter.cpp).
extern const float* shim_weight_sinogram;

// Sinogram3D_CPU: diffSinogram (Sinogram3D_CPU.cu:311-336), multSinogram (:154-169),
// getSinogramL2Norm (:358-374); loadSinogram reads the entry point's weight sinogram in place
// of the file.
template <typename T> class Sinogram3D_CPU {
public:
    Sinogram3D_CPU(unsigned long u, unsigned long v, unsigned long p) : nu_(u), nv_(v), np_(p), d_(u * v * p, T(0)) {}
    T* getDataSinogram() { return d_.data(); }
    unsigned long getDataSinogramSize() const { return (unsigned long)d_.size(); }
    void diffSinogram(Sinogram3D_CPU<T>* s1, Sinogram3D_CPU<T>* s2) {
        for (size_t i = 0; i < d_.size(); ++i) d_[i] = s1->d_[i] - s2->d_[i];
    }
    void multSinogram(Sinogram3D_CPU<T>* s) {
        for (size_t i = 0; i < d_.size(); ++i) d_[i] = d_[i] * s->d_[i];
    }
    void loadSinogram(const string&) {
        if (!shim_weight_sinogram) std::abort();
        for (size_t i = 0; i < d_.size(); ++i) d_[i] = (T)shim_weight_sinogram[i];
    }
    double getSinogramL2Norm() {
        double s = 0.0;
        for (size_t i = 0; i < d_.size(); ++i) s += double(d_[i] * d_[i]);
        return s;
    }
    double getSinogramMeanSquare() { return getSinogramL2Norm() / (double)d_.size(); }

private:
    unsigned long nu_, nv_, np_;
    std::vector<T> d_;
};

// Projector / backprojector over the reference's kernel sources built for the host;
// updateVolume as Projector.cu:110-124.
template <typename T> class RefRSProjector {
public:
    explicit RefRSProjector(const ref_config_ct& c) : c_(c) {}
    void doProjection(Sinogram3D_CPU<T>* s, Volume_CPU<T>* v) { ref_rs_box_project(&c_, v->getVolumeData(), s->getDataSinogram()); }
    void updateVolume(Volume_CPU<T>* out, Volume_CPU<T>* in, double lambda, int positive) {
        if (positive) out->positiveAddVolume(in, lambda);
        else out->addVolume(in, lambda);
    }

private:
    ref_config_ct c_;
};
template <typename T> class RefVIBackProjector {
public:
    explicit RefVIBackProjector(const ref_config_ct& c) : c_(c) {}
    void doBackProjection(Volume_CPU<T>* v, Sinogram3D_CPU<T>* s) { ref_vi_backproject(&c_, s->getDataSinogram(), v->getVolumeData()); }
    void DisableP2P() {}
    void EnableP2P() {}

private:
    ref_config_ct c_;
};

struct ShimConfigIteration {
    void updateLogFile(unsigned, double, double, double, double, double, double) {}
};
struct ShimConfigArch {
    int getGpuNb_proj() { return 1; }
    int getprojectionStreamsNb() { return 1; }
    int getStorage() { return 0; }
    int getPrecision() { return 1; }
};

template <template <typename> class P, template <typename> class BP, template <typename> class R_Huber,
          template <typename> class R_GG, template <typename> class C, template <typename> class V,
          template <typename> class S, typename T>
class Iter3D {
public:
    Iter3D(const ref_config_ct& c, int iterations, int optimal, double lambda, int positivity, kind_reg reg,
           double huber, double beta)
        : cfg_(c), proj_(c), back_(c), gg_(beta), huber_(huber), iterations_(iterations), optimal_(optimal),
          lambda_(lambda), positivity_(positivity), reg_(reg) {}
    P<T>* getProjector() { return &proj_; }
    BP<T>* getBackprojector() { return &back_; }
    R_GG<T>* getRegularizer_GG() { return &gg_; }
    R_Huber<T>* getRegularizer_Huber() { return &huber_; }
    kind_reg getKind_Regularizer() const { return reg_; }
    unsigned int getGradientIterationNb() const { return iterations_; }
    unsigned int getOptimalStepIterationNb() const { return optimal_; }
    unsigned int getGlobalIterationNb() const { return 1; }
    double getLambda() const { return lambda_; }
    char getPositivity() const { return (char)positivity_; }
    string getOutputDirectory() const { return "./"; }
    ShimConfigIteration* getConfigIterationFile() { return &cit_; }
    ShimConfigArch* getConfigComputeArchitectureFile() { return &arch_; }
    V<T>* create_volume() {
        return new V<T>(cfg_.x_volume_size, cfg_.y_volume_size, cfg_.z_volume_size, cfg_.x_volume_pixel_nb,
                        cfg_.y_volume_pixel_nb, cfg_.z_volume_pixel_nb);
    }
    S<T>* create_sinogram3D() {
        return new S<T>(cfg_.u_detector_pixel_nb, cfg_.v_detector_pixel_nb, cfg_.projection_nb);
    }
    void Init1_SG(V<T>* volume, S<T>* sino);
    void Init2_SG(V<T>* volume, V<T>* dJ, S<T>* sino);
    void Init3_SG(S<T>* sino);
    void doSimpleGradient(V<T>* volume, S<T>* realSinogram, V<T>* realVolume);
    void doWeightedGradient(V<T>* volume, S<T>* realSinogram, V<T>* realVolume);
    void doConjugateGradient(V<T>* volume, S<T>* realSinogram, V<T>* realVolume);
    void doProjBack(V<T>* volume);
    string sinogramDirectory = ".";

private:
    ref_config_ct cfg_;
    P<T> proj_;
    BP<T> back_;
    R_GG<T> gg_;
    R_Huber<T> huber_;
    ShimConfigIteration cit_;
    ShimConfigArch arch_;
    unsigned int iterations_, optimal_;
    double lambda_;
    int positivity_;
    kind_reg reg_;
};

typedef Iter3D<RefRSProjector, RefVIBackProjector, HuberRegularizer_CPU, GeneralizedGaussianRegularizer_CPU,
               Convolution3D_CPU, Volume_CPU, Sinogram3D_CPU, float>
    RefIter3D;
