// TomoGPI.hpp -- header-only C++ drop-in for TomoGPI_lib's operator layer, over the C-ABI
// of libtomogpi_b200.so (include/tomogpi_b200.h).
//
// Same class names, constructor arguments and virtuals as the reference (paths inside the
// TomoGPI project):
//   Projector<V,S,T>::doProjection(S<T>*, V<T>*)             src/TomoGPI_lib/inc/Projector.cuh:113-138
//   BackProjector<V,S,T>::doBackProjection(V<T>*, S<T>*)     src/TomoGPI_lib/inc/BackProjector.cuh:139-180
//   RegularSamplingProjector_compute_CUDA_mem_CPU/_mem_GPU   src/TomoGPI_lib/inc/Projector_CPU.cuh:80-98,
//                                                            src/TomoGPI_lib/inc/Projector_GPU.cuh:15-36
//   SiddonProjector_compute_C_mem_CPU                        src/TomoGPI_lib/inc/Projector_CPU.cuh:34-42
//   VIBackProjector_compute_CUDA_mem_CPU/_mem_GPU            src/TomoGPI_lib/inc/BackProjector_CPU.cuh:14-36,
//                                                            src/TomoGPI_lib/inc/BackProjector_GPU.cuh:15-38
//   Acquisition / UniformAcquisition, Detector, Volume_CPU/GPU, Sinogram3D_CPU/GPU.
// Differences a caller sees: T is float only; errors throw tomogpi::Error (the reference
// calls exit); the CUDA*Architecture launch descriptors are accepted and ignored (the
// kernels choose their own launch shapes); SiddonProjector_compute_C_mem_CPU runs the
// Siddon traversal of the reference's C file on the GPU (host buffers in and out).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../tomogpi_b200.h"

namespace tomogpi {

struct Error : std::runtime_error {
    explicit Error(const std::string& m) : std::runtime_error(m) {}
};

inline void check(tomo_status s, const char* what) {
    if (s != TOMO_OK) throw Error(std::string(what) + ": " + tomo_last_error());
}

// Acquisition.hpp: distances (double), start/stop angle in units of pi, P views.
class Acquisition {
  public:
    Acquisition(double focusDetectorDistance, double focusObjectDistance, double startAngle, double stopAngle,
                unsigned long projectionNb)
        : fdd_(focusDetectorDistance), fod_(focusObjectDistance), start_(startAngle), stop_(stopAngle),
          np_(projectionNb) {}
    virtual ~Acquisition() = default;
    double getFocusDetectorDistance() const { return fdd_; }
    double getFocusObjectDistance() const { return fod_; }
    double getStartAngle() const { return start_; }
    double getStopAngle() const { return stop_; }
    unsigned long getProjectionNb() const { return np_; }

  private:
    double fdd_, fod_, start_, stop_;
    unsigned long np_;
};

class UniformAcquisition : public Acquisition {
  public:
    UniformAcquisition(double fdd, double fod, double startAngle, double stopAngle, double /*stepAngle*/,
                       unsigned long projectionNb)
        : Acquisition(fdd, fod, startAngle, stopAngle, projectionNb) {}
};

class Detector {
  public:
    Detector(float uDetectorSize, float vDetectorSize, unsigned long uDetectorPixelNb, unsigned long vDetectorPixelNb)
        : usize_(uDetectorSize), vsize_(vDetectorSize), nu_(uDetectorPixelNb), nv_(vDetectorPixelNb) {}
    float getUDetectorSize() const { return usize_; }
    float getVDetectorSize() const { return vsize_; }
    unsigned long getUDetectorPixelNb() const { return nu_; }
    unsigned long getVDetectorPixelNb() const { return nv_; }

  private:
    float usize_, vsize_;
    unsigned long nu_, nv_;
};

// Launch-shape descriptors of the reference (ComputingArchitecture.cuh:89-170): accepted
// for signature compatibility only.
struct CUDAProjectionArchitecture {};
struct CUDABProjectionArchitecture {};

// Containers. _CPU: host memory; _GPU: CUDA managed memory (as the reference's
// Image3D_GPU, src/TomoGPI_lib/src/CPP/Image3D_GPU.cu:18). Raw headerless files.
template <typename T>
class Volume_CPU {
  public:
    Volume_CPU(float xSize, float ySize, float zSize, unsigned long xNb, unsigned long yNb, unsigned long zNb)
        : xs_(xSize), ys_(ySize), zs_(zSize), nx_(xNb), ny_(yNb), nz_(zNb), data_(xNb * yNb * zNb, T(0)) {}
    virtual ~Volume_CPU() = default;
    T* getVolumeData() { return data_.data(); }
    float getXVolumeSize() const { return xs_; }
    float getYVolumeSize() const { return ys_; }
    float getZVolumeSize() const { return zs_; }
    unsigned long getXVolumePixelNb() const { return nx_; }
    unsigned long getYVolumePixelNb() const { return ny_; }
    unsigned long getZVolumePixelNb() const { return nz_; }
    void setVolume(T v) { std::fill(data_.begin(), data_.end(), v); }
    void saveVolume(const std::string& path) const { save_raw(path, data_.data(), data_.size()); }
    void loadVolume(const std::string& path) { load_raw(path, data_.data(), data_.size()); }

    static void save_raw(const std::string& path, const T* p, size_t n) {
        std::ofstream f(path, std::ios::binary);
        if (!f) throw Error("Unable to open file " + path);
        f.write(reinterpret_cast<const char*>(p), sizeof(T) * n);
    }
    static void load_raw(const std::string& path, T* p, size_t n) {
        std::ifstream f(path, std::ios::binary);
        if (!f) throw Error("Unable to open file " + path);
        f.read(reinterpret_cast<char*>(p), sizeof(T) * n);
        if ((size_t)f.gcount() != sizeof(T) * n) throw Error("short read from " + path);
    }

  protected:
    float xs_, ys_, zs_;
    unsigned long nx_, ny_, nz_;
    std::vector<T> data_;
};

template <typename T>
class Sinogram3D_CPU {
  public:
    Sinogram3D_CPU(unsigned long uNb, unsigned long vNb, unsigned long pNb)
        : nu_(uNb), nv_(vNb), np_(pNb), data_(uNb * vNb * pNb, T(0)) {}
    virtual ~Sinogram3D_CPU() = default;
    T* getDataSinogram() { return data_.data(); }
    unsigned long getUSinogramPixelNb() const { return nu_; }
    unsigned long getVSinogramPixelNb() const { return nv_; }
    unsigned long getProjectionSinogramNb() const { return np_; }
    void saveSinogram(const std::string& path) const { Volume_CPU<T>::save_raw(path, data_.data(), data_.size()); }
    void loadSinogram(const std::string& path) { Volume_CPU<T>::load_raw(path, data_.data(), data_.size()); }

  protected:
    unsigned long nu_, nv_, np_;
    std::vector<T> data_;
};

template <typename T>
class Volume_GPU {
  public:
    Volume_GPU(float xSize, float ySize, float zSize, unsigned long xNb, unsigned long yNb, unsigned long zNb)
        : xs_(xSize), ys_(ySize), zs_(zSize), nx_(xNb), ny_(yNb), nz_(zNb) {
        if (cudaMallocManaged(&d_, sizeof(T) * xNb * yNb * zNb) != cudaSuccess) throw Error("cudaMallocManaged failed");
        cudaMemset(d_, 0, sizeof(T) * xNb * yNb * zNb);
    }
    virtual ~Volume_GPU() { cudaFree(d_); }
    Volume_GPU(const Volume_GPU&) = delete;
    Volume_GPU& operator=(const Volume_GPU&) = delete;
    T* getVolumeData() { return d_; }
    float getXVolumeSize() const { return xs_; }
    float getYVolumeSize() const { return ys_; }
    float getZVolumeSize() const { return zs_; }
    unsigned long getXVolumePixelNb() const { return nx_; }
    unsigned long getYVolumePixelNb() const { return ny_; }
    unsigned long getZVolumePixelNb() const { return nz_; }

  private:
    float xs_, ys_, zs_;
    unsigned long nx_, ny_, nz_;
    T* d_ = nullptr;
};

template <typename T>
class Sinogram3D_GPU {
  public:
    Sinogram3D_GPU(unsigned long uNb, unsigned long vNb, unsigned long pNb) : nu_(uNb), nv_(vNb), np_(pNb) {
        if (cudaMallocManaged(&d_, sizeof(T) * uNb * vNb * pNb) != cudaSuccess) throw Error("cudaMallocManaged failed");
        cudaMemset(d_, 0, sizeof(T) * uNb * vNb * pNb);
    }
    virtual ~Sinogram3D_GPU() { cudaFree(d_); }
    Sinogram3D_GPU(const Sinogram3D_GPU&) = delete;
    Sinogram3D_GPU& operator=(const Sinogram3D_GPU&) = delete;
    T* getDataSinogram() { return d_; }
    unsigned long getUSinogramPixelNb() const { return nu_; }
    unsigned long getVSinogramPixelNb() const { return nv_; }
    unsigned long getProjectionSinogramNb() const { return np_; }

  private:
    unsigned long nu_, nv_, np_;
    T* d_ = nullptr;
};

// One tomo_context per (acquisition, detector, volume) geometry.
class Geometry {
  public:
    template <typename VOL>
    Geometry(Acquisition* a, Detector* d, VOL* v, int device = 0) {
        tomo_config_ct c{};
        c.fod = a->getFocusObjectDistance();
        c.fdd = a->getFocusDetectorDistance();
        c.num_start_angle = a->getStartAngle();
        c.den_start_angle = 1.0;
        c.num_stop_angle = a->getStopAngle();
        c.den_stop_angle = 1.0;
        c.projection_nb = (int32_t)a->getProjectionNb();
        c.u_detector_size = d->getUDetectorSize();
        c.v_detector_size = d->getVDetectorSize();
        c.u_detector_pixel_nb = (int32_t)d->getUDetectorPixelNb();
        c.v_detector_pixel_nb = (int32_t)d->getVDetectorPixelNb();
        c.x_volume_size = v->getXVolumeSize();
        c.y_volume_size = v->getYVolumeSize();
        c.z_volume_size = v->getZVolumeSize();
        c.x_volume_pixel_nb = (int32_t)v->getXVolumePixelNb();
        c.y_volume_pixel_nb = (int32_t)v->getYVolumePixelNb();
        c.z_volume_pixel_nb = (int32_t)v->getZVolumePixelNb();
        tomo_context* ctx = nullptr;
        check(tomo_context_create(&c, device, &ctx), "tomo_context_create");
        ctx_.reset(ctx, [](tomo_context* p) { tomo_context_destroy(p); });
    }
    tomo_context* get() const { return ctx_.get(); }

  private:
    std::shared_ptr<tomo_context> ctx_;
};

template <template <typename> class V, template <typename> class S, typename T>
class Projector {
    static_assert(std::is_same<T, float>::value, "tomogpi_b200 computes in FP32 (T = float)");

  public:
    Projector(Acquisition* acquisition, Detector* detector, V<T>* volume)
        : acquisition_(acquisition), detector_(detector), volume_(volume), geom_(acquisition, detector, volume) {}
    virtual ~Projector() = default;
    virtual void doProjection(S<T>* estimatedSinogram, V<T>* volume) = 0;
    Acquisition* getAcquisition() const { return acquisition_; }
    Detector* getDetector() const { return detector_; }
    V<T>* getVolume() const { return volume_; }
    void setVolume(V<T>* v) { volume_ = v; }
    void EnableP2P() {}
    void DisableP2P() {}

  protected:
    Acquisition* acquisition_;
    Detector* detector_;
    V<T>* volume_;
    Geometry geom_;
};

template <template <typename> class V, template <typename> class S, typename T>
class BackProjector {
  public:
    // fdk != 0: the FDK-weighted backprojection of FDK3D_VIB_kernel_v0_16reg
    // (BackProjector.cu:16-37 stores the flag; setFdk as Mex.cu:434-436 toggles it).
    BackProjector(Acquisition* acquisition, Detector* detector, V<T>* volume, char fdk)
        : acquisition_(acquisition), detector_(detector), volume_(volume), fdk_(fdk),
          geom_(acquisition, detector, volume) {}
    virtual ~BackProjector() = default;
    virtual void doBackProjection(V<T>* estimatedVolume, S<T>* sinogram) = 0;
    void setFdk(char fdk) { fdk_ = fdk; }
    char getFdk() const { return fdk_; }
    void EnableP2P() {}
    void DisableP2P() {}

  protected:
    Acquisition* acquisition_;
    Detector* detector_;
    V<T>* volume_;
    char fdk_;
    Geometry geom_;
};

template <typename T>
class RegularSamplingProjector_compute_CUDA_mem_CPU : public Projector<Volume_CPU, Sinogram3D_CPU, T> {
  public:
    RegularSamplingProjector_compute_CUDA_mem_CPU(Acquisition* a, Detector* d, CUDAProjectionArchitecture*,
                                                  Volume_CPU<T>* v)
        : Projector<Volume_CPU, Sinogram3D_CPU, T>(a, d, v) {}
    void doProjection(Sinogram3D_CPU<T>* s, Volume_CPU<T>* v) override {
        this->setVolume(v);
        check(tomo_project_host(this->geom_.get(), TOMO_PROJ_RS, v->getVolumeData(), s->getDataSinogram()),
              "RegularSamplingProjector_compute_CUDA_mem_CPU::doProjection");
    }
};

template <typename T>
class SiddonProjector_compute_C_mem_CPU : public Projector<Volume_CPU, Sinogram3D_CPU, T> {
  public:
    SiddonProjector_compute_C_mem_CPU(Acquisition* a, Detector* d, Volume_CPU<T>* v)
        : Projector<Volume_CPU, Sinogram3D_CPU, T>(a, d, v) {}
    void doProjection(Sinogram3D_CPU<T>* s, Volume_CPU<T>* v) override {
        this->setVolume(v);
        check(tomo_project_host(this->geom_.get(), TOMO_PROJ_SIDDON_REF, v->getVolumeData(), s->getDataSinogram()),
              "SiddonProjector_compute_C_mem_CPU::doProjection");
    }
};

template <typename T>
class RegularSamplingProjector_compute_CUDA_mem_GPU : public Projector<Volume_GPU, Sinogram3D_GPU, T> {
  public:
    RegularSamplingProjector_compute_CUDA_mem_GPU(Acquisition* a, Detector* d, CUDAProjectionArchitecture*,
                                                  Volume_GPU<T>* v)
        : Projector<Volume_GPU, Sinogram3D_GPU, T>(a, d, v) {}
    void doProjection(Sinogram3D_GPU<T>* s, Volume_GPU<T>* v) override {
        this->setVolume(v);
        check(tomo_project(this->geom_.get(), TOMO_PROJ_RS_UM, v->getVolumeData(), TOMO_F32, s->getDataSinogram(),
                           TOMO_F32, nullptr),
              "RegularSamplingProjector_compute_CUDA_mem_GPU::doProjection");
        if (cudaDeviceSynchronize() != cudaSuccess) throw Error("cudaDeviceSynchronize failed");
    }
};

template <typename T>
class VIBackProjector_compute_CUDA_mem_CPU : public BackProjector<Volume_CPU, Sinogram3D_CPU, T> {
  public:
    VIBackProjector_compute_CUDA_mem_CPU(Acquisition* a, Detector* d, CUDABProjectionArchitecture*, Volume_CPU<T>* v,
                                         char fdk)
        : BackProjector<Volume_CPU, Sinogram3D_CPU, T>(a, d, v, fdk) {}
    void doBackProjection(Volume_CPU<T>* v, Sinogram3D_CPU<T>* s) override {
        check(tomo_backproject_host(this->geom_.get(), this->fdk_ ? TOMO_BACK_FDK : TOMO_BACK_VI, s->getDataSinogram(),
                                    v->getVolumeData()),
              "VIBackProjector_compute_CUDA_mem_CPU::doBackProjection");
    }
};

template <typename T>
class VIBackProjector_compute_CUDA_mem_GPU : public BackProjector<Volume_GPU, Sinogram3D_GPU, T> {
  public:
    VIBackProjector_compute_CUDA_mem_GPU(Acquisition* a, Detector* d, CUDABProjectionArchitecture*, Volume_GPU<T>* v,
                                         char fdk)
        : BackProjector<Volume_GPU, Sinogram3D_GPU, T>(a, d, v, fdk) {}
    void doBackProjection(Volume_GPU<T>* v, Sinogram3D_GPU<T>* s) override {
        // the reference's mem_GPU backprojector keeps the fdk flag but never reads it
        // (VIBackProjector_compute_CUDA_mem_GPU.cu): always the unweighted VI_UM kernel
        check(tomo_backproject(this->geom_.get(), TOMO_BACK_VI_UM, s->getDataSinogram(), TOMO_F32,
                               v->getVolumeData(), TOMO_F32, nullptr),
              "VIBackProjector_compute_CUDA_mem_GPU::doBackProjection");
        if (cudaDeviceSynchronize() != cudaSuccess) throw Error("cudaDeviceSynchronize failed");
    }
};

}  // namespace tomogpi
