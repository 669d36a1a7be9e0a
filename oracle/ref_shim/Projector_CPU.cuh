// Projector_CPU.cuh (host shim) -- TEST INFRASTRUCTURE ONLY.
//
// Stands in for the reference header of the same name so that the reference's
// SiddonProjector_compute_C_mem_CPU.cpp compiles unmodified for the host. It declares
// only what that file uses: the container getters, the geometry getters and the
// Siddon class itself. Like the reference's Projector.cuh it includes <math.h> and
// <cmath>, so the float overloads of fabs/floor/ceil are the ones the file binds to.
#pragma once
#include <math.h>
#include <cmath>
#include <iostream>
#include <sys/types.h>

template <typename T>
class Volume_CPU {
  public:
    T* data;
    float xc, yc, zc, dx;
    unsigned long nx, ny, nz;
    T* getVolumeData() { return data; }
    float getXVolumeCenterPixel() { return xc; }
    float getYVolumeCenterPixel() { return yc; }
    float getZVolumeCenterPixel() { return zc; }
    float getXVolumePixelSize() { return dx; }
    unsigned long int getXVolumePixelNb() { return nx; }
    unsigned long int getYVolumePixelNb() { return ny; }
    unsigned long int getZVolumePixelNb() { return nz; }
};

template <typename T>
class Sinogram3D_CPU {
  public:
    T* data;
    T* getDataSinogram() { return data; }
};

class Acquisition {
  public:
    double fdd, fod;
    unsigned long np;
    double getFocusDetectorDistance() { return fdd; }
    double getFocusObjectDistance() { return fod; }
    unsigned long int getProjectionNb() { return np; }
};

class Detector {
  public:
    float uc, vc, du, dv;
    unsigned long nu, nv;
    float getUDetectorCenterPixel() { return uc; }
    float getVDetectorCenterPixel() { return vc; }
    float getUDetectorPixelSize() { return du; }
    float getVDetectorPixelSize() { return dv; }
    unsigned long int getUDetectorPixelNb() { return nu; }
    unsigned long int getVDetectorPixelNb() { return nv; }
};

template <template <typename> class V, template <typename> class S, typename T>
class Projector {
  public:
    Projector(Acquisition* a, Detector* d, V<T>* v) : acquisition(a), detector(d), volume(v) {}
    virtual ~Projector() {}
    Acquisition* getAcquisition() const { return acquisition; }
    Detector* getDetector() const { return detector; }
    V<T>* getVolume() const { return volume; }
    void setVolume(V<T>* v) { volume = v; }
    float* getAlphaIOcylinderC() { return alpha; }
    float* getBetaIOcylinderC() { return beta; }
    float* alpha = nullptr;
    float* beta = nullptr;

  private:
    Acquisition* acquisition;
    Detector* detector;
    V<T>* volume;
};

template <typename T>
class SiddonProjector_compute_C_mem_CPU : public Projector<Volume_CPU, Sinogram3D_CPU, T> {
  public:
    SiddonProjector_compute_C_mem_CPU(Acquisition* acquisition, Detector* detector, Volume_CPU<T>* volume);
    ~SiddonProjector_compute_C_mem_CPU();
    void doProjection(Sinogram3D_CPU<T>* estimatedSinogram, Volume_CPU<T>* volume);
    void EnableP2P();
    void DisableP2P();
};
