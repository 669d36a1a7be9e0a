// Stand-in for the reference's Volume_CPU.cuh (and the Image3D_CPU / Convolution3D_CPU
// classes it brings in) when the reference's regulariser sources
// (GeneralizedGaussianRegularizer_CPU.cu, HuberRegularizer_CPU.cu) are compiled on the
// host for the oracle. Test infrastructure only.
//
// Volume_CPU<T>: host volume with the element-wise operations the regularisers call,
// restated from Image3D_CPU.cu (addImage :151-170, diffImage :207-285, multImage
// :287-312, scalarProductImage :314-342, getImageL1Norm :344-361, getImageL2Norm :363-392,
// getImageLpNorm :396-413, getImageHuberNorm :415-440; sequential z, y, x order).
// getVolumeSign is getImageSign (:523-546) with the sign of Image3D_GPU_kernel.cuh:10
// (+1, -1, 0); getVolumeAbsPow is the loop body of getImageAbsPow (:564) run over every
// voxel: the reference's z loop there runs a print statement in place of that body (:561),
// so its own CPU form leaves the output unwritten, while the device form
// (Image3D_GPU_kernel.cuh:687-700) writes every voxel.
// Convolution3D_CPU<T>: the sum of the three 1-D convolutions with zero padding, per axis
// tmp = 0; tmp += s[c-1] k[2]; tmp += s[c] k[1]; tmp += s[c+1] k[0], then h + v + p
// (Convolution3D_sep_shared_kernel.cuh:81-90).
// The half-precision classes only need to exist for the sources to compile: their members
// abort (the oracle never calls them).
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>
using namespace std;

class CUDAArchitecture;

template <typename T> class Volume_CPU {
public:
    Volume_CPU(float xs, float ys, float zs, unsigned long nx, unsigned long ny, unsigned long nz)
        : xs_(xs), ys_(ys), zs_(zs), nx_(nx), ny_(ny), nz_(nz), d_(nx * ny * nz, T(0)) {}
    virtual ~Volume_CPU() {}
    float getXVolumeSize() const { return xs_; }
    float getYVolumeSize() const { return ys_; }
    float getZVolumeSize() const { return zs_; }
    unsigned long getXVolumePixelNb() const { return nx_; }
    unsigned long getYVolumePixelNb() const { return ny_; }
    unsigned long getZVolumePixelNb() const { return nz_; }
    T* getVolumeData() { return d_.data(); }
    size_t size() const { return d_.size(); }
    bool isSameSize(Volume_CPU<T>* o) const { return nx_ == o->nx_ && ny_ == o->ny_ && nz_ == o->nz_; }
    void addVolume(Volume_CPU<T>* o, T lambda) { for (size_t i = 0; i < d_.size(); ++i) d_[i] = d_[i] + lambda * o->d_[i]; }
    void diffVolume(Volume_CPU<T>* o) { for (size_t i = 0; i < d_.size(); ++i) d_[i] -= o->d_[i]; }
    void diffVolume(T lambda, Volume_CPU<T>* o) { for (size_t i = 0; i < d_.size(); ++i) d_[i] = lambda * d_[i] - o->d_[i]; }
    void multVolume(Volume_CPU<T>* o) { for (size_t i = 0; i < d_.size(); ++i) d_[i] *= o->d_[i]; }
    double scalarProductVolume(Volume_CPU<T>* o) {
        double t = 0.0;
        for (size_t i = 0; i < d_.size(); ++i) t += (double)d_[i] * (double)o->d_[i];
        return t;
    }
    double getVolumeL1Norm() { double s = 0.0; for (T v : d_) s = s + (double)std::fabs((double)v); return s; }
    double getVolumeL2Norm() { double s = 0.0; for (T v : d_) s += (double)v * (double)v; return s; }
    double getVolumeLpNorm(double p) { double s = 0.0; for (T v : d_) s = s + (double)std::pow(std::fabs((double)v), p); return s; }
    double getVolumeHuberNorm(double thr) {
        double s = 0.0;
        const double t2 = thr * thr;
        for (T v : d_) {
            const double x = double(v);
            if (std::fabs(x) < thr) s += x * x;
            else if (std::fabs(x) >= thr) s += 2.0 * thr * std::fabs(x) - t2;
            else s += x;
        }
        return s;
    }
    void getVolumeSign(Volume_CPU<T>* out) {
        for (size_t i = 0; i < d_.size(); ++i) out->d_[i] = d_[i] > 0 ? T(1) : (d_[i] < 0 ? T(-1) : T(0));
    }
    void getVolumeAbsPow(Volume_CPU<T>* out, double p) {
        for (size_t i = 0; i < d_.size(); ++i) out->d_[i] = (T)std::pow(std::fabs((double)d_[i]), p);
    }
    void positiveAddVolume(Volume_CPU<T>* o, T lambda) {  // Image3D_CPU.cu:176-203
        for (size_t i = 0; i < d_.size(); ++i) {
            d_[i] = d_[i] + lambda * o->d_[i];
            if (d_[i] < (T)0.0) d_[i] = (T)0.0;
        }
    }
    void scalarVolume(T value) { for (auto& v : d_) v = v * value; }  // Image3D_CPU.cu:508-520
    void setVolume(T value) { for (auto& v : d_) v = value; }
    void saveVolume(string) {}
    void saveVolumeIter(string) {}

private:
    float xs_, ys_, zs_;
    unsigned long nx_, ny_, nz_;
    std::vector<T> d_;
};

template <typename T> class Convolution3D_CPU {
public:
    Convolution3D_CPU(T* kh, T* kv, T* kp) {
        for (int i = 0; i < 3; ++i) { h_[i] = kh[i]; v_[i] = kv[i]; p_[i] = kp[i]; }
    }
    void doSeparableConvolution3D(Volume_CPU<T>* in, Volume_CPU<T>* out) {
        const long nx = in->getXVolumePixelNb(), ny = in->getYVolumePixelNb(), nz = in->getZVolumePixelNb();
        const long plane = nx * ny;
        const T* s = in->getVolumeData();
        T* o = out->getVolumeData();
        for (long z = 0; z < nz; ++z)
            for (long y = 0; y < ny; ++y)
                for (long x = 0; x < nx; ++x) {
                    const long i = z * plane + y * nx + x;
                    const T c = s[i];
                    const T xm = x > 0 ? s[i - 1] : T(0), xp = x < nx - 1 ? s[i + 1] : T(0);
                    const T ym = y > 0 ? s[i - nx] : T(0), yp = y < ny - 1 ? s[i + nx] : T(0);
                    const T zm = z > 0 ? s[i - plane] : T(0), zp = z < nz - 1 ? s[i + plane] : T(0);
                    T a = T(0); a += xm * h_[2]; a += c * h_[1]; a += xp * h_[0];
                    T b = T(0); b += ym * v_[2]; b += c * v_[1]; b += yp * v_[0];
                    T d = T(0); d += zm * p_[2]; d += c * p_[1]; d += zp * p_[0];
                    o[i] = (a + b) + d;
                }
    }

private:
    T h_[3], v_[3], p_[3];
};

// ---- half-precision classes: declared so that the sources compile; never called ----
struct half { unsigned short bits; };
inline int singles2halfp(void*, void*, int) { std::abort(); }
inline int halfp2singles(void*, void*, int) { std::abort(); }

class Volume_CPU_half {
public:
    template <class... A> Volume_CPU_half(A...) { std::abort(); }
    unsigned long getXVolumePixelNb() const { std::abort(); }
    unsigned long getYVolumePixelNb() const { std::abort(); }
    unsigned long getZVolumePixelNb() const { std::abort(); }
    float getXVolumeSize() const { std::abort(); }
    float getYVolumeSize() const { std::abort(); }
    float getZVolumeSize() const { std::abort(); }
    half* getVolumeData() { std::abort(); }
    template <class... A> bool isSameSize(A...) { std::abort(); }
    template <class... A> void addVolume(A...) { std::abort(); }
    template <class... A> void diffVolume(A...) { std::abort(); }
    template <class... A> void multVolume(A...) { std::abort(); }
    template <class... A> double scalarProductVolume(A...) { std::abort(); }
    template <class... A> void getVolumeSign(A...) { std::abort(); }
    template <class... A> void getVolumeAbsPow(A...) { std::abort(); }
    template <class... A> void saveVolume(A...) { std::abort(); }
    double getVolumeL1Norm() { std::abort(); }
    double getVolumeL2Norm() { std::abort(); }
    double getVolumeLpNorm(double) { std::abort(); }
    double getVolumeHuberNorm(double) { std::abort(); }
};

class Convolution3D_CPU_half {
public:
    template <class... A> Convolution3D_CPU_half(A...) { std::abort(); }
    template <class... A> void doSeparableConvolution3D(A...) { std::abort(); }
};
