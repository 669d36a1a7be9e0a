// Stand-in for the reference's Sinogram3D_CPU.cuh (host sinogram of u x v x p values,
// zero-initialised here). Test infrastructure only.
#pragma once
#include <vector>
#include "Config.hpp"

template <typename T> class Sinogram3D_CPU {
public:
    Sinogram3D_CPU(unsigned long u, unsigned long v, unsigned long p, CUDAArchitecture*) : data((size_t)u * v * p, T(0)) {}
    T* getDataSinogram() { return data.data(); }
    size_t size() const { return data.size(); }
    void setSinogram(T value) { for (auto& x : data) x = value; }

private:
    std::vector<T> data;
};
