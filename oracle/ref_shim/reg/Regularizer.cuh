// Stand-in for the reference's Regularizer.cuh: the base classes the regularisers derive
// from (no members are needed by the host build of the oracle). Test infrastructure only.
#pragma once
#include "Volume_CPU.cuh"
template <template <typename> class V, typename T> class Regularizer {
public:
    virtual ~Regularizer() {}
};
template <typename V> class Regularizer_half {
public:
    virtual ~Regularizer_half() {}
};
