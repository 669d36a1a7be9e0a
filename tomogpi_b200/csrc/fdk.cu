// fdk.cu -- the ramp filter of filtered backprojection (FDK), for the FDK-weighted VI
// backprojector (vi_device.cuh, FDK = true).
//
// The filter follows the reference's ramp_filter_TOMO8.m (Matlab/Tomo8): a ramp |k| over an
// oversampled length M = oversampling * nu, normalised to 1, times a centred Hann window of
// round(M * cutoff) points (made even), taken back to the spatial domain; the taps of lags
// -round(nu/2) .. round(nu/2) - 1 (those the Matlab code keeps after its 2 nu-point
// circular convolution) are applied to every detector row, zero outside the row, and the
// result divided by 2 du. The taps are computed once per (nu, oversampling, cutoff) on the
// host in double; the convolution runs in FP32, one CTA per detector row, the row and the
// taps staged in shared memory.
#include <cmath>
#include <vector>

#include "tomo_kernels.cuh"

namespace tomo {

// Spatial taps of ramp_filter_TOMO8 for rows of nu pixels, scaled by 1 / (2 du). Returns
// half = round(nu / 2) and taps[l] for lag l - half, l in [0, 2 half).
int ramp_taps(int nu, int oversampling, double cutoff, double du, std::vector<float>& taps) {
    const long M = (long)oversampling * nu;
    // window: hann(Nr) (symmetric), Nr = round(M cutoff) made even, centred in M points,
    // then fftshift (even M: a shift by M/2)
    long nr = (long)std::floor(M * cutoff + 0.5);
    if (nr % 2) --nr;
    std::vector<double> win(M, 0.0), g(M);
    const long off = (M - nr) / 2;
    for (long n = 0; n < nr; ++n)
        win[off + n] = nr > 1 ? 0.5 * (1.0 - std::cos(2.0 * M_PI * n / (double)(nr - 1))) : 1.0;
    for (long k = 0; k < M; ++k) {
        const double ramp = (double)(k <= M / 2 ? k : M - k) / (double)(M / 2);  // |k| in FFT order, max 1
        g[k] = ramp * win[(k + M / 2) % M];
    }
    const int half = (int)std::floor(nu / 2.0 + 0.5);
    const int lo = (int)std::floor(3.0 * nu / 2.0 + 0.5) - 2 * nu;  // most negative kept lag
    taps.assign(2 * half, 0.f);
    for (int l = 0; l < 2 * half; ++l) {
        const int lag = l - half;
        if (lag < lo) continue;
        // real part of the inverse DFT at n = lag mod M
        const long n = lag >= 0 ? lag : M + lag;
        double s = 0.0;
        for (long k = 0; k < M; ++k) s += g[k] * std::cos(2.0 * M_PI * (double)((k * n) % M) / (double)M);
        taps[l] = (float)(s / (double)M / (2.0 * du));
    }
    return half;
}

template <typename Ti>
__global__ void ramp_filter_kernel(const Ti* __restrict__ in, float* __restrict__ out, const float* __restrict__ taps,
                                   int half, int nu) {
    extern __shared__ float sm[];
    float* row = sm;           // nu
    float* tp = sm + nu;       // 2 half
    const long r = blockIdx.x;  // detector row (view, v)
    for (int i = threadIdx.x; i < nu; i += blockDim.x) row[i] = ldp(in + r * nu + i);
    for (int i = threadIdx.x; i < 2 * half; i += blockDim.x) tp[i] = taps[i];
    __syncthreads();
    for (int i = threadIdx.x; i < nu; i += blockDim.x) {
        float acc = 0.f;
        // lag = l - half, source pixel j = i - lag within [0, nu)
        const int l0 = max(0, i - nu + 1 + half), l1 = min(2 * half, i + half + 1);
        for (int l = l0; l < l1; ++l) acc = fmaf(tp[l], row[i - (l - half)], acc);
        out[r * nu + i] = acc;
    }
}

cudaError_t launch_ramp_filter(const void* in, tomo_dtype idt, float* out, const float* taps, int half, int nu, int nv,
                               int np, cudaStream_t st) {
    const long rows = (long)nv * np;
    const size_t smem = (size_t)(nu + 2 * half) * sizeof(float);
    switch (idt) {
        case TOMO_F32: ramp_filter_kernel<float><<<(unsigned)rows, 256, smem, st>>>((const float*)in, out, taps, half, nu); break;
        case TOMO_BF16:
            ramp_filter_kernel<__nv_bfloat16><<<(unsigned)rows, 256, smem, st>>>((const __nv_bfloat16*)in, out, taps, half, nu);
            break;
        case TOMO_F16: ramp_filter_kernel<__half><<<(unsigned)rows, 256, smem, st>>>((const __half*)in, out, taps, half, nu); break;
    }
    return cudaGetLastError();
}

}  // namespace tomo
