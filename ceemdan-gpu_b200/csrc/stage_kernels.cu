// Stage-level kernels of the ICEEMDAN engine: statistics, noise injection, ensemble means.
//
// Reference counterparts (cudaICEEMDAN.cu unless noted):
//   k_canon_mean / k_canon_var  meanD/varianceD + multiplyD (statistics.cu:167-241,
//                               launched :1732-1742, :1874-1878).  The reference reduces with
//                               shuffles and atomicAdd into accumulators it never zeroes; the
//                               carry (acc + sum) * factor is kept, the order is the
//                               canonical one: 256 strided lanes, then a halving tree.
//   k_standardize               standardizeRunning :58-66
//   k_add_noise / k_add_noise2  addNoise :69-78, addNoise2 :81-90
//   k_first_imf                 produceFirstIMF :42-55
//   k_avg_update                produceResidue :583-591 + averageUpdateSignal :594-607
//   k_sub_inplace               updateSignal :610-617
//   k_check_iota / k_fill_iota  the sample coordinates d_x (must be / are made 0..N-1)
//   k_widen_f32 / k_narrow_f64  float data and IMFs of the FP32 entry points
#include <cuda_runtime.h>

#include <cstdint>

#include "canon.cuh"
#include "kernels.h"

namespace ceemdan {

namespace {

constexpr int kUnroll = 8;

// Canonical lane sum of v[0..n): lane t adds v[t], v[t+256], ... in order; then the tree.
// sq = true: lane adds fma(d, d, acc) with d = v - mean.
template <bool kSq>
__device__ double canon_reduce(const double* __restrict__ v, size_t n, double mean) {
    __shared__ double sp[kLanes];
    const int t = threadIdx.x;
    double acc = 0.0;
    size_t i = (size_t)t;
    // loads are issued kUnroll at a time; the additions stay in lane order
    for (; i + (size_t)(kUnroll - 1) * kLanes < n; i += (size_t)kUnroll * kLanes) {
        double x[kUnroll];
#pragma unroll
        for (int k = 0; k < kUnroll; ++k) x[k] = v[i + (size_t)k * kLanes];
#pragma unroll
        for (int k = 0; k < kUnroll; ++k) {
            if (kSq) {
                const double d = x[k] - mean;
                acc = fma(d, d, acc);
            } else {
                acc = acc + x[k];
            }
        }
    }
    for (; i < n; i += kLanes) {
        if (kSq) {
            const double d = v[i] - mean;
            acc = fma(d, d, acc);
        } else {
            acc = acc + v[i];
        }
    }
    sp[t] = acc;
    __syncthreads();
    for (int s = kLanes / 2; s > 0; s >>= 1) {
        if (t < s) sp[t] = sp[t] + sp[t + s];
        __syncthreads();
    }
    const double out = sp[0];
    __syncthreads();
    return out;
}

}  // namespace

// acc[b] = (acc[b] + sum(v_b)) * inv_n   (one CTA of kLanes threads per vector)
__global__ void __launch_bounds__(kLanes)
k_canon_mean(const double* v, size_t n, size_t stride, double* acc, double inv_n) {
    const size_t b = blockIdx.x;
    const double s = canon_reduce<false>(v + b * stride, n, 0.0);
    if (threadIdx.x == 0) acc[b] = (acc[b] + s) * inv_n;
}

// acc[b] = (acc[b] + sum((v_b - mean[b])^2)) * inv_nm1
__global__ void __launch_bounds__(kLanes)
k_canon_var(const double* v, size_t n, size_t stride, const double* mean, double* acc,
            double inv_nm1) {
    const size_t b = blockIdx.x;
    const double s = canon_reduce<true>(v + b * stride, n, mean[b]);
    if (threadIdx.x == 0) acc[b] = (acc[b] + s) * inv_nm1;
}

// Raw canonical sums (stage-level entry point).
__global__ void __launch_bounds__(kLanes)
k_canon_sums(const double* v, size_t n, const double* mean, double* sum, double* sqdev) {
    const size_t b = blockIdx.x;
    const double s = canon_reduce<false>(v + b * n, n, 0.0);
    if (threadIdx.x == 0) sum[b] = s;
    if (mean) {
        const double q = canon_reduce<true>(v + b * n, n, mean[b]);
        if (threadIdx.x == 0) sqdev[b] = q;
    }
}

__global__ void k_standardize(double* x, size_t n, const double* var) {
    const double sc = 1.0 / sqrt(var[0]);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        x[i] = x[i] * sc;
}

// h0_r = x + (nstd * E_r) * (1/sqrt(var(E_r)))   (blockIdx.y = realization)
__global__ void k_add_noise(double* h0, const double* x, const double* E, size_t n, int nr,
                            double nstd, const double* evar) {
    const int r = blockIdx.y;
    const double sc = 1.0 / sqrt(evar[r]);
    const size_t base = (size_t)r * n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        h0[base + i] = fma(nstd * E[base + i], sc, x[i]);
}

// h0_r = r + (nstd * E_r) * sqrt(var(r))
__global__ void k_add_noise2(double* h0, const double* rs, const double* E, size_t n, int nr,
                             double nstd, const double* svar) {
    const int r = blockIdx.y;
    const double sq = sqrt(svar[0]);
    const size_t base = (size_t)r * n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        h0[base + i] = fma(nstd * E[base + i], sq, rs[i]);
}

// aux = sum_r fma(1/NR, h0_r - mode_r, aux) in realization order; IMF_0 = x - aux.
__global__ void k_first_imf(const double* h0, const double* mode, const double* x,
                            double* fornext, double* imf, size_t n, int nr) {
    const double inr = 1.0 / (double)nr;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int r = 0; r < nr; ++r) t = fma(inr, h0[(size_t)r * n + i] - mode[(size_t)r * n + i], t);
        fornext[i] = t;
        imf[i] = x[i] - t;
    }
}

// r_k = (sum_r (h0_r - mode_r)) / NR in realization order; IMF_k = r_{k-1} - r_k.
__global__ void k_avg_update(const double* h0, const double* mode, double* fornext, double* imf,
                             size_t n, int nr) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int r = 0; r < nr; ++r) t = t + (h0[(size_t)r * n + i] - mode[(size_t)r * n + i]);
        const double avg = t / (double)nr;
        imf[i] = fornext[i] - avg;
        fornext[i] = avg;
    }
}

__global__ void k_sub_inplace(double* w, const double* e, size_t count) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x)
        w[i] = w[i] - e[i];
}

// FP32 entry points: float data widened to FP64 (exact) and FP64 results rounded to float.
__global__ void k_widen_f32(const float* src, double* dst, size_t count) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

__global__ void k_narrow_f64(const double* src, float* dst, size_t count) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

// Sample index 0..n-1 (the d_x every reference caller passes), for the batch entry point.
__global__ void k_fill_iota(int32_t* x, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        x[i] = (int32_t)i;
}

__global__ void k_check_iota(const int32_t* x, size_t n, int* err) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        if (x[i] != (int32_t)i) atomicCAS(err, 0, 2);
}

}  // namespace ceemdan
