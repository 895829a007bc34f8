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
//   k_stage_end / k_stage_stats / k_stage_begin / k_commit_plan
//                               the batched engine's stage transitions: the same steps as the
//                               kernels above (same operations, same order), for every channel
//                               whose stage has just finished, inside the device-driven loop
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

// A split channel's ensemble sums (ceemdan_plain_split_f64): tsum (the previous parts' running
// sums) continued over this part's realizations in order -- fma(inr, h0_r - mode_r, t) in the
// first stage (k_first_imf), t + (h0_r - mode_r) after it (k_avg_update).
__global__ void k_ens_accum(const double* h0, const double* mode, double* tsum, size_t n, int nr,
                            bool first_stage, double inr) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        double t = tsum[i];
        if (first_stage) {
            for (int r = 0; r < nr; ++r)
                t = fma(inr, h0[(size_t)r * n + i] - mode[(size_t)r * n + i], t);
        } else {
            for (int r = 0; r < nr; ++r) t = t + (h0[(size_t)r * n + i] - mode[(size_t)r * n + i]);
        }
        tsum[i] = t;
    }
}

// The stage's IMF and next residue from the whole ensemble's sums (as k_first_imf /
// k_avg_update): the first stage's sums are already the mean; later ones divide by NR.
__global__ void k_ens_out(const double* tsum, const double* x, double* fornext, double* imf,
                          size_t n, bool first_stage, double nr_total) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double t = tsum[i];
        if (first_stage) {
            fornext[i] = t;
            imf[i] = x[i] - t;
        } else {
            const double avg = t / nr_total;
            imf[i] = fornext[i] - avg;
            fornext[i] = avg;
        }
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

// =======================================================================================
// Batched engine: stage transitions.  A channel whose stage has finished (ChanState.done, set
// by k_criterion) and that has stages left is "in transition" from the first of these kernels
// to k_commit_plan, which opens its next stage; all four read the same states.
// =======================================================================================
namespace {

__device__ __forceinline__ bool in_transition(const ChanState& cs, int M) {
    return cs.done && cs.stage < 2 * M;
}

// The persistent grid's share of virtual blocks over the channels that satisfy pred (nb(c)
// blocks each, in channel order): CTA b takes the blocks b, b + gridDim.x, ...  Every thread
// of the CTA calls body(c, block) with the same arguments (CTA-uniform).
template <class Pred, class NB, class Body>
__device__ __forceinline__ void channel_blocks(int nchan, Pred pred, NB nb, Body body) {
    long long base = 0;
    const long long G = gridDim.x;
    for (int c = 0; c < nchan; ++c) {
        if (!pred(c)) continue;
        const int cnt = nb(c);
        for (long long v = blockIdx.x + ((base - blockIdx.x + G - 1) / G) * G - base;
             v < cnt; v += G)
            body(c, (int)v);
        base += cnt;
    }
}

__device__ __forceinline__ int sample_blocks(const SiftArgs& a, int c) {
    return (__ldg(&a.chan[c].n) + kTransThreads - 1) / kTransThreads;
}

}  // namespace

// End of a stage (the steps after run_stage in the one-channel engine): the realizations that
// finished in the last iteration export h; then
//   noise stage i:    w -= E_i (updateSignal), and after the last one E_M = w;
//   CEEMDAN stage 0:  r_0 = sum_r fma(1/NR, h0_r - mode_r, .), IMF_0 = x~ - r_0;
//   CEEMDAN stage k:  r_k = (sum_r (h0_r - mode_r)) / NR, IMF_k = r_{k-1} - r_k; after the
//                     last one the residue row = r_M.
// One thread per sample, realizations in order.
__global__ void __launch_bounds__(kTransThreads)
k_stage_end(SiftArgs a, BatchArgs b) {
    const int M = b.M;
    channel_blocks(
        a.nchan, [&](int c) { return in_transition(a.cs[c], M) && a.cs[c].stage >= 0; },
        [&](int c) { return sample_blocks(a, c); },
        [&](int c, int blk) {
            const Chan& ch = a.chan[c];
            const int n = ch.n, nr = ch.nr, row0 = ch.row0;
            const int i = blk * kTransThreads + threadIdx.x;
            if (i >= n) return;
            const ChanState& cs = a.cs[c];
            const int s = cs.stage;
            const double* hf = a.h[cs.iter & 1] + ch.samp0 + i;
            const size_t rn = (size_t)n;
            if (s < M) {
                double* Ei = b.E + (size_t)s * b.S + ch.samp0 + i;
                double* w = b.W + ch.samp0 + i;
                for (int r = 0; r < nr; ++r) {
                    const size_t o = (size_t)r * rn;
                    double m;
                    if (a.mark[row0 + r] == 0) {
                        m = hf[o];
                        Ei[o] = m;
                    } else {
                        m = Ei[o];
                    }
                    const double nw = w[o] - m;
                    w[o] = nw;
                    if (s == M - 1) b.E[(size_t)M * b.S + ch.samp0 + i + o] = nw;
                }
                return;
            }
            const int k = s - M;
            const double* h0 = b.H0 + ch.samp0 + i;
            const double* md = b.MODE + ch.samp0 + i;
            double* fn = b.FN + b.xoff[c] + i;
            double* imf = b.imfs[c] + (size_t)k * rn + i;
            double t = 0.0;
            if (k == 0) {
                const double inr = 1.0 / (double)nr;
                for (int r = 0; r < nr; ++r) {
                    const size_t o = (size_t)r * rn;
                    const double m = a.mark[row0 + r] == 0 ? hf[o] : md[o];
                    t = fma(inr, h0[o] - m, t);
                }
                *fn = t;
                *imf = b.XS[b.xoff[c] + i] - t;
            } else {
                for (int r = 0; r < nr; ++r) {
                    const size_t o = (size_t)r * rn;
                    const double m = a.mark[row0 + r] == 0 ? hf[o] : md[o];
                    t = t + (h0[o] - m);
                }
                const double avg = t / (double)nr;
                *imf = *fn - avg;
                *fn = avg;
                t = avg;
            }
            if (k == M - 1) imf[rn] = t;  // final residue
        });
}

// Statistics that open a CEEMDAN stage, canonical order (k_canon_mean / k_canon_var):
// entering stage 0, the carried mean and variance of x and every realization's first noise
// mode; entering stage k > 0, the carried mean and variance of r_{k-1}.  One CTA of kLanes
// threads per vector.
__global__ void __launch_bounds__(kLanes)
k_stage_stats(SiftArgs a, BatchArgs b) {
    const int M = b.M;
    channel_blocks(
        a.nchan,
        [&](int c) {
            const ChanState& cs = a.cs[c];
            return in_transition(cs, M) && cs.stage + 1 >= M && cs.stage + 1 < 2 * M;
        },
        [&](int c) { return a.cs[c].stage + 1 == M ? 1 + a.chan[c].nr : 1; },
        [&](int c, int item) {
            const Chan& ch = a.chan[c];
            const size_t n = (size_t)ch.n;
            const double inv_n = 1.0 / (double)n, inv_nm1 = 1.0 / (double)(n - 1);
            __shared__ double s_mean;
            const double* v;
            double *mean, *var;
            if (item == 0) {
                v = (a.cs[c].stage + 1 == M ? b.XS : b.FN) + b.xoff[c];
                mean = b.smean + c;
                var = b.svar + c;
            } else {
                const int r = item - 1;
                v = b.E + ch.samp0 + (size_t)r * n;  // first noise mode of realization r
                mean = b.emean + ch.row0 + r;
                var = b.evar + ch.row0 + r;
            }
            const double sm = canon_reduce<false>(v, n, 0.0);
            if (threadIdx.x == 0) {
                const double mv = (*mean + sm) * inv_n;
                *mean = mv;
                s_mean = mv;
            }
            __syncthreads();
            const double sq = canon_reduce<true>(v, n, s_mean);
            if (threadIdx.x == 0) *var = (*var + sq) * inv_nm1;
            __syncthreads();
        });
}

// Input of the next stage into h[0] (and h0 for CEEMDAN stages): the residual noise for a noise
// stage; x~ = x / sqrt(var x) and h0_r = fma(Nstd*E_0, 1/sqrt(var E_0,r), x~) for CEEMDAN
// stage 0 (standardizeRunning, addNoise); h0_r = fma(Nstd*E_k, sqrt(var r_{k-1}), r_{k-1})
// for stage k (addNoise2).
__global__ void __launch_bounds__(kTransThreads)
k_stage_begin(SiftArgs a, BatchArgs b) {
    const int M = b.M;
    channel_blocks(
        a.nchan, [&](int c) { return in_transition(a.cs[c], M) && a.cs[c].stage + 1 < 2 * M; },
        [&](int c) { return sample_blocks(a, c); },
        [&](int c, int blk) {
            const Chan& ch = a.chan[c];
            const int n = ch.n, nr = ch.nr;
            const int i = blk * kTransThreads + threadIdx.x;
            if (i >= n) return;
            const int ns = a.cs[c].stage + 1;
            const size_t rn = (size_t)n;
            double* h = a.h[0] + ch.samp0 + i;
            if (ns < M) {
                const double* w = b.W + ch.samp0 + i;
                for (int r = 0; r < nr; ++r) h[(size_t)r * rn] = w[(size_t)r * rn];
                return;
            }
            const int k = ns - M;
            const double* E = b.E + (size_t)k * b.S + ch.samp0 + i;
            double* h0 = b.H0 + ch.samp0 + i;
            const double nstd = b.nstd;
            if (k == 0) {
                double* xs = b.XS + b.xoff[c] + i;
                const double sc = 1.0 / sqrt(b.svar[c]);
                const double xv = *xs * sc;
                *xs = xv;
                for (int r = 0; r < nr; ++r) {
                    const size_t o = (size_t)r * rn;
                    const double esc = 1.0 / sqrt(b.evar[ch.row0 + r]);
                    const double v = fma(nstd * E[o], esc, xv);
                    h0[o] = v;
                    h[o] = v;
                }
            } else {
                const double sq = sqrt(b.svar[c]);
                const double rv = b.FN[b.xoff[c] + i];
                for (int r = 0; r < nr; ++r) {
                    const size_t o = (size_t)r * rn;
                    const double v = fma(nstd * E[o], sq, rv);
                    h0[o] = v;
                    h[o] = v;
                }
            }
        });
}

// One CTA of 1024 threads: opens the next stage of every channel in transition (iteration
// count of the closed stage recorded; sift cap, mode buffer, iteration 0, no realization
// finished, no update pending), or retires the channel after its last stage; then the
// active-channel plan of the iteration.
__global__ void __launch_bounds__(1024)
k_commit_plan(SiftArgs a, BatchArgs b) {
    const int M = b.M;
    for (int c = 0; c < a.nchan; ++c) {
        ChanState& cs = a.cs[c];
        if (!in_transition(cs, M)) continue;  // uniform: every thread reads the same state
        const int s = cs.stage, ns = s + 1;
        const Chan& ch = a.chan[c];
        if (ns < 2 * M)
            for (int r = threadIdx.x; r < ch.nr; r += blockDim.x) {
                a.mark[ch.row0 + r] = -1;
                a.finish[ch.row0 + r] = 0;
            }
        __syncthreads();  // every thread has read cs before thread 0 changes it
        if (threadIdx.x == 0) {
            if (s >= 0) b.iters[(size_t)c * 2 * M + s] = cs.iter;
            cs.stage = ns;
            if (ns == 2 * M) {
                *b.finished += 1;  // done stays set: the channel never sifts again
            } else {
                cs.done = 0;
                cs.iter = 0;
                cs.cap = ns < M ? b.noise_cap : b.max_iter;
                cs.mode_out = (ns < M ? b.E + (size_t)ns * b.S : b.MODE) + ch.samp0;
            }
        }
        __syncthreads();
    }
    plan_block(a);
}

}  // namespace ceemdan
