// Sifting kernels of the ICEEMDAN engine (sm_100a, FP64).
//
// One sift iteration over all realizations of a stage is:
//   k_extrema        deferred update h -= m (or mode export) + strict-extrema flags +
//                    warp-ballot compaction, tile offsets by decoupled look-back
//                    (find_extrema_shfl_* :93-148, CUB scan, select_extrema_* :151-207,
//                     updateRealizations :528-544 of the previous iteration)
//   k_boundary       end-knot extrapolation (setBoundaryMax/Min :210-291)
//   k_chunk_reduce   level-1 chunk sweeps of the canonical partitioned spline solve
//   k_reduced_solve  per-system reduced solve (levels >= 2), one CTA per spline
//   k_chunk_backsub  level-1 back substitution -> spline coefficients c
//                    (tridiagonal_setup :311-343 + cusparseDgtsv2_nopivot :1622-1641)
//   k_eval           envelopes, mean envelope, sx statistics
//                    (spline_coefficients :383-401, interpolate :404-439,
//                     averageUppperLower :442-454, produceSX :457-467,
//                     thresholdJudge :470-492)
//   k_criterion      sifting fraction carry + stop test + break test
//                    (meanD/multiplyD on sx :1851, siftingCriterion :495-525,
//                     checkBreak :547-580)
// Line numbers refer to the reference's cudaICEEMDAN.cu.
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <cstdint>

#include "canon.cuh"
#include "kernels.h"

namespace ceemdan {

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = kTileSamples / kThreads;  // samples per thread in a tile
constexpr int kChunksPerBlock = kThreads;            // one level-1 chunk per thread

__device__ __forceinline__ int pad17(int j) { return j + (j >> 4); }

// 64-bit look-back status word: [63:62] flag (0 empty, 1 aggregate, 2 inclusive),
// [61:31] maxima count, [30:0] minima count.
__device__ __forceinline__ unsigned long long pack_status(unsigned flag, unsigned cmax,
                                                          unsigned cmin) {
    return ((unsigned long long)flag << 62) | ((unsigned long long)cmax << 31) |
           (unsigned long long)cmin;
}

__device__ __forceinline__ void set_error(int* err, int code) { atomicCAS(err, 0, code); }

// ---------------------------------------------------------------------------------------
// chunk sweep of the canonical partitioned solve (rows produced by a functor)
// ---------------------------------------------------------------------------------------
struct ChunkEnds {
    double ga, aa, ba, gb, ab, bb;
};

// Forward + backward sweep over `len` (1..kChunk) rows produced by row(k).  Returns the
// first/last-row coefficients; when `out` is given, also x_k = g_k + al_k*xl + be_k*xr.
template <class RowFn>
__device__ __forceinline__ ChunkEnds chunk_sweep(int len, RowFn row, double xl, double xr,
                                                 double* out, int out_stride) {
    double cp[kChunk], gp[kChunk], ap[kChunk];
    double iw = 0.0, ub = 0.0;
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
        if (k < len) {
            const Row w = row(k);
            if (k == 0) {
                iw = 1.0 / w.m;
                cp[0] = w.u * iw;
                gp[0] = w.r * iw;
                ap[0] = -w.l * iw;
            } else {
                iw = pivot_rcp(w, cp[k - 1]);
                cp[k] = w.u * iw;
                gp[k] = fma(-w.l, gp[k - 1], w.r) * iw;
                ap[k] = (-w.l * ap[k - 1]) * iw;
            }
            ub = w.u;
        }
    }
    const double bp = -ub * iw;
    ChunkEnds e;
    double g = 0.0, a = 0.0, b = 0.0;
#pragma unroll
    for (int k = kChunk - 1; k >= 0; --k) {
        if (k < len) {
            if (k == len - 1) {
                g = gp[k];
                a = ap[k];
                b = bp;
                e.gb = g;
                e.ab = a;
                e.bb = b;
            } else {
                g = fma(-cp[k], g, gp[k]);
                a = fma(-cp[k], a, ap[k]);
                b = -(cp[k] * b);
            }
            if (out) out[k * out_stride] = fma(b, xr, fma(a, xl, g));
        }
    }
    e.ga = g;
    e.aa = a;
    e.ba = b;
    return e;
}

// Canonical Thomas on n <= kChunk rows (base case), x written with stride.
template <class RowFn>
__device__ __forceinline__ void thomas_small(int n, RowFn row, double* x, int stride) {
    double cp[kChunk], gp[kChunk];
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
        if (k < n) {
            const Row w = row(k);
            double iw;
            if (k == 0) {
                iw = 1.0 / w.m;
                cp[0] = w.u * iw;
                gp[0] = w.r * iw;
            } else {
                iw = pivot_rcp(w, cp[k - 1]);
                cp[k] = w.u * iw;
                gp[k] = fma(-w.l, gp[k - 1], w.r) * iw;
            }
        }
    }
    double xv = 0.0;
#pragma unroll
    for (int k = kChunk - 1; k >= 0; --k) {
        if (k < n) {
            xv = (k == n - 1) ? gp[k] : fma(-cp[k], xv, gp[k]);
            x[k * stride] = xv;
        }
    }
}

// Row i (0..K-1) of the natural-spline system from global knots.
__device__ __forceinline__ Row spline_row_global(int i, int K, const int32_t* kx,
                                                 const double* ky) {
    if (i == 0 || i == K - 1) return identity_row();
    const double sp = seg_slope(kx[i - 1], kx[i], ky[i - 1], ky[i]);
    const double sn = seg_slope(kx[i], kx[i + 1], ky[i], ky[i + 1]);
    return spline_row(kx[i - 1], kx[i], kx[i + 1], sp, sn);
}

}  // namespace

// =======================================================================================
// k_extrema
// =======================================================================================
__global__ void __launch_bounds__(kThreads)
k_extrema(SiftArgs a) {
    __shared__ double sh[kTileSamples + 2];
    __shared__ int s_cnt[2][kPerThread * (kThreads / 32)];
    __shared__ int s_off[2][kPerThread * (kThreads / 32)];
    __shared__ unsigned s_ticket;
    __shared__ int s_prefix[2];
    __shared__ int s_agg[2];

    if (*a.done) return;
    if (threadIdx.x == 0) s_ticket = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const unsigned tk = s_ticket;
    const int r = (int)(tk / (unsigned)a.ntiles);
    const int tile = (int)(tk % (unsigned)a.ntiles);
    if (r >= a.nr) return;
    const int n = a.n;
    const int n0 = tile * kTileSamples;
    const size_t base = (size_t)r * (size_t)n;
    const int mk = a.mark[r];
    const double* hin = a.h_in + base;
    double* hout = a.h_out + base;
    const double* me = a.menv + base;

    // Deferred update of the previous iteration + halo, into shared memory.
    for (int j = threadIdx.x; j < kTileSamples + 2; j += kThreads) {
        const int s = n0 - 1 + j;
        double v = 0.0;
        if (s >= 0 && s < n) {
            const double hv = hin[s];
            v = (mk == 1) ? hv - me[s] : hv;
            if (j >= 1 && j <= kTileSamples) {
                hout[s] = v;
                if (mk == 0) a.mode_out[base + s] = hv;
            }
        }
        sh[j] = v;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    unsigned bmax[kPerThread], bmin[kPerThread];
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int j = k * kThreads + threadIdx.x;  // local sample
        const int s = n0 + j;
        bool fmax = false, fmin = false;
        if (s < n) {
            if (s == 0 || s == n - 1) {
                fmax = fmin = true;
            } else {
                const double v = sh[j + 1], vl = sh[j], vr = sh[j + 2];
                fmax = v > vl && v > vr;
                fmin = v < vl && v < vr;
            }
        }
        bmax[k] = __ballot_sync(0xffffffffu, fmax);
        bmin[k] = __ballot_sync(0xffffffffu, fmin);
        if (lane == 0) {
            s_cnt[0][k * (kThreads / 32) + warp] = __popc(bmax[k]);
            s_cnt[1][k * (kThreads / 32) + warp] = __popc(bmin[k]);
        }
    }
    __syncthreads();

    // Exclusive scan of the 64 (row, warp) counts per envelope: warp 0 -> maxima,
    // warp 1 -> minima, two entries per lane.
    constexpr int kSlots = kPerThread * (kThreads / 32);
    static_assert(kSlots == 64, "scan assumes 64 slots");
    if (warp < 2) {
        const int e = warp;
        const int c0 = s_cnt[e][2 * lane], c1 = s_cnt[e][2 * lane + 1];
        int incl = c0 + c1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int excl = incl - (c0 + c1);
        s_off[e][2 * lane] = excl;
        s_off[e][2 * lane + 1] = excl + c0;
        if (lane == 31) s_agg[e] = incl;
    }
    __syncthreads();

    // Decoupled look-back over the tiles of realization r.
    if (threadIdx.x == 0) {
        const unsigned amax = (unsigned)s_agg[0], amin = (unsigned)s_agg[1];
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> me_st(
            a.status[(size_t)r * a.ntiles + tile]);
        unsigned pmax = 0, pmin = 0;
        if (tile == 0) {
            me_st.store(pack_status(2u, amax, amin), cuda::memory_order_release);
        } else {
            me_st.store(pack_status(1u, amax, amin), cuda::memory_order_release);
            int p = tile - 1;
            int spins = 0;
            while (p >= 0) {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> st(
                    a.status[(size_t)r * a.ntiles + p]);
                const unsigned long long w = st.load(cuda::memory_order_acquire);
                const unsigned flag = (unsigned)(w >> 62);
                if (flag == 0u) {
                    if (++spins > a.spin_limit) {
                        set_error(a.err, kErrTimeout);
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                pmax += (unsigned)((w >> 31) & 0x7fffffffu);
                pmin += (unsigned)(w & 0x7fffffffu);
                if (flag == 2u) break;
                --p;
            }
            me_st.store(pack_status(2u, pmax + amax, pmin + amin), cuda::memory_order_release);
        }
        s_prefix[0] = (int)pmax;
        s_prefix[1] = (int)pmin;
        const size_t to = (size_t)(a.ntiles + 1);
        a.tile_off[(size_t)r * to + tile] = (int)pmax;
        a.tile_off[(size_t)(a.nr + r) * to + tile] = (int)pmin;
        if (tile == a.ntiles - 1) {
            a.kcount[r] = (int)(pmax + amax);
            a.kcount[a.nr + r] = (int)(pmin + amin);
            a.tile_off[(size_t)r * to + a.ntiles] = (int)(pmax + amax);
            a.tile_off[(size_t)(a.nr + r) * to + a.ntiles] = (int)(pmin + amin);
        }
    }
    __syncthreads();

    const unsigned lt = (1u << lane) - 1u;
    const size_t kb = (size_t)r * (size_t)a.cap;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int j = k * kThreads + threadIdx.x;
        const int s = n0 + j;
        const int slot = k * (kThreads / 32) + warp;
        if (bmax[k] & (1u << lane)) {
            const int pos = s_prefix[0] + s_off[0][slot] + __popc(bmax[k] & lt);
            a.kx_max[kb + pos] = s;
            a.ky_max[kb + pos] = sh[j + 1];
        }
        if (bmin[k] & (1u << lane)) {
            const int pos = s_prefix[1] + s_off[1][slot] + __popc(bmin[k] & lt);
            a.kx_min[kb + pos] = s;
            a.ky_min[kb + pos] = sh[j + 1];
        }
    }
}

// =======================================================================================
// k_boundary: end-knot extrapolation, one thread per (envelope, realization)
// =======================================================================================
__global__ void k_boundary(SiftArgs a) {
    if (*a.done) return;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= 2 * a.nr) return;
    const int e = id / a.nr, r = id % a.nr;
    const int K = a.kcount[id];
    if (K - 1 <= 4) return;
    const size_t kb = (size_t)r * (size_t)a.cap;
    const int32_t* x = (e == 0 ? a.kx_max : a.kx_min) + kb;
    double* y = (e == 0 ? a.ky_max : a.ky_min) + kb;
    const int L = K - 1;
    const double y0 = boundary_left(e, x[0], x[1], x[2], y[0], y[1], y[2]);
    const double yL = boundary_right(e, x[L - 2], x[L - 1], x[L], y[L - 2], y[L - 1], y[L]);
    y[0] = y0;
    y[L] = yL;
}

// =======================================================================================
// level-1 chunk kernels (reduce and back substitution share the staging)
// =======================================================================================
namespace {

constexpr int kStageSlots = (kChunksPerBlock * kChunk + 2) + ((kChunksPerBlock * kChunk + 2) >> 4) + 1;
constexpr int kBacksubSlots = (kChunksPerBlock * kChunk) + ((kChunksPerBlock * kChunk) >> 4) + 1;

// Knots staged in padded shared memory (one pad slot per 16 knots keeps the per-thread
// stride of 17 bank-conflict free).  Lives in dynamic shared memory.
struct StagedKnots {
    double y[kStageSlots];
    int32_t x[kStageSlots];
};

// Stage knots [row0-1, row0 + kChunksPerBlock*kChunk] (clamped to [0, K-1]) into padded
// shared memory; relative index j = knot - (row0 - 1).
__device__ __forceinline__ void stage_knots(StagedKnots& sk, int row0, int K, const int32_t* kx,
                                            const double* ky) {
    constexpr int kSpan = kChunksPerBlock * kChunk + 2;
    for (int j = threadIdx.x; j < kSpan; j += kThreads) {
        const int i = row0 - 1 + j;
        if (i >= 0 && i < K) {
            sk.x[pad17(j)] = kx[i];
            sk.y[pad17(j)] = ky[i];
        }
    }
}

// Rows of chunk q from staged knots.  Row i uses knots i-1, i, i+1 (relative j = i-row0+1).
struct StagedRowFn {
    const StagedKnots* sk;
    int first_row;  // global row index of local row 0
    int row0;       // global row of relative knot index 1
    int K;
    __device__ __forceinline__ Row operator()(int k) const {
        const int i = first_row + k;
        if (i == 0 || i == K - 1) return identity_row();
        const int j = i - row0 + 1;
        const int32_t xm = sk->x[pad17(j - 1)], x0 = sk->x[pad17(j)], xp = sk->x[pad17(j + 1)];
        const double ym = sk->y[pad17(j - 1)], y0 = sk->y[pad17(j)], yp = sk->y[pad17(j + 1)];
        return spline_row(xm, x0, xp, seg_slope(xm, x0, ym, y0), seg_slope(x0, xp, y0, yp));
    }
};

__device__ __forceinline__ bool chunk_item(const SiftArgs& a, long item, int& e, int& r, int& b,
                                           int& K, int& P) {
    const long per = (long)a.chunk_blocks;
    const int re = (int)(item / per);
    b = (int)(item % per);
    e = re / a.nr;
    r = re % a.nr;
    K = a.kcount[re];
    if (K <= kChunk) return false;
    P = (K - 1) / kChunk;
    return b * kChunksPerBlock <= P;
}

}  // namespace

__global__ void __launch_bounds__(kThreads)
k_chunk_reduce(SiftArgs a) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    StagedKnots& sk = *reinterpret_cast<StagedKnots*>(dyn_smem);
    if (*a.done) return;
    const long items = (long)2 * a.nr * a.chunk_blocks;
    for (long item = blockIdx.x; item < items; item += gridDim.x) {
        int e, r, b, K, P;
        if (!chunk_item(a, item, e, r, b, K, P)) continue;
        const int re = e * a.nr + r;
        const size_t kb = (size_t)r * (size_t)a.cap;
        const int32_t* kx = (e == 0 ? a.kx_max : a.kx_min) + kb;
        const double* ky = (e == 0 ? a.ky_max : a.ky_min) + kb;
        const int row0 = b * kChunksPerBlock * kChunk;
        __syncthreads();
        stage_knots(sk, row0, K, kx, ky);
        __syncthreads();
        const int q = b * kChunksPerBlock + threadIdx.x;
        if (q <= P) {
            const int first = q * kChunk;
            const int len = (q < P) ? kChunk - 1 : K - first;
            StagedRowFn fn{&sk, first, row0, K};
            const ChunkEnds ce = chunk_sweep(len, fn, 0.0, 0.0, nullptr, 0);
            const size_t o = (size_t)re * (size_t)a.rec_stride + q;
            a.rec[0 * a.rec_plane + o] = ce.ga;
            a.rec[1 * a.rec_plane + o] = ce.aa;
            a.rec[2 * a.rec_plane + o] = ce.ba;
            a.rec[3 * a.rec_plane + o] = ce.gb;
            a.rec[4 * a.rec_plane + o] = ce.ab;
            a.rec[5 * a.rec_plane + o] = ce.bb;
            if (q < P) {
                const Row s = fn(kChunk - 1);  // separator row first + kChunk - 1
                a.rec[6 * a.rec_plane + o] = s.l;
                a.rec[7 * a.rec_plane + o] = s.m;
                a.rec[8 * a.rec_plane + o] = s.u;
                a.rec[9 * a.rec_plane + o] = s.r;
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads)
k_chunk_backsub(SiftArgs a) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    StagedKnots& sk = *reinterpret_cast<StagedKnots*>(dyn_smem);
    double* sc = reinterpret_cast<double*>(dyn_smem + sizeof(StagedKnots));
    if (*a.done) return;
    const long items = (long)2 * a.nr * a.chunk_blocks;
    for (long item = blockIdx.x; item < items; item += gridDim.x) {
        int e, r, b, K, P;
        if (!chunk_item(a, item, e, r, b, K, P)) continue;
        const int re = e * a.nr + r;
        const size_t kb = (size_t)r * (size_t)a.cap;
        const int32_t* kx = (e == 0 ? a.kx_max : a.kx_min) + kb;
        const double* ky = (e == 0 ? a.ky_max : a.ky_min) + kb;
        double* c = (e == 0 ? a.c_max : a.c_min) + kb;
        const int row0 = b * kChunksPerBlock * kChunk;
        __syncthreads();
        stage_knots(sk, row0, K, kx, ky);
        __syncthreads();
        const int q = b * kChunksPerBlock + threadIdx.x;
        const double* X = a.xsep + (size_t)re * (size_t)a.rec_stride;
        if (q <= P) {
            const int first = q * kChunk;
            const int len = (q < P) ? kChunk - 1 : K - first;
            StagedRowFn fn{&sk, first, row0, K};
            const double xl = (q > 0) ? X[q - 1] : 0.0;
            const double xr = (q < P) ? X[q] : 0.0;
            // local rows k -> shared slot pad17(threadIdx.x*kChunk + k)
            double* dst = &sc[pad17(threadIdx.x * kChunk)];
            chunk_sweep(len, fn, xl, xr, dst, 1);
            if (q < P) dst[kChunk - 1] = xr;
        }
        __syncthreads();
        const int rows = min(kChunksPerBlock * kChunk, K - row0);
        for (int j = threadIdx.x; j < rows; j += kThreads) c[row0 + j] = sc[pad17(j)];
    }
}

size_t chunk_reduce_smem() { return sizeof(StagedKnots); }
size_t chunk_backsub_smem() { return sizeof(StagedKnots) + sizeof(double) * kBacksubSlots; }

// =======================================================================================
// k_reduced_solve: levels >= 2 of the partitioned solve, one CTA per spline system.
// Small systems (K <= kChunk) are solved here directly from the knots.
// =======================================================================================
namespace {

struct GlobalRowFn {
    const double *l, *m, *u, *r;
    int first;
    __device__ __forceinline__ Row operator()(int k) const {
        const int i = first + k;
        Row w;
        w.l = l[i];
        w.m = m[i];
        w.u = u[i];
        w.r = r[i];
        return w;
    }
};

struct KnotRowFn {
    const int32_t* kx;
    const double* ky;
    int K;
    __device__ __forceinline__ Row operator()(int k) const {
        return spline_row_global(k, K, kx, ky);
    }
};

// In-CTA canonical partitioned solve of an explicit system stored at sys (4 planes of
// `plane` doubles: l, m, u, r), solution to x.  ws: workspace of >= 8*plane doubles for the
// deeper levels.  All threads of the CTA must call it.
__device__ void cta_partitioned(int n, double* sys, int plane, double* x, double* ws) {
    // level sizes
    int sizes[8];
    int depth = 0;
    sizes[0] = n;
    while (sizes[depth] > kChunk && depth < 7) {
        sizes[depth + 1] = (sizes[depth] - 1) / kChunk;
        ++depth;
    }
    // level k system at sys (k == 0) or in ws; level x vectors in ws
    double* lv[8];
    double* xv[8];
    int off = 0;
    lv[0] = sys;
    for (int k = 1; k <= depth; ++k) {
        lv[k] = ws + off;
        off += 4 * sizes[k];
    }
    xv[0] = x;
    for (int k = 1; k <= depth; ++k) {
        xv[k] = ws + off;
        off += sizes[k];
    }
    double* ends = ws + off;  // 6 * (max chunks) scratch
    // down pass
    for (int k = 0; k < depth; ++k) {
        const int nk = sizes[k];
        const int P = sizes[k + 1];
        const int pl = (k == 0) ? plane : nk;
        const double* L = lv[k];
        for (int q = threadIdx.x; q <= P; q += blockDim.x) {
            const int first = q * kChunk;
            const int len = (q < P) ? kChunk - 1 : nk - first;
            GlobalRowFn fn{L, L + pl, L + 2 * pl, L + 3 * pl, first};
            const ChunkEnds ce = chunk_sweep(len, fn, 0.0, 0.0, nullptr, 0);
            ends[6 * q + 0] = ce.ga;
            ends[6 * q + 1] = ce.aa;
            ends[6 * q + 2] = ce.ba;
            ends[6 * q + 3] = ce.gb;
            ends[6 * q + 4] = ce.ab;
            ends[6 * q + 5] = ce.bb;
        }
        __syncthreads();
        double* R = lv[k + 1];
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            const int s = p * kChunk + kChunk - 1;
            Row sr;
            sr.l = L[s];
            sr.m = L[pl + s];
            sr.u = L[2 * pl + s];
            sr.r = L[3 * pl + s];
            const Row o = reduced_row(sr, ends[6 * p + 3], ends[6 * p + 4], ends[6 * p + 5],
                                      ends[6 * (p + 1) + 0], ends[6 * (p + 1) + 1],
                                      ends[6 * (p + 1) + 2]);
            R[p] = o.l;
            R[P + p] = o.m;
            R[2 * P + p] = o.u;
            R[3 * P + p] = o.r;
        }
        __syncthreads();
    }
    // base case
    if (threadIdx.x == 0) {
        const int nb = sizes[depth];
        const int pl = (depth == 0) ? plane : nb;
        const double* L = lv[depth];
        GlobalRowFn fn{L, L + pl, L + 2 * pl, L + 3 * pl, 0};
        thomas_small(nb, fn, xv[depth], 1);
    }
    __syncthreads();
    // up pass
    for (int k = depth - 1; k >= 0; --k) {
        const int nk = sizes[k];
        const int P = sizes[k + 1];
        const int pl = (k == 0) ? plane : nk;
        const double* L = lv[k];
        const double* Xs = xv[k + 1];
        double* xo = xv[k];
        for (int q = threadIdx.x; q <= P; q += blockDim.x) {
            const int first = q * kChunk;
            const int len = (q < P) ? kChunk - 1 : nk - first;
            GlobalRowFn fn{L, L + pl, L + 2 * pl, L + 3 * pl, first};
            const double xl = (q > 0) ? Xs[q - 1] : 0.0;
            const double xr = (q < P) ? Xs[q] : 0.0;
            chunk_sweep(len, fn, xl, xr, xo + first, 1);
            if (q < P) xo[first + kChunk - 1] = xr;
        }
        __syncthreads();
    }
}

}  // namespace

__global__ void __launch_bounds__(kThreads)
k_reduced_solve(SiftArgs a) {
    if (*a.done) return;
    const int re = blockIdx.x;
    if (re >= 2 * a.nr) return;
    const int e = re / a.nr, r = re % a.nr;
    const int K = a.kcount[re];
    const size_t kb = (size_t)r * (size_t)a.cap;
    if (K <= kChunk) {
        if (threadIdx.x == 0) {
            const int32_t* kx = (e == 0 ? a.kx_max : a.kx_min) + kb;
            const double* ky = (e == 0 ? a.ky_max : a.ky_min) + kb;
            double* c = (e == 0 ? a.c_max : a.c_min) + kb;
            KnotRowFn fn{kx, ky, K};
            thomas_small(K, fn, c, 1);
        }
        return;
    }
    const int P = (K - 1) / kChunk;
    double* sys = a.red + (size_t)re * (size_t)a.red_stride;
    double* ws = sys + 4 * (size_t)a.rec_stride;
    const size_t o = (size_t)re * (size_t)a.rec_stride;
    // level-2 rows from the chunk records
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        Row sr;
        sr.l = a.rec[6 * a.rec_plane + o + p];
        sr.m = a.rec[7 * a.rec_plane + o + p];
        sr.u = a.rec[8 * a.rec_plane + o + p];
        sr.r = a.rec[9 * a.rec_plane + o + p];
        const Row w = reduced_row(sr, a.rec[3 * a.rec_plane + o + p], a.rec[4 * a.rec_plane + o + p],
                                  a.rec[5 * a.rec_plane + o + p],
                                  a.rec[0 * a.rec_plane + o + p + 1],
                                  a.rec[1 * a.rec_plane + o + p + 1],
                                  a.rec[2 * a.rec_plane + o + p + 1]);
        sys[p] = w.l;
        sys[a.rec_stride + p] = w.m;
        sys[2 * (size_t)a.rec_stride + p] = w.u;
        sys[3 * (size_t)a.rec_stride + p] = w.r;
    }
    __syncthreads();
    cta_partitioned(P, sys, a.rec_stride, a.xsep + o, ws);
}

// =======================================================================================
// k_eval: envelopes + mean envelope + sx statistics over one tile of samples
// =======================================================================================
__global__ void __launch_bounds__(kThreads)
k_eval(SiftArgs a) {
    constexpr int kMaxKnots = kTileSamples / 2 + 4;
    __shared__ int32_t sx_[kMaxKnots];
    __shared__ double sy[kMaxKnots], scf[kMaxKnots], sb[kMaxKnots], sd[kMaxKnots];
    __shared__ int s_red[kThreads / 32];
    __shared__ int s_any[kThreads / 32];

    if (*a.done) return;
    const int tile = blockIdx.x;
    const int r = blockIdx.y;
    const int n = a.n;
    const int n0 = tile * kTileSamples;
    const size_t base = (size_t)r * (size_t)n;
    const size_t kb = (size_t)r * (size_t)a.cap;
    const size_t to = (size_t)(a.ntiles + 1);
    double env[2][kPerThread];

    for (int e = 0; e < 2; ++e) {
        const int K = a.kcount[e * a.nr + r];
        const int off0 = a.tile_off[(size_t)(e * a.nr + r) * to + tile];
        const int off1 = a.tile_off[(size_t)(e * a.nr + r) * to + tile + 1];
        const int klo = off0 > 0 ? off0 - 1 : 0;
        const int khi = min(off1, K - 1);
        const int nk = khi - klo + 1;
        const int32_t* kx = (e == 0 ? a.kx_max : a.kx_min) + kb;
        const double* ky = (e == 0 ? a.ky_max : a.ky_min) + kb;
        const double* kc = (e == 0 ? a.c_max : a.c_min) + kb;
        __syncthreads();
        for (int j = threadIdx.x; j < nk; j += kThreads) {
            sx_[j] = kx[klo + j];
            sy[j] = ky[klo + j];
            scf[j] = kc[klo + j];
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nk - 1; j += kThreads)
            seg_coeffs(sx_[j], sx_[j + 1], sy[j], sy[j + 1], scf[j], scf[j + 1], sb[j], sd[j]);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const int s = n0 + k * kThreads + threadIdx.x;
            double v = 0.0;
            if (s < n) {
                // segment: largest j in [0, nk-2] with x_j < s (j = 0 for s = 0)
                int lo = 0, hi = nk - 2;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (sx_[mid] < s) lo = mid; else hi = mid - 1;
                }
                v = seg_eval(sy[lo], sb[lo], scf[lo], sd[lo], (double)(s - sx_[lo]));
            }
            env[e][k] = v;
        }
    }

    const bool valid = a.kcount[r] > 3 && a.kcount[a.nr + r] > 3;
    int cnt = 0, any = 0;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int s = n0 + k * kThreads + threadIdx.x;
        if (s < n) {
            const double up = env[0][k], lo = env[1][k];
            if (valid) a.menv[base + s] = (up + lo) / 2.0;
            const double sx = sx_value(up, lo);
            any |= (sx > a.sd2) ? 1 : 0;
            cnt += (sx > a.sd) ? 1 : 0;
            if (a.dbg_upper) {
                a.dbg_upper[base + s] = up;
                a.dbg_lower[base + s] = lo;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        any |= __shfl_xor_sync(0xffffffffu, any, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_red[threadIdx.x >> 5] = cnt;
        s_any[threadIdx.x >> 5] = any;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int c = 0, y = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
            c += s_red[w];
            y |= s_any[w];
        }
        if (c) atomicAdd(&a.cnt[r], (unsigned)c);
        if (y) atomicOr(&a.any[r], 1);
    }
}

// =======================================================================================
// k_criterion: one CTA over all realizations
// =======================================================================================
__global__ void __launch_bounds__(kThreads)
k_criterion(SiftArgs a) {
    __shared__ int s_all[kThreads / 32];
    if (*a.done) return;
    const int j = *a.iter;
    int all = 1;
    for (int r = threadIdx.x; r < a.nr; r += blockDim.x) {
        const unsigned c = a.cnt[r];
        const int any = a.any[r];
        a.cnt[r] = 0u;
        a.any[r] = 0;
        const double fr = (a.frac[r] + (double)c) * a.inv_n;
        a.frac[r] = fr;
        const bool crit = fr > a.tol || (any != 0 && (a.kcount[r] + a.kcount[a.nr + r]) > 6);
        int fin = a.finish[r];
        int mark;
        if (crit) {
            mark = 1;
            if (fin == 0 && j == a.cap_iter - 1) {
                mark = 0;
                fin = 1;
            }
        } else {
            if (fin == 0) {
                mark = 0;
                fin = 1;
            } else {
                mark = 1;
            }
        }
        a.mark[r] = mark;
        a.finish[r] = fin;
        all &= fin;
    }
    all = __all_sync(0xffffffffu, all);
    if ((threadIdx.x & 31) == 0) s_all[threadIdx.x >> 5] = all;
    __syncthreads();
    if (threadIdx.x == 0) {
        int d = 1;
        for (int w = 0; w < kThreads / 32; ++w) d &= s_all[w];
        *a.iter = j + 1;
        if (d) *a.done = 1;
    }
}

// Mode export of the realizations that finished in the last executed iteration.
__global__ void k_export_final(SiftArgs a, const double* h) {
    const int r = blockIdx.y;
    if (a.mark[r] != 0) return;
    const size_t base = (size_t)r * (size_t)a.n;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < a.n; s += gridDim.x * blockDim.x)
        a.mode_out[base + s] = h[base + s];
}

// =======================================================================================
// generic batched tridiagonal solve (stage-level entry point): one CTA per system
// =======================================================================================
__global__ void __launch_bounds__(kThreads)
k_tridiag_batched(int n, const double* l, const double* m, const double* u, const double* r,
                  double* x, double* sys, double* ws, size_t ws_stride) {
    const size_t b = blockIdx.x;
    double* S = sys + b * 4 * (size_t)n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        S[i] = l[b * n + i];
        S[n + i] = m[b * n + i];
        S[2 * n + i] = u[b * n + i];
        S[3 * n + i] = r[b * n + i];
    }
    __syncthreads();
    cta_partitioned(n, S, n, x + b * n, ws + b * ws_stride);
}

}  // namespace ceemdan
