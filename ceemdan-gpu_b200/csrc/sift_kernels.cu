// Sifting kernels of the ICEEMDAN engine (sm_100a, FP64).
//
// One sift iteration over all realizations of a stage is:
//   k_extrema        deferred update h -= m (or mode export) + strict-extrema flags +
//                    warp-ballot compaction into per-tile knot storage, knot bitmaps
//                    (find_extrema_shfl_* :93-148, select_extrema_* :151-207,
//                     updateRealizations :528-544 of the previous iteration)
//   k_scan_boundary  per-spline scan of the tile knot counts (CUB scan :1582-1604) and the
//                    end-knot extrapolation (setBoundaryMax/Min :210-291)
//   k_chunk_reduce   level-1 chunk end relations of the canonical partitioned spline solve
//   k_reduced_solve  per-system reduced solve (levels >= 2), one CTA per spline
//   k_chunk_backsub  level-1 chunk interiors -> spline coefficients c
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
constexpr int kWords = kPerThread * (kThreads / 32); // ballot words per tile (64)
constexpr int kChunksPerBlock = kThreads;            // one level-1 chunk per thread

__device__ __forceinline__ int pad17(int j) { return j + (j >> 4); }

__device__ __forceinline__ void set_error(int* err, int code) { atomicCAS(err, 0, code); }

// Asynchronous global -> shared copies (cp.async): the whole staging window is in flight at
// once instead of one round trip per loop iteration.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }

// Tile of global knot index i in an offset row off[0..ntiles] (off[t] = knots before tile t):
// the largest t with off[t] <= i, which is the non-empty tile holding knot i.
__device__ __forceinline__ int tile_of(const int* off, int ntiles, int i) {
    int lo = 0, hi = ntiles - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ size_t tile_base(const SiftArgs& a, int r, int t) {
    return ((size_t)r * a.ntiles + t) * kTileCap;
}

// Global address of knot i of spline r: the tile is found by walking from tile `t` (a tile at
// or before the one holding knot i when walking forward, at or after it when backward) --
// one or two steps for the end knots and the neighbours of a tile.
__device__ __forceinline__ size_t knot_addr_fwd(const SiftArgs& a, const int* off, int r, int t,
                                                int i) {
    while (off[t + 1] <= i) ++t;
    return tile_base(a, r, t) + (size_t)(i - off[t]);
}
__device__ __forceinline__ size_t knot_addr_bwd(const SiftArgs& a, const int* off, int r, int t,
                                                int i) {
    while (off[t] > i) --t;
    return tile_base(a, r, t) + (size_t)(i - off[t]);
}

// Exact (y1 - y0) / (x1 - x0) and c / (3 (x1 - x0)) with tabled reciprocals (div_rcp).
__device__ __forceinline__ double slope_t(const SiftArgs& a, int32_t x0, int32_t x1, double y0,
                                          double y1) {
    const int h = x1 - x0;
    const double dy = y1 - y0;
    return h <= kRcpMax ? div_rcp(dy, (double)h, __ldg(a.rcp_h + h)) : dy / (double)h;
}

__device__ __forceinline__ void seg_coeffs_t(const SiftArgs& a, int32_t x0, int32_t x1, double y0,
                                             double y1, double c0, double c1, double& b,
                                             double& d) {
    const int hi = x1 - x0;
    const double h = (double)hi;
    const double q = fma(2.0, c0, c1);
    b = slope_t(a, x0, x1, y0, y1) - div_rcp(h * q, 3.0, kRcp3);
    const double dc = c1 - c0;
    d = hi <= kRcpMax ? div_rcp(dc, 3.0 * h, __ldg(a.rcp_3h + hi)) : dc / (3.0 * h);
}

// ---------------------------------------------------------------------------------------
// chunk primitives of the canonical partitioned solve (rows produced by a functor)
// ---------------------------------------------------------------------------------------
struct ChunkEnds {
    double ga, aa, ba, gb, ab, bb;
};

// End relations of a chunk of `len` rows: top-down elimination gives the last row
// x_b = gb + ab*xL + bb*xR, bottom-up elimination the first row x_a = ga + aa*xL + ba*xR.
// The two sweeps are independent chains and run interleaved.
template <class RowFn>
__device__ __forceinline__ ChunkEnds chunk_ends(int len, const RowFn& row) {
    const Row wa = row(0), wb = row(len - 1);
    double iw = 1.0 / wa.m;
    double cp = wa.u * iw, gp = wa.r * iw, ap = -wa.l * iw;
    double iv = 1.0 / wb.m;
    double cq = wb.l * iv, gq = wb.r * iv, bq = -wb.u * iv;
    for (int k = 1; k < len; ++k) {
        const Row w = row(k);
        const Row v = row(len - 1 - k);
        iw = 1.0 / fma(-w.l, cp, w.m);
        iv = 1.0 / fma(-v.u, cq, v.m);
        cp = w.u * iw;
        gp = fma(-w.l, gp, w.r) * iw;
        ap = (-w.l * ap) * iw;
        cq = v.l * iv;
        gq = fma(-v.u, gq, v.r) * iv;
        bq = (-v.u * bq) * iv;
    }
    ChunkEnds e;
    e.gb = gp;
    e.ab = ap;
    e.bb = -wb.u * iw;
    e.ga = gq;
    e.ba = bq;
    e.aa = -wa.l * iv;
    return e;
}

// Interior of a chunk of `len` rows once its separator values xl, xr are known: coupling
// terms move to the right-hand side, then canonical Thomas; x_k written to out[k*stride].
// kCoupled = false is the plain canonical Thomas (no coupling terms at all).
template <bool kCoupled = true, class RowFn>
__device__ __forceinline__ void chunk_interior(int len, const RowFn& row, double xl, double xr,
                                               double* out, int stride) {
    double cp[kChunk], gp[kChunk];
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
        if (k < len) {
            const Row w = row(k);
            double ri = w.r;
            if (kCoupled && k == 0) ri = fma(-w.l, xl, ri);
            if (kCoupled && k == len - 1) ri = fma(-w.u, xr, ri);
            if (k == 0) {
                const double iw = 1.0 / w.m;
                cp[0] = w.u * iw;
                gp[0] = ri * iw;
            } else {
                const double iw = pivot_rcp(w, cp[k - 1]);
                cp[k] = w.u * iw;
                gp[k] = fma(-w.l, gp[k - 1], ri) * iw;
            }
        }
    }
    double xv = 0.0;
#pragma unroll
    for (int k = kChunk - 1; k >= 0; --k) {
        if (k < len) {
            xv = (k == len - 1) ? gp[k] : fma(-cp[k], xv, gp[k]);
            out[k * stride] = xv;
        }
    }
}

// Canonical Thomas on n <= kChunk rows (base case), x written with stride.
template <class RowFn>
__device__ __forceinline__ void thomas_small(int n, const RowFn& row, double* x, int stride) {
    chunk_interior<false>(n, row, 0.0, 0.0, x, stride);
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
    __shared__ __align__(16) double sh[kTileSamples + 4];  // sh[2 + j] = sample n0 + j
    __shared__ int s_cnt[2][kWords];
    __shared__ int s_off[2][kWords];

    if (*a.done) return;
    const int tile = blockIdx.x;
    const int r = blockIdx.y;
    const int n = a.n;
    const int n0 = tile * kTileSamples;
    const size_t base = (size_t)r * (size_t)n;
    const int mk = a.mark[r];
    const double* __restrict__ hin = a.h_in + base;
    double* __restrict__ hout = a.h_out + base;
    const double* __restrict__ me = a.menv + base;
    double* __restrict__ mo = a.mode_out ? a.mode_out + base : nullptr;

    // Deferred update of the previous iteration (h -= m, or mode export), tile + halo
    // into shared memory.  Even n: each thread moves 8 consecutive samples as 4 double2.
    if ((n & 1) == 0) {
        const int j0 = threadIdx.x * kPerThread;
        double2 hv[kPerThread / 2], mv[kPerThread / 2];
#pragma unroll
        for (int k = 0; k < kPerThread / 2; ++k) {
            const int s = n0 + j0 + 2 * k;
            if (s < n) {
                hv[k] = *reinterpret_cast<const double2*>(hin + s);
                if (mk == 1) mv[k] = *reinterpret_cast<const double2*>(me + s);
            }
        }
#pragma unroll
        for (int k = 0; k < kPerThread / 2; ++k) {
            const int s = n0 + j0 + 2 * k;
            double2 v = make_double2(0.0, 0.0);
            if (s < n) {
                v = hv[k];
                if (mk == 1) {
                    v.x = v.x - mv[k].x;
                    v.y = v.y - mv[k].y;
                }
                *reinterpret_cast<double2*>(hout + s) = v;
                if (mk == 0) *reinterpret_cast<double2*>(mo + s) = hv[k];
            }
            sh[2 + j0 + 2 * k] = v.x;
            sh[2 + j0 + 2 * k + 1] = v.y;
        }
    } else {
        double hv[kPerThread], mv[kPerThread];
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const int s = n0 + k * kThreads + threadIdx.x;
            if (s < n) {
                hv[k] = hin[s];
                if (mk == 1) mv[k] = me[s];
            }
        }
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const int j = k * kThreads + threadIdx.x;
            const int s = n0 + j;
            double v = 0.0;
            if (s < n) {
                v = (mk == 1) ? hv[k] - mv[k] : hv[k];
                hout[s] = v;
                if (mk == 0) mo[s] = hv[k];
            }
            sh[2 + j] = v;
        }
    }
    if (threadIdx.x < 2) {  // halo samples n0-1 and n0+kTileSamples
        const int s = threadIdx.x == 0 ? n0 - 1 : n0 + kTileSamples;
        double v = 0.0;
        if (s >= 0 && s < n) {
            const double hv = hin[s];
            v = (mk == 1) ? hv - me[s] : hv;
        }
        sh[threadIdx.x == 0 ? 1 : 2 + kTileSamples] = v;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const size_t bw0 = ((size_t)r * a.ntiles + tile) * kWords;
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
                const double v = sh[2 + j], vl = sh[1 + j], vr = sh[3 + j];
                fmax = v > vl && v > vr;
                fmin = v < vl && v < vr;
            }
        }
        bmax[k] = __ballot_sync(0xffffffffu, fmax);
        bmin[k] = __ballot_sync(0xffffffffu, fmin);
        if (lane == 0) {
            const int w = k * (kThreads / 32) + warp;
            s_cnt[0][w] = __popc(bmax[k]);
            s_cnt[1][w] = __popc(bmin[k]);
            a.bitmap[bw0 + w] = bmax[k];
            a.bitmap[(size_t)a.nr * a.ntiles * kWords + bw0 + w] = bmin[k];
        }
    }
    __syncthreads();

    // Exclusive scan of the 64 word counts per envelope: warp 0 -> maxima, warp 1 -> minima;
    // the total is the tile's knot count.
    static_assert(kWords == 64, "scan assumes 64 words");
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
        if (lane == 31) a.tile_cnt[((size_t)e * a.nr + r) * a.ntiles + tile] = incl;
    }
    __syncthreads();

    const unsigned lt = (1u << lane) - 1u;
    const size_t kb = tile_base(a, r, tile);
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int j = k * kThreads + threadIdx.x;
        const int s = n0 + j;
        const int w = k * (kThreads / 32) + warp;
        if (bmax[k] & (1u << lane)) {
            const int pos = s_off[0][w] + __popc(bmax[k] & lt);
            a.kx_max[kb + pos] = s;
            a.ky_max[kb + pos] = sh[2 + j];
        }
        if (bmin[k] & (1u << lane)) {
            const int pos = s_off[1][w] + __popc(bmin[k] & lt);
            a.kx_min[kb + pos] = s;
            a.ky_min[kb + pos] = sh[2 + j];
        }
    }
}

// =======================================================================================
// k_scan_boundary: one warp per spline (envelope, realization): exclusive scan of the tile
// knot counts into the offset row, the knot count, and the end-knot extrapolation.
// =======================================================================================
__global__ void __launch_bounds__(kThreads)
k_scan_boundary(SiftArgs a) {
    if (*a.done) return;
    const int lane = threadIdx.x & 31;
    const int id = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
    if (id >= 2 * a.nr) return;
    const int e = id / a.nr, r = id % a.nr;
    const int* cnt = a.tile_cnt + (size_t)id * a.ntiles;
    int* off = a.tile_off + (size_t)id * (a.ntiles + 1);
    int carry = 0;
    for (int t0 = 0; t0 < a.ntiles; t0 += 32) {
        const int t = t0 + lane;
        const int c = t < a.ntiles ? cnt[t] : 0;
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (t < a.ntiles) off[t] = carry + incl - c;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    const int K = carry;
    if (lane == 0) {
        off[a.ntiles] = K;
        a.kcount[id] = K;
    }
    // address of the knot just before each tile (last knot of the nearest non-empty tile
    // before it) and just after it (first knot of the nearest non-empty tile after it)
    long long* nb = a.nbr + (size_t)id * a.ntiles * 2;
    int last = -1;  // nearest non-empty tile before the current chunk
    for (int t0 = 0; t0 < a.ntiles; t0 += 32) {
        const int t = t0 + lane;
        const int c = t < a.ntiles ? cnt[t] : 0;
        int v = c > 0 ? t : -1;  // inclusive max-scan of non-empty tile indices
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v = max(v, u);
        }
        int before = __shfl_up_sync(0xffffffffu, v, 1);
        if (lane == 0) before = -1;
        before = max(before, last);
        if (t < a.ntiles)
            nb[2 * t] = before >= 0 ? (long long)(tile_base(a, r, before) + cnt[before] - 1) : -1;
        last = max(last, __shfl_sync(0xffffffffu, v, 31));
    }
    int first = 0x7fffffff;  // nearest non-empty tile after the current chunk
    for (int t0 = ((a.ntiles - 1) / 32) * 32; t0 >= 0; t0 -= 32) {
        const int t = t0 + lane;
        const int c = t < a.ntiles ? cnt[t] : 0;
        int v = c > 0 ? t : 0x7fffffff;  // inclusive min-scan from the right
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_down_sync(0xffffffffu, v, o);
            if (lane + o < 32) v = min(v, u);
        }
        int after = __shfl_down_sync(0xffffffffu, v, 1);
        if (lane == 31) after = 0x7fffffff;
        after = min(after, first);
        if (t < a.ntiles)
            nb[2 * t + 1] = after < a.ntiles ? (long long)tile_base(a, r, after) : -1;
        first = min(first, __shfl_sync(0xffffffffu, v, 0));
    }
    __syncwarp();
    if (lane == 0 && K - 1 > 4) {
        int32_t* kx = e == 0 ? a.kx_max : a.kx_min;
        double* ky = e == 0 ? a.ky_max : a.ky_min;
        const int L = K - 1;
        const int tl = a.ntiles - 1;
        const size_t p0 = knot_addr_fwd(a, off, r, 0, 0), p1 = knot_addr_fwd(a, off, r, 0, 1),
                     p2 = knot_addr_fwd(a, off, r, 0, 2);
        const size_t q0 = knot_addr_bwd(a, off, r, tl, L - 2),
                     q1 = knot_addr_bwd(a, off, r, tl, L - 1), q2 = knot_addr_bwd(a, off, r, tl, L);
        const double y0 = boundary_left(e, kx[p0], kx[p1], kx[p2], ky[p0], ky[p1], ky[p2]);
        const double yL = boundary_right(e, kx[q0], kx[q1], kx[q2], ky[q0], ky[q1], ky[q2]);
        ky[p0] = y0;
        ky[q2] = yL;
    }
}

// Compacted copy of the knots of envelope e (stage-level entry point): realization r's
// knots to kx/ky[r*n + i].
__global__ void k_gather_knots(SiftArgs a, int e, int32_t* kx, double* ky) {
    const int tile = blockIdx.x, r = blockIdx.y;
    const int* off = a.tile_off + ((size_t)e * a.nr + r) * (a.ntiles + 1);
    const int o = off[tile], c = off[tile + 1] - o;
    const size_t src = tile_base(a, r, tile);
    const int32_t* sx = e == 0 ? a.kx_max : a.kx_min;
    const double* sy = e == 0 ? a.ky_max : a.ky_min;
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
        kx[(size_t)r * a.n + o + j] = sx[src + j];
        ky[(size_t)r * a.n + o + j] = sy[src + j];
    }
}

// =======================================================================================
// level-1 chunk kernels (end relations and interiors share the staging)
// =======================================================================================
namespace {

constexpr int kSpan = kChunksPerBlock * kChunk + 2;        // staged knots per block
constexpr int kStageSlots = kSpan + (kSpan >> 4) + 1;      // with one pad per 16
constexpr int kOutSlots = kChunksPerBlock * kChunk + ((kChunksPerBlock * kChunk) >> 4) + 1;

// Knot positions and segment slopes of the window [row0-1, row0-1+kSpan), padded so that
// each thread's 16 consecutive rows sit at stride 17 (bank-conflict free).  The knot values
// are staged into `slope` first and replaced by the segment slopes.
struct Staged {
    double slope[kStageSlots];  // slope[pad17(j)]: segment between window knots j, j+1
    int32_t x[kStageSlots];
    int t0, t1;                 // tiles holding the first and last knot of the window
};

// Copy (cp.async) knots [i0, i1) of spline r into the window, tile range by tile range; the
// window slot of knot i is pad17(i - wbase).  `off` is the offset row in shared memory.
__device__ __forceinline__ void stage_knots(Staged& sg, const SiftArgs& a, const int* off, int r,
                                            const int32_t* kx, const double* ky, int i0, int i1,
                                            int wbase) {
    if (threadIdx.x == 0) {
        sg.t0 = tile_of(off, a.ntiles, i0);
        sg.t1 = tile_of(off, a.ntiles, i1 - 1);
    }
    __syncthreads();
    for (int T = sg.t0; T <= sg.t1; ++T) {
        const int oT = off[T];
        const int lo = max(i0, oT), hi = min(i1, off[T + 1]);
        const size_t tb = tile_base(a, r, T);
        for (int i = lo + threadIdx.x; i < hi; i += kThreads) {
            const int j = pad17(i - wbase);
            cp_async4(&sg.x[j], kx + tb + (i - oT));
            cp_async8(&sg.slope[j], ky + tb + (i - oT));
        }
    }
    cp_async_wait_all();
    __syncthreads();
}

__device__ __forceinline__ void stage_window(Staged& sg, const SiftArgs& a, const int* off, int r,
                                             int row0, int K, const int32_t* kx,
                                             const double* ky) {
    constexpr int kIt = (kSpan + kThreads - 1) / kThreads;
    const int i0 = max(row0 - 1, 0), i1 = min(row0 - 1 + kSpan, K);
    stage_knots(sg, a, off, r, kx, ky, i0, i1, row0 - 1);
    // slopes replace the knot values in place, in rounds of kRound strided elements: a
    // round only reads values at or after its own first element, which later rounds never
    // rewrite before reading.
    constexpr int kRound = 4;
    for (int t0 = 0; t0 < kIt; t0 += kRound) {
        double sl[kRound];
#pragma unroll
        for (int t = 0; t < kRound; ++t) {
            const int j = threadIdx.x + (t0 + t) * kThreads;
            const int i = row0 - 1 + j;
            sl[t] = 0.0;
            if (j + 1 < kSpan && i >= 0 && i + 1 < K)
                sl[t] = slope_t(a, sg.x[pad17(j)], sg.x[pad17(j + 1)], sg.slope[pad17(j)],
                                sg.slope[pad17(j + 1)]);
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < kRound; ++t) {
            const int j = threadIdx.x + (t0 + t) * kThreads;
            if (j < kSpan) sg.slope[pad17(j)] = sl[t];
        }
    }
    __syncthreads();
}

// Rows of the natural-spline system from the staged window.
struct StagedRowFn {
    const Staged* sg;
    int first_row;  // global row of local row 0
    int row0;       // global row of window knot 1
    int K;
    __device__ __forceinline__ Row operator()(int k) const {
        const int i = first_row + k;
        if (i == 0 || i == K - 1) return identity_row();
        const int j = i - row0 + 1;
        return spline_row(sg->x[pad17(j - 1)], sg->x[pad17(j)], sg->x[pad17(j + 1)],
                          sg->slope[pad17(j - 1)], sg->slope[pad17(j)]);
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

// Dynamic shared memory: the staged window, [the interior output], and the offset row.
size_t chunk_reduce_smem(int ntiles) { return sizeof(Staged) + sizeof(int) * (ntiles + 1); }
size_t eval_smem() { return 0; }
size_t chunk_backsub_smem(int ntiles) {
    return sizeof(Staged) + sizeof(double) * kOutSlots + sizeof(int) * (ntiles + 1);
}

// Copy the offset row of spline re into shared memory.
__device__ __forceinline__ const int* stage_off_row(const SiftArgs& a, int re, int* soff) {
    const int* off = a.tile_off + (size_t)re * (a.ntiles + 1);
    for (int t = threadIdx.x; t <= a.ntiles; t += kThreads) soff[t] = off[t];
    __syncthreads();
    return soff;
}

__global__ void __launch_bounds__(kThreads)
k_chunk_reduce(SiftArgs a) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    Staged& sg = *reinterpret_cast<Staged*>(dyn_smem);
    int* soff = reinterpret_cast<int*>(dyn_smem + sizeof(Staged));
    if (*a.done) return;
    {
        int e, r, b, K, P;
        if (!chunk_item(a, blockIdx.x, e, r, b, K, P)) return;
        const int re = e * a.nr + r;
        const int* off = stage_off_row(a, re, soff);
        const int32_t* kx = e == 0 ? a.kx_max : a.kx_min;
        const double* ky = e == 0 ? a.ky_max : a.ky_min;
        const int row0 = b * kChunksPerBlock * kChunk;
        stage_window(sg, a, off, r, row0, K, kx, ky);
        const int q = b * kChunksPerBlock + threadIdx.x;
        if (q <= P) {
            const int first = q * kChunk;
            const int len = (q < P) ? kChunk - 1 : K - first;
            StagedRowFn fn{&sg, first, row0, K};
            const ChunkEnds ce = chunk_ends(len, fn);
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
    Staged& sg = *reinterpret_cast<Staged*>(dyn_smem);
    double* sc = reinterpret_cast<double*>(dyn_smem + sizeof(Staged));
    int* soff = reinterpret_cast<int*>(dyn_smem + sizeof(Staged) + sizeof(double) * kOutSlots);
    if (*a.done) return;
    {
        int e, r, b, K, P;
        if (!chunk_item(a, blockIdx.x, e, r, b, K, P)) return;
        const int re = e * a.nr + r;
        const int* off = stage_off_row(a, re, soff);
        const int32_t* kx = e == 0 ? a.kx_max : a.kx_min;
        const double* ky = e == 0 ? a.ky_max : a.ky_min;
        double* c = e == 0 ? a.c_max : a.c_min;
        const int row0 = b * kChunksPerBlock * kChunk;
        stage_window(sg, a, off, r, row0, K, kx, ky);
        const int q = b * kChunksPerBlock + threadIdx.x;
        const double* X = a.xsep + (size_t)re * (size_t)a.rec_stride;
        if (q <= P) {
            const int first = q * kChunk;
            const int len = (q < P) ? kChunk - 1 : K - first;
            StagedRowFn fn{&sg, first, row0, K};
            const double xl = (q > 0) ? X[q - 1] : 0.0;
            const double xr = (q < P) ? X[q] : 0.0;
            double* dst = &sc[pad17(threadIdx.x * kChunk)];
            chunk_interior(len, fn, xl, xr, dst, 1);
            if (q < P) dst[kChunk - 1] = xr;
        }
        __syncthreads();
        // copy the block's rows [row0, i1) out to the per-tile layout, tile range by range
        const int i1 = min(row0 + kChunksPerBlock * kChunk, K);
        for (int T = sg.t0; T < a.ntiles; ++T) {
            const int oT = off[T];
            if (oT >= i1) break;
            const int lo = max(row0, oT), hi = min(i1, off[T + 1]);
            const size_t tb = tile_base(a, r, T);
            for (int i = lo + threadIdx.x; i < hi; i += kThreads)
                c[tb + (i - oT)] = sc[pad17(i - row0)];
        }
    }
}

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
// `plane` doubles: l, m, u, r), solution to x.  ws: workspace for the deeper levels
// (<= 0.75*n + 16 doubles).  All threads of the CTA must call it.
__device__ void cta_partitioned(int n, const double* sys, int plane, double* x, double* ws) {
    int sizes[8];
    int depth = 0;
    sizes[0] = n;
    while (sizes[depth] > kChunk && depth < 7) {
        sizes[depth + 1] = (sizes[depth] - 1) / kChunk;
        ++depth;
    }
    const double* lv[8];
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
    double* ends = ws + off;  // 6 * (chunks of the widest level)
    for (int k = 0; k < depth; ++k) {
        const int nk = sizes[k];
        const int P = sizes[k + 1];
        const int pl = (k == 0) ? plane : nk;
        const double* L = lv[k];
        for (int q = threadIdx.x; q <= P; q += blockDim.x) {
            const int first = q * kChunk;
            const int len = (q < P) ? kChunk - 1 : nk - first;
            GlobalRowFn fn{L, L + pl, L + 2 * pl, L + 3 * pl, first};
            const ChunkEnds ce = chunk_ends(len, fn);
            ends[6 * q + 0] = ce.ga;
            ends[6 * q + 1] = ce.aa;
            ends[6 * q + 2] = ce.ba;
            ends[6 * q + 3] = ce.gb;
            ends[6 * q + 4] = ce.ab;
            ends[6 * q + 5] = ce.bb;
        }
        __syncthreads();
        double* R = const_cast<double*>(lv[k + 1]);
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
    if (threadIdx.x == 0) {
        const int nb = sizes[depth];
        const int pl = (depth == 0) ? plane : nb;
        const double* L = lv[depth];
        GlobalRowFn fn{L, L + pl, L + 2 * pl, L + 3 * pl, 0};
        thomas_small(nb, fn, xv[depth], 1);
    }
    __syncthreads();
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
            chunk_interior(len, fn, xl, xr, xo + first, 1);
            if (q < P) xo[first + kChunk - 1] = xr;
        }
        __syncthreads();
    }
}

}  // namespace

namespace {

constexpr int kRedPass = kThreads * kChunk;                   // level-2 rows per pass
constexpr int kRedSlots = kRedPass + (kRedPass >> 4) + 1;    // padded

// Level-2 rows staged in shared memory (4 padded planes).
struct RedStage {
    double l[kRedSlots], m[kRedSlots], u[kRedSlots], r[kRedSlots];
};

struct StageRowFn {
    const RedStage* st;
    int first;  // local row of chunk row 0
    __device__ __forceinline__ Row operator()(int k) const {
        const int j = pad17(first + k);
        Row w;
        w.l = st->l[j];
        w.m = st->m[j];
        w.u = st->u[j];
        w.r = st->r[j];
        return w;
    }
};

// Level-2 row p (separator p of the level-1 partition) from the chunk records.
__device__ __forceinline__ Row level2_row(const SiftArgs& a, size_t o, int p) {
    const double* rc = a.rec;
    const size_t pl = a.rec_plane;
    Row sr;
    sr.l = rc[6 * pl + o + p];
    sr.m = rc[7 * pl + o + p];
    sr.u = rc[8 * pl + o + p];
    sr.r = rc[9 * pl + o + p];
    return reduced_row(sr, rc[3 * pl + o + p], rc[4 * pl + o + p], rc[5 * pl + o + p],
                       rc[0 * pl + o + p + 1], rc[1 * pl + o + p + 1], rc[2 * pl + o + p + 1]);
}

__device__ __forceinline__ void stage_level2(RedStage& st, const SiftArgs& a, size_t o, int p0,
                                             int P) {
    const int rows = min(kRedPass, P - p0);
    constexpr int kB = 4;  // rows per thread whose record loads are in flight together
    for (int j0 = threadIdx.x; j0 < rows; j0 += kB * kThreads) {
        Row w[kB];
#pragma unroll
        for (int t = 0; t < kB; ++t) {
            const int j = j0 + t * kThreads;
            if (j < rows) w[t] = level2_row(a, o, p0 + j);
        }
#pragma unroll
        for (int t = 0; t < kB; ++t) {
            const int j = j0 + t * kThreads;
            if (j < rows) {
                const int q = pad17(j);
                st.l[q] = w[t].l;
                st.m[q] = w[t].m;
                st.u[q] = w[t].u;
                st.r[q] = w[t].r;
            }
        }
    }
}

}  // namespace

size_t reduced_solve_smem(int rec_stride, bool* level3_in_smem) {
    const int pmax = rec_stride;
    const int qmax = pmax > kChunk ? (pmax - 1) / kChunk + 1 : 1;
    const size_t l3 = sizeof(double) * ((size_t)10 * (qmax + 1) + 5 * (size_t)qmax + qmax + 64);
    const size_t base = sizeof(RedStage);
    *level3_in_smem = base + l3 <= (size_t)220 * 1024;
    return *level3_in_smem ? base + l3 : base;
}

// k_reduced_solve: levels >= 2 of the partitioned solve, one CTA per spline system.
// Small systems (K <= kChunk) are solved here directly from the knots.
__global__ void __launch_bounds__(kThreads)
k_reduced_solve(SiftArgs a) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    RedStage& st = *reinterpret_cast<RedStage*>(dyn_smem);
    if (*a.done) return;
    const int re = blockIdx.x;
    if (re >= 2 * a.nr) return;
    const int e = re / a.nr, r = re % a.nr;
    const int K = a.kcount[re];
    if (K <= kChunk) {
        if (threadIdx.x == 0) {
            const int* off = a.tile_off + (size_t)re * (a.ntiles + 1);
            const int32_t* gx = e == 0 ? a.kx_max : a.kx_min;
            const double* gy = e == 0 ? a.ky_max : a.ky_min;
            double* gc = e == 0 ? a.c_max : a.c_min;
            int32_t kx[kChunk];
            double ky[kChunk], c[kChunk];
            size_t ad[kChunk];
            for (int i = 0, t = 0; i < K; ++i) {
                while (off[t + 1] <= i) ++t;
                ad[i] = tile_base(a, r, t) + (size_t)(i - off[t]);
                kx[i] = gx[ad[i]];
                ky[i] = gy[ad[i]];
            }
            KnotRowFn fn{kx, ky, K};
            thomas_small(K, fn, c, 1);
            for (int i = 0; i < K; ++i) gc[ad[i]] = c[i];
        }
        return;
    }
    const int P = (K - 1) / kChunk;  // level-2 size
    const size_t o = (size_t)re * (size_t)a.rec_stride;
    double* X = a.xsep + o;
    if (P <= kChunk) {
        stage_level2(st, a, o, 0, P);
        __syncthreads();
        if (threadIdx.x == 0) thomas_small(P, StageRowFn{&st, 0}, X, 1);
        return;
    }
    const int Q = (P - 1) / kChunk;  // level-3 size
    // level-3 workspace: shared memory after the stage, or the global reduced workspace
    double* w3 = a.red_in_smem ? reinterpret_cast<double*>(dyn_smem + sizeof(RedStage))
                               : a.red + (size_t)re * a.red_stride;
    double* ends = w3;                       // 6 * (Q+1)
    double* sep = ends + 6 * (size_t)(Q + 1);  // 4 * (Q+1)
    double* L3 = sep + 4 * (size_t)(Q + 1);    // 4 * Q
    double* x3 = L3 + 4 * (size_t)Q;           // Q
    double* ws3 = x3 + Q;                     // deeper levels
    for (int p0 = 0; p0 < P; p0 += kRedPass) {
        __syncthreads();
        stage_level2(st, a, o, p0, P);
        __syncthreads();
        const int q = p0 / kChunk + threadIdx.x;
        if (q <= Q) {
            const int first = q * kChunk;
            const int len = (q < Q) ? kChunk - 1 : P - first;
            const StageRowFn fn{&st, first - p0};
            const ChunkEnds ce = chunk_ends(len, fn);
            ends[6 * q + 0] = ce.ga;
            ends[6 * q + 1] = ce.aa;
            ends[6 * q + 2] = ce.ba;
            ends[6 * q + 3] = ce.gb;
            ends[6 * q + 4] = ce.ab;
            ends[6 * q + 5] = ce.bb;
            if (q < Q) {
                const Row s2 = fn(kChunk - 1);
                sep[4 * q + 0] = s2.l;
                sep[4 * q + 1] = s2.m;
                sep[4 * q + 2] = s2.u;
                sep[4 * q + 3] = s2.r;
            }
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < Q; p += kThreads) {
        Row s2;
        s2.l = sep[4 * p + 0];
        s2.m = sep[4 * p + 1];
        s2.u = sep[4 * p + 2];
        s2.r = sep[4 * p + 3];
        const Row w = reduced_row(s2, ends[6 * p + 3], ends[6 * p + 4], ends[6 * p + 5],
                                  ends[6 * (p + 1) + 0], ends[6 * (p + 1) + 1],
                                  ends[6 * (p + 1) + 2]);
        L3[p] = w.l;
        L3[Q + p] = w.m;
        L3[2 * Q + p] = w.u;
        L3[3 * Q + p] = w.r;
    }
    __syncthreads();
    cta_partitioned(Q, L3, Q, x3, ws3);
    for (int p0 = 0; p0 < P; p0 += kRedPass) {
        __syncthreads();
        stage_level2(st, a, o, p0, P);
        __syncthreads();
        const int q = p0 / kChunk + threadIdx.x;
        if (q <= Q) {
            const int first = q * kChunk;
            const int len = (q < Q) ? kChunk - 1 : P - first;
            const double xl = (q > 0) ? x3[q - 1] : 0.0;
            const double xr = (q < Q) ? x3[q] : 0.0;
            chunk_interior(len, StageRowFn{&st, first - p0}, xl, xr, X + first, 1);
            if (q < Q) X[first + kChunk - 1] = xr;
        }
    }
}

// =======================================================================================
// k_eval: envelopes + mean envelope + sx statistics over one tile of samples.  Thread t
// handles local samples k*256 + t (k = 0..7), so every warp access to samples, bitmap words
// and the mean envelope is contiguous.  The spline segment of sample s is
// (#knots at positions < s) - 1, a popc rank in the tile's knot bitmap.
// =======================================================================================
__global__ void __launch_bounds__(kThreads, 4)
k_eval(SiftArgs a) {
    constexpr int kMaxKnots = kTileSamples / 2 + 4;
    __shared__ int32_t sx_[kMaxKnots];
    __shared__ double sy[kMaxKnots], scf[kMaxKnots], sb[kMaxKnots], sd[kMaxKnots];
    __shared__ unsigned sbm[kWords];
    __shared__ int swp[kWords];
    __shared__ int s_red[kThreads / 32];
    __shared__ int s_any[kThreads / 32];

    if (*a.done) return;
    const int tile = blockIdx.x;
    const int r = blockIdx.y;
    const int n = a.n;
    const int n0 = tile * kTileSamples;
    const size_t base = (size_t)r * (size_t)n;
    const size_t to = (size_t)(a.ntiles + 1);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    double up[kPerThread];                    // upper envelope, then the mean envelope
    int cnt = 0, any = 0;

#pragma unroll 1
    for (int e = 0; e < 2; ++e) {
        const int se = e * a.nr + r;
        const int K = a.kcount[se];
        const int* off = a.tile_off + (size_t)se * to;
        const int off0 = off[tile];
        const int off1 = off[tile + 1];
        const long long* nb = a.nbr + ((size_t)se * a.ntiles + tile) * 2;
        const int klo = off0 > 0 ? off0 - 1 : 0;
        const int khi = min(off1, K - 1);
        const int nk = khi - klo + 1;
        const int32_t* kx = e == 0 ? a.kx_max : a.kx_min;
        const double* ky = e == 0 ? a.ky_max : a.ky_min;
        const double* kc = e == 0 ? a.c_max : a.c_min;
        __syncthreads();
        {
            // own knots [off0, off1) sit contiguously in this tile's slots; the knots just
            // before and after come from the precomputed neighbour addresses
            const size_t tb = tile_base(a, r, tile);
            for (int i = off0 + threadIdx.x; i < off1; i += kThreads) {
                const int j = i - klo;
                cp_async4(&sx_[j], kx + tb + (i - off0));
                cp_async8(&sy[j], ky + tb + (i - off0));
                cp_async8(&scf[j], kc + tb + (i - off0));
            }
            if (threadIdx.x == 32 && off0 > 0) {
                const size_t p = (size_t)nb[0];
                cp_async4(&sx_[0], kx + p);
                cp_async8(&sy[0], ky + p);
                cp_async8(&scf[0], kc + p);
            }
            if (threadIdx.x == 64 && off1 <= khi) {
                const size_t p = (size_t)nb[1];
                cp_async4(&sx_[off1 - klo], kx + p);
                cp_async8(&sy[off1 - klo], ky + p);
                cp_async8(&scf[off1 - klo], kc + p);
            }
            if (threadIdx.x < kWords)
                cp_async4(&sbm[threadIdx.x],
                          a.bitmap + (size_t)e * a.nr * a.ntiles * kWords +
                              ((size_t)r * a.ntiles + tile) * kWords + threadIdx.x);
        }
        cp_async_wait_all();
        __syncthreads();
        for (int j = threadIdx.x; j < nk - 1; j += kThreads)
            seg_coeffs_t(a, sx_[j], sx_[j + 1], sy[j], sy[j + 1], scf[j], scf[j + 1], sb[j], sd[j]);
        if (warp == 0) {  // exclusive scan of the 64 bitmap word counts
            const int c0 = __popc(sbm[2 * lane]), c1 = __popc(sbm[2 * lane + 1]);
            int incl = c0 + c1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            swp[2 * lane] = incl - (c0 + c1);
            swp[2 * lane + 1] = incl - c1;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const int s = n0 + k * kThreads + threadIdx.x;
            const int w = k * (kThreads / 32) + warp;  // bitmap word of sample s (warp-uniform)
            const int seg = max(off0 + swp[w] + __popc(sbm[w] & lt) - 1, 0);
            const int j = seg - klo;
            const double v =
                seg_eval(sy[j], sb[j], scf[j], sd[j], (double)(s - sx_[j]));
            if (e == 0) {
                up[k] = v;
            } else {
                const double u = up[k];
                if (a.dbg_upper && s < n) {
                    a.dbg_upper[base + s] = u;
                    a.dbg_lower[base + s] = v;
                }
                const double p = fabs(u + v), q = fabs(u - v);
                const bool live = s < n;
                any |= (live && sx_greater_pq(p, q, u, v, a.sd2)) ? 1 : 0;
                cnt += (live && sx_greater_pq(p, q, u, v, a.sd)) ? 1 : 0;
                up[k] = (u + v) / 2.0;
            }
        }
    }

    if (a.kcount[r] > 3 && a.kcount[a.nr + r] > 3) {
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const int s = n0 + k * kThreads + threadIdx.x;
            if (s < n) a.menv[base + s] = up[k];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        any |= __shfl_xor_sync(0xffffffffu, any, o);
    }
    if (lane == 0) {
        s_red[warp] = cnt;
        s_any[warp] = any;
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
    __shared__ unsigned long long s_knots[kThreads / 32];
    if (*a.done) return;
    const int j = *a.iter;
    int all = 1;
    unsigned long long knots = 0;
    for (int r = threadIdx.x; r < a.nr; r += blockDim.x) {
        const unsigned c = a.cnt[r];
        const int any = a.any[r];
        a.cnt[r] = 0u;
        a.any[r] = 0;
        const int kmax = a.kcount[r], kmin = a.kcount[a.nr + r];
        knots += (unsigned long long)(kmax + kmin);
        const double fr = (a.frac[r] + (double)c) * a.inv_n;
        a.frac[r] = fr;
        const bool crit = fr > a.tol || (any != 0 && (kmax + kmin) > 6);
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
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) knots += __shfl_xor_sync(0xffffffffu, knots, o);
    if ((threadIdx.x & 31) == 0) {
        s_all[threadIdx.x >> 5] = all;
        s_knots[threadIdx.x >> 5] = knots;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int d = 1;
        unsigned long long kt = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
            d &= s_all[w];
            kt += s_knots[w];
        }
        *a.iter = j + 1;
        a.acc[0] += kt;
        a.acc[1] += 1ull;
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
