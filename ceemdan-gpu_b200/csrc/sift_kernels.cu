// Sifting kernels of the ICEEMDAN engine (sm_100a, FP64).
//
// One sift iteration over all realizations of a stage is:
//   k_extrema        deferred update h -= m (or mode export) + strict-extrema flags +
//                    warp-ballot compaction into per-tile knot storage, knot bitmaps
//                    (find_extrema_shfl_* :93-148, select_extrema_* :151-207,
//                     updateRealizations :528-544 of the previous iteration)
//   k_scan_boundary  per-spline scan of the tile knot counts (CUB scan :1582-1604), separator
//                    offsets, neighbour-knot addresses and the end-knot extrapolation
//                    (setBoundaryMax/Min :210-291)
//   k_group_scan     prefix over the splines of their 32-separator warp groups
//   k_chunk_reduce   end relations of the tile-aligned chunks of the canonical partitioned
//                    spline solve and the separator rows (tridiagonal_setup :311-343)
//   k_reduced_solve  per-spline separator solve (levels >= 2), one CTA per spline
//                    (with the chunk kernels: cusparseDgtsv2_nopivot :1622-1641)
//   k_segments       chunk interiors -> spline values -> segment coefficients, one record per
//                    segment (spline_coefficients :383-401)
//   k_eval           envelopes, mean envelope, sx statistics
//                    (interpolate :404-439, averageUppperLower :442-454, produceSX :457-467,
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

__device__ __forceinline__ int pad17(int j) { return j + (j >> 4); }


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
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }

// ---------------------------------------------------------------------------------------
// Geometry of the ragged multi-channel layout (kernels.h: Chan, SiftArgs).
// ---------------------------------------------------------------------------------------
struct Geo {
    int c, r, g;       // channel, realization within the channel, global row
    int n, ntiles;     // samples and tiles of the row
    int tile0;         // first global tile of the row
    size_t base;       // first sample of the row
};

__device__ __forceinline__ Geo geo(const SiftArgs& a, int c, int r) {
    Geo q;
    if (a.nchan == 1) {  // channel 0's geometry from the launch parameters
        q.c = 0;
        q.r = r;
        q.g = r;
        q.n = a.n1;
        q.ntiles = a.ntiles1;
        q.tile0 = r * a.ntiles1;
        q.base = (size_t)r * (size_t)a.n1;
        return q;
    }
    const Chan* ch = a.chan + c;
    q.c = c;
    q.r = r;
    q.n = __ldg(&ch->n);
    q.ntiles = __ldg(&ch->ntiles);
    q.g = __ldg(&ch->row0) + r;
    q.tile0 = __ldg(&ch->tile0) + r * q.ntiles;
    q.base = (size_t)__ldg(&ch->samp0) + (size_t)r * (size_t)q.n;
    return q;
}

// last channel c with pre[c] <= v (pre: nondecreasing exclusive prefix, pre[0] = 0): the
// channel whose range [pre[c], pre[c+1]) holds v
__device__ __forceinline__ int plan_find(const int* pre, int nchan, int v) {
    int lo = 0, hi = nchan - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(pre + mid) <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Rows and tiles of the channels that sift in this iteration.
__device__ __forceinline__ int active_rows(const SiftArgs& a) {
    if (a.nchan == 1) return a.cs[0].done ? 0 : a.nr1;
    return __ldg(a.plan + a.nchan);
}
__device__ __forceinline__ int active_tiles(const SiftArgs& a) {
    if (a.nchan == 1) return a.cs[0].done ? 0 : a.nr1 * a.ntiles1;
    return __ldg(a.plan + 2 * a.nchan + 1);
}

// Active row v -> its geometry.
__device__ __forceinline__ Geo row_geo(const SiftArgs& a, int v) {
    if (a.nchan == 1) return geo(a, 0, v);
    const int c = plan_find(a.plan, a.nchan, v);
    return geo(a, c, v - __ldg(a.plan + c));
}

// Active tile v -> the geometry of its row and its tile index t within the row.
__device__ __forceinline__ Geo tile_geo(const SiftArgs& a, int v, int& t) {
    int c = 0, local = v;
    if (a.nchan > 1) {
        const int* pt = a.plan + a.nchan + 1;
        c = plan_find(pt, a.nchan, v);
        local = v - __ldg(pt + c);
    }
    const int nt = a.nchan == 1 ? a.ntiles1 : __ldg(&a.chan[c].ntiles);
    const int r = local / nt;
    t = local - r * nt;
    return geo(a, c, r);
}

// Active spline v (the maxima splines of the ra active rows, then their minima splines).
__device__ __forceinline__ Geo spline_geo(const SiftArgs& a, int v, int ra, int& e) {
    e = v >= ra ? 1 : 0;
    return row_geo(a, v - e * ra);
}

// Index of tile t of row q's spline e in the per-tile arrays (tile_cnt, bitmap words / 64,
// nbr pairs / 2) and in the per-tile-plus-one arrays (tile_off, sep_off).
__device__ __forceinline__ size_t tix(const SiftArgs& a, int e, const Geo& q, int t) {
    return (size_t)e * a.ntot + (size_t)(q.tile0 + t);
}
__device__ __forceinline__ size_t oix(const SiftArgs& a, int e, const Geo& q) {
    return (size_t)e * (size_t)(a.ntot + a.nrows) + (size_t)(q.tile0 + q.g);
}
__device__ __forceinline__ int spline_id(const SiftArgs& a, int e, const Geo& q) {
    return e * a.nrows + q.g;
}
// first knot slot of global tile gt in the tile-local knot arrays
__device__ __forceinline__ size_t tile_base(int gt) { return (size_t)gt * kTileCap; }
// record / separator-value offset and reduced-workspace offset of row q's spline e
__device__ __forceinline__ size_t rec_base(const SiftArgs& a, int e, const Geo& q) {
    if (a.nchan == 1) return (size_t)e * (size_t)a.rec_total + (size_t)q.r * (size_t)a.rs1;
    const Chan* ch = a.chan + q.c;
    return (size_t)e * (size_t)a.rec_total + (size_t)__ldg(&ch->rec0) +
           (size_t)q.r * (size_t)__ldg(&ch->rec_stride);
}
__device__ __forceinline__ size_t red_base(const SiftArgs& a, int e, const Geo& q) {
    if (a.nchan == 1)
        return (size_t)e * (size_t)a.red_total + (size_t)q.r * (size_t)red_stride_of(a.rs1);
    const Chan* ch = a.chan + q.c;
    return (size_t)e * (size_t)a.red_total + (size_t)__ldg(&ch->red0) +
           (size_t)q.r * (size_t)red_stride_of(__ldg(&ch->rec_stride));
}

// Global address of knot i of a spline whose tile offsets are off[0..ntiles] and whose first
// tile is tile0: the tile is found by walking from tile `t` (a tile at or before the one
// holding knot i when walking forward, at or after it when backward) -- one or two steps for
// the end knots and the neighbours of a tile.
__device__ __forceinline__ size_t knot_addr_fwd(const int* off, int tile0, int t, int i) {
    while (off[t + 1] <= i) ++t;
    return tile_base(tile0 + t) + (size_t)(i - off[t]);
}
__device__ __forceinline__ size_t knot_addr_bwd(const int* off, int tile0, int t, int i) {
    while (off[t] > i) --t;
    return tile_base(tile0 + t) + (size_t)(i - off[t]);
}

// ---------------------------------------------------------------------------------------
// Exact divisions of the spline arithmetic, warp-wide.  Each lane forms div_rcp's quotient from
// a tabled reciprocal (Markstein's correction, correctly rounded in its range); lanes outside
// that range (tiny or huge operands, spacings beyond the table) take the division, under a
// vote of the whole warp so that the division is skipped when no lane needs it -- as a plain
// branch the compiler evaluates it unconditionally.  Every lane of the warp must call these
// together (warp-uniform control flow); `active` = false lanes compute nothing meaningful.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double rcp_fast(double a, double d, double y, bool& slow) {
    const double q0 = a * y;
    const double r = fma(-q0, d, a);
    const double q1 = fma(r, y, q0);
    slow = !(fabs(a) > 0x1p-960) || !(fabs(q1) < 0x1p+1000);
    return q1;
}

// Fast parts alone, for loops that collect the lanes needing the division over all their
// iterations and take it once after the loop (one vote instead of one per iteration).  The
// results equal the divisions' whenever `slow` comes back false.
__device__ __forceinline__ double slope_fast(const SiftArgs& a, int32_t x0, int32_t x1, double y0,
                                             double y1, bool& slow) {
    const int h = x1 - x0;
    const bool tab = h >= 1 && h <= kRcpMax;
    const double q = rcp_fast(y1 - y0, (double)h, __ldg(a.rcp_h + (tab ? h : 1)), slow);
    slow = slow || !tab;
    return q;
}

__device__ __forceinline__ void seg_coeffs_fast(const SiftArgs& a, int32_t x0, int32_t x1,
                                                double slope, double c0, double c1, double& b,
                                                double& d, bool& slow) {
    const int hi = x1 - x0;
    const bool tab = hi >= 1 && hi <= kRcpMax;
    const double h = (double)hi;
    bool slow_b, slow_d;
    const double qb = rcp_fast(h * fma(2.0, c0, c1), 3.0, kRcp3, slow_b);
    d = rcp_fast(c1 - c0, 3.0 * h, __ldg(a.rcp_3h + (tab ? hi : 1)), slow_d);
    b = slope - qb;
    slow = slow_b || slow_d || !tab;
}

// The same coefficients by the divisions themselves (the fallback of seg_coeffs_fast).
__device__ __forceinline__ void seg_coeffs_div(int32_t x0, int32_t x1, double slope, double c0,
                                               double c1, double& b, double& d) {
    const double h = (double)(x1 - x0);
    b = slope - (h * fma(2.0, c0, c1)) / 3.0;
    d = (c1 - c0) / (3.0 * h);
}

// (y1 - y0) / (x1 - x0), the same quotient as seg_slope.
__device__ __forceinline__ double slope_warp(const SiftArgs& a, int32_t x0, int32_t x1, double y0,
                                             double y1, bool active) {
    const int h = x1 - x0;
    const bool tab = h >= 1 && h <= kRcpMax;
    const double dy = y1 - y0;
    bool slow;
    double q = rcp_fast(dy, (double)h, __ldg(a.rcp_h + (tab ? h : 1)), slow);
    slow = active && (slow || !tab);
    if (__any_sync(0xffffffffu, slow)) {
        if (slow) q = dy / (double)h;
    }
    return q;
}

// Segment coefficients b and d (seg_coeffs) from the segment's slope and spline values.
__device__ __forceinline__ void seg_coeffs_warp(const SiftArgs& a, int32_t x0, int32_t x1,
                                                double slope, double c0, double c1, double& b,
                                                double& d, bool active) {
    const int hi = x1 - x0;
    const bool tab = hi >= 1 && hi <= kRcpMax;
    const double h = (double)hi;
    const double hq = h * fma(2.0, c0, c1);
    const double dc = c1 - c0;
    bool slow_b, slow_d;
    double qb = rcp_fast(hq, 3.0, kRcp3, slow_b);
    d = rcp_fast(dc, 3.0 * h, __ldg(a.rcp_3h + (tab ? hi : 1)), slow_d);
    slow_b = active && slow_b;
    slow_d = active && (slow_d || !tab);
    if (__any_sync(0xffffffffu, slow_b || slow_d)) {
        if (slow_b) qb = hq / 3.0;
        if (slow_d) d = dc / (3.0 * h);
    }
    b = slope - qb;
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
template <bool kCoupled = true, class RowFn, class Out>
__device__ __forceinline__ void chunk_interior(int len, const RowFn& row, double xl, double xr,
                                               Out out, int stride) {
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

}  // namespace

// =======================================================================================
// k_extrema
// =======================================================================================
template <int kMinBlocks, bool kLoop>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_extrema_t(SiftArgs a) {
    __shared__ __align__(16) double sh[kTileSamples + 4];  // sh[2 + j] = sample n0 + j
    __shared__ __align__(16) double sm[kTileSamples];      // mean envelope of the tile
    __shared__ int s_cnt[2][kWords];
    __shared__ int s_off[2][kWords];
    __shared__ __align__(16) double s_halo[4];  // h at n0-1 and n0+2048, then the mean there

    const int total = active_tiles(a);
    // kLoop: persistent CTAs, active tiles v, v + gridDim.x, ... (CTA-uniform loop); else the
    // grid covers every tile, one per CTA
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
    int tile;
    const Geo q = tile_geo(a, v, tile);
    const int n = q.n;
    const int n0 = tile * kTileSamples;
    const size_t base = q.base;
    const ChanState& cst = a.cs[q.c];
    const int it = a.par >= 0 ? a.par : cst.iter;
    const int mk = a.mark[q.g];
    const double* __restrict__ hin = a.h[it & 1] + base;
    double* __restrict__ hout = a.h[(it + 1) & 1] + base;
    const double* __restrict__ me = a.menv + base;
    double* __restrict__ mo = mk == 0 ? cst.mode_out + (size_t)q.r * n : nullptr;

    // Deferred update of the previous iteration (h -= m, or mode export).  The tile of h (and
    // of the mean envelope when it is subtracted) is copied to shared memory with cp.async,
    // all copies in flight at once; registers hold nothing while they land.  Even n: the tile
    // moves as 16-byte pieces (sample pairs), piece k*256 + t by thread t, so every warp
    // instruction covers 512 contiguous bytes (n even keeps every piece 16-byte aligned and
    // inside the row; every row starts at an even sample of the channel's block, and blocks
    // start 256-byte aligned).
    const bool even = (n & 1) == 0;
    if (even) {
#pragma unroll
        for (int k = 0; k < kPerThread / 2; ++k) {
            const int j = 2 * (k * kThreads + threadIdx.x);
            const int s = n0 + j;
            if (s < n) {
                cp_async16(&sh[2 + j], hin + s);
                if (mk == 1) cp_async16(&sm[j], me + s);
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const int j = k * kThreads + threadIdx.x;
            const int s = n0 + j;
            if (s < n) {
                cp_async8(&sh[2 + j], hin + s);
                if (mk == 1) cp_async8(&sm[j], me + s);
            }
        }
    }
    if (threadIdx.x < 2) {  // halo samples n0-1 and n0+kTileSamples, with the tile's copies
        const int s = threadIdx.x == 0 ? n0 - 1 : n0 + kTileSamples;
        if (s >= 0 && s < n) {
            cp_async8(&s_halo[threadIdx.x], hin + s);
            if (mk == 1) cp_async8(&s_halo[2 + threadIdx.x], me + s);
        }
    }
    cp_async_wait_all();
    // each thread updates the samples it copied (no other thread reads them before the barrier)
    if (even) {
#pragma unroll
        for (int k = 0; k < kPerThread / 2; ++k) {
            const int j = 2 * (k * kThreads + threadIdx.x);
            const int s = n0 + j;
            double2 val = make_double2(0.0, 0.0);
            if (s < n) {
                const double2 hv = *reinterpret_cast<const double2*>(&sh[2 + j]);
                val = hv;
                if (mk == 1) {
                    const double2 mv = *reinterpret_cast<const double2*>(&sm[j]);
                    val.x = hv.x - mv.x;
                    val.y = hv.y - mv.y;
                }
                *reinterpret_cast<double2*>(hout + s) = val;
                if (mk == 0) *reinterpret_cast<double2*>(mo + s) = hv;
            }
            *reinterpret_cast<double2*>(&sh[2 + j]) = val;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const int j = k * kThreads + threadIdx.x;
            const int s = n0 + j;
            double val = 0.0;
            if (s < n) {
                const double hv = sh[2 + j];
                val = (mk == 1) ? hv - sm[j] : hv;
                hout[s] = val;
                if (mk == 0) mo[s] = hv;
            }
            sh[2 + j] = val;
        }
    }
    if (threadIdx.x < 2) {  // the halo this thread copied
        const int s = threadIdx.x == 0 ? n0 - 1 : n0 + kTileSamples;
        double val = 0.0;
        if (s >= 0 && s < n) {
            const double hv = s_halo[threadIdx.x];
            val = (mk == 1) ? hv - s_halo[2 + threadIdx.x] : hv;
        }
        sh[threadIdx.x == 0 ? 1 : 2 + kTileSamples] = val;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const size_t bw0 = tix(a, 0, q, tile) * kWords;
    const size_t bw1 = tix(a, 1, q, tile) * kWords;
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
                const double x = sh[2 + j], xl = sh[1 + j], xr = sh[3 + j];
                fmax = x > xl && x > xr;
                fmin = x < xl && x < xr;
            }
        }
        bmax[k] = __ballot_sync(0xffffffffu, fmax);
        bmin[k] = __ballot_sync(0xffffffffu, fmin);
        if (lane == 0) {
            const int w = k * (kThreads / 32) + warp;
            s_cnt[0][w] = __popc(bmax[k]);
            s_cnt[1][w] = __popc(bmin[k]);
            a.bitmap[bw0 + w] = bmax[k];
            a.bitmap[bw1 + w] = bmin[k];
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
        if (lane == 31) a.tile_cnt[tix(a, e, q, tile)] = incl;
    }
    __syncthreads();

    const unsigned lt = (1u << lane) - 1u;
    const size_t kb = tile_base(q.tile0 + tile);
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
    if (!kLoop) break;
    __syncthreads();  // shared memory is reused by the CTA's next tile
    }
}

// The register budgets the autotuner chooses between (resident CTAs per SM), persistent or one
// tile per CTA; same results.
template __global__ void k_extrema_t<kExtremaBlocksA, true>(SiftArgs a);
template __global__ void k_extrema_t<kExtremaBlocksB, true>(SiftArgs a);
template __global__ void k_extrema_t<kExtremaBlocksA, false>(SiftArgs a);
template __global__ void k_extrema_t<kExtremaBlocksB, false>(SiftArgs a);

// =======================================================================================
// k_scan_boundary: one warp per spline (envelope, realization): exclusive scan of the tile
// knot counts into the offset row, the knot count, and the end-knot extrapolation.
// =======================================================================================
__global__ void __launch_bounds__(kThreads)
k_scan_boundary(SiftArgs a) {
    const int lane = threadIdx.x & 31;
    const int ra = active_rows(a);
    const int wpb = kThreads / 32;
    // one warp per active spline (warp-uniform loop)
    for (int v = blockIdx.x * wpb + (threadIdx.x >> 5); v < 2 * ra; v += gridDim.x * wpb) {
    int e;
    const Geo q = spline_geo(a, v, ra, e);
    const int id = spline_id(a, e, q);
    const int ntiles = q.ntiles;
    const int* cnt = a.tile_cnt + tix(a, e, q, 0);
    int* off = a.tile_off + oix(a, e, q);
    int carry = 0;
    for (int t0 = 0; t0 < ntiles; t0 += 32) {
        const int t = t0 + lane;
        const int c = t < ntiles ? cnt[t] : 0;
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (t < ntiles) off[t] = carry + incl - c;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    const int K = carry;
    if (lane == 0) {
        off[ntiles] = K;
        a.kcount[id] = K;
    }
    // separators per tile (local 0, 16, 32, ... and the last knot), exclusive scan
    int* soff = a.sep_off + oix(a, e, q);
    int scarry = 0;
    for (int t0 = 0; t0 < ntiles; t0 += 32) {
        const int t = t0 + lane;
        const int c = t < ntiles ? cnt[t] : 0;
        const int ns = c > 0 ? (c + kChunk - 2) / kChunk + 1 : 0;
        int incl = ns;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (t < ntiles) soff[t] = scarry + incl - ns;
        scarry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
        soff[ntiles] = scarry;
        a.pcount[id] = scarry;
        a.gcount[v] = (scarry + 31) >> 5;  // warp groups of k_chunk_reduce / k_segments
    }
    // address of the knot just before each tile (last knot of the nearest non-empty tile
    // before it) and just after it (first knot of the nearest non-empty tile after it)
    long long* nb = a.nbr + tix(a, e, q, 0) * 2;
    int last = -1;  // nearest non-empty tile before the current chunk
    for (int t0 = 0; t0 < ntiles; t0 += 32) {
        const int t = t0 + lane;
        const int c = t < ntiles ? cnt[t] : 0;
        int w = c > 0 ? t : -1;  // inclusive max-scan of non-empty tile indices
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w = max(w, u);
        }
        int before = __shfl_up_sync(0xffffffffu, w, 1);
        if (lane == 0) before = -1;
        before = max(before, last);
        if (t < ntiles)
            nb[2 * t] = before >= 0
                            ? (long long)(tile_base(q.tile0 + before) + cnt[before] - 1)
                            : -1;
        last = max(last, __shfl_sync(0xffffffffu, w, 31));
    }
    int first = 0x7fffffff;  // nearest non-empty tile after the current chunk
    for (int t0 = ((ntiles - 1) / 32) * 32; t0 >= 0; t0 -= 32) {
        const int t = t0 + lane;
        const int c = t < ntiles ? cnt[t] : 0;
        int w = c > 0 ? t : 0x7fffffff;  // inclusive min-scan from the right
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_down_sync(0xffffffffu, w, o);
            if (lane + o < 32) w = min(w, u);
        }
        int after = __shfl_down_sync(0xffffffffu, w, 1);
        if (lane == 31) after = 0x7fffffff;
        after = min(after, first);
        if (t < ntiles)
            nb[2 * t + 1] = after < ntiles ? (long long)tile_base(q.tile0 + after) : -1;
        first = min(first, __shfl_sync(0xffffffffu, w, 0));
    }
    __syncwarp();
    if (lane == 0 && K - 1 > 4) {
        int32_t* kx = e == 0 ? a.kx_max : a.kx_min;
        double* ky = e == 0 ? a.ky_max : a.ky_min;
        const int L = K - 1;
        const int tl = ntiles - 1;
        const size_t p0 = knot_addr_fwd(off, q.tile0, 0, 0),
                     p1 = knot_addr_fwd(off, q.tile0, 0, 1),
                     p2 = knot_addr_fwd(off, q.tile0, 0, 2);
        const size_t q0 = knot_addr_bwd(off, q.tile0, tl, L - 2),
                     q1 = knot_addr_bwd(off, q.tile0, tl, L - 1),
                     q2 = knot_addr_bwd(off, q.tile0, tl, L);
        const double y0 = boundary_left(e, kx[p0], kx[p1], kx[p2], ky[p0], ky[p1], ky[p2]);
        const double yL = boundary_right(e, kx[q0], kx[q1], kx[q2], ky[q0], ky[q1], ky[q2]);
        // a replaced end value differs from the old one in its bits (t > y or t < y)
        if (a.bflags)
            a.bflags[id] = (unsigned char)(
                (__double_as_longlong(y0) != __double_as_longlong(ky[p0]) ? 1 : 0) |
                (__double_as_longlong(yL) != __double_as_longlong(ky[q2]) ? 2 : 0));
        ky[p0] = y0;
        ky[q2] = yL;
    } else if (lane == 0 && a.bflags) {
        a.bflags[id] = 0;
    }
    __syncwarp();
    }
}

// Compacted copy of the knots of envelope e (stage-level entry point, one channel): row r's
// knots to kx/ky[r*n + i].
__global__ void k_gather_knots(SiftArgs a, int e, int32_t* kx, double* ky) {
    const int tile = blockIdx.x;
    const Geo q = geo(a, 0, blockIdx.y);
    const int* off = a.tile_off + oix(a, e, q);
    const int o = off[tile], c = off[tile + 1] - o;
    const size_t src = tile_base(q.tile0 + tile);
    const int32_t* sx = e == 0 ? a.kx_max : a.kx_min;
    const double* sy = e == 0 ? a.ky_max : a.ky_min;
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
        kx[q.base + o + j] = sx[src + j];
        ky[q.base + o + j] = sy[src + j];
    }
}

// =======================================================================================
// Tile-aligned first level of the canonical spline solve.  In each tile, the knots at local
// index 0, 16, 32, ... and the tile's last knot are separators; chunk k of a tile holds the
// knots strictly between its separators k-1 and k and has global chunk index sep_off[t] + k
// (the chunk left of separator sep_off[t] + k; the chunk left of local 0 is empty).
// =======================================================================================
namespace {

__device__ __forceinline__ int sep_local(int k, int cnt) { return min(k * kChunk, cnt - 1); }

}  // namespace

// End relations of a chunk of len >= 1 rows from a slab: x[0] is the knot before row 0,
// rows 0..len-1 are knots 1..len, knot len+1 closes the last row, s[i] is the slope of
// segment i -> i+1.  The operations and their order are those of chunk_ends; the next rows
// of both sweeps are loaded ahead of the reciprocal chain.
__device__ __forceinline__ ChunkEnds chunk_ends_slab(const int32_t* x, const double* s,
                                                     int len) {
    auto row = [&](int k) { return spline_row(x[k], x[k + 1], x[k + 2], s[k], s[k + 1]); };
    const Row wa = row(0), wb = row(len - 1);
    double iw = 1.0 / wa.m;
    double cp = wa.u * iw, gp = wa.r * iw, ap = -wa.l * iw;
    double iv = 1.0 / wb.m;
    double cq = wb.l * iv, gq = wb.r * iv, bq = -wb.u * iv;
    Row wn = wa, vn = wb;
    if (len > 1) {
        wn = row(1);
        vn = row(len - 2);
    }
    for (int k = 1; k < len; ++k) {
        const Row w = wn, v = vn;
        if (k + 1 < len) {
            wn = row(k + 1);
            vn = row(len - 2 - k);
        }
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

// k_group_scan: one CTA of 1024 threads.  gsum[v] = exclusive prefix over the active splines
// (k_scan_boundary's order) of gcount[v] = ceil(pcount / 32), the warp groups of 32 separators
// that k_chunk_reduce and k_segments hand to their warps; gsum[2*ra] is the total.
__global__ void __launch_bounds__(1024)
k_group_scan(SiftArgs a) {
    __shared__ int s_warp[32];
    const int m = 2 * active_rows(a);
    const int per = (m + 1023) / 1024;
    const int i0 = threadIdx.x * per;
    int sum = 0;
    for (int i = i0; i < min(i0 + per, m); ++i) sum += a.gcount[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = s_warp[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += v;
        }
        s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    int run = (warp > 0 ? s_warp[warp - 1] : 0) + incl - sum;
    for (int i = i0; i < min(i0 + per, m); ++i) {
        a.gsum[i] = run;
        run += a.gcount[i];
    }
    if (threadIdx.x == 1023) a.gsum[m] = s_warp[31];
}

// Active spline of warp group gw: the last of the m active splines whose group prefix is <= gw
// (warp-uniform).
__device__ __forceinline__ int group_spline(const SiftArgs& a, int gw, int m) {
    int lo = 0, hi = m - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(a.gsum + mid) <= gw) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

constexpr int kSlab = kChunk + 1;  // knots of one chunk: the one before it .. its separator
constexpr int kReduceWarps = 4;
constexpr int kSegWarps = 2;

// The chunk of a lane: separator p of spline (e, r) (lanes past the spline's last separator
// take the last one).  Its tile is the last tile whose separator offset is <= p (tiles without
// knots own no separators); js is the separator's local knot, jb the knot before the chunk's
// first row (js for the empty chunk left of local knot 0), len the chunk's rows.
struct ChunkLane {
    int t, k, off0, cnt, js, jb, len;
    size_t tb;
};

__device__ __forceinline__ ChunkLane locate_chunk(const SiftArgs& a, int e, const Geo& q, int p) {
    const size_t o1 = oix(a, e, q);
    const int* soff = a.sep_off + o1;
    int lo = 0, hi = q.ntiles - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(soff + mid) <= p) lo = mid;
        else hi = mid - 1;
    }
    ChunkLane c;
    c.t = lo;
    c.k = p - __ldg(soff + lo);
    const int* off = a.tile_off + o1;
    c.off0 = __ldg(off + lo);
    c.cnt = __ldg(off + lo + 1) - c.off0;
    c.tb = tile_base(q.tile0 + lo);
    c.js = sep_local(c.k, c.cnt);
    c.jb = c.k > 0 ? sep_local(c.k - 1, c.cnt) : c.js;
    c.len = c.js - c.jb - 1;
    return c;
}

// Copy each lane's knots first .. first+c-1 into its slab (positions 0..c-1), then replace the
// knot values by the slopes of the slab's c-1 segments.  Warp-collective; sx/sy are the warp's
// slabs (lane l at l*kSlab).  The warp's knots form a few contiguous runs (one per tile
// touched), so the copies go as flattened positions f = 0..total-1, 32 consecutive ones per
// step (coalesced), all in flight together (cp.async); tab (>= 32*kSlab entries) and gs (32)
// are warp scratch mapping f to (lane, position).  The slopes are then computed by each lane
// in its own slab, with one vote for the exact-division fallback after the loop.
__device__ __forceinline__ void stage_slabs(const SiftArgs& a, const int32_t* kx, const double* ky,
                                            int c, size_t first, int32_t* sx, double* sy,
                                            int lane, unsigned short* tab, long long* gs) {
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int excl = incl - c;
    for (int i = 0; i < c; ++i) tab[excl + i] = (unsigned short)((lane << 5) | i);
    gs[lane] = (long long)first;
    __syncwarp();
    for (int f = lane; f < total; f += 32) {
        const unsigned t = tab[f];
        const int ow = (int)(t >> 5), i = (int)(t & 31u);
        const size_t src = (size_t)gs[ow] + i;
        cp_async4(&sx[ow * kSlab + i], kx + src);
        cp_async8(&sy[ow * kSlab + i], ky + src);
    }
    cp_async_wait_all();
    __syncwarp();
    int32_t* x = sx + lane * kSlab;
    double* y = sy + lane * kSlab;
    unsigned slow_i = 0u;
    for (int i = 0; i + 1 < c; ++i) {  // slope i reads knots i, i+1, then replaces knot i
        bool slow;
        const double sl = slope_fast(a, x[i], x[i + 1], y[i], y[i + 1], slow);
        if (slow) slow_i |= 1u << i;
        y[i] = sl;
    }
    if (__any_sync(0xffffffffu, slow_i != 0u)) {
        for (int i = 0; i + 1 < c; ++i)
            if (slow_i >> i & 1u)
                y[i] = (ky[first + i + 1] - ky[first + i]) / (double)(x[i + 1] - x[i]);
    }
    __syncwarp();
}

// k_chunk_reduce: one thread per separator p of a spline; each warp takes groups of 32
// separators of one spline (k_group_scan) until all are done.  The thread writes the
// separator's own row and the end relations of the chunk left of it (identity for an empty
// chunk).  Each warp first
// copies the knots of its 32 chunks -- a few contiguous runs, one per tile touched -- with
// coalesced loads into per-lane slabs of shared memory (stride 17: no bank conflicts when
// every lane reads the same slab position), replaces the knot values by the segment slopes,
// then every lane sweeps its own slab.
__global__ void __launch_bounds__(kReduceWarps * 32)
k_chunk_reduce(SiftArgs a) {
    __shared__ int32_t slab_x[kReduceWarps][32 * kSlab];
    __shared__ double slab_y[kReduceWarps][32 * kSlab];
    __shared__ unsigned short slab_tab[kReduceWarps][32 * kSlab];
    __shared__ long long slab_gs[kReduceWarps][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ra = active_rows(a);
    const int groups = a.gsum[2 * ra];
    for (int gw = blockIdx.x * kReduceWarps + warp; gw < groups;
         gw += gridDim.x * kReduceWarps) {  // warp-uniform
    const int vs = group_spline(a, gw, 2 * ra);
    int e;
    const Geo q = spline_geo(a, vs, ra, e);
    const int se = spline_id(a, e, q);
    const int P = a.pcount[se];
    const int p0 = (gw - __ldg(a.gsum + vs)) * 32;
    const int p = p0 + lane;
    const bool live = p < P;
    const ChunkLane ch = locate_chunk(a, e, q, live ? p : P - 1);
    const int K = a.kcount[se];
    const int32_t* kx = e == 0 ? a.kx_max : a.kx_min;
    const double* ky = e == 0 ? a.ky_max : a.ky_min;
    const int js = ch.js, len = ch.len;
    const size_t tb = ch.tb;
    int32_t* sx = slab_x[warp];
    double* sy = slab_y[warp];
    stage_slabs(a, kx, ky, (live && len > 0) ? len + 2 : 0, tb + ch.jb, sx, sy, lane,
                slab_tab[warp], slab_gs[warp]);

    // separator row; its neighbours may lie in other tiles.  Computed by every lane (lanes past
    // the last separator repeat the last one) so that the slopes' votes see the whole warp.
    const bool ident = ch.off0 + js == 0 || ch.off0 + js == K - 1;
    const long long* nb = a.nbr + tix(a, e, q, ch.t) * 2;
    size_t im = js > 0 ? tb + js - 1 : (size_t)nb[0];
    size_t ip = js < ch.cnt - 1 ? tb + js + 1 : (size_t)nb[1];
    if (ident) im = ip = tb + js;  // end knots: identity row, no neighbours needed
    const int32_t xm = kx[im], xs = kx[tb + js], xp = kx[ip];
    const double ym = ky[im], ys = ky[tb + js], yp = ky[ip];
    const double sm = slope_warp(a, xm, xs, ym, ys, !ident);
    const double sp = slope_warp(a, xs, xp, ys, yp, !ident);
    if (live) {
    const Row sr = ident ? identity_row() : spline_row(xm, xs, xp, sm, sp);

    const size_t o = rec_base(a, e, q) + p;
    double* rc = a.rec;
    const size_t pl = a.rec_plane;
    rc[6 * pl + o] = sr.l;
    rc[7 * pl + o] = sr.m;
    rc[8 * pl + o] = sr.u;
    rc[9 * pl + o] = sr.r;

    ChunkEnds ce;
    if (len > 0) {
        ce = chunk_ends_slab(sx + lane * kSlab, sy + lane * kSlab, len);
    } else {
        ce.ga = 0.0; ce.aa = 0.0; ce.ba = 1.0;
        ce.gb = 0.0; ce.ab = 1.0; ce.bb = 0.0;
    }
    rc[0 * pl + o] = ce.ga;
    rc[1 * pl + o] = ce.aa;
    rc[2 * pl + o] = ce.ba;
    rc[3 * pl + o] = ce.gb;
    rc[4 * pl + o] = ce.ab;
    rc[5 * pl + o] = ce.bb;
    }
    __syncwarp();  // the slabs are reused by the warp's next group
    }
}

// chunk_interior on a slab: row k (k = 0..len-1) is slab knot k+1; the spline values of slab
// knots 1..len are written to cv[1..len], cpw[1..len] holds the Thomas factors meanwhile.  The
// same operations in the same order as chunk_interior<true>.
__device__ __forceinline__ void chunk_interior_slab(int len, const int32_t* x, const double* s,
                                                    double xl, double xr, double* cpw,
                                                    double* cv) {
    double cp = 0.0, gp = 0.0;
    for (int k = 0; k < len; ++k) {
        const Row w = spline_row(x[k], x[k + 1], x[k + 2], s[k], s[k + 1]);
        double ri = w.r;
        if (k == 0) ri = fma(-w.l, xl, ri);
        if (k == len - 1) ri = fma(-w.u, xr, ri);
        double iw;
        if (k == 0) {
            iw = 1.0 / w.m;
            gp = ri * iw;
        } else {
            iw = pivot_rcp(w, cp);
            gp = fma(-w.l, gp, ri) * iw;
        }
        cp = w.u * iw;
        cpw[k + 1] = cp;
        cv[k + 1] = gp;
    }
    double xv = gp;
    for (int k = len - 2; k >= 0; --k) {
        xv = fma(-cpw[k + 1], xv, cv[k + 1]);
        cv[k + 1] = xv;
    }
}

// k_segments: the spline coefficients of every segment (spline_coefficients), one thread per
// separator p, warps taking groups of 32 separators as in k_chunk_reduce.  The lane's chunk spans knots jb..js: their spline values
// are the separator values X[p-1], X[p] at the ends and the chunk interior between, and the
// lane writes b, c, d of the segments starting at knots jb..js-1 at those knots' slots.  The
// lane of the empty chunk left of a tile's first knot writes the segment that crosses into
// the tile (from the last knot of the previous non-empty tile).
__global__ void __launch_bounds__(kSegWarps * 32)
k_segments(SiftArgs a) {
    __shared__ __align__(16) int32_t slab_x[kSegWarps][32 * kSlab];  // later: copy-out table
    __shared__ double slab_s[kSegWarps][32 * kSlab];  // knot values -> slopes -> b
    __shared__ double slab_c[kSegWarps][32 * kSlab];  // spline values
    __shared__ double slab_d[kSegWarps][32 * kSlab];  // Thomas factors -> d
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ra = active_rows(a);
    const int groups = a.gsum[2 * ra];
    for (int gw = blockIdx.x * kSegWarps + warp; gw < groups;
         gw += gridDim.x * kSegWarps) {  // warp-uniform
    const int vs = group_spline(a, gw, 2 * ra);
    int e;
    const Geo q = spline_geo(a, vs, ra, e);
    const int se = spline_id(a, e, q);
    const int P = a.pcount[se];
    const int p0 = (gw - __ldg(a.gsum + vs)) * 32;
    const int p = p0 + lane;
    const bool live = p < P;
    const ChunkLane ch = locate_chunk(a, e, q, live ? p : P - 1);
    const int32_t* kx = e == 0 ? a.kx_max : a.kx_min;
    const double* ky = e == 0 ? a.ky_max : a.ky_min;
    const double* X = a.xsep + rec_base(a, e, q);
    const int c = (live && ch.k > 0) ? ch.js - ch.jb + 1 : 0;  // slab knots (>= 2 if any)
    int32_t* sx = slab_x[warp];
    double* ss = slab_s[warp];
    // the Thomas-factor and spline-value slabs are free until the interior solve: they hold
    // the staging's position table meanwhile
    stage_slabs(a, kx, ky, c, ch.tb + ch.jb, sx, ss, lane,
                reinterpret_cast<unsigned short*>(slab_d[warp]),
                reinterpret_cast<long long*>(slab_c[warp]));
    const int32_t* x = sx + lane * kSlab;
    double* s = ss + lane * kSlab;
    double* cv = slab_c[warp] + lane * kSlab;
    double* dv = slab_d[warp] + lane * kSlab;
    if (c > 0) {
        const double xl = X[p - 1], xr = X[p];
        cv[0] = xl;
        cv[c - 1] = xr;
        if (ch.len > 0) chunk_interior_slab(ch.len, x, s, xl, xr, dv, cv);
    }
    // coefficients of slab segments i = 0..c-2 (loop trip count uniform over the warp)
    // (segments whose quotients need the divisions are marked and redone after the loop, their
    // slope recomputed from the knots in global memory: s[i] then holds b)
    unsigned slow_seg = 0u;
    for (int i = 0; i < kChunk; ++i) {
        if (i < c - 1) {
            double b, d;
            bool slow;
            seg_coeffs_fast(a, x[i], x[i + 1], s[i], cv[i], cv[i + 1], b, d, slow);
            if (slow) slow_seg |= 1u << i;
            s[i] = b;
            dv[i] = d;
        }
    }
    if (__any_sync(0xffffffffu, slow_seg != 0u)) {
        for (int i = 0; i < kChunk; ++i) {
            if (slow_seg >> i & 1u) {
                const size_t src = ch.tb + ch.jb + i;
                const double slope = (ky[src + 1] - ky[src]) / (double)(x[i + 1] - x[i]);
                seg_coeffs_div(x[i], x[i + 1], slope, cv[i], cv[i + 1], s[i], dv[i]);
            }
        }
    }
    // the segment crossing into the tile: last knot of the previous non-empty tile -> local 0
    {
        const bool act = live && ch.k == 0 && ch.off0 > 0;
        const long long* nb = a.nbr + tix(a, e, q, ch.t) * 2;
        const size_t im = act ? (size_t)nb[0] : ch.tb;
        const int32_t x0 = kx[im], x1 = kx[ch.tb];
        const double y0 = ky[im], y1 = ky[ch.tb];
        const double c0 = act ? X[p - 1] : 0.0, c1 = act ? X[p] : 0.0;
        const double sl = slope_warp(a, x0, x1, y0, y1, act);
        double b, d;
        seg_coeffs_warp(a, x0, x1, sl, c0, c1, b, d, act);
        if (act) {
            double2* rec = reinterpret_cast<double2*>(a.seg[e] + 4 * im);
            rec[0] = make_double2(y0, b);
            rec[1] = make_double2(c0, d);
        }
    }
    // copy-out of the slab segments, coalesced: lane l's segments i = 0..c-2 -> the records
    // {y, b, c, d} of slots tb+jb+i.  The knot-position slab is free now and holds the
    // (lane, position) table of the m = c-1 segments per lane.
    __syncwarp();
    const int m = c > 0 ? c - 1 : 0;
    int incl = m;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned short* tab = reinterpret_cast<unsigned short*>(slab_x[warp]);
    long long* gs = reinterpret_cast<long long*>(slab_x[warp] + 16 * kSlab);  // after tab
    for (int i = 0; i < m; ++i) tab[incl - m + i] = (unsigned short)((lane << 5) | i);
    gs[lane] = (long long)(ch.tb + ch.jb);
    __syncwarp();
    double* out = a.seg[e];
    for (int f = lane; f < total; f += 32) {
        const unsigned t = tab[f];
        const int ow = (int)(t >> 5), i = (int)(t & 31u);
        const size_t dst = (size_t)gs[ow] + i;
        const int q = ow * kSlab + i;
        double2* rec = reinterpret_cast<double2*>(out + 4 * dst);
        rec[0] = make_double2(__ldg(ky + dst), ss[q]);
        rec[1] = make_double2(slab_c[warp][q], slab_d[warp][q]);
    }
    __syncwarp();  // the slabs are reused by the warp's next group
    }
}

// =======================================================================================
// k_reduced_solve: levels >= 2 of the partitioned solve (the system on the separators of
// the tile-aligned first level), one CTA per spline system.
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

__device__ void cta_tridiag(int n, const double* sys, int plane, double* x, double* ws) {
    cta_partitioned(n, sys, plane, x, ws);
}

// ---------------------------------------------------------------------------------------
// The same canonical partitioned solve for many systems at once, one level per launch, the
// chunks of every system spread over the grid (blockIdx.y = system, x = chunk): system s has
// nrows[s] rows (0: skipped) at sys + 4*plane*s (planes l, m, u, r), solution to
// x + plane*s, deeper levels in ws + ws_stride*s with cta_partitioned's layout.  Every chunk
// performs cta_partitioned's operations in the same order, so the solution is identical to
// cta_tridiag's; the launches replace its in-CTA barriers.  For long systems whose one CTA
// would otherwise walk thousands of chunks.
// ---------------------------------------------------------------------------------------
namespace {

struct PLevels {
    int depth;
    int sizes[8];
    size_t lv[8], xv[8], ends;  // offsets into the system's workspace (lv[0], xv[0] unused)
};

// Level-0 rows of a spline system rebuilt from its knot positions and right-hand side (the
// adjoint's systems: identity end rows with zero right-hand side, interior rows
// l = x_i - x_{i-1}, m = 2(l + u), u = x_{i+1} - x_i): the values k_adj_rows stores in the
// l, m, u planes, read as 4 bytes per row instead of 24.
struct KnotSysRows {
    const int32_t* x;
    const double* r;
    int K, first;
    __device__ __forceinline__ Row operator()(int k) const {
        const int i = first + k;
        Row w;
        if (i == 0 || i == K - 1) {
            w.l = 0.0;
            w.m = 1.0;
            w.u = 0.0;
            w.r = 0.0;
        } else {
            const int dl = x[i] - x[i - 1], du = x[i + 1] - x[i];
            w.l = (double)dl;
            w.m = (double)(2 * (dl + du));
            w.u = (double)du;
            w.r = r[i];
        }
        return w;
    }
};

__device__ __forceinline__ PLevels plevels(int n) {
    PLevels v;
    v.depth = 0;
    v.sizes[0] = n;
    while (v.sizes[v.depth] > kChunk && v.depth < 7) {
        v.sizes[v.depth + 1] = (v.sizes[v.depth] - 1) / kChunk;
        ++v.depth;
    }
    size_t off = 0;
    for (int k = 1; k <= v.depth; ++k) {
        v.lv[k] = off;
        off += 4 * (size_t)v.sizes[k];
    }
    for (int k = 1; k <= v.depth; ++k) {
        v.xv[k] = off;
        off += (size_t)v.sizes[k];
    }
    v.ends = off;
    return v;
}

}  // namespace

__global__ void __launch_bounds__(kThreads)
k_psolve_ends(int k, const int* nrows, const double* sys, int plane, double* ws,
              size_t ws_stride, const int32_t* kx) {
    const int sidx = blockIdx.y;
    const int n = nrows[sidx];
    if (n <= 0) return;
    const PLevels v = plevels(n);
    if (k >= v.depth) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nk = v.sizes[k], P = v.sizes[k + 1];
    if (q > P) return;
    double* w = ws + ws_stride * sidx;
    const double* L = k == 0 ? sys + (size_t)4 * plane * sidx : w + v.lv[k];
    const int pl = k == 0 ? plane : nk;
    const int first = q * kChunk;
    const int len = (q < P) ? kChunk - 1 : nk - first;
    const ChunkEnds ce =
        (k == 0 && kx) ? chunk_ends(len, KnotSysRows{kx + (size_t)plane * sidx, L + 3 * pl, n,
                                                     first})
                       : chunk_ends(len, GlobalRowFn{L, L + pl, L + 2 * pl, L + 3 * pl, first});
    double* ends = w + v.ends;
    ends[6 * q + 0] = ce.ga;
    ends[6 * q + 1] = ce.aa;
    ends[6 * q + 2] = ce.ba;
    ends[6 * q + 3] = ce.gb;
    ends[6 * q + 4] = ce.ab;
    ends[6 * q + 5] = ce.bb;
}

__global__ void __launch_bounds__(kThreads)
k_psolve_rows(int k, const int* nrows, const double* sys, int plane, double* ws,
              size_t ws_stride, const int32_t* kx) {
    const int sidx = blockIdx.y;
    const int n = nrows[sidx];
    if (n <= 0) return;
    const PLevels v = plevels(n);
    if (k >= v.depth) return;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int nk = v.sizes[k], P = v.sizes[k + 1];
    if (p >= P) return;
    double* w = ws + ws_stride * sidx;
    const double* L = k == 0 ? sys + (size_t)4 * plane * sidx : w + v.lv[k];
    const int pl = k == 0 ? plane : nk;
    const double* ends = w + v.ends;
    const int s = p * kChunk + kChunk - 1;
    Row sr;
    if (k == 0 && kx) {
        sr = KnotSysRows{kx + (size_t)plane * sidx, L + 3 * pl, n, 0}(s);
    } else {
        sr.l = L[s];
        sr.m = L[pl + s];
        sr.u = L[2 * pl + s];
        sr.r = L[3 * pl + s];
    }
    const Row o = reduced_row(sr, ends[6 * p + 3], ends[6 * p + 4], ends[6 * p + 5],
                              ends[6 * (p + 1) + 0], ends[6 * (p + 1) + 1],
                              ends[6 * (p + 1) + 2]);
    double* R = w + v.lv[k + 1];
    R[p] = o.l;
    R[P + p] = o.m;
    R[2 * P + p] = o.u;
    R[3 * P + p] = o.r;
}

__global__ void __launch_bounds__(kThreads)
k_psolve_base(int nsys, const int* nrows, const double* sys, int plane, double* x, double* ws,
              size_t ws_stride, const int32_t* kx) {
    const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= nsys) return;
    const int n = nrows[sidx];
    if (n <= 0) return;
    const PLevels v = plevels(n);
    double* w = ws + ws_stride * sidx;
    const int nb = v.sizes[v.depth];
    const double* L = v.depth == 0 ? sys + (size_t)4 * plane * sidx : w + v.lv[v.depth];
    const int pl = v.depth == 0 ? plane : nb;
    double* xo = v.depth == 0 ? x + (size_t)plane * sidx : w + v.xv[v.depth];
    if (v.depth == 0 && kx)
        thomas_small(nb, KnotSysRows{kx + (size_t)plane * sidx, L + 3 * pl, n, 0}, xo, 1);
    else
        thomas_small(nb, GlobalRowFn{L, L + pl, L + 2 * pl, L + 3 * pl, 0}, xo, 1);
}

__global__ void __launch_bounds__(kThreads)
k_psolve_back(int k, const int* nrows, const double* sys, int plane, double* x, double* ws,
              size_t ws_stride, const int32_t* kx) {
    const int sidx = blockIdx.y;
    const int n = nrows[sidx];
    if (n <= 0) return;
    const PLevels v = plevels(n);
    if (k >= v.depth) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nk = v.sizes[k], P = v.sizes[k + 1];
    if (q > P) return;
    double* w = ws + ws_stride * sidx;
    const double* L = k == 0 ? sys + (size_t)4 * plane * sidx : w + v.lv[k];
    const int pl = k == 0 ? plane : nk;
    const double* Xs = w + v.xv[k + 1];
    double* xo = k == 0 ? x + (size_t)plane * sidx : w + v.xv[k];
    const int first = q * kChunk;
    const int len = (q < P) ? kChunk - 1 : nk - first;
    const double xl = (q > 0) ? Xs[q - 1] : 0.0;
    const double xr = (q < P) ? Xs[q] : 0.0;
    if (k == 0 && kx)
        chunk_interior(len, KnotSysRows{kx + (size_t)plane * sidx, L + 3 * pl, n, first}, xl,
                       xr, xo + first, 1);
    else
        chunk_interior(len, GlobalRowFn{L, L + pl, L + 2 * pl, L + 3 * pl, first}, xl, xr,
                       xo + first, 1);
    if (q < P) xo[first + kChunk - 1] = xr;
}

// Launch sequence of the level kernels for nsys systems of at most max_rows rows (kx: the
// systems' knot positions, plane-strided, when their level-0 rows are spline rows rebuilt from
// the knots and only the right-hand-side plane is stored; null: all four planes stored).
cudaError_t psolve_launch(int nsys, int max_rows, const int* nrows, const double* sys, int plane,
                          double* x, double* ws, size_t ws_stride, cudaStream_t st,
                          int* launches, const int32_t* kx) {
    int sizes[8], depth = 0;
    sizes[0] = max_rows;
    while (sizes[depth] > kChunk && depth < 7) {
        sizes[depth + 1] = (sizes[depth] - 1) / kChunk;
        ++depth;
    }
    int nl = 0;
    for (int k = 0; k < depth; ++k) {
        const dim3 g((unsigned)((sizes[k + 1] + 1 + kThreads - 1) / kThreads), (unsigned)nsys);
        k_psolve_ends<<<g, kThreads, 0, st>>>(k, nrows, sys, plane, ws, ws_stride, kx);
        k_psolve_rows<<<g, kThreads, 0, st>>>(k, nrows, sys, plane, ws, ws_stride, kx);
        nl += 2;
    }
    k_psolve_base<<<(unsigned)((nsys + kThreads - 1) / kThreads), kThreads, 0, st>>>(
        nsys, nrows, sys, plane, x, ws, ws_stride, kx);
    ++nl;
    for (int k = depth - 1; k >= 0; --k) {
        const dim3 g((unsigned)((sizes[k + 1] + 1 + kThreads - 1) / kThreads), (unsigned)nsys);
        k_psolve_back<<<g, kThreads, 0, st>>>(k, nrows, sys, plane, x, ws, ws_stride, kx);
        ++nl;
    }
    if (launches) *launches = nl;
    return cudaGetLastError();
}

namespace {

constexpr int kRedPass = kRedThreads * kChunk;                // level-2 rows per pass
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

// Level-2 row p (separator p of the level-1 partition) from the chunk records; chunk p is the
// chunk left of separator p, chunk p+1 the one right of it (chunk P, after the last knot,
// is empty: x_{s+1} = x_{s_next}).
__device__ __forceinline__ Row level2_row(const double* rc, size_t pl, size_t o, int p, int P) {
    Row sr;
    sr.l = rc[6 * pl + o + p];
    sr.m = rc[7 * pl + o + p];
    sr.u = rc[8 * pl + o + p];
    sr.r = rc[9 * pl + o + p];
    double ga = 0.0, aa = 0.0, ba = 1.0;
    if (p + 1 < P) {
        ga = rc[0 * pl + o + p + 1];
        aa = rc[1 * pl + o + p + 1];
        ba = rc[2 * pl + o + p + 1];
    }
    return reduced_row(sr, rc[3 * pl + o + p], rc[4 * pl + o + p], rc[5 * pl + o + p], ga, aa, ba);
}

__device__ __forceinline__ void stage_level2(RedStage& st, const double* rc, size_t pl, size_t o,
                                             int p0,
                                             int P) {
    const int rows = min(kRedPass, P - p0);
    constexpr int kB = 4;  // rows per thread whose record loads are in flight together
    for (int j0 = threadIdx.x; j0 < rows; j0 += kB * kRedThreads) {
        Row w[kB];
#pragma unroll
        for (int t = 0; t < kB; ++t) {
            const int j = j0 + t * kRedThreads;
            if (j < rows) w[t] = level2_row(rc, pl, o, p0 + j, P);
        }
#pragma unroll
        for (int t = 0; t < kB; ++t) {
            const int j = j0 + t * kRedThreads;
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

// Dynamic shared memory of k_reduced_solve: the level-2 stage plus a level-3 workspace for up
// to *qcap level-3 rows (16*Q + 74 doubles for Q rows), within kRedSmemMax.  Splines with more
// level-3 rows use the global workspace.
size_t reduced_solve_smem(int* qcap) {
    const size_t base = sizeof(RedStage);
    const long avail = (long)(kRedSmemMax - base) / (long)sizeof(double) - 74;
    *qcap = avail > 0 ? (int)(avail / 16) : 0;
    return base + sizeof(double) * (16 * (size_t)*qcap + 74);
}

namespace {

// The reduced solve of one spline system (level-2 size P, records at rc + o of planes pl,
// separator values to X, global level-3 workspace wg).  Every thread of the CTA calls it.
__device__ __forceinline__ void reduced_solve_one(unsigned char* dyn_smem, const double* rc,
                                               size_t pl, size_t o, int P, double* X,
                                               int red_qcap, double* wg) {
    RedStage& st = *reinterpret_cast<RedStage*>(dyn_smem);
    if (P <= kChunk) {
        stage_level2(st, rc, pl, o, 0, P);
        __syncthreads();
        if (threadIdx.x == 0) thomas_small(P, StageRowFn{&st, 0}, X, 1);
        return;
    }
    const int Q = (P - 1) / kChunk;  // level-3 size
    // level-3 workspace: shared memory after the stage, or the global reduced workspace
    double* w3 = Q <= red_qcap ? reinterpret_cast<double*>(dyn_smem + sizeof(RedStage)) : wg;
    double* ends = w3;                       // 6 * (Q+1)
    double* sep = ends + 6 * (size_t)(Q + 1);  // 4 * (Q+1)
    double* L3 = sep + 4 * (size_t)(Q + 1);    // 4 * Q
    double* x3 = L3 + 4 * (size_t)Q;           // Q
    double* ws3 = x3 + Q;                     // deeper levels
    for (int p0 = 0; p0 < P; p0 += kRedPass) {
        __syncthreads();
        stage_level2(st, rc, pl, o, p0, P);
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
    for (int p = threadIdx.x; p < Q; p += kRedThreads) {
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
        if (P > kRedPass) stage_level2(st, rc, pl, o, p0, P);  // else: still staged from pass one
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

}  // namespace

// k_reduced_solve: one CTA of kRedThreads per active spline system (maxima splines first,
// then minima); the grid covers every spline of the engine, CTAs past the active ones exit.
__global__ void __launch_bounds__(kRedThreads)
k_reduced_solve(SiftArgs a) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const int ra = active_rows(a);
    const int vs = blockIdx.x;
    if (vs >= 2 * ra) return;
    int e;
    const Geo gq = spline_geo(a, vs, ra, e);
    const int re = spline_id(a, e, gq);
    const size_t o = rec_base(a, e, gq);
    reduced_solve_one(dyn_smem, a.rec, a.rec_plane, o, a.pcount[re], a.xsep + o, a.red_qcap,
                      a.red + red_base(a, e, gq));
}

// =======================================================================================
// k_eval: envelopes + mean envelope + sx statistics over one tile of samples, both envelopes
// at once.  Thread t handles local samples k*256 + t, so warp accesses to samples and bitmap
// words are contiguous.  The segment of sample s is (#knots at positions < s) - 1, a popc
// rank in the tile's knot bitmap: the word of a warp's 32 samples and the knot count before it
// come by shuffle.  The segment's record {a, b, c, d} (k_segments) and start position are
// read from its start knot's slot, the previous tile's last knot for the samples before the
// tile's first knot.
// =======================================================================================
template <int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_eval_t(SiftArgs a) {
    __shared__ int s_red[kThreads / 32];
    __shared__ int s_any[kThreads / 32];
    const int total = active_tiles(a);
    // persistent CTAs: active tiles v, v + gridDim.x, ... (CTA-uniform loop)
    for (int vt = blockIdx.x; vt < total; vt += gridDim.x) {
    int tile;
    const Geo gq = tile_geo(a, vt, tile);
    const int n = gq.n;
    const int n0 = tile * kTileSamples;
    const size_t base = gq.base;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const size_t tb = tile_base(gq.tile0 + tile);
    // Per envelope: the slot of the knot before the tile, and for k = 0..7 (held by lane k)
    // this warp's bitmap word k*8 + warp with the count of the tile's knots before it.
    size_t pv[2];
    unsigned wk[2];
    int pk[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int off0 = __ldg(a.tile_off + oix(a, e, gq) + tile);
        pv[e] = off0 > 0 ? (size_t)__ldg(a.nbr + tix(a, e, gq, tile) * 2) : tb;
        const unsigned* bm = a.bitmap + tix(a, e, gq, tile) * kWords;
        const unsigned b0 = __ldg(bm + 2 * lane), b1 = __ldg(bm + 2 * lane + 1);
        const int pair = __popc(b0) + __popc(b1);
        int incl = pair;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        // lane k < 8 takes word k*8 + warp from lane (k*8 + warp) / 2
        const int src = (lane & 7) * 4 + (warp >> 1);
        const unsigned a0 = __shfl_sync(0xffffffffu, b0, src);
        const unsigned a1 = __shfl_sync(0xffffffffu, b1, src);
        const int ex = __shfl_sync(0xffffffffu, incl - pair, src);
        const bool odd = (warp & 1) != 0;
        wk[e] = odd ? a1 : a0;
        pk[e] = ex + (odd ? __popc(a0) : 0);
    }
    // envelope e at local sample k*256 + threadIdx.x
    auto env_at = [&](int e, int k) {
        const unsigned word = __shfl_sync(0xffffffffu, wk[e], k);
        const int sl = __shfl_sync(0xffffffffu, pk[e], k) + __popc(word & lt) - 1;
        const size_t q = sl >= 0 ? tb + (size_t)sl : pv[e];
        const double2* rp = reinterpret_cast<const double2*>(a.seg[e] + 4 * q);
        const double2 yb = __ldg(rp), cd = __ldg(rp + 1);
        const int32_t x = __ldg((e == 0 ? a.kx_max : a.kx_min) + q);
        const int s = n0 + k * kThreads + threadIdx.x;
        return seg_eval(yb.x, yb.y, cd.x, cd.y, (double)(s - x));
    };
    // averageUppperLower: the mean envelope keeps its previous value unless both envelopes
    // have more than 3 knots
    const bool write_mean = a.kcount[gq.g] > 3 && a.kcount[a.nrows + gq.g] > 3;
    int cnt = 0, any = 0;
    // sx > t is decided without the division where the products give a margin (sx_bounds);
    // undecided samples are redone exactly after the loop
    unsigned undecided = 0u;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int s = n0 + k * kThreads + threadIdx.x;
        const bool live = s < n;
        const double u = env_at(0, k);
        const double v = env_at(1, k);
        if (live) {
            if (write_mean) a.menv[base + s] = (u + v) / 2.0;
            if (a.dbg_upper) {
                a.dbg_upper[base + s] = u;
                a.dbg_lower[base + s] = v;
            }
        }
        const double p = fabs(u + v), q = fabs(u - v);
        const bool inr = q > 0x1p-800 && q < 0x1p+800;
        const bool any_t = p > q * a.sd2_hi, any_f = p < q * a.sd2_lo;
        const bool cnt_t = p > q * a.sd_hi, cnt_f = p < q * a.sd_lo;
        any |= (live && inr && any_t) ? 1 : 0;
        cnt += (live && inr && cnt_t) ? 1 : 0;
        if (live && !(inr && (any_t || any_f) && (cnt_t || cnt_f))) undecided |= 1u << k;
    }
    if (__any_sync(0xffffffffu, undecided != 0u)) {
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const double u = env_at(0, k);  // every lane: env_at shuffles
            const double v = env_at(1, k);
            if (!(undecided >> k & 1u)) continue;
            const double p = fabs(u + v), q = fabs(u - v);
            const bool inr = q > 0x1p-800 && q < 0x1p+800;
            if (!(inr && (p > q * a.sd2_hi || p < q * a.sd2_lo)))
                any |= sx_value_greater(u, v, a.sd2) ? 1 : 0;
            if (!(inr && (p > q * a.sd_hi || p < q * a.sd_lo)))
                cnt += sx_value_greater(u, v, a.sd) ? 1 : 0;
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
        if (c) atomicAdd(&a.cnt[gq.g], (unsigned)c);
        if (y) atomicOr(&a.any[gq.g], 1);
    }
    __syncthreads();  // s_red / s_any are reused by the CTA's next tile
    }
}

// The register budgets the autotuner chooses between; same results.  (A one-tile-per-CTA
// form, as k_extrema has, spills at budget A and was measured slower.)
template __global__ void k_eval_t<kEvalBlocksA>(SiftArgs a);
template __global__ void k_eval_t<kEvalBlocksB>(SiftArgs a);

// =======================================================================================
// k_criterion: one CTA per channel (persistent over the channels), over the channel's
// realizations; channels whose stage has finished are skipped.
// =======================================================================================
__global__ void __launch_bounds__(kThreads)
k_criterion(SiftArgs a) {
    __shared__ int s_all[kThreads / 32];
    __shared__ unsigned long long s_knots[kThreads / 32];
    for (int c = blockIdx.x; c < a.nchan; c += gridDim.x) {
    ChanState& cst = a.cs[c];
    if (cst.done) continue;  // CTA-uniform
    const Chan* ch = a.chan + c;
    const int nr = __ldg(&ch->nr), row0 = __ldg(&ch->row0);
    const double inv_n = 1.0 / (double)__ldg(&ch->n);
    const int j = cst.iter;
    const int cap = cst.cap;
    int all = 1;
    unsigned long long knots = 0;
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        const int g = row0 + r;
        const unsigned cn = a.cnt[g];
        const int any = a.any[g];
        a.cnt[g] = 0u;
        a.any[g] = 0;
        const int kmax = a.kcount[g], kmin = a.kcount[a.nrows + g];
        knots += (unsigned long long)(kmax + kmin);
        const double fr = (a.frac[g] + (double)cn) * inv_n;
        a.frac[g] = fr;
        const bool crit = fr > a.tol || (any != 0 && (kmax + kmin) > 6);
        int fin = a.finish[g];
        int mark;
        if (crit) {
            mark = 1;
            if (fin == 0 && j == cap - 1) {
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
        a.mark[g] = mark;
        if (a.tape_mark) a.tape_mark[r] = (signed char)mark;
        a.finish[g] = fin;
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
        cst.iter = j + 1;
        cst.knots += kt;
        cst.iters += 1ull;
        if (a.forced > 0 ? j + 1 >= a.forced : d != 0) cst.done = 1;
    }
    __syncthreads();  // s_all / s_knots are reused for the CTA's next channel
    }
}

// Mode export of channel c's realizations that finished in the last executed iteration
// (blockIdx.y = realization).
__global__ void k_export_final(SiftArgs a, int c) {
    const Geo q = geo(a, c, blockIdx.y);
    if (a.mark[q.g] != 0) return;
    const ChanState& cst = a.cs[c];
    const double* h = a.h[cst.iter & 1] + q.base;
    double* mo = cst.mode_out + (size_t)q.r * q.n;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < q.n; s += gridDim.x * blockDim.x)
        mo[s] = h[s];
}

// Start of a stage of channel c (one CTA): the stage's sift cap and mode buffer, iteration 0,
// no realization finished, no update pending.
__global__ void k_begin_stage(SiftArgs a, int c, int cap, double* mode_out) {
    const Chan* ch = a.chan + c;
    const int nr = __ldg(&ch->nr), row0 = __ldg(&ch->row0);
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        a.mark[row0 + r] = -1;
        a.finish[row0 + r] = 0;
    }
    if (threadIdx.x == 0) {
        ChanState& cst = a.cs[c];
        cst.done = 0;
        cst.iter = 0;
        cst.cap = cap;
        cst.mode_out = mode_out;
    }
}

// Active-channel plan of the iteration (several channels): one CTA.  plan[c] = rows and
// plan[nchan+1+c] = tiles of the channels before c whose stage is running (done == 0);
// plan[nchan] and plan[2*nchan+1] are the totals.
__device__ void plan_block(const SiftArgs& a) {
    __shared__ int s_rows[32], s_tiles[32];
    const int m = a.nchan;
    const int per = (m + 1023) / 1024;
    const int i0 = threadIdx.x * per;
    int rows = 0, tiles = 0;
    for (int i = i0; i < min(i0 + per, m); ++i) {
        if (a.cs[i].done) continue;
        const int nr = a.chan[i].nr;
        rows += nr;
        tiles += nr * a.chan[i].ntiles;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int ir = rows, itl = tiles;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, ir, o);
        const int w = __shfl_up_sync(0xffffffffu, itl, o);
        if (lane >= o) {
            ir += u;
            itl += w;
        }
    }
    if (lane == 31) {
        s_rows[warp] = ir;
        s_tiles[warp] = itl;
    }
    __syncthreads();
    if (warp == 0) {
        int u = s_rows[lane], w = s_tiles[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int pu = __shfl_up_sync(0xffffffffu, u, o);
            const int pw = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) {
                u += pu;
                w += pw;
            }
        }
        s_rows[lane] = u;
        s_tiles[lane] = w;
    }
    __syncthreads();
    int pr = (warp > 0 ? s_rows[warp - 1] : 0) + ir - rows;
    int pt = (warp > 0 ? s_tiles[warp - 1] : 0) + itl - tiles;
    for (int i = i0; i < min(i0 + per, m); ++i) {
        a.plan[i] = pr;
        a.plan[m + 1 + i] = pt;
        if (a.cs[i].done) continue;
        const int nr = a.chan[i].nr;
        pr += nr;
        pt += nr * a.chan[i].ntiles;
    }
    if (threadIdx.x == 1023) {
        a.plan[m] = s_rows[31];
        a.plan[2 * m + 1] = s_tiles[31];
    }
}

__global__ void __launch_bounds__(1024)
k_plan(SiftArgs a) {
    plan_block(a);
}

// =======================================================================================
// generic batched tridiagonal solve (stage-level entry point): one CTA per system
// =======================================================================================
__global__ void __launch_bounds__(kTridiagThreads)
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

// =======================================================================================
// k_sift_small: the whole lock-step sift of one stage for rows of at most kSmallMaxN samples,
// in one cooperative launch: CTA r holds realization r's h in shared memory and runs every
// iteration on chip -- the deferred update, extrema and compaction, the end-knot rule, the
// canonical tile-aligned spline solve (chunk end relations, separator rows, the separator
// system by the same level-2/level-3 partition as k_reduced_solve, chunk interiors), segment
// coefficients, both envelopes, the mean envelope, the sx statistics and the stop test -- and
// meets the other CTAs once per iteration at the lock-step test (a counter polled at most
// spin_limit times; when it runs out, the CTA sets CEEMDAN_ERR_TIMEOUT in the channel's error
// word and returns).  Every operation is the one the multi-kernel iteration performs, in the
// same order (canon.cuh; divisions taken as IEEE divisions, which the tabled-reciprocal fast
// paths of the other kernels reproduce exactly), so the results are bit-identical.  Channel 0
// only; the reference loop it replaces is cudaICEEMDAN.cu:1752-1867 (per iteration ~25
// kernel launches and library calls, and a host round trip).
// =======================================================================================
namespace {

struct SmallSmem {
    double *H, *KY, *KS, *KC, *ENDS, *R2, *X2, *W3;
    int *KX, *SEP, *misc, *WP;
    unsigned* BM;
    double* KD;  // segment d's, over the solve's workspace (ENDS .. W3) once the solve is done
    int kcap, pcap, qcap, dcap;
};

// Knot k of the knot arrays KX, KY, KS, KC sits at kp(k): one pad slot after every 16 knots,
// so the chunk chains of the spline solve (lane p walks the knots of chunk p, 16 knots after
// lane p-1's) read different banks.
__host__ __device__ __forceinline__ int kp(int k) { return k + (k >> 4); }

// Spline values written by chunk_interior into the padded knot array from knot `first` on.
struct PadOut {
    double* a;
    int first;
    __device__ __forceinline__ double& operator[](int k) const { return a[kp(first + k)]; }
};

// Layout of the dynamic shared memory for rows of n samples (doubles first, 16-byte aligned).
__host__ __device__ inline size_t small_layout(int n, SmallSmem* L, unsigned char* base) {
    const int ntiles = (n + kTileSamples - 1) / kTileSamples;
    const int kcap = n / 2 + 2;
    const int kpad = kp(kcap) + 1;  // knot arrays, one pad slot per 16 knots
    const int pcap = kcap / kChunk + 2 * ntiles + 8;
    const int qcap = pcap / kChunk + 1;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 15) & ~(size_t)15;
        return o;
    };
    const size_t oH = take(sizeof(double) * n);
    const size_t oKY = take(sizeof(double) * kpad);
    const size_t oKS = take(sizeof(double) * kpad);
    const size_t oKC = take(sizeof(double) * kpad);
    const size_t oE = take(sizeof(double) * 6 * pcap);
    const size_t oR = take(sizeof(double) * 4 * pcap);
    const size_t oX = take(sizeof(double) * pcap);
    const size_t oW = take(sizeof(double) * (16 * (size_t)qcap + 74));
    const size_t oKX = take(sizeof(int) * kpad);
    const size_t oS = take(sizeof(int) * pcap);
    const size_t oM = take(sizeof(int) * 64);
    const int nw = (n + 31) >> 5;
    const size_t oBM = take(sizeof(unsigned) * nw);
    const size_t oWP = take(sizeof(int) * (nw + 1));
    if (L && base) {
        L->H = reinterpret_cast<double*>(base + oH);
        L->KY = reinterpret_cast<double*>(base + oKY);
        L->KS = reinterpret_cast<double*>(base + oKS);
        L->KC = reinterpret_cast<double*>(base + oKC);
        L->ENDS = reinterpret_cast<double*>(base + oE);
        L->R2 = reinterpret_cast<double*>(base + oR);
        L->X2 = reinterpret_cast<double*>(base + oX);
        L->W3 = reinterpret_cast<double*>(base + oW);
        L->KX = reinterpret_cast<int*>(base + oKX);
        L->SEP = reinterpret_cast<int*>(base + oS);
        L->misc = reinterpret_cast<int*>(base + oM);
        L->BM = reinterpret_cast<unsigned*>(base + oBM);
        L->WP = reinterpret_cast<int*>(base + oWP);
        L->KD = L->ENDS;
        L->kcap = kcap;
        L->pcap = pcap;
        L->qcap = qcap;
        L->dcap = (int)((oKX - oE) / sizeof(double));
    }
    return off;
}

// Spline row of knot g from the knot arrays (the slopes of segments g-1 and g).
struct KnotRowFn {
    const int* x;
    const double* s;
    int first;  // knot of row 0 minus 1 (the knot before the chunk)
    __device__ __forceinline__ Row operator()(int k) const {
        const int i = first + k;
        return spline_row(x[kp(i)], x[kp(i + 1)], x[kp(i + 2)], s[kp(i)], s[kp(i + 1)]);
    }
};

// Row p of a system stored as planes l, m, u, r of `plane` doubles.
struct PlaneRowFn {
    const double* L;
    int plane, first;
    __device__ __forceinline__ Row operator()(int k) const {
        const int i = first + k;
        Row w;
        w.l = L[i];
        w.m = L[plane + i];
        w.u = L[2 * plane + i];
        w.r = L[3 * plane + i];
        return w;
    }
};

// Exclusive prefix of v over the CTA's threads in thread order; *total = the sum.  scratch:
// 2 * (kSmallThreads / 32) ints.
__device__ __forceinline__ int block_excl_scan(int v, int* scratch, int* total) {
    constexpr int kW = kSmallThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) scratch[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kW ? scratch[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        if (lane < kW) scratch[kW + lane] = w;
    }
    __syncthreads();
    const int before = warp > 0 ? scratch[kW + warp - 1] : 0;
    *total = scratch[2 * kW - 1];
    __syncthreads();
    return before + incl - v;
}

static_assert(kSmallMaxN / 32 <= kSmallThreads, "one bitmap word per thread in the knot scan");
static_assert(16 + 2 * (kSmallThreads / 32) <= 64, "scan scratch inside the misc ints");

// Knots of envelope e of h[0..n) (its maxima or minima, and both end samples): the bitmap BM
// (bit j of word w: sample 32w + j, one warp ballot per word), the knots before each word WP
// (WP[nw] = K), and the knots in order in KX/KY with the end rule applied; returns K.
__device__ __noinline__ int small_knots(const SmallSmem& S, int n, int e) {
    const double* H = S.H;
    const int nw = (n + 31) >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int w = warp; w < nw; w += kSmallThreads / 32) {
        const int i = (w << 5) + lane;
        bool k = false;
        if (i < n) {
            if (i == 0 || i == n - 1) {
                k = true;
            } else {
                const double v = H[i], vl = H[i - 1], vr = H[i + 1];
                k = e == 0 ? (v > vl && v > vr) : (v < vl && v < vr);
            }
        }
        const unsigned b = __ballot_sync(0xffffffffu, k);
        if (lane == 0) S.BM[w] = b;
    }
    __syncthreads();
    int K;
    const int c = (int)threadIdx.x < nw ? __popc(S.BM[threadIdx.x]) : 0;
    const int ex = block_excl_scan(c, S.misc + 16, &K);
    if ((int)threadIdx.x < nw) S.WP[threadIdx.x] = ex;
    if (threadIdx.x == 0) S.WP[nw] = K;
    __syncthreads();
    for (int w = warp; w < nw; w += kSmallThreads / 32) {
        const unsigned b = S.BM[w];
        if (b >> lane & 1u) {
            const int pos = kp(S.WP[w] + __popc(b & ((1u << lane) - 1u)));
            const int i = (w << 5) + lane;
            S.KX[pos] = i;
            S.KY[pos] = H[i];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // setBoundaryMax/Min, from the original values
        int flags = 0;
        if (K - 1 > 4) {
            const int L = K - 1;
            const int a0 = kp(0), a1 = kp(1), a2 = kp(2);
            const int b0 = kp(L - 2), b1 = kp(L - 1), b2 = kp(L);
            const double y0 =
                boundary_left(e, S.KX[a0], S.KX[a1], S.KX[a2], S.KY[a0], S.KY[a1], S.KY[a2]);
            const double yL =
                boundary_right(e, S.KX[b0], S.KX[b1], S.KX[b2], S.KY[b0], S.KY[b1], S.KY[b2]);
            // the tape's end-rule flags (as k_scan_boundary): a replaced value differs in bits
            flags = (__double_as_longlong(y0) != __double_as_longlong(S.KY[a0]) ? 1 : 0) |
                    (__double_as_longlong(yL) != __double_as_longlong(S.KY[b2]) ? 2 : 0);
            S.KY[a0] = y0;
            S.KY[b2] = yL;
        }
        S.misc[12] = flags;
    }
    __syncthreads();
    return K;
}

// The canonical tile-aligned spline solve of the K knots in KX/KY: spline values to KC.
__device__ __noinline__ void small_spline(const SmallSmem& S, int n, int K) {
    const int ntiles = (n + kTileSamples - 1) / kTileSamples;
    int* toff = S.misc;        // [ntiles+1] first knot of each tile
    int* soff = S.misc + 6;    // [ntiles+1] first separator of each tile
    if (threadIdx.x == 0) {
        // knots before each tile, from the bitmap scan (a tile is a whole number of words)
        for (int t = 0; t < ntiles; ++t) toff[t] = S.WP[t * (kTileSamples / 32)];
        toff[ntiles] = K;
        soff[0] = 0;
        for (int u = 0; u < ntiles; ++u) {
            const int c = toff[u + 1] - toff[u];
            soff[u + 1] = soff[u] + (c > 0 ? (c + kChunk - 2) / kChunk + 1 : 0);
        }
    }
    // slopes of the segments (the exact quotients)
    for (int i = threadIdx.x; i + 1 < K; i += kSmallThreads)
        S.KS[kp(i)] = seg_slope(S.KX[kp(i)], S.KX[kp(i + 1)], S.KY[kp(i)], S.KY[kp(i + 1)]);
    __syncthreads();
    const int P = soff[ntiles];
    // separators: local knots 0, 16, 32, ... and the last of every tile with knots
    for (int p = threadIdx.x; p < P; p += kSmallThreads) {
        int t = 0;
        while (soff[t + 1] <= p) ++t;
        const int c = toff[t + 1] - toff[t];
        S.SEP[p] = toff[t] + sep_local(p - soff[t], c);
    }
    __syncthreads();
    // chunk end relations (the chunk left of each separator; empty left of a tile's first
    // knot) and the separator rows
    double* SROW = S.R2;
    for (int p = threadIdx.x; p < P; p += kSmallThreads) {
        const int gs = S.SEP[p];
        int t = 0;
        while (soff[t + 1] <= p) ++t;
        ChunkEnds ce;
        const int len = p > soff[t] ? gs - S.SEP[p - 1] - 1 : 0;
        if (len > 0) {
            ce = chunk_ends(len, KnotRowFn{S.KX, S.KS, S.SEP[p - 1]});
        } else {
            ce.ga = 0.0; ce.aa = 0.0; ce.ba = 1.0;
            ce.gb = 0.0; ce.ab = 1.0; ce.bb = 0.0;
        }
        double* en = S.ENDS + 6 * p;
        en[0] = ce.ga; en[1] = ce.aa; en[2] = ce.ba;
        en[3] = ce.gb; en[4] = ce.ab; en[5] = ce.bb;
        const Row sr = (gs == 0 || gs == K - 1)
                           ? identity_row()
                           : spline_row(S.KX[kp(gs - 1)], S.KX[kp(gs)], S.KX[kp(gs + 1)],
                                        S.KS[kp(gs - 1)], S.KS[kp(gs)]);
        SROW[p] = sr.l;
        SROW[S.pcap + p] = sr.m;
        SROW[2 * S.pcap + p] = sr.u;
        SROW[3 * S.pcap + p] = sr.r;
    }
    __syncthreads();
    // level-2 rows: the separator rows with the neighbouring chunks eliminated
    for (int p = threadIdx.x; p < P; p += kSmallThreads) {
        Row sr;
        sr.l = SROW[p];
        sr.m = SROW[S.pcap + p];
        sr.u = SROW[2 * S.pcap + p];
        sr.r = SROW[3 * S.pcap + p];
        const double* en = S.ENDS + 6 * p;
        double ga = 0.0, aa = 0.0, ba = 1.0;
        if (p + 1 < P) {
            ga = S.ENDS[6 * (p + 1) + 0];
            aa = S.ENDS[6 * (p + 1) + 1];
            ba = S.ENDS[6 * (p + 1) + 2];
        }
        const Row w = reduced_row(sr, en[3], en[4], en[5], ga, aa, ba);
        SROW[p] = w.l;
        SROW[S.pcap + p] = w.m;
        SROW[2 * S.pcap + p] = w.u;
        SROW[3 * S.pcap + p] = w.r;
    }
    __syncthreads();
    // the separator system, partitioned as k_reduced_solve does
    const PlaneRowFn R2{SROW, S.pcap, 0};
    if (P <= kChunk) {
        if (threadIdx.x == 0) thomas_small(P, R2, S.X2, 1);
    } else {
        const int Q = (P - 1) / kChunk;
        double* ends = S.W3;
        double* sep = ends + 6 * (size_t)(Q + 1);
        double* L3 = sep + 4 * (size_t)(Q + 1);
        double* x3 = L3 + 4 * (size_t)Q;
        double* ws3 = x3 + Q;
        for (int q = threadIdx.x; q <= Q; q += kSmallThreads) {
            const int first = q * kChunk;
            const int len = (q < Q) ? kChunk - 1 : P - first;
            const PlaneRowFn fn{SROW, S.pcap, first};
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
        __syncthreads();
        for (int p = threadIdx.x; p < Q; p += kSmallThreads) {
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
        for (int q = threadIdx.x; q <= Q; q += kSmallThreads) {
            const int first = q * kChunk;
            const int len = (q < Q) ? kChunk - 1 : P - first;
            const double xl = (q > 0) ? x3[q - 1] : 0.0;
            const double xr = (q < Q) ? x3[q] : 0.0;
            chunk_interior(len, PlaneRowFn{SROW, S.pcap, first}, xl, xr, S.X2 + first, 1);
            if (q < Q) S.X2[first + kChunk - 1] = xr;
        }
    }
    __syncthreads();
    // spline values: the separators', then the chunk interiors between them
    for (int p = threadIdx.x; p < P; p += kSmallThreads) {
        const int gs = S.SEP[p];
        S.KC[kp(gs)] = S.X2[p];
        int t = 0;
        while (soff[t + 1] <= p) ++t;
        if (p > soff[t]) {
            const int gb = S.SEP[p - 1];
            const int len = gs - gb - 1;
            if (len > 0)
                chunk_interior(len, KnotRowFn{S.KX, S.KS, gb}, S.X2[p - 1], S.X2[p],
                               PadOut{S.KC, gb + 1}, 1);
        }
    }
    __syncthreads();
}

// Tape of envelope e of realization r at iteration j (taped forward): the knot bitmap in the
// multi-kernel layout (64 words per tile, zero past the row), the knot count and the end-rule
// flags -- what k_tape_record copies from the multi-kernel iteration.
__device__ __forceinline__ void small_tape_knots(const SmallSmem& S, const SmallArgs& sa, int j,
                                                 int r, int n, int e, int K) {
    const TapeLayout& L = sa.tl;
    unsigned char* slot =
        sa.tblocks[j / kTapeBlockSlots] + (size_t)(j % kTapeBlockSlots) * L.stride;
    const int words = L.ntiles * (kTileSamples / 32);
    const int nw = (n + 31) >> 5;
    unsigned* bits = reinterpret_cast<unsigned*>(slot) + (size_t)(e * L.nr + r) * words;
    for (int w = threadIdx.x; w < words; w += kSmallThreads) bits[w] = w < nw ? S.BM[w] : 0u;
    if (threadIdx.x == 0) {
        reinterpret_cast<int*>(slot + L.off_kc)[e * L.nr + r] = K;
        (slot + L.off_bf)[e * L.nr + r] = (unsigned char)S.misc[12];
    }
}

// Segment coefficients after the solve: b of segment i into KS[i] (the slopes are spent) and,
// when the K - 1 segments fit the solve's workspace, d into KD[i]; returns whether d is stored.
__device__ __noinline__ bool small_coeffs(const SmallSmem& S, int K) {
    const bool dk = K - 1 <= S.dcap;
    for (int i = threadIdx.x; i + 1 < K; i += kSmallThreads) {
        const int i0 = kp(i), i1 = kp(i + 1);
        double b, d;
        seg_coeffs(S.KX[i0], S.KX[i1], S.KY[i0], S.KY[i1], S.KC[i0], S.KC[i1], b, d);
        S.KS[i0] = b;
        if (dk) S.KD[i] = d;
    }
    __syncthreads();
    return dk;
}

// Envelope at sample s: segment i holds x_i < s <= x_{i+1} (segment 0 also s = 0), i.e. i is
// the number of knots before s, less one -- a rank in the knot bitmap.  d as seg_coeffs forms
// it when it is not stored.
__device__ __forceinline__ double small_env_at(const SmallSmem& S, int s, bool dk) {
    const int w = s >> 5;
    const int before = S.WP[w] + __popc(S.BM[w] & ((1u << (s & 31)) - 1u));
    const int i = s > 0 ? before - 1 : 0;
    const int i0 = kp(i), i1 = kp(i + 1);
    const int x0 = S.KX[i0];
    const double c0 = S.KC[i0];
    const double d = dk ? S.KD[i] : (S.KC[i1] - c0) / (3.0 * (double)(S.KX[i1] - x0));
    return seg_eval(S.KY[i0], S.KS[i0], c0, d, (double)(s - x0));
}

}  // namespace

size_t small_sift_smem(int n) { return small_layout(n, nullptr, nullptr); }

// Bounded wait of one thread until *word >= target (acquire); false when it gave up.
__device__ __forceinline__ bool small_wait(unsigned* word, unsigned target, int limit) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> w(*word);
    int spins = 0;
    while (w.load(cuda::memory_order_acquire) < target) {
        if (++spins > limit) return false;
        __nanosleep(64);
    }
    return true;
}

__global__ void __launch_bounds__(kSmallThreads, 1)
k_sift_small(SiftArgs a, SmallArgs sa) {
    extern __shared__ __align__(16) unsigned char small_smem[];
    __shared__ int s_red[2][kSmallThreads / 32];
    __shared__ int s_ctl[5];  // mark, finish, all finished, error, the upper knot count
    // Realization r; role 2: one CTA does both envelopes.  Paired (two CTAs per realization):
    // role 0 builds the upper envelope and hands it over through global memory, role 1 the
    // lower one, then the mean, the statistics and the stop decision.  Both keep h.
    const bool pair = sa.pair != 0;
    const int r = pair ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const int role = pair ? (int)(blockIdx.x & 1) : 2;
    const int nreal = pair ? (int)(gridDim.x >> 1) : (int)gridDim.x;
    const Geo q = geo(a, 0, r);
    const int n = q.n;
    SmallSmem S;
    small_layout(n, &S, small_smem);
    ChanState& cst = a.cs[0];
    const int cap = cst.cap;
    double* mode = cst.mode_out + (size_t)q.r * n;
    double* menv = a.menv + q.base;
    double* up = sa.up + q.base;
    const double* hin = a.h[0] + q.base;  // the stage input
    const double inv_n = 1.0 / (double)n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < n; i += kSmallThreads) S.H[i] = hin[i];
    if (threadIdx.x == 0) {
        s_ctl[0] = -1;
        s_ctl[1] = 0;
    }
    __syncthreads();
    int j = 0;
    for (; j < cap; ++j) {
        // deferred update of the previous iteration (updateRealizations); the mean envelope
        // and the upper envelope are read through L2 (the paired CTA wrote them)
        const int mk = s_ctl[0];
        if (mk == 1) {
            // the mean envelope's loads of a round are all issued before the subtractions
            for (int i0 = 0; i0 < n; i0 += kSmallPre * kSmallThreads) {
                double mv[kSmallPre];
#pragma unroll
                for (int k = 0; k < kSmallPre; ++k) {
                    const int i = i0 + k * kSmallThreads + threadIdx.x;
                    mv[k] = i < n ? __ldcg(menv + i) : 0.0;
                }
#pragma unroll
                for (int k = 0; k < kSmallPre; ++k) {
                    const int i = i0 + k * kSmallThreads + threadIdx.x;
                    if (i < n) S.H[i] = S.H[i] - mv[k];
                }
            }
        } else if (mk == 0 && role != 0)
            for (int i = threadIdx.x; i < n; i += kSmallThreads) mode[i] = S.H[i];
        __syncthreads();
        int kmax = 0, kmin = 0;
        if (role != 1) {
            kmax = small_knots(S, n, 0);
            if (sa.tblocks) small_tape_knots(S, sa, j, q.r, n, 0, kmax);
            small_spline(S, n, kmax);
            const bool dmax = small_coeffs(S, kmax);
            for (int s = threadIdx.x; s < n; s += kSmallThreads) up[s] = small_env_at(S, s, dmax);
            __syncthreads();
            if (role == 0 && threadIdx.x == 0) {  // hand the upper envelope over
                sa.pair_kmax[r] = kmax;
                __threadfence();
                cuda::atomic_ref<unsigned, cuda::thread_scope_device> rd(sa.ready[r]);
                rd.store((unsigned)(j + 1), cuda::memory_order_release);
            }
        }
        if (role != 0) {
            kmin = small_knots(S, n, 1);
            if (sa.tblocks) small_tape_knots(S, sa, j, q.r, n, 1, kmin);
            small_spline(S, n, kmin);
            const bool dmin = small_coeffs(S, kmin);
            if (role == 1) {  // the upper envelope of this iteration from the paired CTA
                if (threadIdx.x == 0) {
                    const bool ok = small_wait(sa.ready + r, (unsigned)(j + 1), sa.spin_limit);
                    if (!ok) atomicExch(&cst.err, kErrTimeout);
                    s_ctl[3] = ok ? 0 : 1;
                    s_ctl[4] = ok ? __ldcg(sa.pair_kmax + r) : 0;
                }
                __syncthreads();
                if (s_ctl[3]) return;
                kmax = s_ctl[4];
            }
            const bool write_mean = kmax > 3 && kmin > 3;
            int cnt = 0, any = 0;
            // the upper envelope's loads of a round are all issued first (the mean envelope's
            // stores would otherwise hold each load back behind the previous sample's store)
            for (int s0 = 0; s0 < n; s0 += kSmallPre * kSmallThreads) {
                double uv[kSmallPre];
#pragma unroll
                for (int k = 0; k < kSmallPre; ++k) {
                    const int s = s0 + k * kSmallThreads + threadIdx.x;
                    uv[k] = s < n ? __ldcg(up + s) : 0.0;
                }
#pragma unroll
                for (int k = 0; k < kSmallPre; ++k) {
                    const int s = s0 + k * kSmallThreads + threadIdx.x;
                    if (s < n) {
                        const double v = small_env_at(S, s, dmin);
                        const double u = uv[k];
                        if (write_mean) menv[s] = (u + v) / 2.0;
                        any |= sx_greater(u, v, a.sd2) ? 1 : 0;
                        cnt += sx_greater(u, v, a.sd) ? 1 : 0;
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
                any |= __shfl_xor_sync(0xffffffffu, any, o);
            }
            if (lane == 0) {
                s_red[0][warp] = cnt;
                s_red[1][warp] = any;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int c = 0, y = 0;
                for (int w = 0; w < kSmallThreads / 32; ++w) {
                    c += s_red[0][w];
                    y |= s_red[1][w];
                }
                // the sifting-fraction carry and siftingCriterion (as k_criterion)
                const double fr = (a.frac[q.g] + (double)c) * inv_n;
                a.frac[q.g] = fr;
                const bool crit = fr > a.tol || (y != 0 && (kmax + kmin) > 6);
                int fin = s_ctl[1];
                int mark;
                if (crit) {
                    mark = 1;
                    if (fin == 0 && j == cap - 1) {
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
                s_ctl[0] = mark;
                s_ctl[1] = fin;
                if (pair) sa.pair_mark[r] = mark;
                if (sa.tblocks)
                    reinterpret_cast<signed char*>(sa.tblocks[j / kTapeBlockSlots] +
                                                   (size_t)(j % kTapeBlockSlots) * sa.tl.stride +
                                                   sa.tl.off_mark)[q.r] = (signed char)mark;
                atomicAdd(&cst.knots, (unsigned long long)(kmax + kmin));
                // the lock-step test: every realization's finish flag of this iteration
                if (fin) atomicAdd(sa.nfin + j, 1);
            }
        }
        // every CTA meets the others once per iteration (the stop test's lock step)
        if (threadIdx.x == 0) {
            // the fence orders this CTA's writes before its arrival; the arrival is a
            // reduction that does not wait for the counter's old value (the wait below
            // acquires)
            __threadfence();
            atomicAdd(sa.arrive, 1u);
            const unsigned target = (unsigned)(j + 1) * gridDim.x + sa.extra;
            const bool ok = small_wait(sa.arrive, target, sa.spin_limit);
            if (!ok) atomicExch(&cst.err, kErrTimeout);
            cuda::atomic_ref<int, cuda::thread_scope_device> nf(sa.nfin[j]);
            s_ctl[2] = a.forced > 0 ? (j + 1 >= a.forced ? 1 : 0)
                                    : (nf.load(cuda::memory_order_acquire) == nreal ? 1 : 0);
            s_ctl[3] = ok ? 0 : 1;
            if (role == 0) s_ctl[0] = __ldcg(sa.pair_mark + r);  // the next update's mark
        }
        __syncthreads();
        if (s_ctl[3]) return;  // a wait gave up: the host reports CEEMDAN_ERR_TIMEOUT
        if (s_ctl[2]) {
            ++j;
            break;
        }
    }
    if (j > cap) j = cap;
    // realizations that finished in the last iteration export h (k_export_final)
    if (s_ctl[0] == 0 && role != 0)
        for (int i = threadIdx.x; i < n; i += kSmallThreads) mode[i] = S.H[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cst.iter = j;
        cst.iters += (unsigned long long)j;
        cst.done = 1;
    }
}

}  // namespace ceemdan
