// Sifting kernels of the ICEEMDAN engine (sm_100a, FP64).
//
// One sift iteration over all realizations of a stage is:
//   k_extrema        deferred update h -= m (or mode export) + strict-extrema flags +
//                    warp-ballot compaction, tile offsets by decoupled look-back, per-tile
//                    knot bitmaps
//                    (find_extrema_shfl_* :93-148, CUB scan, select_extrema_* :151-207,
//                     updateRealizations :528-544 of the previous iteration)
//   k_boundary       end-knot extrapolation (setBoundaryMax/Min :210-291)
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

// 64-bit look-back status word: [63:62] flag (0 empty, 1 aggregate, 2 inclusive),
// [61:31] maxima count, [30:0] minima count.
__device__ __forceinline__ unsigned long long pack_status(unsigned flag, unsigned cmax,
                                                          unsigned cmin) {
    return ((unsigned long long)flag << 62) | ((unsigned long long)cmax << 31) |
           (unsigned long long)cmin;
}

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
    __shared__ unsigned s_ticket;
    __shared__ int s_prefix[2];
    __shared__ int s_agg[2];

    if (*a.done) return;
    if (threadIdx.x == 0) s_ticket = atomicAdd(a.ticket, 1u);
    __syncthreads();
    // Tile-major order: tile t of every realization is handed out before tile t+1 of any,
    // so a tile's predecessor has usually published its inclusive prefix already.
    const unsigned tk = s_ticket;
    const int tile = (int)(tk / (unsigned)a.nr);
    const int r = (int)(tk % (unsigned)a.nr);
    if (tile >= a.ntiles) return;
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
            const size_t bw = ((size_t)r * a.ntiles + tile) * kWords + w;
            a.bitmap[bw] = bmax[k];
            a.bitmap[(size_t)a.nr * a.ntiles * kWords + bw] = bmin[k];
        }
    }
    __syncthreads();

    // Exclusive scan of the 64 word counts per envelope: warp 0 -> maxima, warp 1 -> minima.
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
        if (lane == 31) s_agg[e] = incl;
    }
    __syncthreads();

    // Decoupled look-back over the tiles of realization r, 32 predecessors per step by
    // warp 0 (bounded wait: a predecessor that never publishes ends in kErrTimeout).
    if (warp == 0) {
        const unsigned amax = (unsigned)s_agg[0], amin = (unsigned)s_agg[1];
        unsigned long long* st_row = a.status + (size_t)r * a.ntiles;
        unsigned pmax = 0, pmin = 0;
        if (lane == 0) {
            cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> me_st(st_row[tile]);
            me_st.store(pack_status(tile == 0 ? 2u : 1u, amax, amin), cuda::memory_order_release);
        }
        if (tile > 0) {
            int hi = tile - 1;
            int spins = 0;
            bool timed_out = false;
            for (;;) {
                const int p = hi - lane;  // lane 0 = nearest predecessor
                unsigned long long w = pack_status(2u, 0u, 0u);
                unsigned flag = 2u;
                do {
                    if (p >= 0) {
                        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> st(st_row[p]);
                        w = st.load(cuda::memory_order_acquire);
                        flag = (unsigned)(w >> 62);
                    }
                    if (!__any_sync(0xffffffffu, flag == 0u)) break;
                    if (++spins > a.spin_limit) {
                        timed_out = true;
                        break;
                    }
                    __nanosleep(64);
                } while (true);
                if (timed_out) {
                    if (lane == 0) set_error(a.err, kErrTimeout);
                    break;
                }
                const unsigned incl = __ballot_sync(0xffffffffu, flag == 2u);
                const int stop = incl ? __ffs(incl) - 1 : 31;
                unsigned cm = lane <= stop ? (unsigned)((w >> 31) & 0x7fffffffu) : 0u;
                unsigned cn = lane <= stop ? (unsigned)(w & 0x7fffffffu) : 0u;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    cm += __shfl_xor_sync(0xffffffffu, cm, o);
                    cn += __shfl_xor_sync(0xffffffffu, cn, o);
                }
                pmax += cm;
                pmin += cn;
                if (incl) break;
                hi -= 32;
            }
            if (lane == 0) {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> me_st(st_row[tile]);
                me_st.store(pack_status(2u, pmax + amax, pmin + amin), cuda::memory_order_release);
            }
        }
        if (lane == 0) {
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
    }
    __syncthreads();

    const unsigned lt = (1u << lane) - 1u;
    const size_t kb = (size_t)r * (size_t)a.cap;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int j = k * kThreads + threadIdx.x;
        const int s = n0 + j;
        const int w = k * (kThreads / 32) + warp;
        if (bmax[k] & (1u << lane)) {
            const int pos = s_prefix[0] + s_off[0][w] + __popc(bmax[k] & lt);
            a.kx_max[kb + pos] = s;
            a.ky_max[kb + pos] = sh[2 + j];
        }
        if (bmin[k] & (1u << lane)) {
            const int pos = s_prefix[1] + s_off[1][w] + __popc(bmin[k] & lt);
            a.kx_min[kb + pos] = s;
            a.ky_min[kb + pos] = sh[2 + j];
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
// level-1 chunk kernels (end relations and interiors share the staging)
// =======================================================================================
namespace {

constexpr int kSpan = kChunksPerBlock * kChunk + 2;        // staged knots per block
constexpr int kStageSlots = kSpan + (kSpan >> 4) + 1;      // with one pad per 16

// Knot positions and segment slopes of the window [row0-1, row0-1+kSpan), padded so that
// each thread's 16 consecutive rows sit at stride 17 (bank-conflict free).  The knot values
// are staged into `slope` first and replaced by the segment slopes.
struct Staged {
    double slope[kStageSlots];  // slope[pad17(j)]: segment between window knots j, j+1
    int32_t x[kStageSlots];
};

__device__ __forceinline__ void stage_window(Staged& sg, int row0, int K, const int32_t* kx,
                                             const double* ky) {
    constexpr int kIt = (kSpan + kThreads - 1) / kThreads;
    for (int j = threadIdx.x; j < kSpan; j += kThreads) {
        const int i = row0 - 1 + j;
        if (i >= 0 && i < K) {
            cp_async4(&sg.x[pad17(j)], kx + i);
            cp_async8(&sg.slope[pad17(j)], ky + i);
        }
    }
    cp_async_wait_all();
    __syncthreads();
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
                sl[t] = seg_slope(sg.x[pad17(j)], sg.x[pad17(j + 1)], sg.slope[pad17(j)],
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

size_t chunk_reduce_smem() { return sizeof(Staged); }
size_t eval_smem() { return sizeof(double) * kTileSamples; }
size_t chunk_backsub_smem() { return sizeof(Staged); }

__global__ void __launch_bounds__(kThreads)
k_chunk_reduce(SiftArgs a) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    Staged& sg = *reinterpret_cast<Staged*>(dyn_smem);
    if (*a.done) return;
    {
        int e, r, b, K, P;
        if (!chunk_item(a, blockIdx.x, e, r, b, K, P)) return;
        const int re = e * a.nr + r;
        const size_t kb = (size_t)r * (size_t)a.cap;
        const int32_t* kx = (e == 0 ? a.kx_max : a.kx_min) + kb;
        const double* ky = (e == 0 ? a.ky_max : a.ky_min) + kb;
        const int row0 = b * kChunksPerBlock * kChunk;
        stage_window(sg, row0, K, kx, ky);
        __syncthreads();
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
    if (*a.done) return;
    {
        int e, r, b, K, P;
        if (!chunk_item(a, blockIdx.x, e, r, b, K, P)) return;
        const int re = e * a.nr + r;
        const size_t kb = (size_t)r * (size_t)a.cap;
        const int32_t* kx = (e == 0 ? a.kx_max : a.kx_min) + kb;
        const double* ky = (e == 0 ? a.ky_max : a.ky_min) + kb;
        double* c = (e == 0 ? a.c_max : a.c_min) + kb;
        const int row0 = b * kChunksPerBlock * kChunk;
        stage_window(sg, row0, K, kx, ky);
        __syncthreads();
        const int q = b * kChunksPerBlock + threadIdx.x;
        const double* X = a.xsep + (size_t)re * (size_t)a.rec_stride;
        if (q <= P) {
            const int first = q * kChunk;
            const int len = (q < P) ? kChunk - 1 : K - first;
            StagedRowFn fn{&sg, first, row0, K};
            const double xl = (q > 0) ? X[q - 1] : 0.0;
            const double xr = (q < P) ? X[q] : 0.0;
            chunk_interior(len, fn, xl, xr, c + first, 1);
            if (q < P) c[first + kChunk - 1] = xr;
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
// k_eval: envelopes + mean envelope + sx statistics over one tile of samples
// =======================================================================================
__global__ void __launch_bounds__(kThreads, 4)
k_eval(SiftArgs a) {
    constexpr int kMaxKnots = kTileSamples / 2 + 4;
    __shared__ int32_t sx_[kMaxKnots];
    __shared__ double sy[kMaxKnots], scf[kMaxKnots], sb[kMaxKnots], sd[kMaxKnots];
    extern __shared__ __align__(16) double su[];  // [kTileSamples] upper envelope of the tile
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
    const size_t kb = (size_t)r * (size_t)a.cap;
    const size_t to = (size_t)(a.ntiles + 1);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    double env[kPerThread];

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
            cp_async4(&sx_[j], kx + klo + j);
            cp_async8(&sy[j], ky + klo + j);
            cp_async8(&scf[j], kc + klo + j);
        }
        if (threadIdx.x < kWords)
            cp_async4(&sbm[threadIdx.x], a.bitmap + (size_t)e * a.nr * a.ntiles * kWords +
                                             ((size_t)r * a.ntiles + tile) * kWords + threadIdx.x);
        cp_async_wait_all();
        __syncthreads();
        for (int j = threadIdx.x; j < nk - 1; j += kThreads)
            seg_coeffs(sx_[j], sx_[j + 1], sy[j], sy[j + 1], scf[j], scf[j + 1], sb[j], sd[j]);
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
            double v = 0.0;
            if (s < n) {
                // segment of sample s: (#knots at positions < s) - 1, segment 0 at s = 0
                const int w = k * (kThreads / 32) + warp;
                const int rank = swp[w] + __popc(sbm[w] & lt);
                const int seg = max(off0 + rank - 1, 0);
                const int j = seg - klo;
                v = seg_eval(sy[j], sb[j], scf[j], sd[j], (double)(s - sx_[j]));
            }
            if (e == 0)
                su[k * kThreads + threadIdx.x] = v;
            else
                env[k] = v;
        }
    }

    const bool valid = a.kcount[r] > 3 && a.kcount[a.nr + r] > 3;
    int cnt = 0, any = 0;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int s = n0 + k * kThreads + threadIdx.x;
        if (s < n) {
            const double up = su[k * kThreads + threadIdx.x], lo = env[k];
            if (valid) a.menv[base + s] = (up + lo) / 2.0;
            any |= sx_greater(up, lo, a.sd2) ? 1 : 0;
            cnt += sx_greater(up, lo, a.sd) ? 1 : 0;
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
