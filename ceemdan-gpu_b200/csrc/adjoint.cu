// Reverse pass of the decomposition with its structure frozen (ceemdan_backward_f64).
//
// A taped forward call records, for every executed iteration of every signal stage, the knot
// bitmaps and counts of both envelopes, the end-rule flags and the marks (k_tape_record,
// k_scan_boundary, k_criterion).  With that structure fixed, one sift iteration of
// cudaICEEMDAN.cu:1752-2002 is linear in h:
//   knots       y_i = h[x_i], end values replaced by the extrapolation of :210-291
//   spline      natural cubic spline through (x_i, y_i) (:311-343, the cuSPARSE solve :1630)
//   envelope    a + b t + c t^2 + d t^3 on each segment (:383-439)
//   mean        m = (U + L)/2 when both knot counts exceed 3, else the previous m (:442-454)
//   update      h -= m (mark 1) or mode = h (mark 0) (:528-544)
// and these kernels apply the transposed maps in reverse order, one launch per step of one
// iteration over all realizations.  The spline matrix restricted to its interior rows is
// symmetric, so the transposed solve is the forward's canonical partitioned solve with a new
// right-hand side (cta_tridiag).  Every kernel is deterministic (no atomics; fixed summation
// orders), and the arithmetic order is the CPU oracle's (oracle/ceemdan_oracle.cpp,
// env_adjoint, sift_adjoint, vjp).
#include "canon.cuh"
#include "kernels.h"

namespace ceemdan {
namespace {

constexpr int kAdjThreads = 256;
constexpr int kTileWords = kTileSamples / 32;

struct Slot {
    const unsigned* bits;
    const int* kc;
    const unsigned char* bf;
    const signed char* mark;
};

__device__ __forceinline__ Slot view(const unsigned char* s, const TapeLayout& L) {
    return {reinterpret_cast<const unsigned*>(s), reinterpret_cast<const int*>(s + L.off_kc),
            s + L.off_bf, reinterpret_cast<const signed char*>(s + L.off_mark)};
}

// the iteration replaced realization r's mean envelope (both knot counts > 3)
__device__ __forceinline__ bool updated(const Slot& v, int nr, int r) {
    return v.kc[r] > 3 && v.kc[nr + r] > 3;
}

// knot count of spline sp, never above the cap of its knot arrays
__device__ __forceinline__ int knots(const Slot& v, int sp, int cap) {
    return min(v.kc[sp], cap);
}

// Adjoint of knot value i after the transposed end rule (flags bf; the rule applies to
// splines of more than 5 knots): t_left = y1 (1 + rho) - y2 rho with rho = (x1-x0)/(x2-x1),
// t_right = y_{L-1} (1 + rho) - y_{L-2} rho with rho = (x_L-x_{L-1})/(x_{L-1}-x_{L-2}).
__device__ double end_rule_adjoint(const int32_t* x, const double* y2, int K, int bf, int i) {
    double g = y2[i];
    if (K - 1 > 4) {
        const int L = K - 1;
        if (bf & 1) {
            const double rho = (double)(x[1] - x[0]) / (double)(x[2] - x[1]);
            if (i == 0) g = 0.0;
            else if (i == 1) g = y2[1] + y2[0] * (1.0 + rho);
            else if (i == 2) g = y2[2] - y2[0] * rho;
        }
        if (bf & 2) {
            const double rho = (double)(x[L] - x[L - 1]) / (double)(x[L - 1] - x[L - 2]);
            if (i == L) g = 0.0;
            else if (i == L - 1) g = y2[L - 1] + y2[L] * (1.0 + rho);
            else if (i == L - 2) g = y2[L - 2] - y2[L] * rho;
        }
    }
    return g;
}

}  // namespace

// One slot of the tape from the iteration just executed (launched before k_criterion, which
// writes the marks into the slot itself).  Iterations after the stop word record nothing.
__global__ void k_tape_record(SiftArgs a, TapeLayout L, unsigned char* slot) {
    if (a.cs[0].done) return;  // the taped forward has one channel
    const size_t q = L.off_kc / sizeof(uint4);  // bitmap bytes are a multiple of 512
    const uint4* src = reinterpret_cast<const uint4*>(a.bitmap);
    uint4* dst = reinterpret_cast<uint4*>(slot);
    const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = t0; i < q; i += step) dst[i] = src[i];
    int* kc = reinterpret_cast<int*>(slot + L.off_kc);
    unsigned char* bf = slot + L.off_bf;
    for (size_t i = t0; i < (size_t)2 * L.nr; i += step) {
        kc[i] = a.kcount[i];
        bf[i] = a.bflags[i];
    }
}

// Reverse of the update step (mark 1: h_{j+1} = h_j - m; mark 0: mode = h_j, h_{j+1} = h_j)
// and of the mean-envelope overwrite m = (U + L)/2: gh, gm hold the adjoints of h and m;
// eb receives the adjoint of each envelope.  Grid (x: samples, y: realization).
__global__ void k_adj_seed(const unsigned char* slot, TapeLayout L, int n, double* gh,
                           double* gm, double* eb, const double* abar, double inr) {
    const Slot v = view(slot, L);
    const int r = blockIdx.y;
    const bool sub = v.mark[r] == 1;
    const bool upd = updated(v, L.nr, r);
    const size_t base = (size_t)r * n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double m = gm[base + k];
        if (sub) {
            m = m - gh[base + k];
        } else {
            gh[base + k] = gh[base + k] + (-(abar[k] * inr));
        }
        if (upd) {
            eb[base + k] = m * 0.5;
            m = 0.0;
        }
        gm[base + k] = m;
    }
}

// Knot positions of spline sp from its recorded bitmaps (the whole CTA: a scan of the words'
// popcounts, kAdjThreads words per pass).
__device__ __forceinline__ void adj_knots_cta(const Slot& v, const TapeLayout& L, int cap, int sp,
                                              int32_t* kx, int* s_scan) {
    const int W = L.ntiles * kTileWords;
    const unsigned* bw = v.bits + (size_t)sp * W;
    int32_t* out = kx + (size_t)sp * cap;
    int carry = 0;
    for (int c0 = 0; c0 < W; c0 += kAdjThreads) {
        const int wi = c0 + threadIdx.x;
        unsigned w = wi < W ? bw[wi] : 0u;
        const int c = __popc(w);
        s_scan[threadIdx.x] = c;
        __syncthreads();
        for (int o = 1; o < kAdjThreads; o <<= 1) {
            const int t = threadIdx.x >= o ? s_scan[threadIdx.x - o] : 0;
            __syncthreads();
            s_scan[threadIdx.x] += t;
            __syncthreads();
        }
        int pos = carry + s_scan[threadIdx.x] - c;
        const int total = s_scan[kAdjThreads - 1];
        const int base = (wi / kTileWords) * kTileSamples + (wi % kTileWords) * 32;
        while (w) {
            const int b = __ffs(w) - 1;
            if (pos < cap) out[pos] = base + b;
            ++pos;
            w &= w - 1;
        }
        carry += total;
        __syncthreads();
    }
}

// Knot positions of one spline (one CTA per spline e*nr + r) from its recorded bitmaps.
__global__ void __launch_bounds__(kAdjThreads)
k_adj_knots(const unsigned char* slot, TapeLayout L, int cap, int32_t* kx) {
    __shared__ int s_scan[kAdjThreads];
    const Slot v = view(slot, L);
    const int sp = blockIdx.x;
    if (!updated(v, L.nr, sp % L.nr)) return;
    adj_knots_cta(v, L, cap, sp, kx, s_scan);
}

// Segment sums of eb * t^p (p = 0..3) over segment s = (x_s, x_{s+1}] (sample 0 in segment 0),
// in sample order; one thread per segment.  S: 4 planes of [2*nr][cap].
__device__ __forceinline__ void adj_segsum_one(const Slot& v, const TapeLayout& L, int n, int cap,
                                               const int32_t* kx, const double* eb, double* S,
                                               int sp, int s) {
    const int r = sp % L.nr;
    if (s >= knots(v, sp, cap) - 1) return;
    const int32_t* x = kx + (size_t)sp * cap;
    const double* e = eb + (size_t)r * n;
    const int x0 = x[s], x1 = x[s + 1];
    if (x0 < 0 || x1 >= n || x1 <= x0) return;  // knots increase inside 0..n-1
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    for (int i = s == 0 ? x0 : x0 + 1; i <= x1; ++i) {
        const double t = (double)(i - x0);
        const double ev = e[i];
        const double p1 = ev * t, p2 = p1 * t, p3 = p2 * t;
        a0 = a0 + ev;
        a1 = a1 + p1;
        a2 = a2 + p2;
        a3 = a3 + p3;
    }
    const size_t plane = (size_t)2 * L.nr * cap;
    double* o = S + (size_t)sp * cap + s;
    o[0] = a0;
    o[plane] = a1;
    o[2 * plane] = a2;
    o[3 * plane] = a3;
}

__global__ void __launch_bounds__(kAdjThreads)
k_adj_segsums(const unsigned char* slot, TapeLayout L, int n, int cap, const int32_t* kx,
              const double* eb, double* S) {
    const Slot v = view(slot, L);
    const int sp = blockIdx.y;
    if (!updated(v, L.nr, sp % L.nr)) return;
    adj_segsum_one(v, L, n, cap, kx, eb, S, sp, blockIdx.x * blockDim.x + threadIdx.x);
}

// Transposed coefficient maps (a = y_s, b = (y_{s+1}-y_s)/h - h(2c_s+c_{s+1})/3, c = c_s,
// d = (c_{s+1}-c_s)/(3h)): per knot the adjoint of y from its two segments (yb) and of c,
// which becomes the right-hand side of the transposed solve (interior rows; the end rows are
// identity rows with zero right-hand side).  One thread per knot.
__device__ __forceinline__ void adj_rows_one(const Slot& v, const TapeLayout& L, int cap,
                                             const int32_t* kx, const double* S, double* yb,
                                             double* sys, bool rhs_only, int sp, int i) {
    const int K = knots(v, sp, cap);
    if (i >= K) return;
    const int32_t* x = kx + (size_t)sp * cap;
    const size_t plane = (size_t)2 * L.nr * cap;
    const double* s0 = S + (size_t)sp * cap;
    const double* s1 = s0 + plane;
    const double* s2 = s1 + plane;
    const double* s3 = s2 + plane;
    double y = 0.0, cb = 0.0;
    if (i + 1 < K) {
        const double h = (double)(x[i + 1] - x[i]);
        y = s0[i] - s1[i] / h;
        cb = (s2[i] - s1[i] * (2.0 * h / 3.0)) - s3[i] / (3.0 * h);
    }
    if (i > 0) {
        const double h = (double)(x[i] - x[i - 1]);
        y = y + s1[i - 1] / h;
        cb = cb + (s3[i - 1] / (3.0 * h) - s1[i - 1] * (h / 3.0));
    }
    yb[(size_t)sp * cap + i] = y;
    double* R = sys + (size_t)sp * 4 * cap;
    if (rhs_only) {  // the level-by-level solve rebuilds l, m, u from the knots
        R[3 * (size_t)cap + i] = (i == 0 || i == K - 1) ? 0.0 : cb;
        return;
    }
    if (i == 0 || i == K - 1) {
        R[i] = 0.0;
        R[cap + i] = 1.0;
        R[2 * (size_t)cap + i] = 0.0;
        R[3 * (size_t)cap + i] = 0.0;
    } else {
        const int dl = x[i] - x[i - 1], du = x[i + 1] - x[i];
        R[i] = (double)dl;
        R[cap + i] = (double)(2 * (dl + du));
        R[2 * (size_t)cap + i] = (double)du;
        R[3 * (size_t)cap + i] = cb;
    }
}

__global__ void __launch_bounds__(kAdjThreads)
k_adj_rows(const unsigned char* slot, TapeLayout L, int cap, const int32_t* kx, const double* S,
           double* yb, double* sys, int* nrows) {
    const Slot v = view(slot, L);
    const int sp = blockIdx.y;
    const bool upd = updated(v, L.nr, sp % L.nr);
    // the system sizes for the level-by-level solve (0: no solve for this spline)
    if (nrows && blockIdx.x == 0 && threadIdx.x == 0) nrows[sp] = upd ? knots(v, sp, cap) : 0;
    if (!upd) return;
    adj_rows_one(v, L, cap, kx, S, yb, sys, nrows != nullptr, sp,
                 blockIdx.x * blockDim.x + threadIdx.x);
}

// Transposed spline solve: one CTA per spline, the canonical partitioned solve.
__global__ void __launch_bounds__(kAdjThreads)
k_adj_solve(const unsigned char* slot, TapeLayout L, int cap, const double* sys, double* z,
            double* ws, size_t ws_stride) {
    const Slot v = view(slot, L);
    const int sp = blockIdx.x;
    if (!updated(v, L.nr, sp % L.nr)) return;
    cta_tridiag(knots(v, sp, cap), sys + (size_t)sp * 4 * cap, cap, z + (size_t)sp * cap,
                ws + (size_t)sp * ws_stride);
}

// Transposed right-hand side r_i = 3((y_{i+1}-y_i)/du_i - (y_i-y_{i-1})/dl_i), interior i.
__device__ __forceinline__ void adj_rhs_one(const Slot& v, const TapeLayout& L, int cap,
                                            const int32_t* kx, const double* yb, const double* z,
                                            double* y2, int sp, int i) {
    const int K = knots(v, sp, cap);
    if (i >= K) return;
    const int32_t* x = kx + (size_t)sp * cap;
    const double* zz = z + (size_t)sp * cap;
    double y = yb[(size_t)sp * cap + i];
    if (i >= 2) y = y + (3.0 * zz[i - 1]) / (double)(x[i] - x[i - 1]);
    if (i >= 1 && i <= K - 2)
        y = y - ((3.0 * zz[i]) / (double)(x[i + 1] - x[i]) +
                 (3.0 * zz[i]) / (double)(x[i] - x[i - 1]));
    if (i + 1 <= K - 2) y = y + (3.0 * zz[i + 1]) / (double)(x[i + 1] - x[i]);
    y2[(size_t)sp * cap + i] = y;
}

__global__ void __launch_bounds__(kAdjThreads)
k_adj_rhs(const unsigned char* slot, TapeLayout L, int cap, const int32_t* kx, const double* yb,
          const double* z, double* y2) {
    const Slot v = view(slot, L);
    const int sp = blockIdx.y;
    if (!updated(v, L.nr, sp % L.nr)) return;
    adj_rhs_one(v, L, cap, kx, yb, z, y2, sp, blockIdx.x * blockDim.x + threadIdx.x);
}

// Transposed end rule and scatter of the knot adjoints to their samples, both envelopes of
// realization r (grid y).  Interior knots of the two envelopes sit on different samples (a
// strict maximum is no strict minimum); thread 0 adds the two end samples, maxima first.
__global__ void __launch_bounds__(kAdjThreads)
k_adj_scatter(const unsigned char* slot, TapeLayout L, int n, int cap, const int32_t* kx,
              const double* y2, double* gh) {
    const Slot v = view(slot, L);
    const int r = blockIdx.y;
    if (!updated(v, L.nr, r)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double* g = gh + (size_t)r * n;
    for (int e = 0; e < 2; ++e) {
        const int sp = e * L.nr + r;
        const int K = knots(v, sp, cap);
        if (i >= 1 && i <= K - 2) {
            const int32_t* x = kx + (size_t)sp * cap;
            const int xi = x[i];
            if (xi > 0 && xi < n - 1)  // interior knots sit on interior samples
                g[xi] = g[xi] + end_rule_adjoint(x, y2 + (size_t)sp * cap, K, v.bf[sp], i);
        }
    }
    if (i == 0) {
        double g0 = g[0], gl = g[n - 1];
        for (int e = 0; e < 2; ++e) {
            const int sp = e * L.nr + r;
            const int K = knots(v, sp, cap);
            const int32_t* x = kx + (size_t)sp * cap;
            const double* yy = y2 + (size_t)sp * cap;
            g0 = g0 + end_rule_adjoint(x, yy, K, v.bf[sp], 0);
            gl = gl + end_rule_adjoint(x, yy, K, v.bf[sp], K - 1);
        }
        g[0] = g0;
        g[n - 1] = gl;
    }
}

// Adjoint of a stage's ensemble mean f_i: abar = fbar - g_i (IMF_i = f_{i-1} - f_i).
__global__ void k_adj_abar(const double* fbar, const double* g, double* abar, size_t n) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x)
        abar[k] = fbar[k] - g[k];
}

// Adjoint of every realization's stage input h0_r = (sift adjoint) + abar/NR, summed over the
// realizations in order (hs) and weighted by the stage's noise mode (p).
__global__ void k_adj_inject(const double* gh, const double* abar, double inr, const double* E,
                             int nr, size_t n, double* hs, double* p) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double s1 = 0.0, s2 = 0.0;
        for (int r = 0; r < nr; ++r) {
            const double hb = gh[(size_t)r * n + k] + abar[k] * inr;
            s1 = s1 + hb;
            s2 = s2 + hb * E[(size_t)r * n + k];
        }
        hs[k] = s1;
        p[k] = s2;
    }
}

// Reverse of the stage statistics (one CTA of kLanes threads; canonical sums: lane t adds
// elements t, t+256, ... in order, then a halving tree).  Stage i >= 1:
//   h0 = f + nstd*E*sqrt(var), var = (var_prev + sum (f-mu)^2)/(n-1), mu = (mu_prev + sum f)/n
// stage 0: xs = y/sqrt(var), h0 = xs + noise, with var, mu of y.  scal: [0] adjoint of the
// carried variance, [1] of the carried mean (both from the stage above), [2] qbar, [3] mubar,
// [4] 1/sqrt(var) of stage 0.
__global__ void __launch_bounds__(kLanes)
k_adj_stats(int stage, const double* f, const double* stats, const double* p, const double* g,
            const double* hs, size_t n, double nstd, double inv_n, double inv_nm1,
            double* scal) {
    __shared__ double sh[kLanes];
    const int t = threadIdx.x;
    const double mu = stats[2 * stage], var = stats[2 * stage + 1];
    double acc = 0.0;
    for (size_t k = t; k < n; k += kLanes) acc = acc + (f[k] - mu);
    sh[t] = acc;
    __syncthreads();
    for (int s = kLanes / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] = sh[t] + sh[t + s];
        __syncthreads();
    }
    const double D = sh[0];
    __syncthreads();
    acc = 0.0;
    if (stage >= 1) {
        for (size_t k = t; k < n; k += kLanes) acc = acc + p[k];
    } else {
        for (size_t k = t; k < n; k += kLanes) {
            const double xb = g[k] + hs[k];
            acc = acc + xb * f[k];
        }
    }
    sh[t] = acc;
    __syncthreads();
    for (int s = kLanes / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] = sh[t] + sh[t + s];
        __syncthreads();
    }
    if (t == 0) {
        const double P = sh[0];
        double vbar;
        if (stage >= 1) {
            const double sq = sqrt(var);
            vbar = scal[0] + (nstd * P) * (0.5 / sq);
        } else {
            const double sc = 1.0 / sqrt(var);
            scal[4] = sc;
            vbar = scal[0] + P * (-0.5 * sc / var);
        }
        const double qbar = vbar * inv_nm1;
        const double mubar = scal[1] + qbar * (-2.0 * D);
        scal[2] = qbar;
        scal[3] = mubar;
        scal[0] = vbar * inv_nm1;
        scal[1] = mubar * inv_n;
    }
}

// Adjoint of the stage input: f_{i-1} (stage i >= 1, into fbar) or y (stage 0, the result).
__global__ void k_adj_out(int stage, const double* g, const double* hs, const double* f,
                          const double* stats, const double* scal, double* out, size_t n,
                          double inv_n) {
    const double mu = stats[2 * stage];
    const double qbar = scal[2], mubar = scal[3];
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const double dv = f[k] - mu;
        const double tail = qbar * (2.0 * dv) + mubar * inv_n;
        out[k] = stage >= 1 ? (g[k] + hs[k]) + tail : (g[k] + hs[k]) * scal[4] + tail;
    }
}

}  // namespace ceemdan
