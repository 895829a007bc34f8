// Canonical arithmetic of the engine: every floating-point step whose order or fusion
// decides the rounding is written here once, with explicit fma(), and the whole library
// is compiled with -fmad=false so nvcc adds no contraction of its own.
//
// The reference computes these steps in (cudaICEEMDAN.cu):
//   setBoundaryMax/Min          :210-291   (end-knot extrapolation)
//   tridiagonal_setup           :311-343   (natural-spline rows)
//   cusparseDgtsv2_nopivot      :1622-1641 (closed library: replaced by the canonical
//                                           partitioned solve below)
//   spline_coefficients         :383-401
//   interpolate                 :404-439
// A one-ulp difference anywhere changes later extrema and stop decisions (the sifting
// iteration is chaotic at the rounding level), so the CPU oracle evaluates this exact
// sequence too.
#pragma once
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define CEEMDAN_HD __host__ __device__ __forceinline__
#define CEEMDAN_HD_COLD static __host__ __device__ __noinline__
#else
#define CEEMDAN_HD inline
#define CEEMDAN_HD_COLD static inline
using std::fabs;
using std::fma;
#endif

#ifndef CEEMDAN_CHUNK
#define CEEMDAN_CHUNK 16  // rows per chunk of the partitioned spline solve
#endif

namespace ceemdan {

constexpr int kChunk = CEEMDAN_CHUNK;
constexpr int kLanes = 256;  // lanes of the canonical reductions

struct Row {
    double l, m, u, r;
};

// End-knot extrapolation (setBoundaryMax/Min): applied when count-1 > 4.
// kind 0 = maxima (keep the larger value), 1 = minima (keep the smaller value).
CEEMDAN_HD double boundary_left(int kind, int32_t x0, int32_t x1, int32_t x2,
                                                double y0, double y1, double y2) {
    const double sl = (y2 - y1) / (double)(x2 - x1);
    const double t = fma(-sl, (double)(x1 - x0), y1);
    return kind == 0 ? (t > y0 ? t : y0) : (t < y0 ? t : y0);
}
CEEMDAN_HD double boundary_right(int kind, int32_t xa, int32_t xb, int32_t xL,
                                                 double ya, double yb, double yL) {
    // xa = x[L-2], xb = x[L-1], xL = x[L]
    const double sr = (yb - ya) / (double)(xb - xa);
    const double t = fma(sr, (double)(xL - xb), yb);
    return kind == 0 ? (t > yL ? t : yL) : (t < yL ? t : yL);
}

// Correctly rounded a / d from y = RN(1/d) (Markstein's theorem: q0 = RN(a*y) is within one
// ulp of a/d, r = a - d*q0 is exact with one fma, RN(q0 + r*y) = RN(a/d)).  Three FP64 ops in
// place of a division; zero, tiny and non-finite operands take the division (keeps the sign of
// zero and stays clear of underflow, where the theorem's assumptions fail).
CEEMDAN_HD double div_plain(double a, double d) { return a / d; }

CEEMDAN_HD double div_rcp(double a, double d, double y) {
    const double q0 = a * y;
    const double r = fma(-q0, d, a);
    const double q1 = fma(r, y, q0);
    if (!(fabs(a) > 0x1p-960) || !(fabs(q1) < 0x1p+1000)) return div_plain(a, d);
    return q1;
}

constexpr double kRcp3 = 1.0 / 3.0;  // RN(1/3)

// Segment slope (y1-y0)/(x1-x0): shared by the spline rows and the b coefficient.
CEEMDAN_HD double seg_slope(int32_t x0, int32_t x1, double y0, double y1) {
    return (y1 - y0) / (double)(x1 - x0);
}

// Interior row i of the natural spline system from its two adjacent slopes.
CEEMDAN_HD Row spline_row(int32_t xm, int32_t x0, int32_t xp, double s_prev,
                                          double s_next) {
    const int dl = x0 - xm;
    const int du = xp - x0;
    Row w;
    w.l = (double)dl;
    w.u = (double)du;
    w.m = (double)(2 * (dl + du));
    w.r = 3.0 * (s_next - s_prev);
    return w;
}

CEEMDAN_HD Row identity_row() {
    Row w;
    w.l = 0.0;
    w.m = 1.0;
    w.u = 0.0;
    w.r = 0.0;
    return w;
}

// Forward step of the canonical Thomas sweep: returns the reciprocal pivot 1/w.
CEEMDAN_HD double pivot_rcp(const Row& w, double cp_prev) {
    return 1.0 / fma(-w.l, cp_prev, w.m);
}

// Reduced-system row for separator row s, between a left chunk (last-row values gb, ab, bb)
// and a right chunk (first-row values ga, aa, ba).
CEEMDAN_HD Row reduced_row(const Row& s, double gb, double ab, double bb,
                                           double ga, double aa, double ba) {
    Row o;
    o.l = s.l * ab;
    o.m = fma(s.u, aa, fma(s.l, bb, s.m));
    o.u = s.u * ba;
    o.r = fma(-s.u, ga, fma(-s.l, gb, s.r));
    return o;
}

// Spline segment coefficients (spline_coefficients): b and d of segment [x0, x1].
CEEMDAN_HD void seg_coeffs(int32_t x0, int32_t x1, double y0, double y1,
                                           double c0, double c1, double& b, double& d) {
    const double h = (double)(x1 - x0);
    const double q = fma(2.0, c0, c1);
    b = (y1 - y0) / h - (h * q) / 3.0;
    d = (c1 - c0) / (3.0 * h);
}

// Horner evaluation a + t(b + t(c + t d)) as the reference's contracted form.
CEEMDAN_HD double seg_eval(double a, double b, double c, double d, double t) {
    return fma(fma(fma(d, t, c), t, b), t, a);
}

// Sifting statistic |(U+L)/(U-L)| (produceSX).
CEEMDAN_HD double sx_value(double up, double lo) {
    return fabs((up + lo) / (up - lo));
}

CEEMDAN_HD bool sx_value_greater(double up, double lo, double t) {
    return sx_value(up, lo) > t;
}

// Exactly (sx_value(up, lo) > t) for a threshold t > 0, without the division in all but
// near-tie cases (p = |U+L|, q = |U-L| as rounded sums).  With Q = |U+L| / |U-L| (exact), fl(Q) > t holds when Q >= t(1+2^-50) and
// fails when Q <= t(1-2^-50); the products below decide those two cases with margin for
// their own rounding (relative error <= 2^-52 each), and everything else -- near ties,
// zero / infinite / NaN / extreme magnitudes -- takes the division.
CEEMDAN_HD bool sx_greater_pq(double p, double q, double up, double lo, double t) {
    if (q > 0x1p-900 && q < 0x1p+900 && p < 0x1p+900) {
        const double z = t * q;
        if (p > z * (1.0 + 0x1p-49)) return true;
        if (p < z * (1.0 - 0x1p-49)) return false;
    }
    return sx_value_greater(up, lo, t);
}

CEEMDAN_HD bool sx_greater(double up, double lo, double t) {
    return sx_greater_pq(fabs(up + lo), fabs(up - lo), up, lo, t);
}

}  // namespace ceemdan
