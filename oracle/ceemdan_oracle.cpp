/*
 * ORACLE — test infrastructure only (see ceemdan_oracle.h for the contract).
 *
 * Every function below names the reference lines it restates.  Reference paths are
 * relative to the EEGLab-Pannon/CEEMDAN-GPU project root.
 *
 * Build: -O2 -ffp-contract=off -fopenmp (no implicit contraction: every fused
 * multiply-add the reference gets from nvcc's default contraction is an explicit fma()).
 */
#include "ceemdan_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using std::fma;
using std::vector;

/* ------------------------------------------------------------------------------------ */
/* canonical reductions: 256 lanes, lane t sums v[t], v[t+256], ... in order, then a     */
/* halving tree (s = 128 .. 1: p[t] += p[t+s]).  statistics.cu:167-241 reduces with      */
/* shuffles + atomics in an unspecified order; this order is the one the engine uses.    */
/* ------------------------------------------------------------------------------------ */
constexpr int kLanes = 256;

double tree256(double* p) {
    for (int s = kLanes / 2; s > 0; s >>= 1)
        for (int t = 0; t < s; ++t) p[t] = p[t] + p[t + s];
    return p[0];
}

double canon_sum(const double* v, size_t n) {
    double p[kLanes];
    for (int t = 0; t < kLanes; ++t) {
        double acc = 0.0;
        for (size_t i = (size_t)t; i < n; i += kLanes) acc = acc + v[i];
        p[t] = acc;
    }
    return tree256(p);
}

/* varianceD accumulates (x-mean)*(x-mean), contracted to fma(d, d, acc). */
double canon_sqdev(const double* v, size_t n, double mean) {
    double p[kLanes];
    for (int t = 0; t < kLanes; ++t) {
        double acc = 0.0;
        for (size_t i = (size_t)t; i < n; i += kLanes) {
            double d = v[i] - mean;
            acc = fma(d, d, acc);
        }
        p[t] = acc;
    }
    return tree256(p);
}

/* ------------------------------------------------------------------------------------ */
/* extrema: find_extrema_shfl_max/min (cudaICEEMDAN.cu:93-148) + exclusive scan +         */
/* select_extrema_max/min (:151-207).  Strict comparisons; both end samples forced.      */
/* ------------------------------------------------------------------------------------ */
int extrema(const double* h, int n, int kind, int32_t* kx, double* ky) {
    int k = 0;
    for (int i = 0; i < n; ++i) {
        bool f;
        if (i == 0 || i == n - 1) {
            f = true;
        } else if (kind == 0) {
            f = h[i] > h[i - 1] && h[i] > h[i + 1];
        } else {
            f = h[i] < h[i - 1] && h[i] < h[i + 1];
        }
        if (f) {
            kx[k] = i;
            ky[k] = h[i];
            ++k;
        }
    }
    return k;
}

/* setBoundaryMax/Min (cudaICEEMDAN.cu:210-291): applied when scan[N-1] = count-1 > 4.
 * Returns which end values the extrapolation replaced (bit 0 left, bit 1 right). */
int boundary(int count, const int32_t* kx, double* ky, int kind) {
    if (count - 1 <= 4) return 0;
    const int L = count - 1;
    // left end: t = y1 - slope*(x1-x0), contracted to fma(-slope, dx, y1)
    double sl = (ky[2] - ky[1]) / (double)(kx[2] - kx[1]);
    double tl = fma(-sl, (double)(kx[1] - kx[0]), ky[1]);
    // right end: t = y[L-1] + slope*(x[L]-x[L-1])
    double sr = (ky[L - 1] - ky[L - 2]) / (double)(kx[L - 1] - kx[L - 2]);
    double tr = fma(sr, (double)(kx[L] - kx[L - 1]), ky[L - 1]);
    const bool lrep = kind == 0 ? tl > ky[0] : tl < ky[0];
    const bool rrep = kind == 0 ? tr > ky[L] : tr < ky[L];
    if (lrep) ky[0] = tl;
    if (rrep) ky[L] = tr;
    return (lrep ? 1 : 0) | (rrep ? 2 : 0);
}

/* ------------------------------------------------------------------------------------ */
/* tridiagonal solves                                                                    */
/* ------------------------------------------------------------------------------------ */
void thomas(int n, const double* l, const double* m, const double* u, const double* r,
            double* x) {
    vector<double> cp(n), gp(n);
    double w = m[0];
    cp[0] = u[0] / w;
    gp[0] = r[0] / w;
    for (int k = 1; k < n; ++k) {
        w = fma(-l[k], cp[k - 1], m[k]);
        cp[k] = u[k] / w;
        gp[k] = fma(-l[k], gp[k - 1], r[k]) / w;
    }
    x[n - 1] = gp[n - 1];
    for (int k = n - 2; k >= 0; --k) x[k] = fma(-cp[k], x[k + 1], gp[k]);
}

/* Canonical Thomas (base case of the partitioned solve): one reciprocal per row,
 * iw = 1/w, then products; the CUDA engine evaluates the identical sequence. */
void thomas_canon(int n, const double* l, const double* m, const double* u, const double* r,
                  double* x) {
    vector<double> cp(n), gp(n);
    double iw = 1.0 / m[0];
    cp[0] = u[0] * iw;
    gp[0] = r[0] * iw;
    for (int k = 1; k < n; ++k) {
        iw = 1.0 / fma(-l[k], cp[k - 1], m[k]);
        cp[k] = u[k] * iw;
        gp[k] = fma(-l[k], gp[k - 1], r[k]) * iw;
    }
    x[n - 1] = gp[n - 1];
    for (int k = n - 2; k >= 0; --k) x[k] = fma(-cp[k], x[k + 1], gp[k]);
}

/* End relations of one chunk (rows a..b) of the canonical partitioned solve.  With the
 * separator values xL = x[a-1] and xR = x[b+1] moved to the right-hand side,
 *   x_b = gb + ab*xL + bb*xR   (top-down elimination, running values only)
 *   x_a = ga + aa*xL + ba*xR   (bottom-up elimination, running values only). */
struct Ends {
    double ga, aa, ba, gb, ab, bb;
};

Ends chunk_ends(int a, int b, const double* l, const double* m, const double* u,
                const double* r) {
    Ends e;
    // top-down
    double iw = 1.0 / m[a];
    double cp = u[a] * iw, gp = r[a] * iw, ap = -l[a] * iw;
    for (int i = a + 1; i <= b; ++i) {
        iw = 1.0 / fma(-l[i], cp, m[i]);
        cp = u[i] * iw;
        gp = fma(-l[i], gp, r[i]) * iw;
        ap = (-l[i] * ap) * iw;
    }
    e.gb = gp;
    e.ab = ap;
    e.bb = -u[b] * iw;
    // bottom-up
    double iv = 1.0 / m[b];
    double cq = l[b] * iv, gq = r[b] * iv, bq = -u[b] * iv;
    for (int i = b - 1; i >= a; --i) {
        iv = 1.0 / fma(-u[i], cq, m[i]);
        cq = l[i] * iv;
        gq = fma(-u[i], gq, r[i]) * iv;
        bq = (-u[i] * bq) * iv;
    }
    e.ga = gq;
    e.ba = bq;
    e.aa = -l[a] * iv;
    return e;
}

/* Interior of chunk a..b once its separators are known: the coupling terms move to the
 * right-hand side (r_a - l_a*xL, r_b - u_b*xR) and the chunk is solved by canonical Thomas
 * (l_a and u_b no longer enter). */
void chunk_interior(int a, int b, const double* l, const double* m, const double* u,
                    const double* r, double xl, double xr, double* x) {
    const int len = b - a + 1;
    double cp[64] = {0}, gp[64] = {0};  // len >= 1 rows are always written
    for (int k = 0; k < len; ++k) {
        const int i = a + k;
        double ri = r[i];
        if (k == 0) ri = fma(-l[i], xl, ri);
        if (k == len - 1) ri = fma(-u[i], xr, ri);
        if (k == 0) {
            const double iw = 1.0 / m[i];
            cp[0] = u[i] * iw;
            gp[0] = ri * iw;
        } else {
            const double iw = 1.0 / fma(-l[i], cp[k - 1], m[i]);
            cp[k] = u[i] * iw;
            gp[k] = fma(-l[i], gp[k - 1], ri) * iw;
        }
    }
    double xv = gp[len - 1];
    x[a + len - 1] = xv;
    for (int k = len - 2; k >= 0; --k) {
        xv = fma(-cp[k], xv, gp[k]);
        x[a + k] = xv;
    }
}

/* Canonical partitioned solve.  Systems of n <= S rows: canonical Thomas.  Otherwise
 * separators at rows s_p = p*S + S-1 (p = 0..P-1, P = (n-1)/S), chunks of S-1 rows between
 * them and a last chunk of 1..S rows; the reduced tridiagonal system on the separators
 * (built from the chunk end relations) is solved the same way, recursively, and each chunk
 * interior is then solved with its separator values. */
void partitioned(int n, const double* l, const double* m, const double* u, const double* r,
                 double* x, int S) {
    if (n <= S) {
        thomas_canon(n, l, m, u, r, x);
        return;
    }
    const int P = (n - 1) / S;
    vector<Ends> ends(P + 1);
    for (int q = 0; q <= P; ++q) {
        const int a = q * S;
        const int b = (q < P) ? q * S + S - 2 : n - 1;
        ends[q] = chunk_ends(a, b, l, m, u, r);
    }
    vector<double> RL(P), RM(P), RU(P), RR(P), X(P);
    for (int p = 0; p < P; ++p) {
        const int s = p * S + S - 1;
        RL[p] = l[s] * ends[p].ab;
        RM[p] = fma(u[s], ends[p + 1].aa, fma(l[s], ends[p].bb, m[s]));
        RU[p] = u[s] * ends[p + 1].ba;
        RR[p] = fma(-u[s], ends[p + 1].ga, fma(-l[s], ends[p].gb, r[s]));
    }
    partitioned(P, RL.data(), RM.data(), RU.data(), RR.data(), X.data(), S);
    for (int q = 0; q <= P; ++q) {
        const int a = q * S;
        const int b = (q < P) ? q * S + S - 2 : n - 1;
        const double xl = (q > 0) ? X[q - 1] : 0.0;
        const double xr = (q < P) ? X[q] : 0.0;
        chunk_interior(a, b, l, m, u, r, xl, xr, x);
        if (q < P) x[b + 1] = X[q];
    }
}

/* tridiagonal_setup (cudaICEEMDAN.cu:311-343), natural end conditions, on K knots. */
void spline_system(int K, const int32_t* kx, const double* ky, double* l, double* m,
                   double* u, double* r) {
    l[0] = 0.0; m[0] = 1.0; u[0] = 0.0; r[0] = 0.0;
    l[K - 1] = 0.0; m[K - 1] = 1.0; u[K - 1] = 0.0; r[K - 1] = 0.0;
    for (int i = 1; i < K - 1; ++i) {
        const int dl = kx[i] - kx[i - 1];
        const int du = kx[i + 1] - kx[i];
        l[i] = (double)dl;
        u[i] = (double)du;
        m[i] = (double)(2 * (dl + du));
        const double sn = (ky[i + 1] - ky[i]) / (double)du;
        const double sp = (ky[i] - ky[i - 1]) / (double)dl;
        r[i] = 3.0 * (sn - sp);
    }
}

/* Canonical spline solve: the first partition level is aligned to the engine's 2048-sample
 * tiles.  Within the knots of each tile, local indices 0, S, 2S, ... and the tile's last knot
 * are separators, so every chunk lies inside one tile (knot 0 and knot K-1 are separators and
 * the chunks before / after them are empty).  Empty chunks (adjacent separators) have the end
 * relations x_{s-1} = x_{s_prev} and x_{s+1} = x_{s_next}.  The separator system is solved by
 * the index-partitioned recursion (partitioned), then each chunk interior by
 * chunk_interior. */
constexpr int kTileSamples = ORACLE_TILE_SAMPLES;

void spline_solve_tiled(int K, const int32_t* kx, const double* l, const double* m,
                        const double* u, const double* r, double* c, int S) {
    vector<int> sep;
    for (int i = 0; i < K;) {
        const int t = kx[i] / kTileSamples;
        int j = i;
        while (j < K && kx[j] / kTileSamples == t) ++j;
        const int cnt = j - i;
        for (int q = 0; q < cnt; ++q)
            if (q % S == 0 || q == cnt - 1) sep.push_back(i + q);
        i = j;
    }
    const int P = (int)sep.size();
    vector<Ends> ends(P + 1);
    for (int q = 0; q <= P; ++q) {
        const int a = (q == 0) ? 0 : sep[q - 1] + 1;
        const int b = (q == P) ? K - 1 : sep[q] - 1;
        if (a > b) {
            ends[q].ga = 0.0; ends[q].aa = 0.0; ends[q].ba = 1.0;
            ends[q].gb = 0.0; ends[q].ab = 1.0; ends[q].bb = 0.0;
        } else {
            ends[q] = chunk_ends(a, b, l, m, u, r);
        }
    }
    vector<double> RL(P), RM(P), RU(P), RR(P), X(P);
    for (int p = 0; p < P; ++p) {
        const int s = sep[p];
        RL[p] = l[s] * ends[p].ab;
        RM[p] = fma(u[s], ends[p + 1].aa, fma(l[s], ends[p].bb, m[s]));
        RU[p] = u[s] * ends[p + 1].ba;
        RR[p] = fma(-u[s], ends[p + 1].ga, fma(-l[s], ends[p].gb, r[s]));
    }
    partitioned(P, RL.data(), RM.data(), RU.data(), RR.data(), X.data(), S);
    for (int q = 1; q < P; ++q) {
        const int a = sep[q - 1] + 1, b = sep[q] - 1;
        if (a <= b) chunk_interior(a, b, l, m, u, r, X[q - 1], X[q], c);
    }
    for (int p = 0; p < P; ++p) c[sep[p]] = X[p];
}

void spline_solve(int K, const int32_t* kx, const double* ky, double* c, int solver, int S) {
    vector<double> l(K), m(K), u(K), r(K);
    spline_system(K, kx, ky, l.data(), m.data(), u.data(), r.data());
    if (solver == 1)
        spline_solve_tiled(K, kx, l.data(), m.data(), u.data(), r.data(), c, S);
    else
        thomas(K, l.data(), m.data(), u.data(), r.data(), c);
}

/* spline_coefficients (:383-401) + interpolate (:404-439).  Sample n > 0 uses the segment
 * s with x[s] < n <= x[s+1]; sample 0 uses segment 0 at t = 0.  Horner form contracted to
 * fma(fma(fma(d,t,c),t,b),t,a). */
void spline_eval(int n, int /*K*/, const int32_t* kx, const double* ky, const double* c,
                 double* env) {
    int seg = 0;
    double a = 0, b = 0, cc = 0, d = 0;
    int cur = -1;
    for (int i = 0; i < n; ++i) {
        if (i > 0)
            while (kx[seg + 1] < i) ++seg;
        if (seg != cur) {
            const double h = (double)(kx[seg + 1] - kx[seg]);
            const double q = fma(2.0, c[seg], c[seg + 1]);
            b = (ky[seg + 1] - ky[seg]) / h - (h * q) / 3.0;
            d = (c[seg + 1] - c[seg]) / (3.0 * h);
            cc = c[seg];
            a = ky[seg];
            cur = seg;
        }
        const double t = (double)(i - kx[seg]);
        env[i] = fma(fma(fma(d, t, cc), t, b), t, a);
    }
}

/* ------------------------------------------------------------------------------------ */
/* sifting                                                                               */
/* ------------------------------------------------------------------------------------ */
struct Ctx {
    size_t nr, n;
    double sd, sd2, tol;
    double inv_n;   /* 1.0/SignalLength, the multiplyD factor */
    int solver, chunk;
    vector<double> menv;   /* d_meanEnvelope, nr*n, persists for the whole call */
    vector<double> frac;   /* d_chanelMeansSiftingStop, nr, persists for the whole call */
    const oracle_split* split = nullptr;  /* realizations split over parts (nr = this part's) */
};

struct Scratch {
    vector<int32_t> kx;
    vector<double> ky, c, up, lo;
};

/* Frozen structure of one lock-step iteration of one realization: the knot positions of
 * both envelopes, which end values the extrapolation replaced, and the update mark. */
struct Step {
    vector<int32_t> kx[2];
    int bflag[2] = {0, 0};
    int mark = 1;
};

/* Frozen structure of one signal stage: J iterations x nr realizations, iteration-major. */
struct StageTape {
    int J = 0;
    vector<Step> it;
};

/* One sift iteration of one realization up to the criterion inputs (envelope pass,
 * cudaICEEMDAN.cu:1752-1851).  Returns the sx statistics; rec (optional) receives the
 * knots and end-value flags. */
void envelopes(Ctx& cx, size_t rz, const double* h, Scratch& s, int& kmax, int& kmin,
               int& any, long& cnt, Step* rec) {
    const int n = (int)cx.n;
    kmax = extrema(h, n, 0, s.kx.data(), s.ky.data());
    const int fmax = boundary(kmax, s.kx.data(), s.ky.data(), 0);
    if (rec) {
        rec->kx[0].assign(s.kx.begin(), s.kx.begin() + kmax);
        rec->bflag[0] = fmax;
    }
    spline_solve(kmax, s.kx.data(), s.ky.data(), s.c.data(), cx.solver, cx.chunk);
    spline_eval(n, kmax, s.kx.data(), s.ky.data(), s.c.data(), s.up.data());
    kmin = extrema(h, n, 1, s.kx.data(), s.ky.data());
    const int fmin = boundary(kmin, s.kx.data(), s.ky.data(), 1);
    if (rec) {
        rec->kx[1].assign(s.kx.begin(), s.kx.begin() + kmin);
        rec->bflag[1] = fmin;
    }
    spline_solve(kmin, s.kx.data(), s.ky.data(), s.c.data(), cx.solver, cx.chunk);
    spline_eval(n, kmin, s.kx.data(), s.ky.data(), s.c.data(), s.lo.data());
    double* me = cx.menv.data() + rz * cx.n;
    if (kmax > 3 && kmin > 3)  // averageUppperLower (:442-454)
        for (int i = 0; i < n; ++i) me[i] = (s.up[i] + s.lo[i]) / 2.0;
    any = 0;
    cnt = 0;
    for (int i = 0; i < n; ++i) {  // produceSX (:457-467) + thresholdJudge (:470-492)
        const double sx = std::fabs((s.up[i] + s.lo[i]) / (s.up[i] - s.lo[i]));
        if (sx > cx.sd2) any = 1;
        if (sx > cx.sd) ++cnt;
    }
}

/* Lock-step sift of all realizations of one stage (cudaICEEMDAN.cu:1572-1711 for the noise
 * modes, :1750-1867 / :1884-2002 for the signal stages).  h (nr*n) is sifted in place; each
 * realization's mode is written to modes when it finishes.  Returns iterations executed. */
int sift_stage(Ctx& cx, double* h, double* modes, size_t cap, StageTape* tape = nullptr) {
    const size_t nr = cx.nr, n = cx.n;
    vector<int> finish(nr, 0);
    int iters = 0;
    for (size_t j = 0; j < cap; ++j) {
        ++iters;
        if (tape) tape->it.resize((j + 1) * nr);
#pragma omp parallel
        {
            Scratch s;
            s.kx.resize(n); s.ky.resize(n); s.c.resize(n); s.up.resize(n); s.lo.resize(n);
#pragma omp for schedule(dynamic, 1)
            for (long rl = 0; rl < (long)nr; ++rl) {
                const size_t rz = (size_t)rl;
                double* hr = h + rz * n;
                int kmax, kmin, any;
                long cnt;
                Step* rec = tape ? &tape->it[j * nr + rz] : nullptr;
                envelopes(cx, rz, hr, s, kmax, kmin, any, cnt, rec);
                // meanD + multiplyD on the sx flags (:1851-1852): never-reset accumulator
                cx.frac[rz] = (cx.frac[rz] + (double)cnt) * cx.inv_n;
                // siftingCriterion (:495-525), C precedence a || (b && c)
                const bool crit = cx.frac[rz] > cx.tol || (any && (kmax + kmin) > 6);
                int mark;
                if (crit) {
                    mark = 1;
                    if (finish[rz] == 0 && j == cap - 1) {
                        mark = 0;
                        finish[rz] = 1;
                    }
                } else {
                    if (finish[rz] == 0) {
                        mark = 0;
                        finish[rz] = 1;
                    } else {
                        mark = 1;
                    }
                }
                if (rec) rec->mark = mark;
                // updateRealizations (:528-544)
                const double* me = cx.menv.data() + rz * n;
                if (mark == 1) {
                    for (size_t i = 0; i < n; ++i) hr[i] = hr[i] - me[i];
                } else {
                    std::memcpy(modes + rz * n, hr, n * sizeof(double));
                }
            }
        }
        bool all = true;
        for (size_t rz = 0; rz < nr; ++rz) all = all && finish[rz] == 1;
        if (cx.split) all = cx.split->all_finished(cx.split->ctx, all ? 1 : 0) != 0;
        if (all) break;
    }
    if (tape) tape->J = iters;
    return iters;
}

/* ------------------------------------------------------------------------------------ */
/* the decomposition: iceemdanD (cudaICEEMDAN.cu:1340-2059)                               */
/* ------------------------------------------------------------------------------------ */

/* Everything the reverse pass (and a frozen-structure replay) needs from one forward call.
 * The per-stage checkpoint (h0, and the mean-envelope and sifting-fraction carries at the
 * stage's start) is all the state a stage's sift depends on: re-running sift_stage from it
 * reproduces the stage's structure, so a reverse pass may recompute stages instead of
 * keeping their iterations. */
struct Tape {
    size_t nr = 0, n = 0, nimf = 0, max_iter = 0;
    double nstd = 0.0;
    vector<double> E;      /* num_imfs*nr*n noise modes */
    vector<double> menv0;  /* mean envelope left by the noise phase */
    vector<double> fin;    /* (num_imfs-1)*n: stage inputs, y for stage 0, f_{i-1} after */
    vector<double> mu, var;  /* carried stage statistics, as computed */
    vector<StageTape> st;  /* num_imfs-1 signal stages */
    vector<vector<double>> ck_h0, ck_menv, ck_frac;  /* per-stage checkpoints */
};

/* Frozen end-knot rule: the extrapolated end values of boundary(), taken where the
 * recording replaced them (flags bit 0 left, bit 1 right). */
void boundary_frozen(int count, const int32_t* kx, double* ky, int flags) {
    if (count - 1 <= 4) return;
    const int L = count - 1;
    const double sl = (ky[2] - ky[1]) / (double)(kx[2] - kx[1]);
    const double tl = fma(-sl, (double)(kx[1] - kx[0]), ky[1]);
    const double sr = (ky[L - 1] - ky[L - 2]) / (double)(kx[L - 1] - kx[L - 2]);
    const double tr = fma(sr, (double)(kx[L] - kx[L - 1]), ky[L - 1]);
    if (flags & 1) ky[0] = tl;
    if (flags & 2) ky[L] = tr;
}

/* Lock-step sift with the recorded structure (knots, end rule, marks, iteration count):
 * the map h -> modes that the reverse pass differentiates.  On the recorded input it repeats
 * sift_stage's arithmetic exactly. */
void sift_replay(Ctx& cx, double* h, double* modes, const StageTape& t) {
    const size_t nr = cx.nr, n = cx.n;
    for (int j = 0; j < t.J; ++j) {
#pragma omp parallel
        {
            vector<double> ky(n), c(n), up(n), lo(n);
#pragma omp for schedule(dynamic, 1)
            for (long rl = 0; rl < (long)nr; ++rl) {
                const size_t rz = (size_t)rl;
                const Step& s = t.it[(size_t)j * nr + rz];
                double* hr = h + rz * n;
                double* me = cx.menv.data() + rz * n;
                const int k0 = (int)s.kx[0].size(), k1 = (int)s.kx[1].size();
                if (k0 > 3 && k1 > 3) {
                    for (int e = 0; e < 2; ++e) {
                        const int K = e == 0 ? k0 : k1;
                        const int32_t* kx = s.kx[e].data();
                        for (int i = 0; i < K; ++i) ky[i] = hr[kx[i]];
                        boundary_frozen(K, kx, ky.data(), s.bflag[e]);
                        spline_solve(K, kx, ky.data(), c.data(), cx.solver, cx.chunk);
                        spline_eval((int)n, K, kx, ky.data(), c.data(), e == 0 ? up.data() : lo.data());
                    }
                    for (size_t i = 0; i < n; ++i) me[i] = (up[i] + lo[i]) / 2.0;
                }
                if (s.mark == 1) {
                    for (size_t i = 0; i < n; ++i) hr[i] = hr[i] - me[i];
                } else {
                    std::memcpy(modes + rz * n, hr, n * sizeof(double));
                }
            }
        }
    }
}

/* The decomposition.  rec (optional) records the tape; rep (optional) replays one: the noise
 * phase is taken from it and every signal stage runs with its frozen structure.  noise_src
 * (optional): the noise phase's result (noise modes, mean-envelope and sifting-fraction
 * carries) is taken from that recorded call of the same noise, sizes and options instead of
 * being computed; the result is the one computing it would give. */
int run(size_t nr, size_t n, size_t num_imfs, size_t max_iter, const double* y,
        const double* noise, double nstd, double* imfs, const oracle_opts& o, Tape* rec,
        const Tape* rep, const Tape* noise_src = nullptr, const oracle_split* sp = nullptr) {
    if (nr < 1 || n < 4 || num_imfs < 2 || max_iter < 1 || o.noise_sift_cap < 1) return -1;
    if (o.solver == 1 && (o.chunk < 2 || o.chunk > 64)) return -1;
    if (rep && (rep->nr != nr || rep->n != n || rep->nimf != num_imfs)) return -1;
    if (noise_src && (noise_src->nr != nr || noise_src->n != n || noise_src->nimf != num_imfs ||
                      noise_src->ck_frac.empty()))
        return -1;
#ifdef _OPENMP
    if (o.threads > 0) omp_set_num_threads(o.threads);
#endif
    Ctx cx;
    cx.nr = nr;
    cx.n = n;
    cx.sd = o.sd;
    cx.sd2 = o.sd2;
    cx.tol = o.tol;
    cx.inv_n = 1.0 / (double)n;
    cx.solver = o.solver;
    cx.chunk = o.chunk;
    cx.menv.assign(nr * n, 0.0);
    cx.frac.assign(nr, 0.0);
    cx.split = sp;
    const size_t rn = nr * n;
    const double inv_nm1 = 1.0 / (double)(n - 1);
    const size_t nr_all = sp ? sp->nr_total : nr;  // realizations of the whole ensemble
    vector<double> tsum(n);

    /* ---- noise modes E_k(w_r) (:1566-1715) ---- */
    vector<double> E;
    if (rep) {
        E = rep->E;
        cx.menv = rep->menv0;
    } else if (noise_src) {
        E = noise_src->E;
        cx.menv = noise_src->menv0;
        cx.frac = noise_src->ck_frac[0];  // the sifting-fraction carry the noise phase left
        for (size_t i = 0; i + 1 < num_imfs && o.iters_out; ++i) o.iters_out[i] = 0;
    } else {
        vector<double> w(noise, noise + rn), cur(rn);
        E.assign(num_imfs * rn, 0.0);
        for (size_t i = 0; i + 1 < num_imfs; ++i) {
            cur = w;
            double* Ei = E.data() + i * rn;
            int it = sift_stage(cx, cur.data(), Ei, (size_t)o.noise_sift_cap);
            if (o.iters_out) o.iters_out[i] = it;
            for (size_t k = 0; k < rn; ++k) w[k] = w[k] - Ei[k];  // updateSignal (:610-617)
        }
        std::copy(w.begin(), w.end(), E.begin() + (num_imfs - 1) * rn);
    }
    if (o.noise_modes_out) std::copy(E.begin(), E.end(), o.noise_modes_out);
    if (rec) {
        rec->nr = nr;
        rec->n = n;
        rec->nimf = num_imfs;
        rec->nstd = nstd;
        rec->E = E;
        rec->menv0 = cx.menv;
        rec->fin.assign((num_imfs - 1) * n, 0.0);
        rec->mu.assign(num_imfs - 1, 0.0);
        rec->var.assign(num_imfs - 1, 0.0);
        rec->st.assign(num_imfs - 1, StageTape());
        rec->max_iter = max_iter;
        rec->ck_h0.assign(num_imfs - 1, vector<double>());
        rec->ck_menv.assign(num_imfs - 1, vector<double>());
        rec->ck_frac.assign(num_imfs - 1, vector<double>());
    }

    /* ---- CEEMDAN stages (:1722-2019) ---- */
    vector<double> xs(y, y + n), h0(rn), hcur(rn), mode(rn), fornext(n);
    double s_mean = 0.0, s_var = 0.0;  // d_singleChannelMean / Variance: carried, never reset
    for (size_t i = 0; i + 1 < num_imfs; ++i) {
        const double* Ei = E.data() + i * rn;
        if (rec)
            std::copy_n(i == 0 ? xs.data() : fornext.data(), n, rec->fin.begin() + i * n);
        if (i == 0) {
            s_mean = (s_mean + canon_sum(xs.data(), n)) * cx.inv_n;
            s_var = (s_var + canon_sqdev(xs.data(), n, s_mean)) * inv_nm1;
            const double sc = 1.0 / std::sqrt(s_var);
            for (size_t k = 0; k < n; ++k) xs[k] = xs[k] * sc;  // standardizeRunning (:58-66)
            for (size_t rz = 0; rz < nr; ++rz) {
                const double* er = Ei + rz * n;
                const double em = canon_sum(er, n) * cx.inv_n;
                const double ev = canon_sqdev(er, n, em) * inv_nm1;
                const double es = 1.0 / std::sqrt(ev);
                for (size_t k = 0; k < n; ++k)  // addNoise (:69-78)
                    h0[rz * n + k] = fma(nstd * er[k], es, xs[k]);
            }
        } else {
            s_mean = (s_mean + canon_sum(fornext.data(), n)) * cx.inv_n;
            s_var = (s_var + canon_sqdev(fornext.data(), n, s_mean)) * inv_nm1;
            const double sq = std::sqrt(s_var);
            for (size_t rz = 0; rz < nr; ++rz)  // addNoise2 (:81-90)
                for (size_t k = 0; k < n; ++k)
                    h0[rz * n + k] = fma(nstd * Ei[rz * n + k], sq, fornext[k]);
        }
        if (rec) {
            rec->mu[i] = s_mean;
            rec->var[i] = s_var;
            rec->ck_h0[i] = h0;
            rec->ck_menv[i] = cx.menv;
            rec->ck_frac[i] = cx.frac;
        }
        hcur = h0;
        if (rep) {
            sift_replay(cx, hcur.data(), mode.data(), rep->st[i]);
        } else {
            int it = sift_stage(cx, hcur.data(), mode.data(), max_iter, rec ? &rec->st[i] : nullptr);
            if (o.iters_out) o.iters_out[(num_imfs - 1) + i] = it;
        }
        // ensemble sums in realization order, continued across the parts of a split
        std::fill(tsum.begin(), tsum.end(), 0.0);
        if (sp && sp->rank > 0) sp->recv_partial(sp->ctx, tsum.data(), n);
        if (i == 0) {
            const double inr = 1.0 / (double)nr_all;  // produceFirstIMF (:42-55)
            for (size_t k = 0; k < n; ++k) {
                double t = tsum[k];
                for (size_t rz = 0; rz < nr; ++rz)
                    t = fma(inr, h0[rz * n + k] - mode[rz * n + k], t);
                tsum[k] = t;
            }
        } else {
            for (size_t k = 0; k < n; ++k) {  // produceResidue + averageUpdateSignal (:583-607)
                double t = tsum[k];
                for (size_t rz = 0; rz < nr; ++rz) t = t + (h0[rz * n + k] - mode[rz * n + k]);
                tsum[k] = t;
            }
        }
        if (sp && sp->rank + 1 < sp->world) sp->send_partial(sp->ctx, tsum.data(), n);
        if (sp) sp->broadcast_last(sp->ctx, tsum.data(), n);
        if (i == 0) {
            for (size_t k = 0; k < n; ++k) {
                fornext[k] = tsum[k];
                imfs[k] = xs[k] - tsum[k];
            }
        } else {
            for (size_t k = 0; k < n; ++k) {
                const double avg = tsum[k] / (double)nr_all;
                imfs[i * n + k] = fornext[k] - avg;
                fornext[k] = avg;
            }
        }
    }
    std::copy(fornext.begin(), fornext.end(), imfs + (num_imfs - 1) * n);
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* reverse pass with the structure frozen (knots, end rule, stale-mean choices, marks and  */
/* iteration counts of the recorded forward call).  With that structure every sift is      */
/* linear in h; the stage statistics (x/std(x), sqrt(var) of the residue, carried) are the */
/* only nonlinear steps.                                                                   */
/* ------------------------------------------------------------------------------------ */

/* Adds (d envelope / d h)^T eb to gh for one envelope with knots kx and end flags bf.
 * Envelope on segment s (x_s < i <= x_{s+1}, sample 0 in segment 0):
 * a + b t + c t^2 + d t^3 with a = y_s, b = (y_{s+1}-y_s)/h - h(2c_s+c_{s+1})/3, c = c_s,
 * d = (c_{s+1}-c_s)/(3h); c solves the natural-spline system, whose interior rows form a
 * symmetric matrix, so the transposed solve is the same solve with a new right-hand side. */
void env_adjoint(int n, const vector<int32_t>& kxv, int bf, const double* eb, double* gh,
                 int S) {
    (void)n;
    const int K = (int)kxv.size();
    const int32_t* kx = kxv.data();
    vector<double> s0(K), s1(K), s2(K), s3(K), yb(K), l(K), m(K), u(K), r(K), z(K);
    for (int s = 0; s + 1 < K; ++s) {  // segment sums of eb * t^p
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        const int first = s == 0 ? kx[0] : kx[s] + 1;
        for (int i = first; i <= kx[s + 1]; ++i) {
            const double t = (double)(i - kx[s]);
            const double e = eb[i];
            const double p1 = e * t, p2 = p1 * t, p3 = p2 * t;
            a0 = a0 + e;
            a1 = a1 + p1;
            a2 = a2 + p2;
            a3 = a3 + p3;
        }
        s0[s] = a0;
        s1[s] = a1;
        s2[s] = a2;
        s3[s] = a3;
    }
    for (int i = 0; i < K; ++i) {  // transposed coefficient maps; system rows
        double y = 0.0, cb = 0.0;
        if (i + 1 < K) {
            const double h = (double)(kx[i + 1] - kx[i]);
            y = s0[i] - s1[i] / h;
            cb = (s2[i] - s1[i] * (2.0 * h / 3.0)) - s3[i] / (3.0 * h);
        }
        if (i > 0) {
            const double h = (double)(kx[i] - kx[i - 1]);
            y = y + s1[i - 1] / h;
            cb = cb + (s3[i - 1] / (3.0 * h) - s1[i - 1] * (h / 3.0));
        }
        yb[i] = y;
        if (i == 0 || i == K - 1) {
            l[i] = 0.0; m[i] = 1.0; u[i] = 0.0; r[i] = 0.0;
        } else {
            const int dl = kx[i] - kx[i - 1], du = kx[i + 1] - kx[i];
            l[i] = (double)dl;
            u[i] = (double)du;
            m[i] = (double)(2 * (dl + du));
            r[i] = cb;
        }
    }
    partitioned(K, l.data(), m.data(), u.data(), r.data(), z.data(), S);
    for (int i = 0; i < K; ++i) {  // transposed right-hand side 3*(slope_i - slope_{i-1})
        double y = yb[i];
        if (i >= 2) y = y + (3.0 * z[i - 1]) / (double)(kx[i] - kx[i - 1]);
        if (i >= 1 && i <= K - 2)
            y = y - ((3.0 * z[i]) / (double)(kx[i + 1] - kx[i]) +
                     (3.0 * z[i]) / (double)(kx[i] - kx[i - 1]));
        if (i + 1 <= K - 2) y = y + (3.0 * z[i + 1]) / (double)(kx[i + 1] - kx[i]);
        r[i] = y;
    }
    for (int i = 0; i < K; ++i) {  // transposed end rule, scatter to the knot samples
        double g = r[i];
        if (K - 1 > 4) {
            const int L = K - 1;
            if (bf & 1) {
                const double rho = (double)(kx[1] - kx[0]) / (double)(kx[2] - kx[1]);
                if (i == 0) g = 0.0;
                else if (i == 1) g = r[1] + r[0] * (1.0 + rho);
                else if (i == 2) g = r[2] - r[0] * rho;
            }
            if (bf & 2) {
                const double rho = (double)(kx[L] - kx[L - 1]) / (double)(kx[L - 1] - kx[L - 2]);
                if (i == L) g = 0.0;
                else if (i == L - 1) g = r[L - 1] + r[L] * (1.0 + rho);
                else if (i == L - 2) g = r[L - 2] - r[L] * rho;
            }
        }
        gh[kx[i]] = gh[kx[i]] + g;
    }
}

/* Reverse of one signal stage.  mbar: adjoint of every realization's mode (the same for all
 * of them); gm (nr*n): adjoint of the mean envelope at the end of the stage, on return at
 * its start; gh (nr*n): on return the adjoint of the stage's sift input h0 through the sift. */
void sift_adjoint(const Tape& T, const StageTape& st, const double* mbar, double* gm,
                  double* gh, int S) {
    const size_t nr = T.nr, n = T.n;
#pragma omp parallel
    {
        vector<double> eb(n);
#pragma omp for schedule(dynamic, 1)
        for (long rl = 0; rl < (long)nr; ++rl) {
            const size_t rz = (size_t)rl;
            double* g = gh + rz * n;
            double* m = gm + rz * n;
            std::fill(g, g + n, 0.0);
            for (int j = st.J - 1; j >= 0; --j) {
                const Step& s = st.it[(size_t)j * nr + rz];
                if (s.mark == 1) {
                    for (size_t k = 0; k < n; ++k) m[k] = m[k] - g[k];
                } else {
                    for (size_t k = 0; k < n; ++k) g[k] = g[k] + mbar[k];
                }
                if (s.kx[0].size() > 3 && s.kx[1].size() > 3) {
                    for (size_t k = 0; k < n; ++k) {
                        eb[k] = m[k] * 0.5;
                        m[k] = 0.0;
                    }
                    env_adjoint((int)n, s.kx[0], s.bflag[0], eb.data(), g, S);
                    env_adjoint((int)n, s.kx[1], s.bflag[1], eb.data(), g, S);
                }
            }
        }
    }
}

/* Stage i's structure re-computed from its checkpoint (the forward's sift_stage on the stage's
 * input h0 with the carries it started from). */
StageTape recompute_stage(const Tape& T, const oracle_opts& o, size_t i) {
    Ctx cx;
    cx.nr = T.nr;
    cx.n = T.n;
    cx.sd = o.sd;
    cx.sd2 = o.sd2;
    cx.tol = o.tol;
    cx.inv_n = 1.0 / (double)T.n;
    cx.solver = o.solver;
    cx.chunk = o.chunk;
    cx.menv = T.ck_menv[i];
    cx.frac = T.ck_frac[i];
    vector<double> h = T.ck_h0[i], modes(T.nr * T.n);
    StageTape st;
    sift_stage(cx, h.data(), modes.data(), T.max_iter, &st);
    return st;
}

/* Vector-Jacobian product: gy = (d imfs / d y)^T gimfs with the recorded structure.  With
 * `recompute` (o required) every stage's structure is re-computed from its checkpoint just
 * before its reverse pass instead of being read from the recorded iterations. */
void vjp(const Tape& T, const double* gimfs, double* gy, int S, const oracle_opts* recompute) {
    const size_t nr = T.nr, n = T.n, nimf = T.nimf, rn = nr * n;
    const size_t ns = nimf - 1;
    const double inr = 1.0 / (double)nr, inv_n = 1.0 / (double)n;
    const double inv_nm1 = 1.0 / (double)(n - 1);
    vector<double> fbar(gimfs + ns * n, gimfs + (ns + 1) * n);  // adjoint of f_{ns-1}
    vector<double> gm(rn, 0.0), gh(rn), abar(n), mbar(n), hs(n), p(n), dv(n);
    double vcarry = 0.0, mucarry = 0.0;
    for (long i = (long)ns - 1; i >= 0; --i) {
        const double* gi = gimfs + (size_t)i * n;
        for (size_t k = 0; k < n; ++k) {
            abar[k] = fbar[k] - gi[k];  // adjoint of the ensemble mean f_i
            mbar[k] = -(abar[k] * inr);
        }
        if (recompute) {
            const StageTape st = recompute_stage(T, *recompute, (size_t)i);
            sift_adjoint(T, st, mbar.data(), gm.data(), gh.data(), S);
        } else {
            sift_adjoint(T, T.st[(size_t)i], mbar.data(), gm.data(), gh.data(), S);
        }
        const double* Ei = T.E.data() + (size_t)i * rn;
        for (size_t k = 0; k < n; ++k) {  // adjoint of h0_r, summed over r (and times E_r)
            double s1 = 0.0, s2 = 0.0;
            for (size_t rz = 0; rz < nr; ++rz) {
                const double hb = gh[rz * n + k] + abar[k] * inr;
                s1 = s1 + hb;
                s2 = s2 + hb * Ei[rz * n + k];
            }
            hs[k] = s1;
            p[k] = s2;
        }
        const double* f = T.fin.data() + (size_t)i * n;
        const double mu = T.mu[(size_t)i], var = T.var[(size_t)i];
        for (size_t k = 0; k < n; ++k) dv[k] = f[k] - mu;
        const double D = canon_sum(dv.data(), n);
        if (i >= 1) {
            // h0 = f + nstd*E*sqrt(var); var = (var_prev + sum (f-mu)^2)/(n-1);
            // mu = (mu_prev + sum f)/n
            const double sq = std::sqrt(var);
            const double vbar = vcarry + (T.nstd * canon_sum(p.data(), n)) * (0.5 / sq);
            const double qbar = vbar * inv_nm1;
            const double mubar = mucarry + qbar * (-2.0 * D);
            for (size_t k = 0; k < n; ++k)
                fbar[k] = (gi[k] + hs[k]) + (qbar * (2.0 * dv[k]) + mubar * inv_n);
            vcarry = vbar * inv_nm1;
            mucarry = mubar * inv_n;
        } else {
            // xs = y / sqrt(var), h0 = xs + noise; mu = sum y / n; var = sum (y-mu)^2/(n-1)
            const double sc = 1.0 / std::sqrt(var);
            for (size_t k = 0; k < n; ++k) {
                hs[k] = gi[k] + hs[k];  // adjoint of xs
                p[k] = hs[k] * f[k];
            }
            const double vbar = vcarry + canon_sum(p.data(), n) * (-0.5 * sc / var);
            const double qbar = vbar * inv_nm1;
            const double mubar = mucarry + qbar * (-2.0 * D);
            for (size_t k = 0; k < n; ++k)
                gy[k] = hs[k] * sc + (qbar * (2.0 * dv[k]) + mubar * inv_n);
        }
    }
}

}  // namespace

struct oracle_tape {
    Tape t;
    oracle_opts o;
};

extern "C" {

void oracle_default_opts(oracle_opts* o) {
    std::memset(o, 0, sizeof(*o));
    o->noise_sift_cap = 2000;
    o->sd = 0.05;
    o->sd2 = 0.5;
    o->tol = 0.05;
    o->solver = 0;
    o->chunk = 16;
    o->threads = 0;
}

int oracle_iceemdan_f64(size_t nr, size_t n, size_t num_imfs, size_t max_iter,
                        const double* y, const double* noise, double nstd, double* imfs,
                        const oracle_opts* oin) {
    oracle_opts o;
    if (oin) o = *oin; else oracle_default_opts(&o);
    return run(nr, n, num_imfs, max_iter, y, noise, nstd, imfs, o, nullptr, nullptr);
}

int oracle_iceemdan_split_f64(size_t nr_local, size_t n, size_t num_imfs, size_t max_iter,
                              const double* y, const double* noise_local, double nstd,
                              double* imfs, const oracle_opts* oin, const oracle_split* sp) {
    oracle_opts o;
    if (oin) o = *oin; else oracle_default_opts(&o);
    if (sp && (sp->world < 1 || sp->rank < 0 || sp->rank >= sp->world || !sp->all_finished ||
               !sp->recv_partial || !sp->send_partial || !sp->broadcast_last ||
               sp->nr_total < nr_local))
        return -1;
    return run(nr_local, n, num_imfs, max_iter, y, noise_local, nstd, imfs, o, nullptr, nullptr,
               nullptr, sp);
}

oracle_tape* oracle_tape_forward_f64(size_t nr, size_t n, size_t num_imfs, size_t max_iter,
                                     const double* y, const double* noise, double nstd,
                                     double* imfs, const oracle_opts* oin) {
    oracle_tape* t = new oracle_tape();
    if (oin) t->o = *oin; else oracle_default_opts(&t->o);
    t->o.iters_out = oin ? oin->iters_out : nullptr;
    if (run(nr, n, num_imfs, max_iter, y, noise, nstd, imfs, t->o, &t->t, nullptr) != 0) {
        delete t;
        return nullptr;
    }
    t->o.iters_out = nullptr;
    t->o.noise_modes_out = nullptr;
    return t;
}

oracle_tape* oracle_tape_forward_shared_f64(size_t nr, size_t n, size_t num_imfs,
                                            size_t max_iter, const double* y, double nstd,
                                            double* imfs, const oracle_opts* oin,
                                            const oracle_tape* noise_from) {
    if (!noise_from) return nullptr;
    oracle_tape* t = new oracle_tape();
    if (oin) t->o = *oin; else oracle_default_opts(&t->o);
    t->o.iters_out = oin ? oin->iters_out : nullptr;
    if (run(nr, n, num_imfs, max_iter, y, nullptr, nstd, imfs, t->o, &t->t, nullptr,
            &noise_from->t) != 0) {
        delete t;
        return nullptr;
    }
    t->o.iters_out = nullptr;
    t->o.noise_modes_out = nullptr;
    return t;
}

int oracle_tape_replay_f64(const oracle_tape* t, const double* y, double* imfs) {
    if (!t) return -1;
    return run(t->t.nr, t->t.n, t->t.nimf, 1, y, nullptr, t->t.nstd, imfs, t->o, nullptr,
               &t->t);
}

int oracle_tape_vjp_f64(const oracle_tape* t, const double* gimfs, double* gy) {
    if (!t) return -1;
#ifdef _OPENMP
    if (t->o.threads > 0) omp_set_num_threads(t->o.threads);
#endif
    vjp(t->t, gimfs, gy, 16, nullptr);
    return 0;
}

int oracle_tape_vjp_recompute_f64(const oracle_tape* t, const double* gimfs, double* gy) {
    if (!t) return -1;
#ifdef _OPENMP
    if (t->o.threads > 0) omp_set_num_threads(t->o.threads);
#endif
    vjp(t->t, gimfs, gy, 16, &t->o);
    return 0;
}

int oracle_tape_recompute_mismatches(const oracle_tape* t) {
    if (!t) return -1;
    int bad = 0;
    for (size_t i = 0; i < t->t.st.size(); ++i) {
        const StageTape a = recompute_stage(t->t, t->o, i);
        const StageTape& b = t->t.st[i];
        if (a.J != b.J || a.it.size() != b.it.size()) {
            ++bad;
            continue;
        }
        for (size_t k = 0; k < a.it.size(); ++k)
            for (int e = 0; e < 2; ++e)
                if (a.it[k].kx[e] != b.it[k].kx[e] || a.it[k].bflag[e] != b.it[k].bflag[e] ||
                    a.it[k].mark != b.it[k].mark)
                    ++bad;
    }
    return bad;
}

int oracle_tape_iterations(const oracle_tape* t, int stage) {
    if (!t || stage < 0 || (size_t)stage >= t->t.st.size()) return -1;
    return t->t.st[(size_t)stage].J;
}

int oracle_tape_step(const oracle_tape* t, int stage, int iter, int r, int e, int32_t* kx,
                     int* bflag, int* mark) {
    if (!t || stage < 0 || (size_t)stage >= t->t.st.size() || r < 0 || (size_t)r >= t->t.nr ||
        e < 0 || e > 1)
        return -1;
    const StageTape& st = t->t.st[(size_t)stage];
    if (iter < 0 || iter >= st.J) return -1;
    const Step& s = st.it[(size_t)iter * t->t.nr + (size_t)r];
    if (kx) std::copy(s.kx[e].begin(), s.kx[e].end(), kx);
    if (bflag) *bflag = s.bflag[e];
    if (mark) *mark = s.mark;
    return (int)s.kx[e].size();
}

void oracle_tape_free(oracle_tape* t) { delete t; }

int oracle_extrema_f64(const double* h, int n, int kind, int32_t* kx, double* ky) {
    return extrema(h, n, kind, kx, ky);
}

void oracle_boundary_f64(int count, const int32_t* kx, double* ky, int kind) {
    boundary(count, kx, ky, kind);
}

void oracle_spline_solve_f64(int count, const int32_t* kx, const double* ky, double* c,
                             int solver, int chunk) {
    spline_solve(count, kx, ky, c, solver, chunk);
}

void oracle_spline_eval_f64(int n, int count, const int32_t* kx, const double* ky,
                            const double* c, double* env) {
    spline_eval(n, count, kx, ky, c, env);
}

double oracle_canonical_sum_f64(const double* v, size_t n) { return canon_sum(v, n); }

double oracle_canonical_sqdev_f64(const double* v, size_t n, double mean) {
    return canon_sqdev(v, n, mean);
}

void oracle_tridiag_partitioned_f64(int n, const double* l, const double* m, const double* u,
                                    const double* r, double* x, int chunk) {
    partitioned(n, l, m, u, r, x, chunk);
}

}  // extern "C"
