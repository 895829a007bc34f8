/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement (C++17 + OpenMP, FP64) of the ICEEMDAN decomposition performed by
 * iceemdanD in the reference (cudaICEEMDAN.cu:1340-2059, kernels :41-617, statistics
 * kernels statistics.cu:167-241).  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py may load this library, and only as the checker or the timed
 * CPU baseline.  The product (ceemdan-gpu_b200) never links or calls it.
 *
 * Semantics ("compat" = what the reference computes, with its undefined behaviour pinned):
 *   - every accumulator the reference never zeroes (mean / variance carries, the sifting
 *     fraction accumulator) starts at 0.0, as on a fresh allocation;
 *   - the mean-envelope buffer starts at 0.0 and keeps its last value whenever a
 *     realization has <= 3 maxima or <= 3 minima (stale mean, cudaICEEMDAN.cu:442-454);
 *   - reductions whose order the reference leaves to atomics use one canonical order
 *     (256 strided lanes, then a halving tree), shared with the CUDA engine;
 *   - all realizations of a stage iterate in lock step until every one has finished
 *     (checkBreak, cudaICEEMDAN.cu:547-580, read as the intended AND over realizations);
 *   - floating-point contractions follow nvcc's default fused multiply-add placement
 *     in the reference kernels, written out with explicit fma() calls.
 *
 * Parity pinning: the reference has no golden vectors or tests.  The spline solve is a
 * closed library call there (cuSPARSE gtsv2_nopivot) whose rounding cannot be restated;
 * this oracle offers a plain Thomas solve (solver = 0) and the canonical partitioned
 * solve the CUDA engine uses (solver = 1: first level aligned to ORACLE_TILE_SAMPLES-sample
 * tiles, deeper levels index-based).
 */
#ifndef CEEMDAN_ORACLE_H
#define CEEMDAN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Samples per tile of the engine's extrema/evaluation passes; the first level of the
 * canonical spline partition is aligned to these tiles. */
#define ORACLE_TILE_SAMPLES 2048

typedef struct oracle_opts {
    int noise_sift_cap;   /* sift cap of the noise-mode precompute (reference: 2000) */
    double sd;            /* threshold_1 (0.05) */
    double sd2;           /* threshold_2 (0.5)  */
    double tol;           /* threshold_3 (0.05) */
    int solver;           /* 0 = Thomas, 1 = canonical tile-aligned partitioned solve */
    int chunk;            /* rows per chunk of the partitioned solve */
    int threads;          /* OpenMP threads; 0 = runtime default */
    int32_t* iters_out;   /* optional [2*(num_imfs-1)]: lock-step iterations per noise stage,
                             then per signal stage */
    double* noise_modes_out; /* optional [num_imfs*nr*n]: the noise modes E_k(w_r) */
} oracle_opts;

void oracle_default_opts(oracle_opts* o);

/* Realizations of one channel split over ranks (parts in rank order, each a contiguous block
 * of realizations).  The decomposition needs three exchanges, supplied by the caller:
 *   all_finished   the lock-step stop test of every sift iteration: the AND over the parts
 *                  of "all my realizations have finished" (the same value on every part);
 *   recv_partial / send_partial
 *                  the ensemble sums at the end of a CEEMDAN stage continue across the parts
 *                  in realization order: part k receives the running sums of the samples
 *                  (n doubles) from part k-1 (part 0 starts from zeros), adds its own
 *                  realizations in order and sends them to part k+1 -- the same operations
 *                  in the same order as one part holding every realization;
 *   broadcast_last the last part's sums to every part.
 * Every part returns the whole channel's IMFs. */
typedef struct oracle_split {
    size_t nr_total;      /* realizations of the whole ensemble */
    int rank, world;      /* this part and the number of parts */
    void* ctx;
    int (*all_finished)(void* ctx, int local_all);
    void (*recv_partial)(void* ctx, double* t, size_t n);
    void (*send_partial)(void* ctx, const double* t, size_t n);
    void (*broadcast_last)(void* ctx, double* t, size_t n);
} oracle_split;

/* The decomposition of one part (nr_local realizations, their noise rows): see oracle_split.
 * With world = 1 it is oracle_iceemdan_f64. */
int oracle_iceemdan_split_f64(size_t nr_local, size_t n, size_t num_imfs, size_t max_iter,
                              const double* y, const double* noise_local, double nstd,
                              double* imfs, const oracle_opts* o, const oracle_split* sp);

/* Full decomposition.  noise: nr*n N(0,1) samples (realization-major), as the reference's
 * cuRAND call produces them.  imfs: num_imfs*n, row k = IMF k, last row = residue, in
 * units of x/std(x).  Returns 0 on success, a negative code on invalid arguments. */
int oracle_iceemdan_f64(size_t nr, size_t n, size_t num_imfs, size_t max_iter,
                        const double* y, const double* noise, double nstd,
                        double* imfs, const oracle_opts* o);

/* ---- frozen-structure tape and reverse pass ----
 * oracle_tape_forward_f64 runs oracle_iceemdan_f64 and records, for every signal-stage
 * iteration and realization, the knot positions of both envelopes, which end values the
 * end-knot rule replaced, and the update mark (1 subtract, 0 mode export), plus each stage's
 * iteration count, the noise modes and the carried stage statistics.  With that structure
 * frozen, the decomposition is a differentiable map y -> imfs (linear sifts; the stage
 * statistics are the nonlinear steps):
 *   oracle_tape_replay_f64  evaluates it at another y (identical to the forward at the
 *                           recorded y), the function finite differences are taken of;
 *   oracle_tape_vjp_f64     gy = (d imfs / d y)^T gimfs (gimfs: num_imfs*n). */
typedef struct oracle_tape oracle_tape;

oracle_tape* oracle_tape_forward_f64(size_t nr, size_t n, size_t num_imfs, size_t max_iter,
                                     const double* y, const double* noise, double nstd,
                                     double* imfs, const oracle_opts* o);
/* The same taped forward for another input of the same length, noise and options, starting
 * from noise_from's noise phase (noise modes, mean-envelope and sifting-fraction carries)
 * instead of computing it: the result a full call gives.  noise_from's options should equal
 * o's. */
oracle_tape* oracle_tape_forward_shared_f64(size_t nr, size_t n, size_t num_imfs,
                                            size_t max_iter, const double* y, double nstd,
                                            double* imfs, const oracle_opts* o,
                                            const oracle_tape* noise_from);
int oracle_tape_replay_f64(const oracle_tape* t, const double* y, double* imfs);
int oracle_tape_vjp_f64(const oracle_tape* t, const double* gimfs, double* gy);
/* The same vjp, each stage's structure re-computed from its checkpoint (the stage input and
 * the mean-envelope and sifting-fraction carries at its start) instead of read from the
 * recorded iterations: the checkpoint-and-recompute form of the reverse pass. */
int oracle_tape_vjp_recompute_f64(const oracle_tape* t, const double* gimfs, double* gy);
/* Recorded steps that a re-computation from the checkpoints does not reproduce (0 expected). */
int oracle_tape_recompute_mismatches(const oracle_tape* t);
/* Iterations of signal stage `stage`, or -1. */
int oracle_tape_iterations(const oracle_tape* t, int stage);
/* Knots (kx, optional) of envelope e (0 max, 1 min) in iteration iter of realization r of
 * signal stage `stage`, its end-rule flags (bit 0 left, bit 1 right) and the mark; returns
 * the knot count, or -1. */
int oracle_tape_step(const oracle_tape* t, int stage, int iter, int r, int e, int32_t* kx,
                     int* bflag, int* mark);
void oracle_tape_free(oracle_tape* t);

/* ---- stage-level primitives (one realization) ---- */

/* Strict local maxima (kind 0) or minima (kind 1) with both end samples forced, compacted
 * in order.  kx/ky need room for n entries.  Returns the knot count. */
int oracle_extrema_f64(const double* h, int n, int kind, int32_t* kx, double* ky);

/* End-knot linear extrapolation applied when count-1 > 4 (setBoundaryMax/Min). */
void oracle_boundary_f64(int count, const int32_t* kx, double* ky, int kind);

/* Natural cubic spline second-derivative/2 coefficients c[0..count). */
void oracle_spline_solve_f64(int count, const int32_t* kx, const double* ky, double* c,
                             int solver, int chunk);

/* Envelope value at every sample 0..n-1 (interpolate kernel semantics). */
void oracle_spline_eval_f64(int n, int count, const int32_t* kx, const double* ky,
                            const double* c, double* env);

/* Canonical sum / sum of squared deviations (shared with the CUDA engine). */
double oracle_canonical_sum_f64(const double* v, size_t n);
double oracle_canonical_sqdev_f64(const double* v, size_t n, double mean);

/* Generic tridiagonal solve with the canonical partitioned method (for solver tests). */
void oracle_tridiag_partitioned_f64(int n, const double* l, const double* m, const double* u,
                                    const double* r, double* x, int chunk);

#ifdef __cplusplus
}
#endif

#endif
