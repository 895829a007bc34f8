/*
 * ceemdan_b200 — C ABI of the B200 (sm_100a) ICEEMDAN engine.
 *
 * Plain pointers and sizes only.  Device pointers are prefixed d_, host pointers h_.
 * Every entry point returns a ceemdan_status; none of them falls back to the CPU.
 *
 * Reference interface replaced (EEGLab-Pannon/CEEMDAN-GPU):
 *   double iceemdanD(size_t numNoise, size_t SignalLength, size_t num_IMFs, size_t max_iter,
 *                    int* d_x, double* d_y, double* d_IMFs, double noiseStrength);
 *     cudaICEEMDAN.cuh:26, implemented at cudaICEEMDAN.cu:1340-2059.
 * The C++-linkage drop-in with that exact signature is declared in cudaICEEMDAN.cuh
 * (this directory) and exported by the same library.
 */
#ifndef CEEMDAN_B200_H
#define CEEMDAN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ceemdan_status {
    CEEMDAN_OK = 0,
    CEEMDAN_ERR_INVALID_ARG = 1,   /* sizes/pointers rejected before any GPU work */
    CEEMDAN_ERR_COORD = 2,         /* d_x is not the sample index 0..N-1 */
    CEEMDAN_ERR_CUDA = 3,          /* a CUDA runtime call failed (see ceemdan_last_error) */
    CEEMDAN_ERR_NO_MEMORY = 4,     /* device or pinned allocation failed */
    CEEMDAN_ERR_TIMEOUT = 5,       /* a bounded in-kernel wait ran out (the kernel returned) */
    CEEMDAN_ERR_CANCELLED = 6      /* the host cancel word was set between sift iterations */
} ceemdan_status;

/* Options of the extended entry points.  ceemdan_default_options() gives the reference's
 * hard-coded values (cudaICEEMDAN.cu:1461-1467 and :1572). */
typedef struct ceemdan_options {
    uint32_t struct_size;        /* sizeof(ceemdan_options) */
    int32_t noise_sift_cap;      /* sift cap of the noise-mode precompute (2000) */
    double sd;                   /* sx threshold of the sifting fraction (0.05) */
    double sd2;                  /* sx threshold of the "any" test (0.5) */
    double tol;                  /* sifting fraction threshold (0.05) */
    uint64_t seed;               /* cuRAND XORWOW seed of the white noise (1234) */
    const double* d_noise;       /* optional [nr*n] N(0,1) noise; NULL = generate with cuRAND */
    double* d_noise_modes_out;   /* optional [num_imfs*nr*n]: receives the noise modes E_k */
    int32_t* h_iters_out;        /* optional [2*(num_imfs-1)]: lock-step sift iterations of
                                    each noise stage, then of each signal stage */
    volatile int32_t* h_cancel;  /* optional host word; nonzero aborts between iterations */
    int32_t group;               /* sift iterations launched between host checks; 0 = auto */
    int32_t spin_limit;          /* polls of an in-kernel wait before it gives up and the call
                                    returns CEEMDAN_ERR_TIMEOUT (0 = auto, about a second): the
                                    lock-step stop test of the on-chip path for short rows.  A
                                    negative value -k is a test of that failure path: the wait
                                    expects one arrival more than the launch has, so it always
                                    gives up after k polls */
    double* h_kernel_ms;         /* optional [CEEMDAN_NUM_KERNEL_KINDS]: accumulated device time
                                    per kernel kind (CUDA events around every launch) */
    uint64_t* h_counters;        /* optional [CEEMDAN_NUM_COUNTERS]: accumulated work counters */
    double* d_noise_state_out;   /* optional [(num_imfs+1)*nr*n + nr]: the state the noise phase
                                    leaves for the CEEMDAN stages -- the noise modes E_k
                                    ([num_imfs][nr][n]), then the mean-envelope carry
                                    ([nr][n]), then the sifting-fraction carry ([nr]) */
    const double* d_noise_state_in; /* optional, same layout: start the CEEMDAN stages from this
                                    state and skip the noise phase (no noise is generated; the
                                    noise entries of h_iters_out are 0).  The noise phase
                                    depends only on the noise, nr, n and num_imfs, so channels
                                    of equal length decomposed with the same noise share it:
                                    the result equals a full call's bit for bit. */
} ceemdan_options;

/* Kernel kinds of h_kernel_ms. */
enum {
    CEEMDAN_K_EXTREMA = 0,       /* deferred update + extrema + compaction */
    CEEMDAN_K_BOUNDARY = 1,      /* end-knot extrapolation */
    CEEMDAN_K_CHUNK_REDUCE = 2,  /* chunk end relations of the spline solve + separator rows */
    CEEMDAN_K_REDUCED_SOLVE = 3, /* per-spline separator solve */
    CEEMDAN_K_SEGMENTS = 4,      /* chunk interiors -> segment coefficients b, c, d */
    CEEMDAN_K_EVAL = 5,          /* envelopes, mean envelope, sx statistics */
    CEEMDAN_K_CRITERION = 6,     /* stop test */
    CEEMDAN_K_SIFT_SMALL = 7,    /* a whole stage on chip (rows of at most 8192 samples) */
    CEEMDAN_NUM_KERNEL_KINDS = 8
};

/* Counters of h_counters. */
enum {
    CEEMDAN_C_KNOTS = 0,         /* sum over executed sift iterations and realizations of
                                    (maxima + minima knot counts) */
    CEEMDAN_C_ITERATIONS = 1,    /* executed lock-step sift iterations (all stages) */
    CEEMDAN_C_LAUNCHES = 2,      /* kernels launched by the engine */
    CEEMDAN_C_WAVES = 3,         /* ceemdan_batched_f64: waves of channels run */
    CEEMDAN_C_PEAK_BYTES = 4,    /* ceemdan_batched_f64: peak device bytes of the library's
                                    memory pool during a wave (maximum over the waves) */
    CEEMDAN_NUM_COUNTERS = 5
};

void ceemdan_default_options(ceemdan_options* opt);

/* Plain ICEEMDAN of one channel (the iceemdanD computation, cudaICEEMDAN.cu:1340-2059).
 * d_x: int32[n], must be 0..n-1 (every reference caller passes this; the reference's
 * spline search assumes it).  d_y: f64[n].  d_imfs: f64[num_imfs*n], row k = IMF k, last row
 * = final residue, in units of y/std(y).  stream: a cudaStream_t (NULL = legacy default).
 * Synchronous: returns after the result is in d_imfs.
 * Requires nr >= 1, n >= 4, num_imfs >= 2, max_iter >= 1. */
ceemdan_status ceemdan_plain_f64(size_t nr, size_t n, size_t num_imfs, size_t max_iter,
                                 const int32_t* d_x, const double* d_y, double* d_imfs,
                                 double nstd, const ceemdan_options* opt, void* stream);

/* One channel whose realizations are split over the ranks of a group (parts in rank order,
 * each a contiguous block of realizations: this part holds realizations first ..
 * first + nr_local - 1 of nr_total).  Within a stage the realizations sift independently except
 * for the lock-step stop test, and the stage's ensemble mean sums h0_r - mode_r over the
 * realizations in order (cudaICEEMDAN.cu:42-55, :583-607, the reference's reduction over
 * realizations :1869, :2005-2006).  The caller supplies the exchanges:
 *   all_finished    every sift iteration: the AND over the parts of "all my realizations have
 *                   finished" (local_all 0/1), the same value returned on every part;
 *   recv_partial    (part k > 0) the running sums of the n samples from part k-1 into d_t;
 *   send_partial    (part k < world-1) this part's running sums on to part k+1;
 *   broadcast_last  the last part's sums to every part (the last part sends d_t, the others
 *                   receive into it).
 * d_t is a device buffer of n doubles; no work is pending on the call's stream when a callback
 * runs, and the callback's writes must be complete when it returns.  all_finished returns the
 * AND (0 or 1), or a negative value to abort the call; the other three return 0, or nonzero to
 * abort it (both CEEMDAN_ERR_CUDA).  opt->h_cancel is read after each iteration's all_finished:
 * a caller that cancels sets the word on every part, since a part that stops alone leaves the
 * others waiting in their next all_finished.  The running sums continue across the parts in
 * realization order, so every part returns the whole channel's IMFs bit for bit as one
 * ceemdan_plain_f64 call holding all nr_total realizations. */
typedef struct ceemdan_split {
    size_t nr_total;  /* realizations of the whole ensemble */
    size_t first;     /* this part's first realization */
    int rank, world;  /* this part and the number of parts */
    void* ctx;
    int (*all_finished)(void* ctx, int local_all);
    int (*recv_partial)(void* ctx, double* d_t, size_t n);
    int (*send_partial)(void* ctx, const double* d_t, size_t n);
    int (*broadcast_last)(void* ctx, double* d_t, size_t n);
} ceemdan_split;

/* ceemdan_plain_f64 of this part's nr_local realizations of a split channel (ceemdan_split).
 * Noise: opt->d_noise holds this part's nr_local rows; otherwise cuRAND with opt->seed draws
 * the whole ensemble's nr_total rows (as the one-part call would) and the part takes its own.
 * Every sift iteration exchanges its stop flag through the host, so a stage runs iteration by
 * iteration (no on-chip short-row path, no per-iteration pipelining); no tape, no noise-state
 * input or output.  The same arguments and rules as ceemdan_plain_f64 otherwise. */
ceemdan_status ceemdan_plain_split_f64(size_t nr_local, size_t n, size_t num_imfs,
                                       size_t max_iter, const int32_t* d_x, const double* d_y,
                                       double* d_imfs, double nstd, const ceemdan_options* opt,
                                       const ceemdan_split* split, void* stream);

/* The same decomposition for float data (the iceemdanS computation, cudaICEEMDAN.cu:619-1338):
 * d_y f32[n] and d_imfs f32[num_imfs*n].  The data are widened exactly to FP64 and decomposed
 * by the FP64 engine; the default noise is cuRAND's float normals (curandGenerateNormal, the
 * FP32 path's generator, cudaICEEMDAN.cu:741) widened exactly, or opt->d_noise (f64) when
 * given; the IMFs are rounded to float at the end.  Same arguments and rules otherwise. */
ceemdan_status ceemdan_plain_f32(size_t nr, size_t n, size_t num_imfs, size_t max_iter,
                                 const int32_t* d_x, const float* d_y, float* d_imfs,
                                 float nstd, const ceemdan_options* opt, void* stream);

/* A batch of channels of different lengths, each decomposed as ceemdan_plain_f64 with NR = nr
 * realizations: channel c reads d_y[c] (f64[lengths[c]], device) and writes d_imfs[c]
 * (f64[num_imfs*lengths[c]], device); its sample coordinates are 0..lengths[c]-1 and its noise
 * is cuRAND XORWOW with seed opt->seed + c.  `streams` host threads (1..64) each run one
 * channel at a time on their own CUDA stream of the current device, longest channels first,
 * so small ensembles fill the GPU together; every channel allocates its own workspace.
 * Returns after all channels are done, or with the first failure (ceemdan_last_error names
 * the channel).  opt->d_noise, d_noise_modes_out, h_iters_out, h_kernel_ms and h_counters
 * must be NULL.  The reference decomposes one channel per call (iceemdanD,
 * cudaICEEMDAN.cu:1340); this is the batched form of that call. */
ceemdan_status ceemdan_batch_f64(size_t channels, const size_t* lengths,
                                 const double* const* d_y, double* const* d_imfs, size_t nr,
                                 size_t num_imfs, size_t max_iter, double nstd,
                                 const ceemdan_options* opt, int streams);

/* Batched ICEEMDAN of many channels of different lengths: channel c reads d_y[c]
 * (f64[lengths[c]], device) and writes d_imfs[c] (f64[num_imfs*lengths[c]], device), each
 * bit-identical to ceemdan_plain_f64 of that channel with NR = nr, sample coordinates
 * 0..lengths[c]-1 and cuRAND XORWOW noise with seed opt->seed + c.  All channels of a wave
 * sift together: one device-driven loop (transition kernels + one sift iteration of every
 * channel, replayed as a CUDA graph) moves each channel through its own stages, so channels
 * whose stages end at different iterations never wait for each other.  Channels that do not
 * fit together are run in waves, longest first, each wave within wave_bytes of device memory
 * (0 = 85% of the free memory).  Persistent grid sizes are autotuned on the first wave of a
 * shape (environment CEEMDAN_BATCH_TUNE=0: defaults).  opt->h_iters_out, when given, receives
 * [channels][2*(num_imfs-1)] iteration counts (the channel's noise stages, then its CEEMDAN
 * stages); opt->h_kernel_ms and opt->h_counters accumulate as for the plain call (iterations =
 * iterations of the shared loop); opt->group = iterations per graph replay (0 = auto);
 * opt->h_cancel is read between replays.  opt->d_noise, d_noise_modes_out and the noise-phase
 * state must be NULL.  Work queued on `stream` before the call is waited for; synchronous.
 * The reference decomposes one channel per call (iceemdanD, cudaICEEMDAN.cu:1340-2059); this
 * is the batched form of that call. */
ceemdan_status ceemdan_batched_f64(size_t channels, const size_t* lengths,
                                   const double* const* d_y, double* const* d_imfs, size_t nr,
                                   size_t num_imfs, size_t max_iter, double nstd,
                                   const ceemdan_options* opt, size_t wave_bytes,
                                   void* stream);

/* Noise-phase cache for repeated calls (for example one call per EEG channel, as every
 * reference caller does).  Calls that pass no d_noise, d_noise_state_in or d_noise_state_out
 * draw their noise from cuRAND with opt->seed, so their noise phase (noise modes plus the
 * carries it leaves, about half of a decomposition) repeats whenever the device, seed, noise
 * type, nr, n, num_imfs, noise sift cap and thresholds repeat.  With the cache enabled, the
 * library keeps the last such state on the device (one entry of (num_imfs+1)*nr*n + nr
 * doubles, allocated with cudaMalloc) and later calls with the same key skip the noise phase
 * (same results bit for bit; the noise entries of h_iters_out are then 0).  One call at a
 * time computes a new entry (into a fresh buffer, published when it returns); concurrent
 * calls that miss meanwhile run without the cache.  max_bytes = 0
 * disables the cache and frees the entry; states larger than max_bytes are not kept.  The
 * initial limit is the environment variable CEEMDAN_NOISE_CACHE_BYTES (0 when unset), which
 * also reaches callers of the drop-in iceemdanS/iceemdanD.  Returns the previous limit. */
size_t ceemdan_noise_cache(size_t max_bytes);

/* ---- reverse pass (backward entry) ------------------------------------------------
 * The decomposition with its structure frozen -- knot positions of every sift iteration,
 * the end-rule choices, the stale-mean choices, the update marks and the iteration counts of
 * one forward call -- is a differentiable map y -> imfs: every sift is linear in h, and the
 * stage statistics (y/std(y), sqrt of the carried residue variance) are smooth.  The reference
 * has no backward entry; this is its vector-Jacobian product.
 *
 * ceemdan_forward_taped_f64: ceemdan_plain_f64 (same arguments and result, bit for bit) that
 * also records that structure into a tape (*tape_out, owned by the caller): per executed
 * iteration of every signal stage the knot bitmaps and counts, end-rule flags and marks
 * (2*nr*ceil(n/2048)*256 + 5*nr bytes, rounded up to 256), plus the noise modes and stage
 * inputs ((num_imfs*nr*n + num_imfs*n) doubles); ceemdan_tape_bytes reports the total.
 * Requires nr <= 32767.  The noise cache is not used.
 * ceemdan_backward_f64: d_grad_y (f64[n]) = (d imfs / d y)^T d_grad_imfs (f64[num_imfs*n]),
 * on the device the tape was recorded on.  Deterministic: the same arithmetic order as the
 * CPU oracle's reverse pass.  Synchronous. */
typedef struct ceemdan_tape ceemdan_tape;

ceemdan_status ceemdan_forward_taped_f64(size_t nr, size_t n, size_t num_imfs,
                                         size_t max_iter, const int32_t* d_x, const double* d_y,
                                         double* d_imfs, double nstd,
                                         const ceemdan_options* opt, void* stream,
                                         ceemdan_tape** tape_out);
/* Checkpointed form of the taped forward (same arguments and result): instead of every
 * iteration it keeps, per signal stage, the stage input and the mean-envelope and
 * sifting-fraction carries it started from ((2*nr*n + nr) doubles per stage, independent of the
 * iteration counts); ceemdan_backward_f64 then re-runs each stage from its checkpoint (same
 * kernels, options and sift cap: the same structure, checked by its iteration count) before
 * reversing it.  Gradients are identical to the full tape's; the backward costs one more
 * forward pass of the signal stages. */
ceemdan_status ceemdan_forward_checkpointed_f64(size_t nr, size_t n, size_t num_imfs,
                                                size_t max_iter, const int32_t* d_x,
                                                const double* d_y, double* d_imfs, double nstd,
                                                const ceemdan_options* opt, void* stream,
                                                ceemdan_tape** tape_out);
ceemdan_status ceemdan_backward_f64(const ceemdan_tape* tape, const double* d_grad_imfs,
                                    double* d_grad_y, void* stream);
/* Device bytes held by the tape; executed iterations of signal stage `stage` (-1 if none). */
size_t ceemdan_tape_bytes(const ceemdan_tape* tape);
int ceemdan_tape_iterations(const ceemdan_tape* tape, size_t stage);
void ceemdan_tape_free(ceemdan_tape* tape);

/* Device memory of the library's stream-ordered memory pool on the current device (every
 * entry point allocates its workspace there): bytes held by calls in progress, their
 * high-water mark, and bytes the pool has reserved from the device (in use + cached for the
 * next calls, up to 16 GiB kept).  reset_peak != 0 restarts the high-water mark.  Any pointer
 * may be NULL.  No counterpart in the reference (it allocates and frees per call). */
ceemdan_status ceemdan_memory_stats(uint64_t* used, uint64_t* peak, uint64_t* reserved,
                                    int reset_peak);

/* Human-readable text of a status, and of the last CUDA error seen by this thread. */
const char* ceemdan_status_string(ceemdan_status s);
const char* ceemdan_last_error(void);

/* Build identification (arch, chunk rows of the canonical spline solve, tile size). */
const char* ceemdan_build_info(void);

/* Kernels launched by this library in this process so far. */
uint64_t ceemdan_kernel_launches(void);

/* ---- stage-level entry points (same kernels as the full decomposition) ------------- */

/* One envelope pass over nr realizations of length n (d_h: f64[nr*n]): the upper and lower
 * cubic-spline envelopes (d_upper, d_lower: f64[nr*n]) and the knot counts
 * (d_counts: int32[2*nr], maxima counts then minima counts).  Knots are the strict local
 * extrema plus both end samples, end knots extrapolated as setBoundaryMax/Min do. */
ceemdan_status ceemdan_envelopes_f64(size_t nr, size_t n, const double* d_h, double* d_upper,
                                     double* d_lower, int32_t* d_counts, void* stream);

/* Extrema compaction only: knot positions/values of the maxima and minima of every
 * realization (d_kx_*: int32[nr*n], d_ky_*: f64[nr*n], realization r at offset r*n) after the
 * end-knot extrapolation, and the counts (d_counts: int32[2*nr]). */
ceemdan_status ceemdan_extrema_f64(size_t nr, size_t n, const double* d_h, int32_t* d_kx_max,
                                   double* d_ky_max, int32_t* d_kx_min, double* d_ky_min,
                                   int32_t* d_counts, void* stream);

/* The canonical partitioned tridiagonal solve of `batch` independent systems of n rows
 * (d_l, d_m, d_u, d_r, d_x: f64[batch*n]; l[0] and u[n-1] are ignored). */
ceemdan_status ceemdan_tridiag_f64(size_t batch, size_t n, const double* d_l, const double* d_m,
                                   const double* d_u, const double* d_r, double* d_x,
                                   void* stream);

/* The same solve as ceemdan_tridiag_f64 without any allocation, for callers that must not
 * allocate device memory while they run (real-time loops where an allocator call may
 * synchronise the device, hosts that own all device memory, framework plugins that must not
 * bypass the framework's memory pool).  No counterpart in the reference.  Scratch: a fixed
 * 8 MiB array in the library's device image, reserved on a device when the library's device
 * code is loaded there (with lazy module loading: during the first call on that device, which
 * may therefore allocate it) and held until the process exits; requires
 * batch*(5*n+64) <= 1048576 (else CEEMDAN_ERR_INVALID_ARG, nothing launched).  All calls
 * share it: calls that overlap on the GPU race.  The first call on a device looks up the
 * array's address and keeps it for the process; make it before any stream capture, and do
 * not use this entry point on a device after cudaDeviceReset.  Synchronous, like
 * ceemdan_tridiag_f64. */
ceemdan_status ceemdan_tridiag_noalloc_f64(size_t batch, size_t n, const double* d_l,
                                           const double* d_m, const double* d_u,
                                           const double* d_r, double* d_x, void* stream);

/* Canonical sums (256 strided lanes, then a halving tree) of `batch` vectors of n values:
 * d_sum[b] = sum(v_b), d_sqdev[b] = sum((v_b - d_mean[b])^2) (d_mean may be NULL: skipped). */
ceemdan_status ceemdan_canonical_sums_f64(size_t batch, size_t n, const double* d_v,
                                          const double* d_mean, double* d_sum,
                                          double* d_sqdev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CEEMDAN_B200_H */
