// Internal declarations shared by the kernels and the host engine.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ceemdan {

constexpr int kTileSamples = 2048;  // samples per extrema / evaluation tile
constexpr int kTileCap = 1028;      // knot slots per tile and envelope (max 1025 knots)
constexpr int kRcpMax = 4096;       // reciprocal tables cover knot spacings 1..kRcpMax

// Static description of one channel (device array, read-only while the channel sifts): nr
// realizations ("rows") of n samples.  Rows of all channels are numbered globally (channel c
// owns rows row0 .. row0+nr-1), and so are the 2048-sample tiles of the rows (row g of channel
// c owns tiles tile0 + (g-row0)*ntiles + t).  Per-spline arrays are indexed by the spline
// se = e*nrows + g (e = 0 maxima, 1 minima).  With one channel every array has the layout of a
// single decomposition: row r at r*n, tile t of row r at r*ntiles + t.
struct Chan {
    int n, ntiles, nr, row0;
    int cap;               // knot capacity of a spline: n/2 + 2
    int rec_stride;        // per-spline stride of chunk records / separator values
    int tile0;             // first global tile
    int pad;
    long long samp0;       // first sample of row row0 in the row-major sample arrays
    long long rec0;        // record offset of row row0 (within one envelope's half)
    long long red0;        // reduced-workspace offset of row row0 (within one envelope's half)
};

// Dynamic state of one channel.  The first four ints are read by the host between groups of
// iterations (done, iter, err, cap).
struct ChanState {
    int done;              // the current stage has finished: the sift kernels skip the channel
    int iter;              // executed iterations of the current stage (h[iter&1] is current)
    int err;               // device error word (0 = none)
    int cap;               // sift cap of the current stage
    int stage;             // batched engine: current stage (2*(num_imfs-1) = all done)
    int pad[3];
    double* mode_out;      // modes of the current stage (row r of the channel at r*n)
    unsigned long long knots;  // knots summed over executed iterations (both envelopes)
    unsigned long long iters;  // executed iterations, all stages
};

// Everything one sift iteration touches (device pointers unless noted).
struct SiftArgs {
    int nrows, nchan;      // rows and channels
    // channel 0's geometry as launch parameters (used when nchan == 1, so that the kernels
    // need no load of the channel table), and the parity of the iteration when the host knows
    // it (one channel, host-driven iterations; -1: read the channel's iteration counter)
    int n1, ntiles1, nr1, rs1;
    int par;
    // one channel re-run for a known number of iterations (a block of the realizations of a
    // recorded stage): the stage ends after `forced` iterations whatever the block's own
    // lock-step test says; 0: the stop test decides
    int forced;
    int ntot;              // tiles over all rows
    int red_qcap;          // level-3 rows whose workspace fits the reduced solve's shared memory
    long long rec_total;   // record slots of one envelope (sum of the rows' rec_stride)
    long long red_total;   // reduced-workspace doubles of one envelope
    size_t rec_plane;      // stride between record fields (2*rec_total)
    int spin_limit;        // cap of in-kernel waits (reserved: no kernel waits today)
    double sd, sd2, tol;
    // margins of the division-free sx tests (sx_bounds): sx > t is true when |U+L| > |U-L|*t_hi
    // and false when |U+L| < |U-L|*t_lo, for |U-L| in (2^-800, 2^800)
    double sd_hi, sd_lo, sd2_hi, sd2_lo;
    const Chan* chan;      // [nchan]
    ChanState* cs;         // [nchan]
    // active-channel plan of the iteration (nchan > 1; written by k_plan): exclusive prefixes
    // over the channels of the rows [0..nchan] and of the tiles [nchan+1..2*nchan+1] of the
    // channels that sift in this iteration (done == 0).  With one channel the kernels read the
    // channel's done word instead.
    int* plan;
    int* gcount;           // [2*nrows] warp groups of each active spline, active-spline order
    double* h[2];          // sift state ping / pong: iteration j of a stage reads h[j%2]
    double* menv;          // mean envelope, persists for the whole decomposition
    int* mark;             // [nrows] -1 none, 0 export, 1 subtract
    int* finish;
    double* frac;          // sifting fraction accumulator, persists
    unsigned* cnt;
    int* any;
    int* kcount;           // [2*nrows] maxima counts, minima counts (by spline)
    int* tile_cnt;         // [2*ntot] knots found in each tile
    int* tile_off;         // [2*(ntot+nrows)] exclusive prefix of tile_cnt (global knot index)
    int* sep_off;          // [2*(ntot+nrows)] exclusive prefix of the separators per tile
    int* pcount;           // [2*nrows] separators per spline
    int* gsum;             // [2*nrows+1] exclusive prefix of gcount (active-spline order)
    unsigned* bitmap;      // [2][ntot][64] knot flags of each tile (word j/32, bit j%32)
    long long* nbr;        // [2][ntot][2] address of the knot before / after each tile
                           //   (-1 if none)
    // knots, tile-local: knot i of global tile gt at gt*kTileCap + (i - tile_off[t])
    int32_t *kx_max, *kx_min;
    double *ky_max, *ky_min;
    // record {a = y, b, c, d} of the segment starting at each knot (same slots, 4 doubles
    // each, 32-byte aligned)
    double* seg[2];
    const double* rcp_h;   // [kRcpMax+1] RN(1/h)
    const double* rcp_3h;  // [kRcpMax+1] RN(1/(3h))
    double* rec;           // 10 planes of chunk records: 6 end relations of the chunk left of
                           //   each separator, then the separator's own row (l, m, u, r)
    double* xsep;          // [2*rec_total] spline values at the separators
    double* red;           // [2*red_total] reduced-solve workspace
    double* dbg_upper;     // optional envelope outputs (stage-level entry point, one channel)
    double* dbg_lower;
    // taped forward only (one channel; null otherwise): end-rule flags of each spline [2*nr]
    // written by k_scan_boundary (bit 0: the left end value was replaced by the extrapolation,
    // bit 1: the right one), and the tape slot's mark array [nr] that k_criterion fills
    unsigned char* bflags;
    signed char* tape_mark;
};

// Per-channel stage state of the batched engine (stage_kernels.cu: transition kernels): the
// channels sift their stages independently; when a channel's stage has finished (done), the
// transition kernels at the start of the next iteration close it and open the next one.
// Stages 0..M-1 are the noise modes, M..2M-1 the CEEMDAN stages (M = num_imfs - 1); a channel
// starts at stage -1 (done) and ends at stage 2M.
struct BatchArgs {
    int nimf, M;
    int noise_cap, max_iter;
    double nstd;
    size_t S;                  // samples of one plane (all channels' row blocks)
    double* W;                 // residual noise [S] (cuRAND normals at the start)
    double* E;                 // noise modes [nimf][S]
    double* H0;                // inputs of the current CEEMDAN stage [S]
    double* MODE;              // modes of the current CEEMDAN stage [S]
    double* XS;                // standardized signals (x / std(x)) [X]
    double* FN;                // running ensemble means r_k [X]
    const long long* xoff;     // [nchan] offset of channel c's signal in XS / FN
    double* const* imfs;       // [nchan] the caller's output of channel c: [nimf][n]
    double* smean;             // [nchan] carried stage mean
    double* svar;              // [nchan] carried stage variance
    double* emean;             // [nrows] mean of the first noise mode of each realization
    double* evar;              // [nrows] its variance
    int* iters;                // [nchan][2M] executed iterations of every stage
    int* finished;             // channels that have finished every stage
};

// Short rows: the whole lock-step sift of a stage in one cooperative launch, one CTA per
// realization of channel 0 (k_sift_small).  Grid-wide state of the launch, zeroed per stage.
constexpr int kSmallMaxN = 8192;       // longest row the on-chip path takes
constexpr int kSmallThreads = 512;
constexpr int kSmallPre = 8;  // samples per thread whose global loads k_sift_small issues at once
constexpr int kSmallSpreadSmem = 120 * 1024;  // dynamic shared memory that fits one CTA per SM
constexpr int kErrTimeout = 5;         // CEEMDAN_ERR_TIMEOUT, written to ChanState.err
// Per-spline stride of the reduced-solve workspace.
__host__ __device__ inline long long red_stride_of(int rec_stride) {
    return 5LL * rec_stride + 64;
}

// Tape of one executed sift iteration of a signal stage (taped forward, reverse pass), in one
// slot of `stride` bytes: the knot bitmaps of every spline (spline e*nr + r, same layout as
// SiftArgs::bitmap), the knot counts [2*nr] (int), the end-rule flags [2*nr] (byte) and the
// marks [nr] (1 subtract the mean envelope, 0 export the mode; signed byte).
struct TapeLayout {
    int nr, ntiles;
    size_t off_kc, off_bf, off_mark, stride;
};
inline TapeLayout tape_layout(int nr, int ntiles) {
    TapeLayout L;
    L.nr = nr;
    L.ntiles = ntiles;
    L.off_kc = (size_t)2 * nr * ntiles * (kTileSamples / 32) * sizeof(unsigned);
    L.off_bf = L.off_kc + (size_t)2 * nr * sizeof(int);
    L.off_mark = L.off_bf + (size_t)2 * nr;
    L.stride = (L.off_mark + (size_t)nr + 255) & ~(size_t)255;
    return L;
}

// The on-chip stage kernel's own arguments (k_sift_small).
struct SmallArgs {
    unsigned* arrive;      // [1] CTAs arrived at the stop test, all iterations of the stage
    int* nfin;             // [cap] realizations finished after each iteration
    double* up;            // [nrows*n] upper envelope of the current iteration
    int spin_limit;        // polls of the stop-test barrier before giving up (CEEMDAN_ERR_TIMEOUT)
    unsigned extra;        // arrivals the barrier waits for beyond the launch's CTAs: 0, or 1 to
                           // make every wait give up (the timeout path's test)
    // taped forward: the stage's tape blocks (slot j at tblocks[j / kTapeBlockSlots] +
    // (j % kTapeBlockSlots) * tl.stride), null otherwise
    unsigned char* const* tblocks;
    TapeLayout tl;
    // two CTAs per realization (upper / lower envelope) when the launch has room for them:
    // per realization the iteration whose upper envelope is ready, its knot count, and the
    // stop decision's mark for the upper CTA
    int pair;
    unsigned* ready;
    int* pair_kmax;
    int* pair_mark;
};
constexpr int kTapeBlockSlots = 32;  // tape slots per allocation block

// The tile kernels come in two register budgets (minimum resident CTAs per SM, the
// __launch_bounds__ of each variant); the batched engine's autotuner picks one, the results
// are the same.  A is the default.
constexpr int kExtremaBlocksA = 6, kExtremaBlocksB = 4;
constexpr int kEvalBlocksA = 5, kEvalBlocksB = 4;
template <int kMinBlocks, bool kLoop>
__global__ void k_extrema_t(SiftArgs a);
template <int kMinBlocks>
__global__ void k_eval_t(SiftArgs a);
__global__ void k_scan_boundary(SiftArgs a);
__global__ void k_gather_knots(SiftArgs a, int e, int32_t* kx, double* ky);
__global__ void k_chunk_reduce(SiftArgs a);
__global__ void k_group_scan(SiftArgs a);
__global__ void k_reduced_solve(SiftArgs a);
__global__ void k_segments(SiftArgs a);

__global__ void k_criterion(SiftArgs a);
__global__ void k_export_final(SiftArgs a, int c);
__global__ void k_plan(SiftArgs a);
__global__ void k_begin_stage(SiftArgs a, int c, int cap, double* mode_out);
// the active-channel plan of k_plan, computed by every thread of one CTA of 1024 threads
__device__ void plan_block(const SiftArgs& a);
// batched engine: stage transitions (stage_kernels.cu); k_stage_end and k_stage_begin run
// kTransThreads threads per CTA, k_stage_stats kLanes, k_commit_plan 1024
constexpr int kTransThreads = 256;
__global__ void k_stage_end(SiftArgs a, BatchArgs b);
__global__ void k_stage_stats(SiftArgs a, BatchArgs b);
__global__ void k_stage_begin(SiftArgs a, BatchArgs b);
__global__ void k_commit_plan(SiftArgs a, BatchArgs b);
// threads per CTA of k_tridiag_batched (its __launch_bounds__); every launch uses this value
constexpr int kTridiagThreads = 256;
__global__ void k_tridiag_batched(int n, const double* l, const double* m, const double* u,
                                  const double* r, double* x, double* sys, double* ws,
                                  size_t ws_stride);
// In-CTA canonical partitioned solve (sift_kernels.cu): system in 4 planes of `plane` doubles
// (l, m, u, r) at sys, solution to x, workspace ws of >= 0.75*n + 16 doubles; every thread of
// the CTA calls it.
__device__ void cta_tridiag(int n, const double* sys, int plane, double* x, double* ws);
// cta_tridiag's solve for nsys systems at once, one level per launch (sift_kernels.cu)
cudaError_t psolve_launch(int nsys, int max_rows, const int* nrows, const double* sys, int plane,
                          double* x, double* ws, size_t ws_stride, cudaStream_t st,
                          int* launches, const int32_t* kx);

// reverse pass (adjoint.cu)
__global__ void k_tape_record(SiftArgs a, TapeLayout L, unsigned char* slot);
__global__ void k_adj_seed(const unsigned char* slot, TapeLayout L, int n, double* gh,
                           double* gm, double* eb, const double* abar, double inr);
__global__ void k_adj_knots(const unsigned char* slot, TapeLayout L, int cap, int32_t* kx);
__global__ void k_adj_segsums(const unsigned char* slot, TapeLayout L, int n, int cap,
                              const int32_t* kx, const double* eb, double* S);
__global__ void k_adj_rows(const unsigned char* slot, TapeLayout L, int cap, const int32_t* kx,
                           const double* S, double* yb, double* sys, int* nrows);
__global__ void k_adj_solve(const unsigned char* slot, TapeLayout L, int cap, const double* sys,
                            double* z, double* ws, size_t ws_stride);
__global__ void k_adj_rhs(const unsigned char* slot, TapeLayout L, int cap, const int32_t* kx,
                          const double* yb, const double* z, double* y2);
__global__ void k_adj_scatter(const unsigned char* slot, TapeLayout L, int n, int cap,
                              const int32_t* kx, const double* y2, double* gh);
__global__ void k_adj_abar(const double* fbar, const double* g, double* abar, size_t n);
__global__ void k_adj_inject(const double* gh, const double* abar, double inr, const double* E,
                             int nr, size_t n, double* hs, double* p);
__global__ void k_adj_stats(int stage, const double* f, const double* stats, const double* p,
                            const double* g, const double* hs, size_t n, double nstd,
                            double inv_n, double inv_nm1, double* scal);
__global__ void k_adj_out(int stage, const double* g, const double* hs, const double* f,
                          const double* stats, const double* scal, double* out, size_t n,
                          double inv_n);

// dynamic shared memory of k_sift_small for rows of n samples
size_t small_sift_smem(int n);
__global__ void k_sift_small(SiftArgs a, SmallArgs sa);

// dynamic shared memory of the reduced solve
size_t reduced_solve_smem(int* qcap);
constexpr int kRedThreads = 128;  // threads per CTA of k_reduced_solve
// Upper bound of reduced_solve_smem(): the function attribute is always set to this value, so
// that decompositions of different sizes running concurrently agree on it.  70 KB keeps three
// CTAs per SM (measured best); level-3 systems beyond what fits use global memory.
constexpr size_t kRedSmemMax = (size_t)70 * 1024;

// stage kernels (stage_kernels.cu)
__global__ void k_canon_mean(const double* v, size_t n, size_t stride, double* acc,
                             double inv_n);
__global__ void k_canon_var(const double* v, size_t n, size_t stride, const double* mean,
                            double* acc, double inv_nm1);
__global__ void k_canon_sums(const double* v, size_t n, const double* mean, double* sum,
                             double* sqdev);
__global__ void k_standardize(double* x, size_t n, const double* var);
__global__ void k_add_noise(double* h0, const double* x, const double* E, size_t n, int nr,
                            double nstd, const double* evar);
__global__ void k_add_noise2(double* h0, const double* r, const double* E, size_t n, int nr,
                             double nstd, const double* svar);
__global__ void k_first_imf(const double* h0, const double* mode, const double* x,
                            double* fornext, double* imf, size_t n, int nr);
__global__ void k_avg_update(const double* h0, const double* mode, double* fornext,
                             double* imf, size_t n, int nr);
__global__ void k_ens_accum(const double* h0, const double* mode, double* tsum, size_t n, int nr,
                            bool first_stage, double inr);
__global__ void k_ens_out(const double* tsum, const double* x, double* fornext, double* imf,
                          size_t n, bool first_stage, double nr_total);
__global__ void k_sub_inplace(double* w, const double* e, size_t count);
__global__ void k_check_iota(const int32_t* x, size_t n, int* err);
__global__ void k_fill_iota(int32_t* x, size_t n);
__global__ void k_widen_f32(const float* src, double* dst, size_t count);
__global__ void k_narrow_f64(const double* src, float* dst, size_t count);

}  // namespace ceemdan
