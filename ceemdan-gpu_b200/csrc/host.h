// Host-side internals shared by the engine's translation units (engine.cu, batch.cu): error
// text and launch counter, the library's stream-ordered memory pool, workspaces, the tape of
// the reverse pass and the sift engine that launches one iteration of the sift kernels.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ceemdan_b200.h"
#include "canon.cuh"
#include "kernels.h"

namespace ceemdan {

extern thread_local std::string g_last_error;  // last error text of the calling thread
extern std::atomic<uint64_t> g_launches;        // kernels launched by the library

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);         \
            return e_ == cudaErrorMemoryAllocation ? CEEMDAN_ERR_NO_MEMORY            \
                                                   : CEEMDAN_ERR_CUDA;                 \
        }                                                                              \
    } while (0)

#define CKS(expr)                              \
    do {                                       \
        ceemdan_status s_ = (expr);            \
        if (s_ != CEEMDAN_OK) return s_;       \
    } while (0)

constexpr int kThreads = 256;

const double* rcp_tables();
int sm_count();
cudaMemPool_t engine_pool();
ceemdan_status pool_alloc(void** p, size_t bytes, cudaStream_t st);
int* pinned_state();
void release_pinned_state(int* p);
void sx_bounds(double t, double* hi, double* lo);
int grid_for(size_t count);
ceemdan_status generate_noise(double* w, size_t count, uint64_t seed, cudaStream_t st);

// Device allocations owned by one decomposition (or one stage-level call), stream-ordered on
// the call's stream: freed after the work queued on it.
struct Workspace {
    cudaStream_t st;
    std::vector<void*> blocks;
    explicit Workspace(cudaStream_t s) : st(s) {}
    Workspace(const Workspace&) = delete;
    Workspace& operator=(const Workspace&) = delete;
    ceemdan_status alloc(void** p, size_t bytes) {
        const ceemdan_status s = pool_alloc(p, bytes, st);
        if (s == CEEMDAN_OK) blocks.push_back(*p);
        return s;
    }
    template <class T>
    ceemdan_status alloc_n(T** p, size_t count) {
        return alloc(reinterpret_cast<void**>(p), count * sizeof(T));
    }
    ~Workspace() {
        for (void* p : blocks) cudaFreeAsync(p, st);
    }
};

}  // namespace ceemdan

// Frozen structure of one taped forward call (opaque in the C ABI): one tape slot per executed
// iteration of every signal stage (ceemdan::TapeLayout), in device blocks of kBlockSlots
// slots, plus what the reverse pass of the stage statistics needs: the noise modes, each
// stage's input (y for stage 0, the previous ensemble mean after it) and its carried mean and
// variance.  All of it comes from the library's memory pool.
struct ceemdan_tape {
    static constexpr int kBlockSlots = ceemdan::kTapeBlockSlots;
    struct Stage {
        int J = 0;
        std::vector<unsigned char*> blocks;
    };
    int device = 0;
    size_t nr = 0, n = 0, nimf = 0;
    double nstd = 0.0;
    ceemdan::TapeLayout L{};
    std::vector<Stage> stages;
    double* E = nullptr;      // num_imfs*nr*n
    double* fin = nullptr;    // (num_imfs-1)*n
    double* stats = nullptr;  // 2*(num_imfs-1): mean, variance
    size_t bytes = 0;
    // checkpointed form: instead of the iterations, each stage's input h0 [nr*n] and the
    // mean-envelope [nr*n] and sifting-fraction [nr] carries it started from (the whole state
    // its sift depends on); the reverse pass re-runs the stage from them with the forward's
    // options and sift cap
    bool checkpointed = false;
    double* ck = nullptr;     // (num_imfs-1) * (2*nr*n + nr)
    ceemdan_options opts{};
    size_t max_iter = 0;

    size_t ck_stride() const { return 2 * nr * n + nr; }

    const unsigned char* slot(size_t stage, long j) const {
        return stages[stage].blocks[(size_t)j / kBlockSlots] + (size_t)(j % kBlockSlots) * L.stride;
    }
    ceemdan_status alloc(void** p, size_t b, cudaStream_t st) {
        const ceemdan_status s = ceemdan::pool_alloc(p, b, st);
        if (s == CEEMDAN_OK) bytes += b;
        return s;
    }
    // slot j of a stage being recorded (its block allocated on first use, on st); null when
    // out of device memory
    unsigned char* grow(size_t stage, long j, cudaStream_t st) {
        auto& b = stages[stage].blocks;
        while (b.size() <= (size_t)j / kBlockSlots) {
            void* p = nullptr;
            if (alloc(&p, (size_t)kBlockSlots * L.stride, st) != CEEMDAN_OK) return nullptr;
            b.push_back(static_cast<unsigned char*>(p));
        }
        return b[(size_t)j / kBlockSlots] + (size_t)(j % kBlockSlots) * L.stride;
    }
    // free the blocks past the stage's J executed iterations (after the work queued on st)
    void trim(size_t stage, cudaStream_t st) {
        auto& b = stages[stage].blocks;
        const size_t keep = ((size_t)stages[stage].J + kBlockSlots - 1) / kBlockSlots;
        while (b.size() > keep) {
            cudaFreeAsync(b.back(), st);
            b.pop_back();
            bytes -= (size_t)kBlockSlots * L.stride;
        }
    }
    // free every block after the work queued on st (the tape keeps its other buffers)
    void free_blocks(cudaStream_t st) {
        for (size_t i = 0; i < stages.size(); ++i) {
            for (unsigned char* p : stages[i].blocks) cudaFreeAsync(p, st);
            bytes -= stages[i].blocks.size() * (size_t)kBlockSlots * L.stride;
            stages[i].blocks.clear();
        }
    }
    // every call that used the tape has returned (they are synchronous): free on this
    // thread's stream of the tape's device
    ~ceemdan_tape() {
        int cur = -1;
        const bool other = cudaGetDevice(&cur) == cudaSuccess && cur != device;
        if (other) cudaSetDevice(device);
        for (auto& s : stages)
            for (unsigned char* p : s.blocks) cudaFreeAsync(p, cudaStreamPerThread);
        for (void* p : {(void*)E, (void*)fin, (void*)stats, (void*)ck})
            if (p) cudaFreeAsync(p, cudaStreamPerThread);
        if (other) cudaSetDevice(cur);
    }
};

namespace ceemdan {

// One channel of a sift engine: nr realizations of n samples.
struct ChanSpec {
    int n, nr;
};

// Sifting state of one or several channels (shared by all stages of a call).  With one
// channel, run_stage drives the lock-step sift of a stage from the host; the batched engine
// (batch.cu) drives several channels from the device.
struct SiftEngine {
    SiftArgs a{};
    double* h[2] = {nullptr, nullptr};
    ChanState* cs = nullptr;  // device [nchan]
    int* state = nullptr;     // channel 0's (done, iter, err, cap) = the first words of cs[0]
    int* hstate = nullptr;    // pinned host mirror: two slots of (done, iter, err, cap)
    std::vector<Chan> hchan;  // host copy of the channel table
    int nr = 0, n = 0, ntiles = 0;  // channel 0
    cudaEvent_t group_ev[2] = {nullptr, nullptr};
    int group = 4;
    size_t red_smem = 0;
    // persistent grids: resident CTAs x SMs (the separator kernels), or the work itself
    int reduce_grid = 0, segments_grid = 0, red_grid = 0, tile_grid = 0, eval_grid = 0,
        scan_grid = 0;
    double* kernel_ms = nullptr;           // host accumulators (optional)
    std::vector<cudaEvent_t> ev;           // [group][kinds][2] when timing
    ceemdan_tape* tape = nullptr;          // taped forward: the stage being recorded
    size_t tape_stage = 0;
    bool plan_by_caller = false;           // the batched loop computes the plan (k_commit_plan)
    bool extrema_b = false, eval_b = false;  // the tile kernels' second register budgets

    ceemdan_status init(Workspace& ws, int nr_, int n_, const ceemdan_options& o) {
        return init(ws, std::vector<ChanSpec>{{n_, nr_}}, o);
    }

    ceemdan_status init(Workspace& ws, const std::vector<ChanSpec>& chans,
                        const ceemdan_options& o) {
        const int nchan = (int)chans.size();
        hchan.resize(chans.size());
        long long rows = 0, tiles = 0, samp = 0, rec = 0, red = 0;
        for (int c = 0; c < nchan; ++c) {
            Chan& ch = hchan[c];
            std::memset(&ch, 0, sizeof(ch));
            ch.n = chans[c].n;
            ch.nr = chans[c].nr;
            ch.ntiles = (ch.n + kTileSamples - 1) / kTileSamples;
            ch.cap = ch.n / 2 + 2;
            // separators per spline: per tile with c knots (c + 14)/16 + 1, so at most
            // K/16 + 2*ntiles over the spline (K <= cap)
            ch.rec_stride = ((ch.cap + kChunk - 1) / kChunk + 2 * ch.ntiles + 8 + 3) & ~3;
            ch.row0 = (int)rows;
            ch.tile0 = (int)tiles;
            ch.samp0 = samp;
            ch.rec0 = rec;
            ch.red0 = red;
            rows += ch.nr;
            tiles += (long long)ch.nr * ch.ntiles;
            // every channel's block of rows starts 256-byte aligned (16-byte sample pairs)
            samp += ((long long)ch.nr * ch.n + 31) & ~31LL;
            rec += (long long)ch.nr * ch.rec_stride;
            red += (long long)ch.nr * red_stride_of(ch.rec_stride);
        }
        if (rows > 0x3fffffffLL || tiles > 0x3fffffffLL) {
            g_last_error = "too many realizations or tiles for one engine";
            return CEEMDAN_ERR_INVALID_ARG;
        }
        nr = hchan[0].nr;
        n = hchan[0].n;
        ntiles = hchan[0].ntiles;
        a.n1 = n;
        a.ntiles1 = ntiles;
        a.nr1 = nr;
        a.rs1 = hchan[0].rec_stride;
        a.par = -1;
        a.nrows = (int)rows;
        a.nchan = nchan;
        a.ntot = (int)tiles;
        a.rec_total = rec;
        a.red_total = red;
        a.rec_plane = (size_t)2 * (size_t)rec;
        a.spin_limit = o.spin_limit > 0 ? o.spin_limit : (1 << 22);
        a.sd = o.sd;
        a.sd2 = o.sd2;
        sx_bounds(o.sd, &a.sd_hi, &a.sd_lo);
        sx_bounds(o.sd2, &a.sd2_hi, &a.sd2_lo);
        a.tol = o.tol;
        const size_t R = (size_t)rows, T = (size_t)tiles, S = (size_t)samp;
        const size_t kn = T * kTileCap;  // per-tile knot slots
        CKS(ws.alloc_n(&h[0], S));
        CKS(ws.alloc_n(&h[1], S));
        a.h[0] = h[0];
        a.h[1] = h[1];
        CKS(ws.alloc_n(&a.menv, S));
        CKS(ws.alloc_n(&a.mark, R));
        CKS(ws.alloc_n(&a.finish, R));
        CKS(ws.alloc_n(&a.frac, R));
        CKS(ws.alloc_n(&a.cnt, R));
        CKS(ws.alloc_n(&a.any, R));
        CKS(ws.alloc_n(&a.kcount, 2 * R));
        CKS(ws.alloc_n(&a.tile_cnt, 2 * T));
        CKS(ws.alloc_n(&a.tile_off, 2 * (T + R)));
        CKS(ws.alloc_n(&a.sep_off, 2 * (T + R)));
        CKS(ws.alloc_n(&a.pcount, 2 * R));
        CKS(ws.alloc_n(&a.gcount, 2 * R));
        CKS(ws.alloc_n(&a.gsum, 2 * R + 1));
        CKS(ws.alloc_n(&a.plan, 2 * (size_t)nchan + 2));
        CKS(ws.alloc_n(&a.bitmap, 2 * T * (kTileSamples / 32)));
        CKS(ws.alloc_n(&a.nbr, 2 * T * 2));
        CKS(ws.alloc_n(&a.kx_max, kn));
        CKS(ws.alloc_n(&a.kx_min, kn));
        CKS(ws.alloc_n(&a.ky_max, kn));
        CKS(ws.alloc_n(&a.ky_min, kn));
        for (int e = 0; e < 2; ++e) CKS(ws.alloc_n(&a.seg[e], 4 * kn));
        CKS(ws.alloc_n(&a.rec, 10 * a.rec_plane));
        CKS(ws.alloc_n(&a.xsep, 2 * (size_t)rec));
        CKS(ws.alloc_n(&a.red, 2 * (size_t)red));
        double* rcp = nullptr;
        CKS(ws.alloc_n(&rcp, 2 * (size_t)(kRcpMax + 1)));
        CK(cudaMemcpyAsync(rcp, rcp_tables(), sizeof(double) * 2 * (kRcpMax + 1),
                           cudaMemcpyHostToDevice, ws.st));
        a.rcp_h = rcp;
        a.rcp_3h = rcp + (kRcpMax + 1);
        Chan* dchan = nullptr;
        CKS(ws.alloc_n(&dchan, (size_t)nchan));
        CK(cudaMemcpyAsync(dchan, hchan.data(), sizeof(Chan) * nchan, cudaMemcpyHostToDevice,
                           ws.st));
        a.chan = dchan;
        CKS(ws.alloc_n(&cs, (size_t)nchan));
        a.cs = cs;
        state = reinterpret_cast<int*>(cs);
        hstate = pinned_state();
        if (!hstate) {
            g_last_error = "cudaMallocHost failed";
            return CEEMDAN_ERR_NO_MEMORY;
        }
        CK(cudaEventCreateWithFlags(&group_ev[0], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&group_ev[1], cudaEventDisableTiming));
        const size_t rn = (size_t)samp;
        if (o.group > 0) {
            group = o.group;
        } else {
            group = rn >= (size_t)(1 << 22) ? 4 : (rn >= (size_t)(1 << 18) ? 8 : 32);
        }
        int dev = 0, sms = 0, per = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_chunk_reduce, 128, 0));
        reduce_grid = std::max(1, per) * sms;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_segments, 64, 0));
        segments_grid = std::max(1, per) * sms;
        red_smem = reduced_solve_smem(&a.red_qcap);
        // the bound, not this call's size: concurrent calls of other sizes set the same value
        CK(cudaFuncSetAttribute(k_reduced_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kRedSmemMax));
        // one CTA per tile / spline when every channel sifts (the whole work in one wave of
        // launches); the batched engine caps these at a few waves of resident CTAs
        tile_grid = (int)std::max<size_t>(1, T);
        eval_grid = tile_grid;
        // the tile kernels' second register budgets (the batched engine's tuner chooses them;
        // CEEMDAN_TILE_BUDGET=B selects them for the one-channel engine)
        if (const char* e = std::getenv("CEEMDAN_TILE_BUDGET"))
            if (e[0] == 'B') extrema_b = eval_b = true;
        red_grid = (int)std::max<size_t>(1, 2 * R);
        scan_grid = (int)std::max<size_t>(1, (2 * R + 7) / 8);
        return CEEMDAN_OK;
    }

    ~SiftEngine() {
        if (hstate) release_pinned_state(hstate);
        for (cudaEvent_t e : group_ev)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }

    // kinds timed per iteration (the on-chip stage kernel is timed per launch)
    static constexpr int kIterKinds = CEEMDAN_K_SIFT_SMALL;

    ceemdan_status enable_timing(double* ms) {
        kernel_ms = ms;
        ev.resize((size_t)2 * group * kIterKinds * 2 + 2);
        for (auto& e : ev) CK(cudaEventCreate(&e));
        return CEEMDAN_OK;
    }

    cudaEvent_t event(int it, int kind, int end) {
        return ev[((size_t)it * kIterKinds + kind) * 2 + end];
    }

    // Add the event-timed durations of iterations [first, first+count) (completed).
    void harvest_timing(long first, long count) {
        if (!kernel_ms) return;
        for (long j = first; j < first + count; ++j) {
            const int it = (int)(j % (2 * group));
            for (int k = 0; k < kIterKinds; ++k) {
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, event(it, k, 0), event(it, k, 1)) == cudaSuccess)
                    kernel_ms[k] += ms;
            }
        }
    }

    // Zero the whole-call carries: mean envelope and sifting fraction accumulator, and the
    // channels' states.
    ceemdan_status reset_carries(cudaStream_t st) {
        const Chan& last = hchan.back();
        const size_t S = (size_t)last.samp0 + (size_t)last.nr * last.n;
        CK(cudaMemsetAsync(a.menv, 0, sizeof(double) * S, st));
        CK(cudaMemsetAsync(a.frac, 0, sizeof(double) * a.nrows, st));
        CK(cudaMemsetAsync(a.cnt, 0, sizeof(unsigned) * a.nrows, st));
        CK(cudaMemsetAsync(a.any, 0, sizeof(int) * a.nrows, st));
        CK(cudaMemsetAsync(cs, 0, sizeof(ChanState) * a.nchan, st));
        return CEEMDAN_OK;
    }

    // Launch one sift iteration of every channel whose stage runs (channel c reads
    // h[iter_c%2], writes h[(iter_c+1)%2]).
    ceemdan_status launch_iteration(long j, cudaStream_t st) {
        unsigned char* slot = nullptr;
        if (tape) {
            slot = tape->grow(tape_stage, j, st);
            if (!slot) {
                g_last_error = "out of device memory for the tape";
                return CEEMDAN_ERR_NO_MEMORY;
            }
        }
        a.tape_mark = slot ? reinterpret_cast<signed char*>(slot + tape->L.off_mark) : nullptr;
        // one channel driven from the host: iteration j of the stage reads h[j%2] (the device
        // counter equals j until the stage has finished, and then the kernels return at once)
        a.par = (a.nchan == 1 && !plan_by_caller) ? (int)(j & 1) : -1;
        const bool timed = kernel_ms != nullptr;
        const int ti = (int)(j % (2 * group));
        // inside a stream capture an event record becomes a graph node only as an external
        // event (a plain record would only order the capture)
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (timed) cudaStreamIsCapturing(st, &cap);
        const unsigned ev_flags =
            cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
        auto mark_ev = [&](int kind, int end) {
            if (timed) cudaEventRecordWithFlags(event(ti, kind, end), st, ev_flags);
        };
        if (a.nchan > 1 && !plan_by_caller) {
            k_plan<<<1, 1024, 0, st>>>(a);
            ++g_launches;
        }
        mark_ev(CEEMDAN_K_EXTREMA, 0);
        // a grid that covers every tile runs one tile per CTA (no persistent loop)
        const bool loop = tile_grid < a.ntot;
        if (extrema_b && loop)
            k_extrema_t<kExtremaBlocksB, true><<<tile_grid, kThreads, 0, st>>>(a);
        else if (extrema_b)
            k_extrema_t<kExtremaBlocksB, false><<<tile_grid, kThreads, 0, st>>>(a);
        else if (loop)
            k_extrema_t<kExtremaBlocksA, true><<<tile_grid, kThreads, 0, st>>>(a);
        else
            k_extrema_t<kExtremaBlocksA, false><<<tile_grid, kThreads, 0, st>>>(a);
        mark_ev(CEEMDAN_K_EXTREMA, 1);
        mark_ev(CEEMDAN_K_BOUNDARY, 0);
        k_scan_boundary<<<scan_grid, kThreads, 0, st>>>(a);
        mark_ev(CEEMDAN_K_BOUNDARY, 1);
        mark_ev(CEEMDAN_K_CHUNK_REDUCE, 0);
        k_group_scan<<<1, 1024, 0, st>>>(a);
        k_chunk_reduce<<<reduce_grid, 128, 0, st>>>(a);
        mark_ev(CEEMDAN_K_CHUNK_REDUCE, 1);
        mark_ev(CEEMDAN_K_REDUCED_SOLVE, 0);
        k_reduced_solve<<<red_grid, kRedThreads, red_smem, st>>>(a);
        mark_ev(CEEMDAN_K_REDUCED_SOLVE, 1);
        mark_ev(CEEMDAN_K_SEGMENTS, 0);
        k_segments<<<segments_grid, 64, 0, st>>>(a);
        mark_ev(CEEMDAN_K_SEGMENTS, 1);
        mark_ev(CEEMDAN_K_EVAL, 0);
        if (eval_b)
            k_eval_t<kEvalBlocksB><<<eval_grid, kThreads, 0, st>>>(a);
        else
            k_eval_t<kEvalBlocksA><<<eval_grid, kThreads, 0, st>>>(a);
        mark_ev(CEEMDAN_K_EVAL, 1);
        if (slot) {
            const size_t pieces = tape->L.off_kc / 16;  // 16-byte pieces of the bitmaps
            const unsigned g = (unsigned)std::min<size_t>((pieces + kThreads - 1) / kThreads,
                                                          (size_t)sm_count() * 8);
            k_tape_record<<<g, kThreads, 0, st>>>(a, tape->L, slot);
            ++g_launches;
        }
        mark_ev(CEEMDAN_K_CRITERION, 0);
        if (!a.dbg_upper) k_criterion<<<std::min(a.nchan, 4 * sm_count()), kThreads, 0, st>>>(a);
        mark_ev(CEEMDAN_K_CRITERION, 1);
        g_launches += a.dbg_upper ? 7 : 8;
        CK(cudaGetLastError());
        return CEEMDAN_OK;
    }

    // Lock-step sift of all realizations of channel 0 until every one has finished (or cap).
    // h[0] holds the stage input; modes are written to mode_out.  Iterations are launched in
    // groups; the host reads the stop word of group g while group g+1 is already queued, so
    // the device never waits for the host.  Iterations after the stop word is set return
    // at once.
    // Short rows (one channel, n <= kSmallMaxN, every realization a CTA resident at once):
    // a stage runs as one cooperative launch of k_sift_small instead of groups of iterations.
    bool small = false;
    SmallArgs sa{};
    size_t small_smem = 0;

    ceemdan_status enable_small(Workspace& ws, int max_cap, int spin_limit) {
        if (a.nchan != 1 || n > kSmallMaxN) return CEEMDAN_OK;
        if (const char* e = std::getenv("CEEMDAN_SMALL"))
            if (e[0] == '0') return CEEMDAN_OK;
        int dev = 0, coop = 0, sms = 0, per = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (!coop) return CEEMDAN_OK;
        small_smem = small_sift_smem(n);
        CK(cudaFuncSetAttribute(k_sift_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)small_sift_smem(kSmallMaxN)));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sift_small, kSmallThreads,
                                                         small_smem));
        if (per < 1 || nr > per * sms) return CEEMDAN_OK;
        // two CTAs per realization when they fit one per SM (CEEMDAN_SMALL_PAIR=0: one CTA)
        sa.pair = 2 * nr <= sms ? 1 : 0;
        if (const char* e = std::getenv("CEEMDAN_SMALL_PAIR"))
            if (e[0] == '0') sa.pair = 0;
        // the CTAs are latency-bound: when the launch has at most one CTA per SM, ask for more
        // than half an SM's shared memory so that no two of them share an SM
        if ((sa.pair ? 2 * nr : nr) <= sms)
            small_smem = std::max(small_smem, (size_t)kSmallSpreadSmem);
        CKS(ws.alloc_n(&sa.ready, (size_t)nr));
        CKS(ws.alloc_n(&sa.pair_kmax, (size_t)nr));
        CKS(ws.alloc_n(&sa.pair_mark, (size_t)nr));
        CKS(ws.alloc_n(&sa.arrive, 1));
        CKS(ws.alloc_n(&sa.nfin, (size_t)std::max(1, max_cap)));
        CKS(ws.alloc_n(&sa.up, (size_t)nr * n));
        // device copy of a taped stage's block table (blocks of kTapeBlockSlots slots)
        CKS(ws.alloc_n(&tblocks_dev, (size_t)(std::max(1, max_cap) + kTapeBlockSlots - 1) /
                                         kTapeBlockSlots));
        // a negative limit -k: the test of the timeout path (every wait gives up after k polls)
        sa.spin_limit = spin_limit > 0 ? spin_limit : (spin_limit < 0 ? -spin_limit : (1 << 22));
        sa.extra = spin_limit < 0 ? 1u : 0u;
        small_cap = std::max(1, max_cap);
        small = true;
        return CEEMDAN_OK;
    }
    int small_cap = 0;
    unsigned char** tblocks_dev = nullptr;

    // One stage on chip (k_sift_small); the realizations that finish in the last iteration
    // export their modes inside the kernel.
    ceemdan_status run_stage_small(double* mode_out, int cap, cudaStream_t st, int* iters_out) {
        sa.tblocks = nullptr;
        if (tape) {  // every slot the stage may fill (the caller trims past the iterations run)
            if (!tape->grow(tape_stage, (long)cap - 1, st)) {
                g_last_error = "out of device memory for the tape";
                return CEEMDAN_ERR_NO_MEMORY;
            }
            const auto& blocks = tape->stages[tape_stage].blocks;
            CK(cudaMemcpyAsync(tblocks_dev, blocks.data(), blocks.size() * sizeof(unsigned char*),
                               cudaMemcpyHostToDevice, st));
            sa.tblocks = tblocks_dev;
            sa.tl = tape->L;
        }
        k_begin_stage<<<1, kThreads, 0, st>>>(a, 0, cap, mode_out);
        ++g_launches;
        CK(cudaMemsetAsync(sa.arrive, 0, sizeof(unsigned), st));
        CK(cudaMemsetAsync(sa.ready, 0, sizeof(unsigned) * (size_t)nr, st));
        CK(cudaMemsetAsync(sa.nfin, 0, sizeof(int) * (size_t)std::min(cap, small_cap), st));
        void* args[] = {(void*)&a, (void*)&sa};
        cudaEvent_t* sev = kernel_ms ? &ev[ev.size() - 2] : nullptr;
        if (sev) CK(cudaEventRecord(sev[0], st));
        CK(cudaLaunchCooperativeKernel((const void*)k_sift_small,
                                       dim3((unsigned)(sa.pair ? 2 * nr : nr)),
                                       dim3(kSmallThreads), args, small_smem, st));
        ++g_launches;
        if (sev) CK(cudaEventRecord(sev[1], st));
        CK(cudaMemcpyAsync(hstate, state, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (sev) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, sev[0], sev[1]));
            kernel_ms[CEEMDAN_K_SIFT_SMALL] += ms;
        }
        if (hstate[2] != 0) {
            g_last_error = hstate[2] == CEEMDAN_ERR_TIMEOUT
                               ? "the lock-step stop test of the on-chip sift ran out of polls"
                               : "a sift kernel reported an error in the device error word";
            return (ceemdan_status)hstate[2];
        }
        if (iters_out) *iters_out = hstate[1];
        return CEEMDAN_OK;
    }

    // Realizations split over parts: the stop test of every iteration is the AND over the
    // parts (ceemdan_split::all_finished), so the stage runs iteration by iteration with the
    // flag read back after each one.
    const ceemdan_split* split = nullptr;

    ceemdan_status run_stage_split(double* mode_out, int cap, cudaStream_t st, int* iters_out,
                                   volatile int32_t* cancel) {
        k_begin_stage<<<1, kThreads, 0, st>>>(a, 0, cap, mode_out);
        ++g_launches;
        CK(cudaGetLastError());
        for (long j = 0; j < cap; ++j) {
            CKS(launch_iteration(j, st));
            CK(cudaMemcpyAsync(hstate, state, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            harvest_timing(j, 1);
            if (hstate[2] != 0) {
                g_last_error = "a sift kernel reported an error in the device error word";
                return (ceemdan_status)hstate[2];
            }
            const int local = hstate[0] != 0 ? 1 : 0;  // this part's realizations all finished
            const int all = split->all_finished(split->ctx, local);
            if (all < 0) {
                g_last_error = "the split's all_finished exchange failed";
                return CEEMDAN_ERR_CUDA;
            }
            if (all) break;
            // another part still sifts: so do this part's realizations (lock step)
            if (local) CK(cudaMemsetAsync(state, 0, sizeof(int), st));
            if (cancel && *cancel) {
                cudaStreamSynchronize(st);
                g_last_error = "cancelled by the host cancel word";
                return CEEMDAN_ERR_CANCELLED;
            }
        }
        if (iters_out) *iters_out = hstate[1];
        const int bx = std::max(1, std::min((n + kThreads - 1) / kThreads, 64));
        k_export_final<<<dim3(bx, nr), kThreads, 0, st>>>(a, 0);
        ++g_launches;
        CK(cudaGetLastError());
        return CEEMDAN_OK;
    }

    ceemdan_status run_stage(double* mode_out, int cap, cudaStream_t st, int* iters_out,
                             volatile int32_t* cancel) {
        if (split) return run_stage_split(mode_out, cap, st, iters_out, cancel);
        if (small && cap <= small_cap) {
            if (cancel && *cancel) {
                g_last_error = "cancelled by the host cancel word";
                return CEEMDAN_ERR_CANCELLED;
            }
            return run_stage_small(mode_out, cap, st, iters_out);
        }
        k_begin_stage<<<1, kThreads, 0, st>>>(a, 0, cap, mode_out);
        ++g_launches;
        CK(cudaGetLastError());
        long launched = 0;
        int slot = 0;
        long group_first[2] = {0, 0};
        auto launch_group = [&](int sl) -> ceemdan_status {
            group_first[sl] = launched;
            for (int g = 0; g < group; ++g) CKS(launch_iteration(launched++, st));
            CK(cudaMemcpyAsync(hstate + 4 * sl, state, 4 * sizeof(int), cudaMemcpyDeviceToHost,
                               st));
            CK(cudaEventRecord(group_ev[sl], st));
            return CEEMDAN_OK;
        };
        CKS(launch_group(slot));
        for (;;) {
            CKS(launch_group(slot ^ 1));
            CK(cudaEventSynchronize(group_ev[slot]));
            harvest_timing(group_first[slot], group);
            const int* hs = hstate + 4 * slot;
            if (hs[2] != 0) {
                cudaStreamSynchronize(st);
                g_last_error = "a sift kernel reported an error in the device error word";
                return (ceemdan_status)hs[2];
            }
            if (hs[0]) break;
            if (cancel && *cancel) {
                cudaStreamSynchronize(st);
                g_last_error = "cancelled by the host cancel word";
                return CEEMDAN_ERR_CANCELLED;
            }
            slot ^= 1;
        }
        CK(cudaStreamSynchronize(st));
        harvest_timing(group_first[slot ^ 1], group);
        const int iters = hstate[4 * (slot ^ 1) + 1];  // final value (latest copy)
        if (iters_out) *iters_out = iters;
        const int bx = std::max(1, std::min((n + kThreads - 1) / kThreads, 64));
        k_export_final<<<dim3(bx, nr), kThreads, 0, st>>>(a, 0);
        ++g_launches;
        CK(cudaGetLastError());
        return CEEMDAN_OK;
    }
};

}  // namespace ceemdan
