// Batched engine: many channels of different lengths, each decomposed exactly as
// ceemdan_plain_f64 decomposes it, sifted together by one device-driven loop.
//
// The reference decomposes one channel per call (iceemdanD, cudaICEEMDAN.cu:1340-2059), with
// its stages in sequence and a host round trip per sift iteration.  Here every channel of a
// wave owns its rows of one ragged layout (kernels.h: Chan) and runs its own sequence of
// stages; one iteration of the loop is
//   k_stage_end, k_stage_stats, k_stage_begin, k_commit_plan   (channels whose stage finished
//                                                               move to their next stage)
//   k_extrema ... k_criterion                                  (one sift iteration of every
//                                                               channel whose stage runs)
// so channels never wait for each other: a channel that finishes a stage starts the next one
// at the next iteration, in the same launches as the others.  G iterations are captured once
// in a CUDA graph (two copies, so that the host reads the finished-channel count of one while
// the other runs) and replayed until every channel has finished; the host never launches
// single kernels inside the loop.  The persistent grid sizes are chosen by a small autotuner
// that times the first replays of the wave with each candidate (the candidates compute the
// same results: only the assignment of tiles and splines to CTAs and the tile kernels'
// register budgets differ) and keeps the fastest for later waves and calls of the same shape.
//
// Channels that do not fit the device memory together are processed in waves, longest first.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "host.h"

namespace ceemdan {
namespace {

struct BatchChannel {
    size_t n;
    const double* y;
    double* imfs;
    uint64_t seed;
    size_t index;               // position in the caller's list
    const double* noise = nullptr;  // [nr*n] N(0,1) noise; null = cuRAND with `seed`
};

// Launch shapes of one wave: persistent grid sizes (in multiples of the resident CTAs of the
// whole GPU) and the register budgets of the tile kernels.  Every choice computes the same
// results: only the assignment of tiles and splines to CTAs and the registers differ.
struct TuneConfig {
    int tile_mult;    // k_extrema / k_eval: 1, 2 or 4 waves of resident CTAs
    int split_mult;   // k_chunk_reduce / k_segments: 1 or 2
    int extrema_b;    // k_extrema with its second register budget
    int eval_b;       // k_eval with its second register budget
    bool operator<(const TuneConfig& o) const {
        return std::tie(tile_mult, split_mult, extrema_b, eval_b) <
               std::tie(o.tile_mult, o.split_mult, o.extrema_b, o.eval_b);
    }
    bool operator==(const TuneConfig& o) const { return !(*this < o) && !(o < *this); }
};

constexpr TuneConfig kDefaultConfig = {1, 1, 0, 0};

// kernels of one loop iteration: four transitions and eight sift kernels
constexpr int kLoopKernels = 12;

// Tuned configurations by shape: channels, realizations, total samples (log2 bucket).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, TuneConfig> g_tuned;

std::tuple<int, int, int> shape_key(const std::vector<BatchChannel>& ch, size_t nr) {
    size_t tot = 0;
    for (const auto& c : ch) tot += c.n;
    int lg = 0;
    while (((size_t)1 << (lg + 1)) <= tot) ++lg;
    return std::make_tuple((int)ch.size(), (int)nr, lg);
}

// Device bytes of one channel in a wave (sift state, noise modes, knots, records).
size_t channel_bytes(size_t n, size_t nr, size_t nimf) {
    const size_t rn = nr * n;
    const size_t tiles = nr * ((n + kTileSamples - 1) / kTileSamples);
    const size_t planes = (nimf + 6) * rn * 8;          // h x2, menv, W, H0, MODE, E
    const size_t knots = tiles * kTileCap * (2 * 12 + 2 * 32);  // kx, ky, records (x2)
    const size_t rec = nr * (n / 2 / kChunk + 64) * 8 * 2 * 17;  // chunk records, X, workspace
    return planes + knots + rec + tiles * 1024;
}

struct Wave {
    cudaStream_t st;
    SiftEngine eng;
    BatchArgs b{};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int G = 8;
    explicit Wave(cudaStream_t s) : st(s) {}
    ~Wave() {
        if (exec[0] || exec[1]) cudaStreamSynchronize(st);  // no replay still running
        for (auto& e : exec)
            if (e) cudaGraphExecDestroy(e);
    }
};

// Capture G iterations of the batched loop into an executable graph; iteration numbers
// first..first+G-1 select the timing events (when timing is on).
ceemdan_status capture(Wave& w, cudaStream_t st, long first, cudaGraphExec_t* out) {
    SiftEngine& eng = w.eng;
    const int sms = sm_count();
    const unsigned gT = (unsigned)std::max(1, 4 * sms);
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    ceemdan_status rc = CEEMDAN_OK;
    for (int j = 0; j < w.G && rc == CEEMDAN_OK; ++j) {
        k_stage_end<<<gT, kTransThreads, 0, st>>>(eng.a, w.b);
        k_stage_stats<<<gT, kLanes, 0, st>>>(eng.a, w.b);
        k_stage_begin<<<gT, kTransThreads, 0, st>>>(eng.a, w.b);
        k_commit_plan<<<1, 1024, 0, st>>>(eng.a, w.b);
        rc = eng.launch_iteration(first + j, st);
    }
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (rc != CEEMDAN_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess) {
        g_last_error = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce);
        return CEEMDAN_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        g_last_error = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie);
        return CEEMDAN_ERR_CUDA;
    }
    return CEEMDAN_OK;
}

void apply_config(SiftEngine& eng, const TuneConfig& t) {
    const int sms = sm_count();
    int per = 0;
    eng.extrema_b = t.extrema_b != 0;
    eng.eval_b = t.eval_b != 0;
    if (eng.extrema_b)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_extrema_t<kExtremaBlocksB, true>,
                                                      kThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_extrema_t<kExtremaBlocksA, true>,
                                                      kThreads, 0);
    eng.tile_grid = std::max(1, std::min(eng.a.ntot, t.tile_mult * std::max(1, per) * sms));
    if (eng.eval_b)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_eval_t<kEvalBlocksB>, kThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_eval_t<kEvalBlocksA>, kThreads, 0);
    eng.eval_grid = std::max(1, std::min(eng.a.ntot, t.tile_mult * std::max(1, per) * sms));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_chunk_reduce, 128, 0);
    eng.reduce_grid = t.split_mult * std::max(1, per) * sms;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_segments, 64, 0);
    eng.segments_grid = t.split_mult * std::max(1, per) * sms;
    cudaGetLastError();
}

ceemdan_status run_wave(const std::vector<BatchChannel>& ch, size_t nr, size_t nimf,
                        size_t max_iter, double nstd, const ceemdan_options& o,
                        cudaStream_t st, int32_t* h_iters, size_t* peak_bytes) {
    const int nchan = (int)ch.size();
    const int M = (int)nimf - 1;
    Workspace ws(st);
    Wave w(st);
    SiftEngine& eng = w.eng;
    std::vector<ChanSpec> specs(ch.size());
    for (int c = 0; c < nchan; ++c) specs[c] = ChanSpec{(int)ch[c].n, (int)nr};
    cudaMemPool_t pool = engine_pool();
    if (pool) {
        uint64_t zero = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero);
    }
    CKS(eng.init(ws, specs, o));
    const Chan& lastc = eng.hchan.back();
    const size_t S = (size_t)lastc.samp0 + (((size_t)lastc.nr * lastc.n + 31) & ~(size_t)31);
    BatchArgs& b = w.b;
    b.nimf = (int)nimf;
    b.M = M;
    b.noise_cap = o.noise_sift_cap;
    b.max_iter = (int)std::min<size_t>(max_iter, 0x7fffffff);
    b.nstd = nstd;
    b.S = S;
    std::vector<long long> xoff(ch.size());
    size_t X = 0;
    for (int c = 0; c < nchan; ++c) {
        xoff[c] = (long long)X;
        X += (ch[c].n + 31) & ~(size_t)31;
    }
    CKS(ws.alloc_n(&b.W, S));
    CKS(ws.alloc_n(&b.E, nimf * S));
    CKS(ws.alloc_n(&b.H0, S));
    CKS(ws.alloc_n(&b.MODE, S));
    CKS(ws.alloc_n(&b.XS, X));
    CKS(ws.alloc_n(&b.FN, X));
    long long* dxoff = nullptr;
    double** dimfs = nullptr;
    CKS(ws.alloc_n(&dxoff, ch.size()));
    CKS(ws.alloc_n(&dimfs, ch.size()));
    b.xoff = dxoff;
    b.imfs = dimfs;
    double* stat = nullptr;
    CKS(ws.alloc_n(&stat, 2 * ch.size() + 2 * (size_t)eng.a.nrows));
    b.smean = stat;
    b.svar = stat + nchan;
    b.emean = stat + 2 * nchan;
    b.evar = stat + 2 * nchan + eng.a.nrows;
    int* words = nullptr;
    CKS(ws.alloc_n(&words, (size_t)nchan * 2 * M + 4));
    b.iters = words;
    b.finished = words + (size_t)nchan * 2 * M;
    std::vector<double*> himfs(ch.size());
    for (int c = 0; c < nchan; ++c) himfs[c] = ch[c].imfs;
    CK(cudaMemcpyAsync(dxoff, xoff.data(), sizeof(long long) * nchan, cudaMemcpyHostToDevice,
                       st));
    CK(cudaMemcpyAsync(dimfs, himfs.data(), sizeof(double*) * nchan, cudaMemcpyHostToDevice,
                       st));
    CK(cudaMemsetAsync(stat, 0, sizeof(double) * (2 * ch.size() + 2 * (size_t)eng.a.nrows), st));
    CK(cudaMemsetAsync(words, 0, sizeof(int) * ((size_t)nchan * 2 * M + 4), st));
    CKS(eng.reset_carries(st));
    // every channel starts "finished" at stage -1: the first iteration's transitions open
    // its first noise stage
    std::vector<ChanState> cs0(ch.size());
    for (auto& s : cs0) {
        std::memset(&s, 0, sizeof(s));
        s.done = 1;
        s.stage = -1;
    }
    CK(cudaMemcpyAsync(eng.cs, cs0.data(), sizeof(ChanState) * nchan, cudaMemcpyHostToDevice,
                       st));
    for (int c = 0; c < nchan; ++c) {
        const Chan& hc = eng.hchan[c];
        const size_t rn = (size_t)hc.nr * hc.n;
        // the channel's block has room for the pair-rounded count (rn rounded up to 32)
        if (ch[c].noise)
            CK(cudaMemcpyAsync(b.W + hc.samp0, ch[c].noise, rn * sizeof(double),
                               cudaMemcpyDeviceToDevice, st));
        else
            CKS(generate_noise(b.W + hc.samp0, (rn + 1) & ~(size_t)1, ch[c].seed, st));
        CK(cudaMemcpyAsync(b.XS + xoff[c], ch[c].y, ch[c].n * sizeof(double),
                           cudaMemcpyDeviceToDevice, st));
    }
    eng.plan_by_caller = true;

    // iterations per replay: enough that the host check is rare, few enough that the loop
    // overshoots the last channel's end by little
    const size_t work = S;
    w.G = o.group > 0 ? o.group : (work >= ((size_t)1 << 26) ? 8 : 16);
    eng.group = w.G;
    if (o.h_kernel_ms) CKS(eng.enable_timing(o.h_kernel_ms));

    // autotune (first wave of a shape) or reuse
    const auto key = shape_key(ch, nr);
    TuneConfig cfg = kDefaultConfig;
    bool tuned = false;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            cfg = it->second;
            tuned = true;
        }
    }
    const char* tune_env = std::getenv("CEEMDAN_BATCH_TUNE");
    if (tune_env && tune_env[0] == '0') tuned = true;

    int* hs = eng.hstate;  // two slots of (finished, err, -, -)
    cudaEvent_t done_ev[2] = {eng.group_ev[0], eng.group_ev[1]};
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evg{t0, t1};

    long launched = 0;  // iterations launched
    // executable graphs of every configuration built so far (the tuner compares several)
    std::map<TuneConfig, std::pair<cudaGraphExec_t, cudaGraphExec_t>> built;
    struct BuiltGuard {
        std::map<TuneConfig, std::pair<cudaGraphExec_t, cudaGraphExec_t>>& m;
        Wave& w;
        ~BuiltGuard() {
            cudaStreamSynchronize(w.st);
            for (auto& kv : m) {
                if (kv.second.first && kv.second.first != w.exec[0])
                    cudaGraphExecDestroy(kv.second.first);
                if (kv.second.second && kv.second.second != w.exec[1])
                    cudaGraphExecDestroy(kv.second.second);
            }
        }
    } bg{built, w};
    auto use = [&](const TuneConfig& t) -> ceemdan_status {
        auto it = built.find(t);
        if (it == built.end()) {
            apply_config(eng, t);
            std::pair<cudaGraphExec_t, cudaGraphExec_t> ex{nullptr, nullptr};
            CKS(capture(w, st, 0, &ex.first));
            const ceemdan_status s2 = capture(w, st, (long)w.G, &ex.second);
            if (s2 != CEEMDAN_OK) {
                cudaGraphExecDestroy(ex.first);
                return s2;
            }
            it = built.emplace(t, ex).first;
        }
        w.exec[0] = it->second.first;
        w.exec[1] = it->second.second;
        return CEEMDAN_OK;
    };
    auto replay = [&](int slot) -> ceemdan_status {
        CK(cudaGraphLaunch(w.exec[slot], st));
        launched += w.G;
        g_launches += (uint64_t)w.G * kLoopKernels;
        CK(cudaMemcpyAsync(hs + 4 * slot, b.finished, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(done_ev[slot], st));
        return CEEMDAN_OK;
    };
    // one timed replay of configuration t (synchronous; its events harvested)
    auto cancelled = [&]() -> bool { return o.h_cancel && *o.h_cancel; };
    auto timed_replay = [&](const TuneConfig& t, float* ms) -> ceemdan_status {
        if (cancelled()) {
            cudaStreamSynchronize(st);
            g_last_error = "cancelled by the host cancel word";
            return CEEMDAN_ERR_CANCELLED;
        }
        CKS(use(t));
        CK(cudaEventRecord(t0, st));
        CKS(replay(0));
        CK(cudaEventRecord(t1, st));
        CK(cudaEventSynchronize(t1));
        eng.harvest_timing(0, w.G);
        float m = 0.f;
        CK(cudaEventElapsedTime(&m, t0, t1));
        *ms += m;
        return CEEMDAN_OK;
    };

    if (!tuned) {
        // coordinate descent over the four choices: each challenger against the best so far,
        // timed in the order best, challenger, challenger, best on the wave's own iterations
        // (the work drifts slowly as the stages advance; the symmetric order cancels that)
        const TuneConfig axes[][3] = {
            {{2, 1, 0, 0}, {4, 1, 0, 0}, {0, 0, 0, 0}},
            {{0, 2, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
            {{0, 0, 1, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
            {{0, 0, 0, 1}, {0, 0, 0, 0}, {0, 0, 0, 0}}};
        TuneConfig best = kDefaultConfig;
        float dummy = 0.f;
        CKS(timed_replay(best, &dummy));  // warm
        for (int ax = 0; ax < 4; ++ax) {
            for (int v = 0; v < 3; ++v) {
                const TuneConfig& d = axes[ax][v];
                if (d.tile_mult == 0 && d.split_mult == 0 && d.extrema_b == 0 && d.eval_b == 0)
                    continue;
                TuneConfig c = best;
                if (ax == 0) c.tile_mult = d.tile_mult;
                if (ax == 1) c.split_mult = d.split_mult;
                if (ax == 2) c.extrema_b = d.extrema_b;
                if (ax == 3) c.eval_b = d.eval_b;
                if (c == best) continue;
                CKS(timed_replay(c, &dummy));  // warm the challenger's graphs
                float tb = 0.f, tc = 0.f;
                CKS(timed_replay(best, &tb));
                CKS(timed_replay(c, &tc));
                CKS(timed_replay(c, &tc));
                CKS(timed_replay(best, &tb));
                if (tc < 0.99f * tb) best = c;
            }
        }
        cfg = best;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[key] = cfg;
    }
    CKS(use(cfg));
    int slot = 0;
    // double-buffered loop: replay slot s^1 is queued before the host waits for slot s
    CKS(replay(slot));
    int finished = 0;
    for (;;) {
        CKS(replay(slot ^ 1));
        CK(cudaEventSynchronize(done_ev[slot]));
        eng.harvest_timing((long)slot * w.G, w.G);
        finished = hs[4 * slot];
        if (cancelled()) {
            cudaStreamSynchronize(st);
            g_last_error = "cancelled by the host cancel word";
            return CEEMDAN_ERR_CANCELLED;
        }
        if (finished >= nchan) break;
        slot ^= 1;
    }
    CK(cudaStreamSynchronize(st));
    eng.harvest_timing((long)(slot ^ 1) * w.G, w.G);
    if (peak_bytes && pool) {
        uint64_t high = 0;
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &high) == cudaSuccess)
            *peak_bytes = std::max(*peak_bytes, (size_t)high);
    }
    std::vector<ChanState> csh(ch.size());
    CK(cudaMemcpy(csh.data(), eng.cs, sizeof(ChanState) * nchan, cudaMemcpyDeviceToHost));
    for (int c = 0; c < nchan; ++c) {
        if (csh[c].err) {
            g_last_error = "a sift kernel reported an error in the device error word";
            return (ceemdan_status)csh[c].err;
        }
    }
    if (o.h_counters) {
        for (int c = 0; c < nchan; ++c) {
            o.h_counters[CEEMDAN_C_KNOTS] += csh[c].knots;
        }
        // lock-step iterations of the loop (all channels together)
        o.h_counters[CEEMDAN_C_ITERATIONS] += (uint64_t)launched;
    }
    if (h_iters) {
        std::vector<int> it((size_t)nchan * 2 * M);
        CK(cudaMemcpy(it.data(), b.iters, sizeof(int) * it.size(), cudaMemcpyDeviceToHost));
        for (int c = 0; c < nchan; ++c)
            for (int s = 0; s < 2 * M; ++s)
                h_iters[ch[c].index * 2 * M + s] = it[(size_t)c * 2 * M + s];
    }
    return CEEMDAN_OK;
}

}  // namespace
}  // namespace ceemdan

using namespace ceemdan;

extern "C" ceemdan_status ceemdan_batched_f64(size_t channels, const size_t* lengths,
                                              const double* const* d_y, double* const* d_imfs,
                                              size_t nr, size_t num_imfs, size_t max_iter,
                                              double nstd, const ceemdan_options* opt,
                                              size_t wave_bytes, void* stream) {
    ceemdan_options o;
    if (opt && opt->struct_size == sizeof(ceemdan_options)) {
        o = *opt;
    } else if (opt) {
        g_last_error = "ceemdan_options.struct_size mismatch";
        return CEEMDAN_ERR_INVALID_ARG;
    } else {
        ceemdan_default_options(&o);
    }
    if (channels < 1 || channels > 4096 || !lengths || !d_y || !d_imfs || nr < 1 ||
        nr > 65535 || num_imfs < 2 || num_imfs > 64 || max_iter < 1 || o.noise_sift_cap < 1) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    if (o.d_noise || o.d_noise_modes_out || o.d_noise_state_out || o.d_noise_state_in) {
        g_last_error = "batched: external noise and noise-phase state are not supported";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    for (size_t c = 0; c < channels; ++c) {
        if (!d_y[c] || !d_imfs[c] || lengths[c] < 4 || lengths[c] > ((size_t)1 << 30) ||
            nr * lengths[c] > ((size_t)1 << 40)) {
            g_last_error = "invalid argument (channel " + std::to_string(c) + ")";
            return CEEMDAN_ERR_INVALID_ARG;
        }
    }
    // the loop runs on a stream of its own (a graph cannot be captured on the legacy default
    // stream), ordered after the work the caller queued on `stream`
    cudaStream_t cst = (cudaStream_t)stream;
    cudaStream_t st = nullptr;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } sg{st};
    {
        cudaEvent_t in = nullptr;
        CK(cudaEventCreateWithFlags(&in, cudaEventDisableTiming));
        cudaEventRecord(in, cst);
        cudaStreamWaitEvent(st, in, 0);
        cudaEventDestroy(in);
    }
    size_t budget = wave_bytes;
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        budget = (size_t)((double)fr * 0.85);
    }
    // longest channels first, greedily packed into waves that fit the budget
    std::vector<size_t> order(channels);
    std::iota(order.begin(), order.end(), (size_t)0);
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t p, size_t q) { return lengths[p] > lengths[q]; });
    std::vector<std::vector<BatchChannel>> waves;
    size_t used = 0;
    for (size_t k : order) {
        const size_t need = channel_bytes(lengths[k], nr, num_imfs);
        if (waves.empty() || (used + need > budget && !waves.back().empty())) {
            waves.emplace_back();
            used = 0;
        }
        waves.back().push_back(BatchChannel{lengths[k], d_y[k], d_imfs[k], o.seed + k, k});
        used += need;
    }
    size_t peak = 0;
    const uint64_t launches0 = g_launches.load();
    for (const auto& wv : waves) {
        const ceemdan_status s = run_wave(wv, nr, num_imfs, max_iter, nstd, o, st,
                                          o.h_iters_out, &peak);
        if (s != CEEMDAN_OK) {
            cudaStreamSynchronize(st);
            return s;
        }
    }
    if (o.h_counters) {
        o.h_counters[CEEMDAN_C_LAUNCHES] += g_launches.load() - launches0;
        o.h_counters[CEEMDAN_C_WAVES] += waves.size();
        o.h_counters[CEEMDAN_C_PEAK_BYTES] =
            std::max<uint64_t>(o.h_counters[CEEMDAN_C_PEAK_BYTES], peak);
    }
    return CEEMDAN_OK;
}
