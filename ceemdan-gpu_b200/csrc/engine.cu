// Host orchestration of the ICEEMDAN engine and its C ABI.
//
// Follows the call structure of iceemdanD (cudaICEEMDAN.cu:1340-2059), all in decompose():
//   noise-mode precompute  :1566-1715   -> one SiftEngine::run_stage per noise mode
//   CEEMDAN stage 0        :1729-1870   -> stage statistics, addNoise, run_stage, first IMF
//   CEEMDAN stages i >= 1  :1871-2014   -> addNoise2, run_stage, ensemble mean, IMF i
//   final residue          :2019
// The FP32 entry points (iceemdanS, ceemdan_plain_f32) widen the data and noise and narrow
// the IMFs around the same FP64 path; ceemdan_batch_f64 runs several decompose() calls on
// host threads with their own streams.
// with every per-iteration host synchronisation of the reference replaced by a device-side
// stop word that the host reads once per group of iterations.
#include <cuda_runtime.h>

#include <cmath>
#include <curand.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/ceemdan_b200.h"
#include "canon.cuh"
#include "kernels.h"
#include "host.h"

namespace ceemdan {

static_assert(kErrTimeout == CEEMDAN_ERR_TIMEOUT, "the kernels' timeout code is the ABI's");

thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};



// RN(1/h) and RN(1/(3h)) for h = 0..kRcpMax (entry 0 unused): the reciprocals the evaluation
// and spline kernels divide with (div_rcp gives correctly rounded quotients from them).
const double* rcp_tables() {
    // initialised once, thread-safe (concurrent decompositions from several host threads)
    static const std::vector<double> tab = [] {
        std::vector<double> t(2 * (kRcpMax + 1), 0.0);
        for (int h = 1; h <= kRcpMax; ++h) {
            t[h] = 1.0 / (double)h;
            t[kRcpMax + 1 + h] = 1.0 / (3.0 * (double)h);
        }
        return t;
    }();
    return tab.data();
}

int sm_count() {
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }();
    return sms;
}

// The library's stream-ordered memory pool of the current device (created on first use, kept
// for the process).  Calls allocate and free on their own stream, so a call never waits for
// other streams' work (cudaFree synchronises the device), and repeated calls reuse the pool's
// memory up to kPoolKeep bytes.  Freed memory is reused across streams only once its free has
// completed (no dependencies inserted between streams).
constexpr uint64_t kPoolKeep = (uint64_t)16 << 30;

cudaMemPool_t engine_pool() {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if ((size_t)dev >= pools.size()) pools.resize((size_t)dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = kPoolKeep;
        int no = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
        pools[dev] = pool;
    }
    return pools[dev];
}

ceemdan_status pool_alloc(void** p, size_t bytes, cudaStream_t st) {
    cudaMemPool_t pool = engine_pool();
    if (!pool) {
        g_last_error = "no memory pool on the current device";
        return CEEMDAN_ERR_CUDA;
    }
    const cudaError_t e = cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, st);
    if (e != cudaSuccess) {
        g_last_error = std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? CEEMDAN_ERR_NO_MEMORY : CEEMDAN_ERR_CUDA;
    }
    return CEEMDAN_OK;
}


// Pinned host words for the device stop word (two slots of done, iter, err, pad): a process-
// wide free list, so that calls do not pay a pinned allocation (and its free) each time.
namespace {
std::mutex g_pin_mu;
std::vector<int*> g_pin_free;
}  // namespace

int* pinned_state() {
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        if (!g_pin_free.empty()) {
            int* p = g_pin_free.back();
            g_pin_free.pop_back();
            return p;
        }
    }
    int* p = nullptr;
    if (cudaMallocHost(reinterpret_cast<void**>(&p), 16 * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void release_pinned_state(int* p) {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back(p);
}

}  // namespace ceemdan


namespace ceemdan {

// Multipliers of the division-free sx tests.  For p = |U+L|, q = |U-L| (doubles) and a
// threshold t, fl(p/q) > t holds when p/q >= t(1+2^-51) (the quotient then rounds to a double
// above t, whose spacing is at most 2^-52 t) and fails when p/q <= t.  With hi >= t(1+2^-50)
// and lo <= t(1-2^-51), p > RN(q*hi) implies p/q >= t(1+2^-51) and p < RN(q*lo) implies
// p/q < t, as long as q*hi and q*lo are normal: q in (2^-800, 2^800), t in [2^-100, 2^100].
// Outside that threshold range no sample is decided this way (hi = inf, lo = -1).
void sx_bounds(double t, double* hi, double* lo) {
    if (!(t >= 0x1p-100 && t <= 0x1p+100)) {
        *hi = INFINITY;
        *lo = -1.0;
        return;
    }
    *hi = std::nextafter(t * (1.0 + 0x1p-50), INFINITY);  // RN(x) + ulp >= x
    *lo = std::nextafter(t * (1.0 - 0x1p-51), 0.0);       // RN(x) - ulp <= x
}

int grid_for(size_t count) {
    size_t b = (count + kThreads - 1) / kThreads;
    return (int)std::max<size_t>(1, std::min<size_t>(b, (size_t)sm_count() * 16));
}

namespace {

ceemdan_status check_coords(const int32_t* d_x, size_t n, int* d_err, cudaStream_t st) {
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    k_check_iota<<<grid_for(n), kThreads, 0, st>>>(d_x, n, d_err);
    ++g_launches;
    int h = 0;
    CK(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h) {
        g_last_error = "d_x must hold the sample index 0..N-1";
        return CEEMDAN_ERR_COORD;
    }
    return CEEMDAN_OK;
}

}  // namespace

ceemdan_status generate_noise(double* w, size_t count, uint64_t seed, cudaStream_t st) {
    curandGenerator_t gen;
    if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS) {
        g_last_error = "curandCreateGenerator failed";
        return CEEMDAN_ERR_CUDA;
    }
    ceemdan_status rc = CEEMDAN_OK;
    if (curandSetPseudoRandomGeneratorSeed(gen, seed) != CURAND_STATUS_SUCCESS ||
        curandSetStream(gen, st) != CURAND_STATUS_SUCCESS ||
        curandGenerateNormalDouble(gen, w, count, 0.0, 1.0) != CURAND_STATUS_SUCCESS) {
        g_last_error = "curandGenerateNormalDouble failed";
        rc = CEEMDAN_ERR_CUDA;
    }
    curandDestroyGenerator(gen);
    return rc;
}

namespace {

// N(0,1) floats from cuRAND's generator (curandGenerateNormal, the FP32 reference path
// cudaICEEMDAN.cu:741), widened exactly to doubles.
ceemdan_status generate_noise_f32(Workspace& ws, double* w, size_t count, uint64_t seed,
                                  cudaStream_t st) {
    float* f = nullptr;
    CKS(ws.alloc_n(&f, count));
    curandGenerator_t gen;
    if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS) {
        g_last_error = "curandCreateGenerator failed";
        return CEEMDAN_ERR_CUDA;
    }
    ceemdan_status rc = CEEMDAN_OK;
    if (curandSetPseudoRandomGeneratorSeed(gen, seed) != CURAND_STATUS_SUCCESS ||
        curandSetStream(gen, st) != CURAND_STATUS_SUCCESS ||
        curandGenerateNormal(gen, f, count, 0.0f, 1.0f) != CURAND_STATUS_SUCCESS) {
        g_last_error = "curandGenerateNormal failed";
        rc = CEEMDAN_ERR_CUDA;
    }
    curandDestroyGenerator(gen);
    if (rc != CEEMDAN_OK) return rc;
    k_widen_f32<<<grid_for(count), kThreads, 0, st>>>(f, w, count);
    ++g_launches;
    CK(cudaGetLastError());
    return CEEMDAN_OK;
}

// The ensemble sums closing CEEMDAN stage k of a split channel: the running sums from the
// previous part (zeros on part 0), this part's realizations added in order, passed on, the
// last part's sums to every part, then IMF_k and the next residue -- the operations of
// k_first_imf / k_avg_update in the same order.
ceemdan_status split_stage_sums(const ceemdan_split* sp, bool first_stage, const double* h0,
                                const double* mode, const double* xs, double* fornext,
                                double* imf, double* tsum, size_t n, size_t nr,
                                cudaStream_t st) {
    auto failed = [](const char* what) {
        g_last_error = std::string("the split's ") + what + " exchange failed";
        return CEEMDAN_ERR_CUDA;
    };
    CK(cudaMemsetAsync(tsum, 0, n * sizeof(double), st));
    if (sp->rank > 0) {
        CK(cudaStreamSynchronize(st));
        if (sp->recv_partial(sp->ctx, tsum, n) != 0) return failed("recv_partial");
    }
    const double inr = 1.0 / (double)sp->nr_total;
    k_ens_accum<<<grid_for(n), kThreads, 0, st>>>(h0, mode, tsum, n, (int)nr, first_stage, inr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    if (sp->rank + 1 < sp->world && sp->send_partial(sp->ctx, tsum, n) != 0)
        return failed("send_partial");
    if (sp->broadcast_last(sp->ctx, tsum, n) != 0) return failed("broadcast_last");
    k_ens_out<<<grid_for(n), kThreads, 0, st>>>(tsum, xs, fornext, imf, n, first_stage,
                                                (double)sp->nr_total);
    g_launches += 2;
    CK(cudaGetLastError());
    return CEEMDAN_OK;
}

ceemdan_status decompose_impl(size_t nr, size_t n, size_t nimf, size_t max_iter,
                              const int32_t* d_x, const double* d_y, double* d_imfs, double nstd,
                              const ceemdan_options& o, cudaStream_t st, double* stage_seconds,
                              bool float_noise, ceemdan_tape* tape = nullptr,
                              const ceemdan_split* sp = nullptr) {
    if (sp && (tape || o.d_noise_state_in || o.d_noise_state_out || sp->world < 1 ||
               sp->rank < 0 || sp->rank >= sp->world || !sp->all_finished ||
               !sp->recv_partial || !sp->send_partial || !sp->broadcast_last ||
               sp->first + nr > sp->nr_total || sp->nr_total > 65535)) {
        g_last_error = "invalid realization split";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    if (tape && nr > 32767) {  // the reverse pass launches 2*nr CTAs in a grid's y dimension
        g_last_error = "the taped forward takes at most 32767 realizations";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    if (nr < 1 || n < 4 || nimf < 2 || max_iter < 1 || !d_x || !d_y || !d_imfs ||
        o.noise_sift_cap < 1 || n > (size_t)(1u << 30) || nr > 65535 ||
        nr * n > ((size_t)1 << 40)) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    if (max_iter > (size_t)0x7fffffff) max_iter = 0x7fffffff;
    Workspace ws(st);
    SiftEngine eng;
    CKS(eng.init(ws, (int)nr, (int)n, o));
    if (o.h_kernel_ms) CKS(eng.enable_timing(o.h_kernel_ms));
    if (sp) {
        eng.split = sp;  // the stop test of every iteration spans the parts
    } else {
        CKS(eng.enable_small(ws, (int)std::max<size_t>(std::min<size_t>(max_iter, 0x7fffffff),
                                                           (size_t)o.noise_sift_cap),
                                 o.spin_limit));
    }
    const uint64_t launches0 = g_launches.load();
    CKS(check_coords(d_x, n, &eng.cs[0].err, st));
    const size_t rn = nr * n;
    const bool state_in = o.d_noise_state_in != nullptr;
    if (state_in && o.d_noise) {
        g_last_error = "d_noise and d_noise_state_in are exclusive";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    double *w = nullptr, *E = nullptr, *h0, *mode, *xs, *fornext, *stat;
    if (state_in) {
        E = const_cast<double*>(o.d_noise_state_in);  // read only below
    } else {
        CKS(ws.alloc_n(&w, rn + 1));  // cuRAND normals come in pairs
        CKS(ws.alloc_n(&E, nimf * rn));
    }
    CKS(ws.alloc_n(&h0, rn));
    CKS(ws.alloc_n(&mode, rn));
    CKS(ws.alloc_n(&xs, n));
    CKS(ws.alloc_n(&fornext, n));
    CKS(ws.alloc_n(&stat, 2 + 2 * nr));
    double* tsum = nullptr;  // a split's running ensemble sums
    if (sp) CKS(ws.alloc_n(&tsum, n));
    double* s_mean = stat;
    double* s_var = stat + 1;
    double* e_mean = stat + 2;
    double* e_var = stat + 2 + nr;
    CK(cudaMemsetAsync(stat, 0, sizeof(double) * (2 + 2 * nr), st));
    if (state_in) {
        // no noise: the noise phase's result comes with the state
    } else if (o.d_noise) {
        CK(cudaMemcpyAsync(w, o.d_noise, rn * sizeof(double), cudaMemcpyDeviceToDevice, st));
    } else if (sp) {  // the whole ensemble's cuRAND sequence, then this part's rows
        const size_t all = sp->nr_total * n;
        double* wall = nullptr;
        CKS(ws.alloc_n(&wall, all + 1));
        CKS(generate_noise(wall, (all + 1) & ~(size_t)1, o.seed, st));
        CK(cudaMemcpyAsync(w, wall + sp->first * n, rn * sizeof(double), cudaMemcpyDeviceToDevice,
                           st));
    } else {
        if (float_noise) {
            CKS(generate_noise_f32(ws, w, (rn + 1) & ~(size_t)1, o.seed, st));
        } else {
            CKS(generate_noise(w, (rn + 1) & ~(size_t)1, o.seed, st));
        }
    }
    CKS(eng.reset_carries(st));

    // ---- noise modes E_k(w_r) (:1566-1715) ----
    for (size_t i = 0; i + 1 < nimf && state_in; ++i)
        if (o.h_iters_out) o.h_iters_out[i] = 0;
    for (size_t i = 0; i + 1 < nimf && !state_in; ++i) {
        CK(cudaMemcpyAsync(eng.h[0], w, rn * sizeof(double), cudaMemcpyDeviceToDevice, st));
        int it = 0;
        CKS(eng.run_stage(E + i * rn, o.noise_sift_cap, st, &it, o.h_cancel));
        if (o.h_iters_out) o.h_iters_out[i] = it;
        k_sub_inplace<<<grid_for(rn), kThreads, 0, st>>>(w, E + i * rn, rn);
        ++g_launches;
        CK(cudaGetLastError());
    }
    if (!state_in)
        CK(cudaMemcpyAsync(E + (nimf - 1) * rn, w, rn * sizeof(double), cudaMemcpyDeviceToDevice,
                           st));
    // the carries the noise phase leaves (mean envelope, sifting fraction): restored from the
    // given state, or exported with the modes
    if (state_in) {
        CK(cudaMemcpyAsync(eng.a.menv, o.d_noise_state_in + nimf * rn, rn * sizeof(double),
                           cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(eng.a.frac, o.d_noise_state_in + (nimf + 1) * rn, nr * sizeof(double),
                           cudaMemcpyDeviceToDevice, st));
    }
    if (o.d_noise_state_out) {
        CK(cudaMemcpyAsync(o.d_noise_state_out, E, nimf * rn * sizeof(double),
                           cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(o.d_noise_state_out + nimf * rn, eng.a.menv, rn * sizeof(double),
                           cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(o.d_noise_state_out + (nimf + 1) * rn, eng.a.frac,
                           nr * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }

    if (tape) {  // what the reverse pass of the stage statistics reads
        tape->nr = nr;
        tape->n = n;
        tape->nimf = nimf;
        tape->nstd = nstd;
        tape->L = tape_layout((int)nr, eng.ntiles);
        tape->stages.assign(nimf - 1, ceemdan_tape::Stage());
        CKS(tape->alloc(reinterpret_cast<void**>(&tape->E), nimf * rn * sizeof(double), st));
        CKS(tape->alloc(reinterpret_cast<void**>(&tape->fin), (nimf - 1) * n * sizeof(double),
                        st));
        CKS(tape->alloc(reinterpret_cast<void**>(&tape->stats),
                        2 * (nimf - 1) * sizeof(double), st));
        tape->opts = o;
        tape->max_iter = max_iter;
        if (tape->checkpointed)
            CKS(tape->alloc(reinterpret_cast<void**>(&tape->ck),
                            (nimf - 1) * tape->ck_stride() * sizeof(double), st));
        CK(cudaMemcpyAsync(tape->E, E, nimf * rn * sizeof(double), cudaMemcpyDeviceToDevice,
                           st));
        CKS(ws.alloc_n(&eng.a.bflags, 2 * nr));
    }

    // ---- CEEMDAN stages (:1722-2019) ----
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    CK(cudaMemcpyAsync(xs, d_y, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CK(cudaEventRecord(ev0, st));
    const double inv_n = 1.0 / (double)n;
    const double inv_nm1 = 1.0 / (double)(n - 1);
    const dim3 gnr(std::max(1, std::min((int)((n + kThreads - 1) / kThreads), 64)), (unsigned)nr);
    ceemdan_status rc = CEEMDAN_OK;
    for (size_t i = 0; i + 1 < nimf && rc == CEEMDAN_OK; ++i) {
        const double* Ei = E + i * rn;
        if (tape &&
            cudaMemcpyAsync(tape->fin + i * n, i == 0 ? xs : fornext, n * sizeof(double),
                            cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            rc = CEEMDAN_ERR_CUDA;
            break;
        }
        if (i == 0) {
            k_canon_mean<<<1, kLanes, 0, st>>>(xs, n, n, s_mean, inv_n);
            k_canon_var<<<1, kLanes, 0, st>>>(xs, n, n, s_mean, s_var, inv_nm1);
            k_canon_mean<<<(unsigned)nr, kLanes, 0, st>>>(Ei, n, n, e_mean, inv_n);
            k_canon_var<<<(unsigned)nr, kLanes, 0, st>>>(Ei, n, n, e_mean, e_var, inv_nm1);
            k_standardize<<<grid_for(n), kThreads, 0, st>>>(xs, n, s_var);
            k_add_noise<<<gnr, kThreads, 0, st>>>(h0, xs, Ei, n, (int)nr, nstd, e_var);
            g_launches += 6;
        } else {
            k_canon_mean<<<1, kLanes, 0, st>>>(fornext, n, n, s_mean, inv_n);
            k_canon_var<<<1, kLanes, 0, st>>>(fornext, n, n, s_mean, s_var, inv_nm1);
            k_add_noise2<<<gnr, kThreads, 0, st>>>(h0, fornext, Ei, n, (int)nr, nstd, s_var);
            g_launches += 3;
        }
        if (cudaGetLastError() != cudaSuccess) {
            g_last_error = "stage kernel launch failed";
            rc = CEEMDAN_ERR_CUDA;
            break;
        }
        if (cudaMemcpyAsync(eng.h[0], h0, rn * sizeof(double), cudaMemcpyDeviceToDevice, st) !=
            cudaSuccess) {
            rc = CEEMDAN_ERR_CUDA;
            break;
        }
        if (tape && cudaMemcpyAsync(tape->stats + 2 * i, stat, 2 * sizeof(double),
                                    cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            rc = CEEMDAN_ERR_CUDA;
            break;
        }
        if (tape && tape->checkpointed) {
            double* c = tape->ck + i * tape->ck_stride();
            if (cudaMemcpyAsync(c, eng.h[0], rn * sizeof(double), cudaMemcpyDeviceToDevice, st) !=
                    cudaSuccess ||
                cudaMemcpyAsync(c + rn, eng.a.menv, rn * sizeof(double),
                                cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
                cudaMemcpyAsync(c + 2 * rn, eng.a.frac, nr * sizeof(double),
                                cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
                rc = CEEMDAN_ERR_CUDA;
                break;
            }
        }
        eng.tape = (tape && !tape->checkpointed) ? tape : nullptr;
        eng.tape_stage = i;
        int it = 0;
        rc = eng.run_stage(mode, (int)max_iter, st, &it, o.h_cancel);
        eng.tape = nullptr;
        if (tape && rc == CEEMDAN_OK) {  // run_stage synchronised the stream
            tape->stages[i].J = it;
            tape->trim(i, st);
        }
        if (rc != CEEMDAN_OK) break;
        if (o.h_iters_out) o.h_iters_out[(nimf - 1) + i] = it;
        ++g_launches;
        if (sp) {
            rc = split_stage_sums(sp, i == 0, h0, mode, xs, fornext, d_imfs + i * n, tsum, n, nr,
                                  st);
        } else if (i == 0) {
            k_first_imf<<<grid_for(n), kThreads, 0, st>>>(h0, mode, xs, fornext, d_imfs, n,
                                                          (int)nr);
        } else {
            k_avg_update<<<grid_for(n), kThreads, 0, st>>>(h0, mode, fornext, d_imfs + i * n, n,
                                                           (int)nr);
        }
    }
    if (rc == CEEMDAN_OK) {
        cudaEventRecord(ev1, st);
        cudaMemcpyAsync(d_imfs + (nimf - 1) * n, fornext, n * sizeof(double),
                        cudaMemcpyDeviceToDevice, st);
        if (o.d_noise_modes_out)
            cudaMemcpyAsync(o.d_noise_modes_out, E, nimf * rn * sizeof(double),
                            cudaMemcpyDeviceToDevice, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            g_last_error = std::string("decomposition: ") + cudaGetErrorString(e);
            rc = CEEMDAN_ERR_CUDA;
        } else {
            if (stage_seconds) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev0, ev1);
                *stage_seconds = ms * 1e-3;
            }
            if (o.h_counters) {
                ChanState c0;
                if (cudaMemcpy(&c0, eng.cs, sizeof(c0), cudaMemcpyDeviceToHost) == cudaSuccess) {
                    o.h_counters[CEEMDAN_C_KNOTS] += c0.knots;
                    o.h_counters[CEEMDAN_C_ITERATIONS] += c0.iters;
                }
                o.h_counters[CEEMDAN_C_LAUNCHES] += g_launches.load() - launches0;
            }
        }
    } else {
        cudaStreamSynchronize(st);
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    return rc;
}

// Realizations per block of a checkpointed reverse pass: as many as the free device memory
// (the device's free memory plus what the library's pool holds unused, 80 % of it) takes with
// their stage re-run (engine rows, a one-stage tape of the longest stage) and their share of the
// reverse kernels' work arrays.  CEEMDAN_BACKWARD_BLOCK=k sets k.
int checkpoint_block(const ceemdan_tape& T) {
    const int nr = (int)T.nr;
    if (const char* e = std::getenv("CEEMDAN_BACKWARD_BLOCK")) {
        const int k = std::atoi(e);
        if (k > 0) return std::min(k, nr);
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return nr;
    }
    if (cudaMemPool_t pool = engine_pool()) {
        uint64_t used = 0, reserved = 0;
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) ==
                cudaSuccess &&
            reserved > used)
            free_b += (size_t)(reserved - used);
    }
    const size_t n = T.n;
    int jmax = 1;
    for (const auto& stg : T.stages) jmax = std::max(jmax, stg.J);
    const size_t slots = ((size_t)jmax + kTapeBlockSlots - 1) / kTapeBlockSlots * kTapeBlockSlots;
    const size_t tape_row = (size_t)2 * T.L.ntiles * (kTileSamples / 32) * sizeof(unsigned) + 16;
    // the reverse work arrays (eb; per spline knots, four segment sums, yb, the system, z, its
    // workspace: a bound of 128 bytes per sample) and the rows of the two re-run engines (h,
    // mean envelope, modes, knots, records, reduced workspaces: 160 bytes per sample each)
    const size_t per_row = slots * tape_row + 128 * n + 2 * 160 * n;
    const size_t fixed = 2 * T.nr * n * sizeof(double) + ((size_t)64 << 20);  // gh, gm, margin
    const size_t usable = (size_t)(0.8 * (double)free_b);
    const int most = usable <= fixed ? 1
                                     : (int)std::max<size_t>(
                                           1, std::min<size_t>((size_t)nr,
                                                               (usable - fixed) / per_row));
    // blocks of nearly equal size
    const int blocks = (nr + most - 1) / most;
    return (nr + blocks - 1) / blocks;
}

// Reverse pass (vector-Jacobian product) of a taped decomposition: gy = (d imfs/d y)^T g with
// the recorded structure, stage by stage from the last, iteration by iteration from the last
// (adjoint.cu); same arithmetic order as the CPU oracle's vjp.  A checkpointed tape re-runs
// each stage from its checkpoint a block of realizations at a time, every block for exactly
// the stage's recorded iteration count (within a stage a realization's sift depends only on
// its own state; the lock-step test only decides how long the stage runs), records the block's
// one-stage tape and reverses it; the stage-level sums then run over all realizations.
ceemdan_status backward_impl(const ceemdan_tape& T, const double* g, double* gy,
                             cudaStream_t st) {
    const int nr = (int)T.nr, n = (int)T.n;
    const size_t ns = T.nimf - 1, rn = T.nr * T.n;
    const int cap = n / 2 + 2;
    const int nb = T.checkpointed ? checkpoint_block(T) : nr;  // realizations per block
    const int nsp = 2 * nb;
    const size_t pc = (size_t)nsp * cap, ws_stride = (size_t)cap + 64;
    Workspace ws(st);
    double *gh, *gm, *eb, *abar, *fbar, *hs, *p, *scal, *S, *yb, *sys, *z, *wsp;
    int32_t* kx;
    CKS(ws.alloc_n(&gh, rn));
    CKS(ws.alloc_n(&gm, rn));
    CKS(ws.alloc_n(&eb, (size_t)nb * T.n));
    CKS(ws.alloc_n(&abar, T.n));
    CKS(ws.alloc_n(&fbar, T.n));
    CKS(ws.alloc_n(&hs, T.n));
    CKS(ws.alloc_n(&p, T.n));
    CKS(ws.alloc_n(&scal, 8));
    CKS(ws.alloc_n(&kx, pc));
    CKS(ws.alloc_n(&S, 4 * pc));
    CKS(ws.alloc_n(&yb, pc));
    CKS(ws.alloc_n(&sys, 4 * pc));
    CKS(ws.alloc_n(&z, pc));
    CKS(ws.alloc_n(&wsp, (size_t)nsp * ws_stride));
    // the transposed spline solves: one CTA per spline (cta_tridiag), or for long splines the
    // same solve level by level over the whole grid (psolve_launch); CEEMDAN_ADJ_SOLVE=cta or
    // grid chooses
    bool grid_solve = cap > 16384;
    if (const char* e = std::getenv("CEEMDAN_ADJ_SOLVE")) {
        if (std::strcmp(e, "grid") == 0) grid_solve = true;
        if (std::strcmp(e, "cta") == 0) grid_solve = false;
    }
    int* nrows = nullptr;
    if (grid_solve) CKS(ws.alloc_n(&nrows, (size_t)nsp));
    CK(cudaMemsetAsync(gm, 0, rn * sizeof(double), st));
    CK(cudaMemsetAsync(scal, 0, 8 * sizeof(double), st));
    CK(cudaMemcpyAsync(fbar, g + ns * T.n, T.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    const double inr = 1.0 / (double)nr, inv_n = 1.0 / (double)n;
    const double inv_nm1 = 1.0 / (double)(n - 1);
    const unsigned kb = (unsigned)((cap + kThreads - 1) / kThreads);
    // checkpointed tape: engines that re-run a block of realizations of one stage from its
    // checkpoint into a one-stage tape (the forward's kernels, options and sift cap: the same
    // structure); one for blocks of nb rows and one for a last, shorter block
    Workspace rws(st), rws2(st);
    SiftEngine reng, reng2;
    ceemdan_tape one;
    struct FreeOnStream {  // the one-stage tape's blocks go back after the work queued on st
        ceemdan_tape& t;
        cudaStream_t s;
        ~FreeOnStream() { t.free_blocks(s); }
    } one_guard{one, st};
    double *rmode = nullptr, *rmode2 = nullptr;
    const int rem = nr % nb;
    auto init_rerun = [&](Workspace& w, SiftEngine& e, double** mode, int rows) -> ceemdan_status {
        CKS(e.init(w, rows, n, T.opts));
        CKS(e.enable_small(w, (int)T.max_iter, T.opts.spin_limit));
        CKS(e.reset_carries(st));
        CKS(w.alloc_n(&e.a.bflags, (size_t)2 * rows));
        CKS(w.alloc_n(mode, (size_t)rows * T.n));
        return CEEMDAN_OK;
    };
    if (T.checkpointed) {
        CKS(init_rerun(rws, reng, &rmode, nb));
        if (rem > 0) CKS(init_rerun(rws2, reng2, &rmode2, rem));
        one.device = T.device;
        one.n = T.n;
        one.stages.assign(1, ceemdan_tape::Stage());
    }
    for (long i = (long)ns - 1; i >= 0; --i) {
        const double* gi = g + (size_t)i * T.n;
        k_adj_abar<<<grid_for(T.n), kThreads, 0, st>>>(fbar, gi, abar, T.n);
        CK(cudaMemsetAsync(gh, 0, rn * sizeof(double), st));
        for (int r0 = 0; r0 < nr; r0 += nb) {
            const int rows = std::min(nb, nr - r0);
            const ceemdan_tape* src = &T;
            size_t si = (size_t)i;
            if (T.checkpointed) {
                SiftEngine& E = rows == nb ? reng : reng2;
                double* rm = rows == nb ? rmode : rmode2;
                const double* c = T.ck + (size_t)i * T.ck_stride();
                const size_t off = (size_t)r0 * T.n, bn = (size_t)rows * T.n;
                CK(cudaMemcpyAsync(E.h[0], c + off, bn * sizeof(double), cudaMemcpyDeviceToDevice,
                                   st));
                CK(cudaMemcpyAsync(E.a.menv, c + rn + off, bn * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st));
                CK(cudaMemcpyAsync(E.a.frac, c + 2 * rn + r0, rows * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st));
                one.nr = (size_t)rows;
                one.L = tape_layout(rows, T.L.ntiles);
                const int J = T.stages[(size_t)i].J;
                E.a.forced = J;
                E.tape = &one;
                E.tape_stage = 0;
                int it = 0;
                const ceemdan_status rs = E.run_stage(rm, (int)T.max_iter, st, &it, nullptr);
                E.tape = nullptr;
                E.a.forced = 0;
                if (rs != CEEMDAN_OK) return rs;
                one.stages[0].J = it;
                if (it != J) {
                    g_last_error = "a stage re-run from its checkpoint took another iteration count";
                    return CEEMDAN_ERR_CUDA;
                }
                src = &one;
                si = 0;
            }
            const TapeLayout& L = src->L;
            const int bsp = 2 * rows;
            double* ghb = gh + (size_t)r0 * T.n;
            double* gmb = gm + (size_t)r0 * T.n;
            const dim3 gseed((unsigned)std::max(1, std::min((n + kThreads - 1) / kThreads, 64)),
                             (unsigned)rows);
            const dim3 gknot(kb, (unsigned)bsp), gscat(kb, (unsigned)rows);
            for (long j = (long)src->stages[si].J - 1; j >= 0; --j) {
                const unsigned char* slot = src->slot(si, j);
                k_adj_seed<<<gseed, kThreads, 0, st>>>(slot, L, n, ghb, gmb, eb, abar, inr);
                k_adj_knots<<<(unsigned)bsp, kThreads, 0, st>>>(slot, L, cap, kx);
                k_adj_segsums<<<gknot, kThreads, 0, st>>>(slot, L, n, cap, kx, eb, S);
                k_adj_rows<<<gknot, kThreads, 0, st>>>(slot, L, cap, kx, S, yb, sys, nrows);
                if (grid_solve) {
                    int nl = 0;
                    CK(psolve_launch(bsp, cap, nrows, sys, cap, z, wsp, ws_stride, st, &nl,
                                     kx));
                    g_launches += (uint64_t)nl - 1;
                } else {
                    k_adj_solve<<<(unsigned)bsp, kThreads, 0, st>>>(slot, L, cap, sys, z, wsp,
                                                                    ws_stride);
                }
                k_adj_rhs<<<gknot, kThreads, 0, st>>>(slot, L, cap, kx, yb, z, S);
                k_adj_scatter<<<gscat, kThreads, 0, st>>>(slot, L, n, cap, kx, S, ghb);
                g_launches += 7;
            }
            if (T.checkpointed) one.free_blocks(st);  // after the reverse kernels that read them
            CK(cudaGetLastError());
        }
        k_adj_inject<<<grid_for(T.n), kThreads, 0, st>>>(gh, abar, inr, T.E + (size_t)i * rn,
                                                         nr, T.n, hs, p);
        k_adj_stats<<<1, kLanes, 0, st>>>((int)i, T.fin + (size_t)i * T.n, T.stats, p, gi, hs,
                                          T.n, T.nstd, inv_n, inv_nm1, scal);
        k_adj_out<<<grid_for(T.n), kThreads, 0, st>>>((int)i, gi, hs, T.fin + (size_t)i * T.n,
                                                      T.stats, scal, i >= 1 ? fbar : gy, T.n,
                                                      inv_n);
        g_launches += 4;
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(st));
    return CEEMDAN_OK;
}

}  // namespace

void set_last_error(const std::string& what) { g_last_error = what; }

}  // namespace ceemdan

using namespace ceemdan;

// ---------------------------------------------------------------------------------------
// Noise-phase cache.  Calls without explicit noise options draw their noise from cuRAND with
// the options' seed, so for equal (device, seed, noise type, nr, n, num_imfs, noise sift cap,
// thresholds) the noise phase -- noise modes plus the carries it leaves -- is the same every
// time.  When enabled (ceemdan_noise_cache, or CEEMDAN_NOISE_CACHE_BYTES at first use), one
// such state is kept on the device: a call with the same key starts from it and skips the
// noise phase (same result bit for bit); a call with another key computes its state into a
// fresh buffer that replaces the entry once the call has finished.  Readers hold a shared
// reference, so a replaced entry stays valid until they are done.
// ---------------------------------------------------------------------------------------
namespace {

struct NoiseKey {
    int device;
    uint64_t seed;
    bool float_noise;
    size_t nr, n, nimf;
    int cap;
    double sd, sd2, tol;
    bool operator==(const NoiseKey& k) const {
        return device == k.device && seed == k.seed && float_noise == k.float_noise &&
               nr == k.nr && n == k.n && nimf == k.nimf && cap == k.cap && sd == k.sd &&
               sd2 == k.sd2 && tol == k.tol;
    }
};

std::mutex g_nc_mu;
bool g_nc_init = false;
size_t g_nc_limit = 0;
bool g_nc_valid = false;
bool g_nc_filling = false;  // one call at a time computes a new entry; others bypass
NoiseKey g_nc_key{};
std::shared_ptr<double> g_nc_buf;

size_t noise_cache_limit_locked() {
    if (!g_nc_init) {
        g_nc_init = true;
        if (const char* e = std::getenv("CEEMDAN_NOISE_CACHE_BYTES"))
            g_nc_limit = (size_t)std::strtoull(e, nullptr, 10);
    }
    return g_nc_limit;
}

std::shared_ptr<double> device_buffer(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();  // an unavailable cache buffer only disables caching for this call
        return nullptr;
    }
    return std::shared_ptr<double>(static_cast<double*>(p), [](double* q) { cudaFree(q); });
}

ceemdan_status decompose(size_t nr, size_t n, size_t nimf, size_t max_iter, const int32_t* d_x,
                         const double* d_y, double* d_imfs, double nstd,
                         const ceemdan_options& o, cudaStream_t st, double* stage_seconds,
                         bool float_noise = false) {
    if (o.d_noise || o.d_noise_state_in || o.d_noise_state_out || nr < 1 || n < 4 || nimf < 2)
        return decompose_impl(nr, n, nimf, max_iter, d_x, d_y, d_imfs, nstd, o, st,
                              stage_seconds, float_noise);
    const size_t bytes = ((nimf + 1) * nr * n + nr) * sizeof(double);
    NoiseKey key{0, o.seed, float_noise, nr, n, nimf, o.noise_sift_cap, o.sd, o.sd2, o.tol};
    cudaGetDevice(&key.device);
    std::shared_ptr<double> hit, fill;
    bool filler = false;
    {
        std::lock_guard<std::mutex> lk(g_nc_mu);
        if (noise_cache_limit_locked() >= bytes) {
            if (g_nc_valid && g_nc_key == key) {
                hit = g_nc_buf;
            } else if (!g_nc_filling) {
                g_nc_filling = filler = true;
            }
        }
    }
    if (filler) fill = device_buffer(bytes);
    ceemdan_options oc = o;
    if (hit) oc.d_noise_state_in = hit.get();
    if (fill) oc.d_noise_state_out = fill.get();
    const ceemdan_status s = decompose_impl(nr, n, nimf, max_iter, d_x, d_y, d_imfs, nstd, oc,
                                            st, stage_seconds, float_noise);
    if (filler) {
        std::lock_guard<std::mutex> lk(g_nc_mu);
        if (s == CEEMDAN_OK && fill && g_nc_limit >= bytes) {  // the stream is synchronised
            g_nc_key = key;
            g_nc_buf = fill;
            g_nc_valid = true;
        }
        g_nc_filling = false;
    }
    return s;
}

}  // namespace

extern "C" {

void ceemdan_default_options(ceemdan_options* o) {
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(ceemdan_options);
    o->noise_sift_cap = 2000;
    o->sd = 0.05;
    o->sd2 = 0.5;
    o->tol = 0.05;
    o->seed = 1234ULL;
}

const char* ceemdan_status_string(ceemdan_status s) {
    switch (s) {
        case CEEMDAN_OK: return "ok";
        case CEEMDAN_ERR_INVALID_ARG: return "invalid argument";
        case CEEMDAN_ERR_COORD: return "d_x is not the sample index 0..N-1";
        case CEEMDAN_ERR_CUDA: return "CUDA error";
        case CEEMDAN_ERR_NO_MEMORY: return "out of device memory";
        case CEEMDAN_ERR_TIMEOUT: return "bounded in-kernel wait ran out";
        case CEEMDAN_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

const char* ceemdan_last_error(void) { return g_last_error.c_str(); }

uint64_t ceemdan_kernel_launches(void) { return g_launches.load(); }

const char* ceemdan_build_info(void) {
    static const std::string info = "sm_100a fp64 chunk=" + std::to_string(kChunk) +
                                    " tile=" + std::to_string(kTileSamples) +
                                    " lanes=" + std::to_string(kLanes);
    return info.c_str();
}

ceemdan_status ceemdan_plain_f64(size_t nr, size_t n, size_t num_imfs, size_t max_iter,
                                 const int32_t* d_x, const double* d_y, double* d_imfs,
                                 double nstd, const ceemdan_options* opt, void* stream) {
    ceemdan_options o;
    if (opt && opt->struct_size == sizeof(ceemdan_options)) {
        o = *opt;
    } else if (opt) {
        g_last_error = "ceemdan_options.struct_size mismatch";
        return CEEMDAN_ERR_INVALID_ARG;
    } else {
        ceemdan_default_options(&o);
    }
    return decompose(nr, n, num_imfs, max_iter, d_x, d_y, d_imfs, nstd, o,
                     (cudaStream_t)stream, nullptr);
}

ceemdan_status ceemdan_plain_split_f64(size_t nr_local, size_t n, size_t num_imfs,
                                       size_t max_iter, const int32_t* d_x, const double* d_y,
                                       double* d_imfs, double nstd, const ceemdan_options* opt,
                                       const ceemdan_split* split, void* stream) {
    ceemdan_options o;
    if (opt && opt->struct_size == sizeof(ceemdan_options)) {
        o = *opt;
    } else if (opt) {
        g_last_error = "ceemdan_options.struct_size mismatch";
        return CEEMDAN_ERR_INVALID_ARG;
    } else {
        ceemdan_default_options(&o);
    }
    if (!split) {
        g_last_error = "split is null";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    return decompose_impl(nr_local, n, num_imfs, max_iter, d_x, d_y, d_imfs, nstd, o,
                          (cudaStream_t)stream, nullptr, false, nullptr, split);
}

// FP32 data through the FP64 engine: y widened exactly, noise = cuRAND float normals widened
// exactly (the FP32 reference path's generator), IMFs rounded to float at the end.
ceemdan_status ceemdan_forward_taped_f64(size_t nr, size_t n, size_t num_imfs,
                                         size_t max_iter, const int32_t* d_x, const double* d_y,
                                         double* d_imfs, double nstd,
                                         const ceemdan_options* opt, void* stream,
                                         ceemdan_tape** tape_out) {
    if (!tape_out) {
        g_last_error = "tape_out is null";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    *tape_out = nullptr;
    ceemdan_options o;
    if (opt && opt->struct_size == sizeof(ceemdan_options)) {
        o = *opt;
    } else if (opt) {
        g_last_error = "ceemdan_options.struct_size mismatch";
        return CEEMDAN_ERR_INVALID_ARG;
    } else {
        ceemdan_default_options(&o);
    }
    std::unique_ptr<ceemdan_tape> t(new ceemdan_tape());
    cudaGetDevice(&t->device);
    const ceemdan_status s = decompose_impl(nr, n, num_imfs, max_iter, d_x, d_y, d_imfs, nstd, o,
                                            (cudaStream_t)stream, nullptr, false, t.get());
    if (s == CEEMDAN_OK) {
        *tape_out = t.release();
    } else {
        cudaStreamSynchronize((cudaStream_t)stream);  // iterations still queued write the tape
    }
    return s;
}

ceemdan_status ceemdan_forward_checkpointed_f64(size_t nr, size_t n, size_t num_imfs,
                                                size_t max_iter, const int32_t* d_x,
                                                const double* d_y, double* d_imfs, double nstd,
                                                const ceemdan_options* opt, void* stream,
                                                ceemdan_tape** tape_out) {
    if (!tape_out) {
        g_last_error = "tape_out is null";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    *tape_out = nullptr;
    ceemdan_options o;
    if (opt && opt->struct_size == sizeof(ceemdan_options)) {
        o = *opt;
    } else if (opt) {
        g_last_error = "ceemdan_options.struct_size mismatch";
        return CEEMDAN_ERR_INVALID_ARG;
    } else {
        ceemdan_default_options(&o);
    }
    std::unique_ptr<ceemdan_tape> t(new ceemdan_tape());
    t->checkpointed = true;
    cudaGetDevice(&t->device);
    const ceemdan_status s = decompose_impl(nr, n, num_imfs, max_iter, d_x, d_y, d_imfs, nstd, o,
                                            (cudaStream_t)stream, nullptr, false, t.get());
    if (s == CEEMDAN_OK) {
        *tape_out = t.release();
    } else {
        cudaStreamSynchronize((cudaStream_t)stream);
    }
    return s;
}

ceemdan_status ceemdan_backward_f64(const ceemdan_tape* tape, const double* d_grad_imfs,
                                    double* d_grad_y, void* stream) {
    if (!tape || !d_grad_imfs || !d_grad_y || tape->stages.empty()) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != tape->device) {
        g_last_error = "the tape belongs to another device";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    return backward_impl(*tape, d_grad_imfs, d_grad_y, (cudaStream_t)stream);
}

size_t ceemdan_tape_bytes(const ceemdan_tape* tape) { return tape ? tape->bytes : 0; }

int ceemdan_tape_iterations(const ceemdan_tape* tape, size_t stage) {
    if (!tape || stage >= tape->stages.size()) return -1;
    return tape->stages[stage].J;
}

void ceemdan_tape_free(ceemdan_tape* tape) { delete tape; }

static ceemdan_status decompose_f32(size_t nr, size_t n, size_t nimf, size_t max_iter,
                             const int32_t* d_x, const float* d_y, float* d_imfs, double nstd,
                             const ceemdan_options& o, cudaStream_t st, double* stage_seconds) {
    if (nr < 1 || n < 4 || nimf < 2 || max_iter < 1 || !d_x || !d_y || !d_imfs ||
        n > (size_t)(1u << 30) || nimf > ((size_t)1 << 20)) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    Workspace ws(st);
    double *y64 = nullptr, *imfs64 = nullptr;
    CKS(ws.alloc_n(&y64, n));
    CKS(ws.alloc_n(&imfs64, nimf * n));
    k_widen_f32<<<grid_for(n), kThreads, 0, st>>>(d_y, y64, n);
    ++g_launches;
    CK(cudaGetLastError());
    CKS(decompose(nr, n, nimf, max_iter, d_x, y64, imfs64, nstd, o, st, stage_seconds,
                  /*float_noise=*/true));
    k_narrow_f64<<<grid_for(nimf * n), kThreads, 0, st>>>(imfs64, d_imfs, nimf * n);
    ++g_launches;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return CEEMDAN_OK;
}

ceemdan_status ceemdan_plain_f32(size_t nr, size_t n, size_t num_imfs, size_t max_iter,
                                 const int32_t* d_x, const float* d_y, float* d_imfs, float nstd,
                                 const ceemdan_options* opt, void* stream) {
    ceemdan_options o;
    if (opt && opt->struct_size == sizeof(ceemdan_options)) {
        o = *opt;
    } else if (opt) {
        g_last_error = "ceemdan_options.struct_size mismatch";
        return CEEMDAN_ERR_INVALID_ARG;
    } else {
        ceemdan_default_options(&o);
    }
    return decompose_f32(nr, n, num_imfs, max_iter, d_x, d_y, d_imfs, (double)nstd, o,
                         (cudaStream_t)stream, nullptr);
}

ceemdan_status ceemdan_envelopes_f64(size_t nr, size_t n, const double* d_h, double* d_upper,
                                     double* d_lower, int32_t* d_counts, void* stream) {
    if (nr < 1 || n < 4 || !d_h || !d_upper || !d_lower || nr > 65535) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    ceemdan_options o;
    ceemdan_default_options(&o);
    Workspace ws(st);
    SiftEngine eng;
    CKS(eng.init(ws, (int)nr, (int)n, o));
    CKS(eng.reset_carries(st));
    CK(cudaMemsetAsync(eng.a.mark, 0xff, sizeof(int) * nr, st));
    CK(cudaMemcpyAsync(eng.h[0], d_h, nr * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    eng.a.dbg_upper = d_upper;
    eng.a.dbg_lower = d_lower;
    CKS(eng.launch_iteration(0, st));
    if (d_counts)
        CK(cudaMemcpyAsync(d_counts, eng.a.kcount, 2 * nr * sizeof(int), cudaMemcpyDeviceToDevice,
                           st));
    CK(cudaMemcpyAsync(eng.hstate, eng.state, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (eng.hstate[2]) return (ceemdan_status)eng.hstate[2];
    return CEEMDAN_OK;
}

ceemdan_status ceemdan_extrema_f64(size_t nr, size_t n, const double* d_h, int32_t* d_kx_max,
                                   double* d_ky_max, int32_t* d_kx_min, double* d_ky_min,
                                   int32_t* d_counts, void* stream) {
    if (nr < 1 || n < 4 || !d_h || !d_kx_max || !d_ky_max || !d_kx_min || !d_ky_min ||
        !d_counts || nr > 65535) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    ceemdan_options o;
    ceemdan_default_options(&o);
    Workspace ws(st);
    SiftEngine eng;
    CKS(eng.init(ws, (int)nr, (int)n, o));
    CKS(eng.reset_carries(st));
    CK(cudaMemsetAsync(eng.a.mark, 0xff, sizeof(int) * nr, st));
    CK(cudaMemcpyAsync(eng.h[0], d_h, nr * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    SiftArgs& a = eng.a;
    const dim3 grid_tiles((unsigned)eng.ntiles, (unsigned)nr);
    k_extrema_t<kExtremaBlocksA, false><<<eng.tile_grid, kThreads, 0, st>>>(a);
    k_scan_boundary<<<eng.scan_grid, kThreads, 0, st>>>(a);
    k_gather_knots<<<grid_tiles, kThreads, 0, st>>>(a, 0, d_kx_max, d_ky_max);
    k_gather_knots<<<grid_tiles, kThreads, 0, st>>>(a, 1, d_kx_min, d_ky_min);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(d_counts, a.kcount, 2 * nr * sizeof(int), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(eng.hstate, eng.state, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (eng.hstate[2]) return (ceemdan_status)eng.hstate[2];
    return CEEMDAN_OK;
}

ceemdan_status ceemdan_tridiag_f64(size_t batch, size_t n, const double* d_l, const double* d_m,
                                   const double* d_u, const double* d_r, double* d_x,
                                   void* stream) {
    if (batch < 1 || n < 1 || batch > 65535 || n > (size_t)(1 << 26) || !d_l || !d_m || !d_u ||
        !d_r || !d_x) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    Workspace ws(st);
    double *sys, *wsp;
    const size_t ws_stride = n + 64;
    CKS(ws.alloc_n(&sys, batch * 4 * n));
    CKS(ws.alloc_n(&wsp, batch * ws_stride));
    k_tridiag_batched<<<(unsigned)batch, kTridiagThreads, 0, st>>>((int)n, d_l, d_m, d_u, d_r, d_x, sys,
                                                            wsp, ws_stride);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return CEEMDAN_OK;
}

ceemdan_status ceemdan_canonical_sums_f64(size_t batch, size_t n, const double* d_v,
                                          const double* d_mean, double* d_sum,
                                          double* d_sqdev, void* stream) {
    if (batch < 1 || n < 1 || !d_v || !d_sum || (d_mean && !d_sqdev) || batch > 65535) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    k_canon_sums<<<(unsigned)batch, kLanes, 0, st>>>(d_v, n, d_mean, d_sum, d_sqdev);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return CEEMDAN_OK;
}

ceemdan_status ceemdan_memory_stats(uint64_t* used, uint64_t* peak, uint64_t* reserved,
                                    int reset_peak) {
    cudaMemPool_t pool = engine_pool();
    if (!pool) {
        g_last_error = "no memory pool on the current device";
        return CEEMDAN_ERR_CUDA;
    }
    uint64_t v = 0;
    if (used) CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, used));
    if (peak) CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, peak));
    if (reserved) CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, reserved));
    if (reset_peak) CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &v));
    return CEEMDAN_OK;
}

size_t ceemdan_noise_cache(size_t max_bytes) {
    std::lock_guard<std::mutex> lk(g_nc_mu);
    const size_t prev = noise_cache_limit_locked();
    g_nc_limit = max_bytes;
    if (max_bytes == 0 || (g_nc_valid && !g_nc_buf)) {
        g_nc_valid = false;
        g_nc_buf.reset();
    }
    return prev;
}

ceemdan_status ceemdan_batch_f64(size_t channels, const size_t* lengths,
                                 const double* const* d_y, double* const* d_imfs, size_t nr,
                                 size_t num_imfs, size_t max_iter, double nstd,
                                 const ceemdan_options* opt, int streams) {
    ceemdan_options o;
    if (opt && opt->struct_size == sizeof(ceemdan_options)) {
        o = *opt;
    } else if (opt) {
        g_last_error = "ceemdan_options.struct_size mismatch";
        return CEEMDAN_ERR_INVALID_ARG;
    } else {
        ceemdan_default_options(&o);
    }
    if (channels < 1 || !lengths || !d_y || !d_imfs || streams < 1 || streams > 64) {
        g_last_error = "invalid argument";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    if (o.d_noise || o.d_noise_modes_out || o.h_iters_out || o.h_kernel_ms || o.h_counters ||
        o.d_noise_state_out || o.d_noise_state_in) {
        g_last_error = "batch: per-channel outputs and external noise are not supported";
        return CEEMDAN_ERR_INVALID_ARG;
    }
    for (size_t c = 0; c < channels; ++c) {
        if (!d_y[c] || !d_imfs[c] || lengths[c] < 4) {
            g_last_error = "invalid argument (channel " + std::to_string(c) + ")";
            return CEEMDAN_ERR_INVALID_ARG;
        }
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    // longest channels first; workers take the next one until none is left
    std::vector<size_t> order(channels);
    for (size_t c = 0; c < channels; ++c) order[c] = c;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t p, size_t q) { return lengths[p] > lengths[q]; });
    std::atomic<size_t> next{0};
    std::mutex mu;
    ceemdan_status first = CEEMDAN_OK;
    std::string first_msg;
    auto worker = [&]() {
        cudaSetDevice(dev);
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            if (first == CEEMDAN_OK) {
                first = CEEMDAN_ERR_CUDA;
                first_msg = "cudaStreamCreateWithFlags failed";
            }
            return;
        }
        for (;;) {
            {
                std::lock_guard<std::mutex> lk(mu);
                if (first != CEEMDAN_OK) break;
            }
            const size_t k = next.fetch_add(1);
            if (k >= channels) break;
            const size_t c = order[k];
            ceemdan_options oc = o;
            oc.seed = o.seed + c;
            ceemdan_status s = CEEMDAN_OK;
            {
                Workspace ws(st);
                int32_t* x = nullptr;
                s = ws.alloc_n(&x, lengths[c]);
                if (s == CEEMDAN_OK) {
                    k_fill_iota<<<grid_for(lengths[c]), kThreads, 0, st>>>(x, lengths[c]);
                    ++g_launches;
                    // per-channel seeds never repeat a key: bypass the noise-phase cache
                    s = decompose_impl(nr, lengths[c], num_imfs, max_iter, x, d_y[c], d_imfs[c],
                                       nstd, oc, st, nullptr, false);
                }
                if (s == CEEMDAN_OK && cudaStreamSynchronize(st) != cudaSuccess)
                    s = CEEMDAN_ERR_CUDA;
            }
            if (s != CEEMDAN_OK) {
                std::lock_guard<std::mutex> lk(mu);
                if (first == CEEMDAN_OK) {
                    first = s;
                    first_msg = "channel " + std::to_string(c) + ": " + g_last_error;
                }
                break;
            }
        }
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    };
    const int nthreads = (int)std::min<size_t>((size_t)streams, channels);
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    if (first != CEEMDAN_OK) g_last_error = first_msg;
    return first;
}

}  // extern "C"

// Drop-in for cudaICEEMDAN.cuh:26 (C++ linkage, same mangled name as the reference).
double iceemdanS(size_t numNoise, size_t SignalLength, size_t num_IMFs, size_t max_iter,
                 int* d_x, float* d_y, float* d_IMFs, float noiseStrength) {
    ceemdan_options o;
    ceemdan_default_options(&o);
    double secs = 0.0;
    ceemdan_status s = decompose_f32(numNoise, SignalLength, num_IMFs, max_iter,
                                     reinterpret_cast<const int32_t*>(d_x), d_y, d_IMFs,
                                     (double)noiseStrength, o, (cudaStream_t)0, &secs);
    if (s != CEEMDAN_OK) return -(double)s;
    return secs;
}

double iceemdanD(size_t numNoise, size_t SignalLength, size_t num_IMFs, size_t max_iter,
                 int* d_x, double* d_y, double* d_IMFs, double noiseStrength) {
    ceemdan_options o;
    ceemdan_default_options(&o);
    double secs = 0.0;
    ceemdan_status s = decompose(numNoise, SignalLength, num_IMFs, max_iter,
                                 reinterpret_cast<const int32_t*>(d_x), d_y, d_IMFs,
                                 noiseStrength, o, (cudaStream_t)0, &secs);
    if (s != CEEMDAN_OK) return -(double)s;
    return secs;
}
