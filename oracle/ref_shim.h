/*
 * ORACLE build support (test infrastructure only).  Force-included (-include) when the
 * reference's own CUDA sources are compiled into oracle/_ref.  Every cudaMalloc of the
 * reference is padded to twice its size and zero-filled:
 *   - iceemdanD allocates d_running with N*sizeof(float) and writes N doubles into it
 *     (cudaICEEMDAN.cu:1346 vs :1722, :1744); the padding keeps that write inside the block;
 *   - the reference's accumulators (statistics.cu atomicAdd targets, d_meanEnvelope, the sift
 *     fraction) are never initialised; zero-filling gives them the fresh-allocation value the
 *     oracle and the engine assume.
 * The reference sources themselves are compiled unmodified from where they lie.
 */
#ifndef CEEMDAN_REF_SHIM_H
#define CEEMDAN_REF_SHIM_H
#include <cuda_runtime.h>

static inline cudaError_t ceemdan_ref_shim_malloc(void** p, size_t bytes) {
    const size_t padded = 2 * bytes + 256;
    cudaError_t e = cudaMalloc(p, padded);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, padded);
    return e;
}
#define cudaMalloc(p, n) ceemdan_ref_shim_malloc((void**)(p), (size_t)(n))

#endif
