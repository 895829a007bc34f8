/*
 * ORACLE driver (test infrastructure only): runs the reference's own CUDA implementation,
 * compiled from its sources (build_ref.sh), on the GPU.  Two entry points:
 *   ref_iceemdan_f64   a full iceemdanD call (cudaICEEMDAN.cu:1340-2059) on host buffers;
 *   ref_envelopes_f64  one envelope pass of one sift iteration over nr realizations with the
 *                      reference's kernels, CUB scans and cuSPARSE solves, launched exactly as
 *                      iceemdanD launches them (cudaICEEMDAN.cu:1574-1660, grid dimensions
 *                      :1487-1557);
 *   ref_knots_f64      the knots of that pass: extrema flags, CUB scans, compaction and the
 *                      end-knot rule (cudaICEEMDAN.cu:1574-1618), positions and values of every
 *                      realization's maxima and minima as the reference's compacted arrays
 *                      hold them (realization r's knot i at r*n + i).
 * The reference translation unit is included from the reference directory (-I); nothing of
 * it is copied here.
 */
#include "cudaICEEMDAN.cu"

#include <vector>

extern "C" int ref_iceemdan_f64(size_t nr, size_t n, size_t nimf, size_t max_iter,
                                const double* h_y, double* h_imfs, double nstd, double* secs) {
    int* d_x = nullptr;
    double *d_y = nullptr, *d_imfs = nullptr;
    cudaMalloc(&d_x, n * sizeof(int));
    cudaMalloc(&d_y, n * sizeof(double));
    cudaMalloc(&d_imfs, nimf * n * sizeof(double));
    std::vector<int> x(n);
    for (size_t i = 0; i < n; ++i) x[i] = (int)i;
    cudaMemcpy(d_x, x.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(d_y, h_y, n * sizeof(double), cudaMemcpyHostToDevice);
    const double t = iceemdanD(nr, n, nimf, max_iter, d_x, d_y, d_imfs, nstd);
    cudaMemcpy(h_imfs, d_imfs, nimf * n * sizeof(double), cudaMemcpyDeviceToHost);
    if (secs) *secs = t;
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_imfs);
    return (int)cudaGetLastError();
}

extern "C" int ref_envelopes_f64(size_t nr, size_t n, const double* h_h, double* h_upper,
                                 double* h_lower, int* h_counts) {
    const size_t rn = nr * n;
    double *d_h, *d_val, *d_up, *d_mid, *d_lo, *d_right, *d_envMax, *d_envMin;
    int *d_idx, *d_flag, *d_scan, *d_cidx, *d_kmax, *d_kmin;
    cudaMalloc(&d_h, rn * sizeof(double));
    cudaMalloc(&d_idx, rn * sizeof(int));
    cudaMalloc(&d_flag, rn * sizeof(int));
    cudaMalloc(&d_scan, rn * sizeof(int));
    cudaMalloc(&d_val, rn * sizeof(double));
    cudaMalloc(&d_cidx, rn * sizeof(int));
    cudaMalloc(&d_kmax, nr * sizeof(int));
    cudaMalloc(&d_kmin, nr * sizeof(int));
    cudaMalloc(&d_up, rn * sizeof(double));
    cudaMalloc(&d_mid, rn * sizeof(double));
    cudaMalloc(&d_lo, rn * sizeof(double));
    cudaMalloc(&d_right, rn * sizeof(double));
    cudaMalloc(&d_envMax, rn * sizeof(double));
    cudaMalloc(&d_envMin, rn * sizeof(double));
    void* d_tmp = nullptr;
    const size_t tmp_bytes = 128 * 1024 * 1024 * sizeof(double);
    cudaMalloc(&d_tmp, tmp_bytes);
    double* d_gtsv = nullptr;
    cudaMalloc(&d_gtsv, 128 * 1024 * 1024 * sizeof(double));
    cusparseHandle_t sp;
    cusparseCreate(&sp);

    cudaMemcpy(d_h, h_h, rn * sizeof(double), cudaMemcpyHostToDevice);
    std::vector<int> x(rn);
    for (size_t r = 0; r < nr; ++r)
        for (size_t i = 0; i < n; ++i) x[r * n + i] = (int)i;
    cudaMemcpy(d_idx, x.data(), rn * sizeof(int), cudaMemcpyHostToDevice);

    // grid dimensions as iceemdanD computes them
    const dim3 b256(256);
    const size_t nthr = (n / 30 + 1) * 32;
    const dim3 gShfl(nthr / 256 + (nthr % 256 == 0 ? 0 : 1), nr);
    const dim3 gN(n / 256 + (n % 256 == 0 ? 0 : 1), nr);
    const dim3 gBnd(nr), bBnd(2);
    const int m = (int)(n * 0.5 + 2);

    for (int env = 0; env < 2; ++env) {
        int* d_k = env == 0 ? d_kmax : d_kmin;
        cudaMemset(d_flag, 0, rn * sizeof(int));
        if (env == 0)
            find_extrema_shfl_max<<<gShfl, b256>>>(d_idx, d_h, d_flag, n);
        else
            find_extrema_shfl_min<<<gShfl, b256>>>(d_idx, d_h, d_flag, n);
        for (size_t k = 0; k < nr; ++k) {
            size_t bytes = tmp_bytes;
            cub::DeviceScan::ExclusiveSum(d_tmp, bytes, d_flag + k * n, d_scan + k * n, (int)n);
        }
        if (env == 0) {
            select_extrema_max<<<gN, b256>>>(d_flag, d_h, d_idx, d_scan, d_val, d_cidx, n, d_k);
            setBoundaryMax<<<gBnd, bBnd>>>(d_val, d_cidx, d_scan, n);
        } else {
            select_extrema_min<<<gN, b256>>>(d_flag, d_h, d_idx, d_scan, d_val, d_cidx, n, d_k);
            setBoundaryMin<<<gBnd, bBnd>>>(d_val, d_cidx, d_scan, n);
        }
        preSetTridiagonalMatrix<<<gN, b256>>>(d_up, d_mid, d_lo, d_right, n);
        tridiagonal_setup<<<gN, b256>>>(d_k, d_cidx, d_val, d_up, d_mid, d_lo, d_right, n);
        for (size_t k = 0; k < nr; ++k)
            cusparseDgtsv2_nopivot(sp, m, 1, d_lo + k * n, d_mid + k * n, d_up + k * n,
                                   d_right + k * n, m, d_gtsv);
        spline_coefficients<<<gN, b256>>>(d_val, d_up, d_mid, d_lo, d_cidx, n, d_k, d_right);
        interpolate<<<gN, b256>>>(d_val, d_up, d_mid, d_lo, d_idx, env == 0 ? d_envMax : d_envMin,
                                  d_cidx, n, d_k);
    }
    cudaDeviceSynchronize();
    cudaMemcpy(h_upper, d_envMax, rn * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(h_lower, d_envMin, rn * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(h_counts, d_kmax, nr * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(h_counts + nr, d_kmin, nr * sizeof(int), cudaMemcpyDeviceToHost);
    const int err = (int)cudaGetLastError();
    cusparseDestroy(sp);
    void* bufs[] = {d_h, d_idx, d_flag, d_scan, d_val, d_cidx, d_kmax, d_kmin, d_up, d_mid,
                    d_lo, d_right, d_envMax, d_envMin, d_tmp, d_gtsv};
    for (void* b : bufs) cudaFree(b);
    return err;
}

extern "C" int ref_knots_f64(size_t nr, size_t n, const double* h_h, int* h_kx_max,
                             double* h_ky_max, int* h_kx_min, double* h_ky_min, int* h_counts) {
    const size_t rn = nr * n;
    double *d_h, *d_val;
    int *d_idx, *d_flag, *d_scan, *d_cidx, *d_k;
    cudaMalloc(&d_h, rn * sizeof(double));
    cudaMalloc(&d_idx, rn * sizeof(int));
    cudaMalloc(&d_flag, rn * sizeof(int));
    cudaMalloc(&d_scan, rn * sizeof(int));
    cudaMalloc(&d_val, rn * sizeof(double));
    cudaMalloc(&d_cidx, rn * sizeof(int));
    cudaMalloc(&d_k, 2 * nr * sizeof(int));
    void* d_tmp = nullptr;
    const size_t tmp_bytes = 128 * 1024 * 1024 * sizeof(double);
    cudaMalloc(&d_tmp, tmp_bytes);
    cudaMemcpy(d_h, h_h, rn * sizeof(double), cudaMemcpyHostToDevice);
    std::vector<int> x(rn);
    for (size_t r = 0; r < nr; ++r)
        for (size_t i = 0; i < n; ++i) x[r * n + i] = (int)i;
    cudaMemcpy(d_idx, x.data(), rn * sizeof(int), cudaMemcpyHostToDevice);
    const dim3 b256(256);
    const size_t nthr = (n / 30 + 1) * 32;
    const dim3 gShfl(nthr / 256 + (nthr % 256 == 0 ? 0 : 1), nr);
    const dim3 gN(n / 256 + (n % 256 == 0 ? 0 : 1), nr);
    const dim3 gBnd(nr), bBnd(2);
    for (int env = 0; env < 2; ++env) {
        int* kc = d_k + env * nr;
        cudaMemset(d_flag, 0, rn * sizeof(int));
        if (env == 0)
            find_extrema_shfl_max<<<gShfl, b256>>>(d_idx, d_h, d_flag, n);
        else
            find_extrema_shfl_min<<<gShfl, b256>>>(d_idx, d_h, d_flag, n);
        for (size_t k = 0; k < nr; ++k) {
            size_t bytes = tmp_bytes;
            cub::DeviceScan::ExclusiveSum(d_tmp, bytes, d_flag + k * n, d_scan + k * n, (int)n);
        }
        if (env == 0) {
            select_extrema_max<<<gN, b256>>>(d_flag, d_h, d_idx, d_scan, d_val, d_cidx, n, kc);
            setBoundaryMax<<<gBnd, bBnd>>>(d_val, d_cidx, d_scan, n);
        } else {
            select_extrema_min<<<gN, b256>>>(d_flag, d_h, d_idx, d_scan, d_val, d_cidx, n, kc);
            setBoundaryMin<<<gBnd, bBnd>>>(d_val, d_cidx, d_scan, n);
        }
        cudaMemcpy(env == 0 ? h_kx_max : h_kx_min, d_cidx, rn * sizeof(int),
                   cudaMemcpyDeviceToHost);
        cudaMemcpy(env == 0 ? h_ky_max : h_ky_min, d_val, rn * sizeof(double),
                   cudaMemcpyDeviceToHost);
    }
    cudaMemcpy(h_counts, d_k, 2 * nr * sizeof(int), cudaMemcpyDeviceToHost);
    const int err = (int)cudaGetLastError();
    void* bufs[] = {d_h, d_idx, d_flag, d_scan, d_val, d_cidx, d_k, d_tmp};
    for (void* b : bufs) cudaFree(b);
    return err;
}
