// A caller written against the reference's header contract: it includes cudaICEEMDAN.cuh,
// passes device pointers (coordinates 0..N-1, the float signal, a num_IMFs x N output) to
// iceemdanS or iceemdanD, and reads the IMFs back.  Built by tests/test_dropin_caller.py and
// linked against libceemdan_b200.so only: a reference caller relinks without source changes.
//
// usage: dropin_caller INPUT OUTPUT NR NUM_IMFS MAX_ITER [d]
//   INPUT  raw float32 samples (float64 with the trailing "d": iceemdanD)
//   OUTPUT raw IMFs, same type
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cudaICEEMDAN.cuh"

template <class T>
static int run(const char* in, const char* out, size_t nr, size_t nimf, size_t mi) {
    FILE* f = std::fopen(in, "rb");
    if (!f) return 2;
    std::vector<T> y;
    T v;
    while (std::fread(&v, sizeof(T), 1, f) == 1) y.push_back(v);
    std::fclose(f);
    const size_t n = y.size();
    std::vector<int> x(n);
    for (size_t i = 0; i < n; ++i) x[i] = (int)i;
    int* d_x = nullptr;
    T *d_y = nullptr, *d_imfs = nullptr;
    cudaMalloc(&d_x, n * sizeof(int));
    cudaMalloc(&d_y, n * sizeof(T));
    cudaMalloc(&d_imfs, nimf * n * sizeof(T));
    cudaMemcpy(d_x, x.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(d_y, y.data(), n * sizeof(T), cudaMemcpyHostToDevice);
    double secs;
    if constexpr (sizeof(T) == sizeof(float))
        secs = iceemdanS(nr, n, nimf, mi, d_x, d_y, d_imfs, 0.2f);
    else
        secs = iceemdanD(nr, n, nimf, mi, d_x, d_y, d_imfs, 0.2);
    std::printf("Execution time: %f\n", secs);
    if (secs < 0) return 3;
    std::vector<T> imfs(nimf * n);
    cudaMemcpy(imfs.data(), d_imfs, imfs.size() * sizeof(T), cudaMemcpyDeviceToHost);
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_imfs);
    FILE* g = std::fopen(out, "wb");
    if (!g) return 2;
    std::fwrite(imfs.data(), sizeof(T), imfs.size(), g);
    std::fclose(g);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 6) return 1;
    const size_t nr = std::strtoul(argv[3], nullptr, 10), nimf = std::strtoul(argv[4], nullptr, 10),
                 mi = std::strtoul(argv[5], nullptr, 10);
    if (argc > 6 && argv[6][0] == 'd') return run<double>(argv[1], argv[2], nr, nimf, mi);
    return run<float>(argv[1], argv[2], nr, nimf, mi);
}
