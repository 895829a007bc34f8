// ceemdan_file: decompose a raw float32 signal file into a raw float32 modes file.
//
// The file-level driver of the reference (sample_binary_file.cu:36-83): the input is N
// little-endian float32 samples (N = file size / 4), the output is num_IMFs x N float32 (row k
// = IMF k, last row = residue, in units of y/std(y)), and the decomposition is iceemdanS with
// the driver's defaults NR = 200, num_IMFs = 12, MaxIter = 300, Nstd = 0.2.  Options change
// those, choose FP64 data (--f64: float64 in and out, iceemdanD semantics) and the noise seed
// (default 1234, the reference's).  Unlike the reference driver, every failure -- unreadable
// or short input, invalid sizes, a CUDA or engine error -- ends with a message and a non-zero
// exit status, and nothing touches the GPU before the arguments and the input are checked.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ceemdan_b200.h"

namespace {

struct Args {
    std::string in, out;
    size_t nr = 200, nimf = 12, max_iter = 300, noise_cap = 2000;
    double nstd = 0.2;
    uint64_t seed = 1234;
    bool f64 = false;
};

void usage(FILE* f) {
    std::fprintf(f,
                 "usage: ceemdan_file INPUT OUTPUT [--nr N] [--imfs K] [--max-iter M]\n"
                 "                    [--nstd S] [--seed X] [--noise-cap C] [--f64]\n"
                 "  INPUT   raw little-endian float32 samples (float64 with --f64)\n"
                 "  OUTPUT  raw modes, K rows of N samples (IMF 0..K-2, residue), same type\n"
                 "  defaults: --nr 200 --imfs 12 --max-iter 300 --nstd 0.2 --seed 1234\n"
                 "            --noise-cap 2000 (sift cap of the noise modes)\n");
}

bool parse_size(const char* s, size_t* v) {
    char* end = nullptr;
    const unsigned long long x = std::strtoull(s, &end, 10);
    if (!end || *end || s[0] == '-') return false;
    *v = (size_t)x;
    return true;
}

// 0: ok, 1: usage error, 2: help shown
int parse(int argc, char** argv, Args* a) {
    std::vector<std::string> pos;
    for (int i = 1; i < argc; ++i) {
        const std::string k = argv[i];
        auto val = [&](const char** out) {
            if (i + 1 >= argc) return false;
            *out = argv[++i];
            return true;
        };
        const char* v = nullptr;
        if (k == "-h" || k == "--help") return 2;
        if (k == "--f64") {
            a->f64 = true;
        } else if (k == "--nr") {
            if (!val(&v) || !parse_size(v, &a->nr)) return 1;
        } else if (k == "--imfs") {
            if (!val(&v) || !parse_size(v, &a->nimf)) return 1;
        } else if (k == "--max-iter") {
            if (!val(&v) || !parse_size(v, &a->max_iter)) return 1;
        } else if (k == "--noise-cap") {
            if (!val(&v) || !parse_size(v, &a->noise_cap)) return 1;
        } else if (k == "--seed") {
            size_t s = 0;
            if (!val(&v) || !parse_size(v, &s)) return 1;
            a->seed = s;
        } else if (k == "--nstd") {
            if (!val(&v)) return 1;
            char* end = nullptr;
            a->nstd = std::strtod(v, &end);
            if (!end || *end || !(a->nstd >= 0.0)) return 1;
        } else if (!k.empty() && k[0] == '-') {
            return 1;
        } else {
            pos.push_back(k);
        }
    }
    if (pos.size() != 2) return 1;
    a->in = pos[0];
    a->out = pos[1];
    if (a->nr < 1 || a->nimf < 2 || a->max_iter < 1 || a->noise_cap < 1) return 1;
    return 0;
}

bool read_file(const std::string& path, std::vector<char>* buf) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 0) {
        std::fclose(f);
        return false;
    }
    buf->resize((size_t)size);
    const size_t got = size ? std::fread(buf->data(), 1, (size_t)size, f) : 0;
    std::fclose(f);
    return got == (size_t)size;
}

int fail(const char* what, const char* detail) {
    std::fprintf(stderr, "ceemdan_file: %s%s%s\n", what, detail ? ": " : "", detail ? detail : "");
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    Args a;
    const int pr = parse(argc, argv, &a);
    if (pr == 2) {
        usage(stdout);
        return 0;
    }
    if (pr != 0) {
        usage(stderr);
        return 2;
    }
    std::vector<char> raw;
    if (!read_file(a.in, &raw)) return fail("cannot read", a.in.c_str());
    const size_t esz = a.f64 ? sizeof(double) : sizeof(float);
    if (raw.size() % esz) return fail("input size is not a whole number of samples", nullptr);
    const size_t n = raw.size() / esz;
    if (n < 4) return fail("input has fewer than 4 samples", nullptr);
    {
        FILE* probe = std::fopen(a.out.c_str(), "wb");  // fail before any GPU work
        if (!probe) return fail("cannot write", a.out.c_str());
        std::fclose(probe);
    }

    std::vector<int32_t> x(n);
    for (size_t i = 0; i < n; ++i) x[i] = (int32_t)i;
    void *d_x = nullptr, *d_y = nullptr, *d_imfs = nullptr;
    const size_t out_bytes = a.nimf * n * esz;
    if (cudaMalloc(&d_x, n * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&d_y, raw.size()) != cudaSuccess ||
        cudaMalloc(&d_imfs, out_bytes) != cudaSuccess)
        return fail("cudaMalloc", cudaGetErrorString(cudaGetLastError()));
    if (cudaMemcpy(d_x, x.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_y, raw.data(), raw.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail("cudaMemcpy", cudaGetErrorString(cudaGetLastError()));

    ceemdan_options o;
    ceemdan_default_options(&o);
    o.seed = a.seed;
    o.noise_sift_cap = (int)a.noise_cap;
    const auto t0 = std::chrono::steady_clock::now();
    const ceemdan_status s =
        a.f64 ? ceemdan_plain_f64(a.nr, n, a.nimf, a.max_iter, (const int32_t*)d_x,
                                  (const double*)d_y, (double*)d_imfs, a.nstd, &o, nullptr)
              : ceemdan_plain_f32(a.nr, n, a.nimf, a.max_iter, (const int32_t*)d_x,
                                  (const float*)d_y, (float*)d_imfs, (float)a.nstd, &o, nullptr);
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (s != CEEMDAN_OK) return fail(ceemdan_status_string(s), ceemdan_last_error());
    std::printf("Execution time: %f \n", secs);

    std::vector<char> out(out_bytes);
    if (cudaMemcpy(out.data(), d_imfs, out_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail("cudaMemcpy", cudaGetErrorString(cudaGetLastError()));
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_imfs);
    FILE* f = std::fopen(a.out.c_str(), "wb");
    if (!f) return fail("cannot write", a.out.c_str());
    const size_t put = std::fwrite(out.data(), 1, out_bytes, f);
    if (std::fclose(f) != 0 || put != out_bytes) return fail("short write", a.out.c_str());
    return 0;
}
