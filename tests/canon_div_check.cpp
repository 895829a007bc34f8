// Checks ceemdan::div_rcp (division by a divisor with a correctly rounded reciprocal, used by
// the evaluation and spline kernels) against IEEE division: random and near-tie dividends,
// zero / tiny / huge / non-finite dividends, divisors 3, h and 3h for h = 1..4096.
// Built and run by tests/test_canon_host.py.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>

#include "../ceemdan-gpu_b200/csrc/canon.cuh"

int main() {
    std::mt19937_64 rng(11);
    long bad = 0, total = 0;
    for (int h = 1; h <= 4096; ++h) {
        const double divs[3] = {(double)h, 3.0 * h, 3.0};
        for (double d : divs) {
            const double y = 1.0 / d;
            for (int it = 0; it < 2000; ++it) {
                double a;
                const int mode = it % 6;
                if (mode == 0) {
                    uint64_t bits = (rng() & 0x800FFFFFFFFFFFFFull) |
                                    ((uint64_t)(1023 + (int)(rng() % 300) - 150) << 52);
                    std::memcpy(&a, &bits, 8);
                } else if (mode == 1) {
                    a = d * (double)(int64_t)(rng() % 1000000) * std::ldexp(1.0, (int)(rng() % 40) - 20);
                    a = std::nextafter(a, (rng() & 1) ? INFINITY : -INFINITY);
                } else if (mode == 2) {
                    const double sp[7] = {0.0, -0.0, 0x1p-1000, -0x1p-1070, 0x1p+1020, INFINITY, NAN};
                    a = sp[rng() % 7];
                } else {
                    std::uniform_real_distribution<double> u(-1e3, 1e3);
                    a = u(rng) * std::ldexp(1.0, (int)(rng() % 80) - 40);
                }
                const double got = ceemdan::div_rcp(a, d, y);
                const double ex = a / d;
                const bool same = (std::isnan(got) && std::isnan(ex)) || std::memcmp(&got, &ex, 8) == 0;
                if (!same) ++bad;
                ++total;
            }
        }
    }
    std::printf("total %ld mismatches %ld\n", total, bad);
    return bad == 0 ? 0 : 1;
}
