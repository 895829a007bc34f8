// Checks ceemdan::sx_greater (division-free sx threshold test used by the evaluation kernel)
// against the exact division it stands for, on random and adversarial near-tie inputs.
// Built and run by tests/test_canon_host.py.
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <random>

#include "../ceemdan-gpu_b200/csrc/canon.cuh"

int main() {
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    const double ths[2] = {0.05, 0.5};
    long bad = 0, total = 0, near = 0;
    for (int it = 0; it < 4000000; ++it) {
        const double t = ths[it & 1];
        double up, lo;
        const int mode = it % 7;
        if (mode == 0) {  // generic
            up = u(rng) * std::pow(10.0, 6 * u(rng));
            lo = u(rng) * std::pow(10.0, 6 * u(rng));
        } else if (mode <= 3) {  // |U+L|/|U-L| within a few ulps of t
            const double d = std::pow(10.0, 4 * u(rng)) * (u(rng) > 0 ? 1 : -1);
            const double s = d * t * (1.0 + (double)((int64_t)(rng() % 64) - 32) * 0x1p-52);
            up = 0.5 * (s + d);
            lo = 0.5 * (s - d);
            ++near;
        } else if (mode == 4) {  // exact zeros / equal envelopes
            up = (rng() & 1) ? 0.0 : u(rng);
            lo = (rng() & 1) ? up : -up;
        } else if (mode == 5) {  // extreme magnitudes
            up = u(rng) * std::ldexp(1.0, (int)(rng() % 2000) - 1000);
            lo = u(rng) * std::ldexp(1.0, (int)(rng() % 2000) - 1000);
        } else {  // non-finite
            const double sp[4] = {INFINITY, -INFINITY, NAN, 0.0};
            up = sp[rng() % 4];
            lo = (rng() & 1) ? sp[rng() % 4] : u(rng);
        }
        const bool exact = std::fabs((up + lo) / (up - lo)) > t;
        if (ceemdan::sx_greater(up, lo, t) != exact) ++bad;
        ++total;
    }
    std::printf("total %ld near %ld mismatches %ld\n", total, near, bad);
    return bad == 0 ? 0 : 1;
}
