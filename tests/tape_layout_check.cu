// Host-only check of the tape slot layout (TapeLayout in csrc/kernels.h) that the taped forward
// and the reverse-pass kernels rely on: the bitmap region is copied as 16-byte pieces, slots
// start 256-byte aligned inside blocks, and every field lies inside its slot.  No device code
// runs.  Built and run by tests/test_adjoint_gpu.py.
#include <cstdio>

#include "../ceemdan-gpu_b200/csrc/kernels.h"

int main() {
    long bad = 0, cases = 0;
    for (int nr = 1; nr <= 4096; nr = nr < 64 ? nr + 1 : nr * 2 + 1) {
        for (int ntiles = 1; ntiles <= 600; ntiles = ntiles < 8 ? ntiles + 1 : ntiles * 3) {
            const ceemdan::TapeLayout L = ceemdan::tape_layout(nr, ntiles);
            ++cases;
            const size_t bits = (size_t)2 * nr * ntiles * (ceemdan::kTileSamples / 32) * 4;
            bool ok = L.off_kc == bits && bits % 16 == 0 &&      // uint4 copies of the bitmaps
                      L.off_kc % alignof(int) == 0 &&             // int knot counts
                      L.off_bf == L.off_kc + (size_t)2 * nr * 4 &&
                      L.off_mark == L.off_bf + (size_t)2 * nr &&
                      L.off_mark + (size_t)nr <= L.stride &&      // marks inside the slot
                      L.stride % 256 == 0 && L.stride - (L.off_mark + nr) < 256;
            if (!ok) {
                ++bad;
                std::printf("bad layout nr=%d ntiles=%d\n", nr, ntiles);
            }
        }
    }
    std::printf("cases %ld mismatches %ld\n", cases, bad);
    return bad == 0 ? 0 : 1;
}
