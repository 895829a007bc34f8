#!/bin/bash
# Builds the reference's own CUDA implementation of the ICEEMDAN path (test infrastructure:
# a second oracle) from its sources where they lie, plus our driver, into oracle/_ref/; also
# the reference's unmodified file-based sample driver (sample_binary_file.cu) relinked against
# libceemdan_b200.so (the drop-in check), the fopen shim it runs under in the tests, and copies
# of the reference's two sample EEG recordings (read by the parity tests).
# Nothing is copied from the reference's sources; they are compiled in place, the reference's
# own implementation with oracle/ref_shim.h force-included (padded, zero-filled allocations).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
# the reference checkout: CEEMDAN_REFERENCE_DIR, else a sibling "reference" directory of the repo
REF="${CEEMDAN_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
PKG="$(cd "$HERE/../ceemdan-gpu_b200" && pwd)"
NVCC=/usr/local/cuda/bin/nvcc
ARCH=(-gencode arch=compute_100a,code=sm_100a)
FLAGS=("${ARCH[@]}" -O3 -std=c++17 -Xcompiler -fPIC
       -Xcompiler -fopenmp -include "$HERE/ref_shim.h" -I"$REF" -w)
if [ ! -f "$REF/cudaICEEMDAN.cu" ]; then
    echo "reference sources not found at $REF" >&2
    exit 1
fi
mkdir -p "$OUT" "$OUT/data"
# newer(target, deps...): true when target is missing or older than a dependency
stale() { local t="$1"; shift; [ ! -e "$t" ] && return 0; for d in "$@"; do [ "$d" -nt "$t" ] && return 0; done; return 1; }
if stale "$OUT/libref_iceemdan.so" "$HERE/ref_driver.cu" "$HERE/ref_shim.h" "$REF/cudaICEEMDAN.cu"; then
    "$NVCC" "${FLAGS[@]}" -c "$REF/statistics.cu" -o "$OUT/statistics.o"
    "$NVCC" "${FLAGS[@]}" -c "$HERE/ref_driver.cu" -o "$OUT/ref_driver.o"
    "$NVCC" "${ARCH[@]}" -shared -o "$OUT/libref_iceemdan.so" \
        "$OUT/ref_driver.o" "$OUT/statistics.o" -L/usr/local/cuda/lib64 -lcusparse -lcurand -lcublas \
        -lgomp -Xlinker -rpath -Xlinker /usr/local/cuda/lib64
fi
if [ -f "$PKG/libceemdan_b200.so" ] && stale "$OUT/sample_binary_file" "$PKG/libceemdan_b200.so" "$REF/sample_binary_file.cu"; then
    "$NVCC" "${ARCH[@]}" -O2 -w "$REF/sample_binary_file.cu" -I"$HERE/../include" -L"$PKG" \
        -lceemdan_b200 -Xlinker -rpath -Xlinker "$PKG" -o "$OUT/sample_binary_file"
fi
if stale "$OUT/path_shim.so" "$HERE/../tests/path_shim.c"; then
    gcc -shared -fPIC -O2 "$HERE/../tests/path_shim.c" -o "$OUT/path_shim.so" -ldl
fi
for f in eegSampleDataCH4.bin eegSampleDataCH1_244032.bin; do
    if [ -f "$REF/$f" ] && stale "$OUT/data/$f" "$REF/$f"; then cp "$REF/$f" "$OUT/data/$f"; fi
done
