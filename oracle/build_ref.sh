#!/bin/bash
# Builds the reference's own CUDA implementation of the ICEEMDAN path (test infrastructure:
# a second oracle) from its sources where they lie, plus our driver, into oracle/_ref/.
# Nothing is copied from the reference; its sources are compiled in place, with
# oracle/ref_shim.h force-included (padded, zero-filled allocations).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
# the reference checkout: CEEMDAN_REFERENCE_DIR, else a sibling "reference" directory of the repo
REF="${CEEMDAN_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
NVCC=/usr/local/cuda/bin/nvcc
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Xcompiler -fPIC
       -Xcompiler -fopenmp -include "$HERE/ref_shim.h" -I"$REF" -w)
if [ ! -f "$REF/cudaICEEMDAN.cu" ]; then
    echo "reference sources not found at $REF" >&2
    exit 1
fi
mkdir -p "$OUT"
if [ "$OUT/libref_iceemdan.so" -nt "$HERE/ref_driver.cu" ] && [ "$OUT/libref_iceemdan.so" -nt "$HERE/ref_shim.h" ]; then
    exit 0
fi
"$NVCC" "${FLAGS[@]}" -c "$REF/statistics.cu" -o "$OUT/statistics.o"
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_driver.cu" -o "$OUT/ref_driver.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libref_iceemdan.so" \
    "$OUT/ref_driver.o" "$OUT/statistics.o" -L/usr/local/cuda/lib64 -lcusparse -lcurand -lcublas \
    -lgomp -Xlinker -rpath -Xlinker /usr/local/cuda/lib64
