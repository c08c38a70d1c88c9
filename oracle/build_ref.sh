#!/usr/bin/env bash
# Build recipe for oracle/_ref/libcirrus_ref.so: the reference's own CUDA implementation of the
# Poisson path, compiled from its unmodified sources where they lie, plus oracle/ref_harness.cu.
# The library links nothing of this project.  A second library, libcirrus_ref_dropin.so, adds
# oracle/ref_dropin_harness.cu (the product's drop-in header on the reference's grids) and links
# both libcirrus_ref.so and the product library; only tests load it.
# Test infrastructure only.  Needs the reference tree (CIRRUS_REFERENCE_DIR, else a directory
# named reference beside this repository) and nvcc; the
# output directory oracle/_ref/ is git-ignored and travels to the GPU box as a built file.
#
# Include paths: fmt (header-only) from torch's bundled headers and nlohmann/json from
# cudnn_frontend's third-party tree, both inside this image's Python environment; Eigen is
# included by src/PoissonSolver.h but unused on this path, so an empty shim header stands in.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${CIRRUS_REFERENCE_DIR:-$HERE/../../reference}"  # default: the reference tree beside this repository
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
  echo "build_ref: reference tree not found at $REF" >&2
  exit 2
fi
SITE="$(python -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')"
FMT_INC="$SITE/torch/include"
JSON_INC="$SITE/include/cudnn_frontend/thirdparty"
mkdir -p "$OUT/obj" "$OUT/shim/Eigen"
: > "$OUT/shim/Eigen/Dense"
NVCC="${NVCC:-nvcc}"
FLAGS=(-std=c++17 -O3 -extended-lambda -lineinfo -gencode arch=compute_100a,code=sm_100a
       -Xcompiler -fPIC -DFMT_HEADER_ONLY -w
       -I"$REF/src" -I"$REF/common" -I"$REF/ext" -I"$FMT_INC" -I"$JSON_INC" -I"$OUT/shim")
pids=()
for src in src/GMGSolver.cu src/PoissonSolver.cu src/PoissonGrid.cu src/HAGrid.cu; do
  obj="$OUT/obj/$(basename "$src").o"
  "$NVCC" "${FLAGS[@]}" -dc -c "$REF/$src" -o "$obj" &
  pids+=($!)
done
"$NVCC" "${FLAGS[@]}" -x cu -dc -c "$REF/common/Common.cpp" -o "$OUT/obj/Common.cpp.o" &
pids+=($!)
"$NVCC" "${FLAGS[@]}" -dc -c "$HERE/ref_harness.cu" -o "$OUT/obj/ref_harness.cu.o" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
"$NVCC" -shared -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC "$OUT"/obj/*.o -o "$OUT/libcirrus_ref.so"
echo "built $OUT/libcirrus_ref.so"
# the drop-in harness: the product's header on the reference grid (tests only)
PRODUCT_LIB="$HERE/../cirrus_b200/_lib"
if [ ! -f "$PRODUCT_LIB/libcirrus_b200.so" ]; then
  echo "build_ref: build the product library first (python cirrus_b200/build.py) for libcirrus_ref_dropin.so" >&2
  exit 3
fi
mkdir -p "$OUT/dropin"
"$NVCC" "${FLAGS[@]}" -I"$HERE/../include" -c "$HERE/ref_dropin_harness.cu" -o "$OUT/dropin/ref_dropin_harness.cu.o"
"$NVCC" -shared -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC "$OUT/dropin/ref_dropin_harness.cu.o" \
  -o "$OUT/libcirrus_ref_dropin.so" -L"$OUT" -lcirrus_ref -L"$PRODUCT_LIB" -lcirrus_b200 \
  -Xlinker -rpath -Xlinker '$ORIGIN' -Xlinker -rpath -Xlinker '$ORIGIN/../../cirrus_b200/_lib'
echo "built $OUT/libcirrus_ref_dropin.so"
