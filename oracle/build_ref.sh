#!/usr/bin/env bash
# Build recipe for oracle/_ref/libcirrus_ref.so: the reference's own CUDA implementation of the
# Poisson path, compiled from its unmodified sources where they lie, plus oracle/ref_harness.cu.
# Test infrastructure only.  Needs the reference tree (default /root/reference) and nvcc;
# the output directory oracle/_ref/ is git-ignored and travels to the GPU box as a built file.
#
# Include paths: fmt (header-only) from torch's bundled headers and nlohmann/json from
# cudnn_frontend's third-party tree, both inside this image's Python environment; Eigen is
# included by src/PoissonSolver.h but unused on this path, so an empty shim header stands in.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${CIRRUS_REFERENCE_DIR:-/root/reference}"
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
"$NVCC" "${FLAGS[@]}" -I"$HERE/../include" -dc -c "$HERE/ref_harness.cu" -o "$OUT/obj/ref_harness.cu.o" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
# the harness also exercises the product's header-only drop-in, so it links the product library
PRODUCT_LIB="$HERE/../cirrus_b200/_lib"
if [ ! -f "$PRODUCT_LIB/libcirrus_b200.so" ]; then
  echo "build_ref: build the product library first (python cirrus_b200/build.py)" >&2
  exit 3
fi
"$NVCC" -shared -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC "$OUT"/obj/*.o -o "$OUT/libcirrus_ref.so" \
  -L"$PRODUCT_LIB" -lcirrus_b200 -Xlinker -rpath -Xlinker '$ORIGIN/../../cirrus_b200/_lib'
echo "built $OUT/libcirrus_ref.so"
