#!/usr/bin/env bash
# Test infrastructure: builds the UNMODIFIED reference (Xshuaizhang/Retainwall_code)
# from its own sources where they lie, into oracle/_ref/ (git-ignored; travels to
# the GPU box with the rest of the tree). Nothing is copied from the reference.
#   oracle/_ref/ref_driver_f32, ref_driver_f64  : reference CUDA step (sm_100a) +
#       oracle/ref_driver.cu in place of src/main.cpp (per-stage dumps, timing)
#   oracle/_ref/libref_hypo_f32.so, _f64.so     : host build of src/functions.h +
#       src/constitutive_model.h (known answers for the oracle's restatement)
# Usage: oracle/build_ref.sh [REFERENCE_SRC_DIR]
#   the directory defaults to $RW_REFERENCE_SRC, else to the read-only reference checkout
#   of the development machine; without sources the prebuilt files are kept.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
SRC="${1:-${RW_REFERENCE_SRC:-/root/reference/src}}"
OUT="$HERE/_ref"
if [ ! -f "$SRC/loquat.cu" ]; then
  echo "reference sources not found at $SRC; keeping prebuilt files in $OUT" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC="${NVCC:-nvcc}"
CU_SRCS="loquat.cu loquat_grid.cu loquat_io.cu adami_boundary.cu particle_interaction.cu predictor_corrector.cu field_smoothing.cu utilities.cu"

build_driver() {  # $1 = suffix, $2 = extra defines
  local tag="$1" def="$2" objs=""
  local tmp="$OUT/obj_$tag"
  mkdir -p "$tmp"
  for f in $CU_SRCS; do
    "$NVCC" -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a $def \
      -I "$HERE/ref_shims" -I "$SRC" -c "$SRC/$f" -o "$tmp/${f%.cu}.o" -w &
  done
  "$NVCC" -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a $def \
    -I "$HERE/ref_shims" -I "$SRC" -c "$HERE/ref_driver.cu" -o "$tmp/ref_driver.o" -w &
  g++ -std=c++17 -O2 $def -c "$SRC/tinyxml2.cpp" -o "$tmp/tinyxml2.o" -w &
  wait
  for f in $CU_SRCS; do objs="$objs $tmp/${f%.cu}.o"; done
  "$NVCC" -gencode arch=compute_100a,code=sm_100a -o "$OUT/ref_driver_$tag" $objs "$tmp/ref_driver.o" "$tmp/tinyxml2.o"
  rm -rf "$tmp"
}

build_hypo() {  # $1 = suffix, $2 = extra defines
  g++ -std=c++17 -O2 -ffp-contract=off -fPIC -shared $2 -I /usr/local/cuda/include -I "$SRC" \
    "$HERE/ref_hypo.cpp" -o "$OUT/libref_hypo_$1.so" -w
}

if ! command -v "$NVCC" >/dev/null 2>&1; then
  echo "nvcc not found; keeping prebuilt files in $OUT" >&2
  exit 0
fi
build_hypo f32 "" &
build_hypo f64 "-DDOUBLE_PRECISION" &
build_driver f32 ""
build_driver f64 "-DDOUBLE_PRECISION"
wait
echo "reference build done: $(ls "$OUT")"
