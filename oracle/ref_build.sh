#!/bin/bash
# Builds oracle/_ref/ref_harness: the reference's own GPU kernel
# (wfa_dispatcher in wfa_gpu.cu, compiled unchanged for sm_100a from the
# reference tree) linked with this project's harness (ref_harness.cu), the
# CPU model that certifies inputs before any launch (ref_kernel_model.c),
# the seeded generator (wfa_gen.c) and a stand-in for the four WFA2-lib
# names wfa_gpu.cu declares (ref_stub/).  Outputs go to oracle/_ref/ only.
# TEST INFRASTRUCTURE ONLY.
#
#   REF=/path/to/reference oracle/ref_build.sh     (default: /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${REF:-/root/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
ARCH="-gencode arch=compute_100a,code=sm_100a"
if [ ! -f "$REF/wfa_gpu.cu" ]; then
  echo "ref_build: $REF/wfa_gpu.cu not found; keeping any prebuilt $OUT" >&2
  exit 0
fi
mkdir -p "$OUT"
# The reference's own flags (Makefile:3,9) plus the target architecture;
# its main is renamed so the harness owns main.
"$NVCC" -std=c++14 -O3 $ARCH -I"$HERE/ref_stub" -I"$REF" -Dmain=tsu_reference_main_unused \
  -Xcompiler -fopenmp -diag-suppress 940,177,550,1650 -Xcompiler -Wno-unused-result -c "$REF/wfa_gpu.cu" -o "$OUT/wfa_gpu.o"
gcc -O2 -fopenmp -std=c11 -I"$HERE/ref_stub" -c "$HERE/ref_stub/ref_stub.c" -o "$OUT/ref_stub.o"
gcc -O2 -fopenmp -std=c11 -c "$HERE/ref_kernel_model.c" -o "$OUT/ref_kernel_model.o"
gcc -O2 -fopenmp -std=c11 -c "$HERE/wfa_gen.c" -o "$OUT/wfa_gen.o"
"$NVCC" -std=c++17 -O2 $ARCH -I"$HERE" -c "$HERE/ref_harness.cu" -o "$OUT/ref_harness.o"
"$NVCC" $ARCH -o "$OUT/ref_harness" "$OUT/ref_harness.o" "$OUT/wfa_gpu.o" "$OUT/ref_stub.o" \
  "$OUT/ref_kernel_model.o" "$OUT/wfa_gen.o" -Xcompiler -fopenmp -lm
echo "ref_build: $OUT/ref_harness"
