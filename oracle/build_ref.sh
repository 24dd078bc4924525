#!/usr/bin/env bash
# Builds oracle/_ref/libsdx_ref.so (FP64 mode) and oracle/_ref/libsdx_ref_f32.so (FP32 mode) from the
# REFERENCE's own sources (read in place, never copied):
# the Smith Neo-Hookean, St. Venant-Kirchhoff, linear-elastic and ARAP translation units plus the header-only StressWork, PCG, PolyReLU and penalty
# contact code and BlockSparseMatrix / BlockJacobiPrec (run without a task scheduler, ref_serial_scheduler.cpp), behind the C shim oracle/ref_shim.cpp.
# Runs only where the reference tree exists; the GPU box uses the prebuilt .so.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
# the reference tree: SDX_REFERENCE_ROOT (no default path; without it nothing is built)
REF="${SDX_REFERENCE_ROOT:-}"
if [ -z "$REF" ]; then
  echo "SDX_REFERENCE_ROOT is not set; skipping oracle/_ref" >&2
  exit 0
fi
M="$REF/superdex_physics/libraries/mochi"
if [ ! -d "$M/mochi_core/include" ]; then
  echo "reference tree not found at $REF; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
# the reference's two floating-point modes: MOCHI_USE_DOUBLE_PRECISION=1 (mochi::real = double, the FP64
# oracle) and =0 (mochi::real = float, the FP32 mode; energies stay double as in the reference)
pids=()
for mode in 1 0; do
  out="$HERE/_ref/libsdx_ref.so"
  [ "$mode" = 0 ] && out="$HERE/_ref/libsdx_ref_f32.so"
  "${REF_CXX:-/usr/bin/g++}" -std=c++20 -O2 -w -fPIC -shared -DMOCHI_USE_DOUBLE_PRECISION=$mode \
    -I"$M/mochi_core/include" -I"$M/third_party/eigen" \
    "$HERE/ref_shim.cpp" "$HERE/ref_serial_scheduler.cpp" "$M/mochi_core/src/materials/batched_smith_neo_hookean.cpp" \
    "$M/mochi_core/src/materials/batched_st_venant_kirchhoff.cpp" \
    "$M/mochi_core/src/materials/batched_linear_elastic.cpp" \
    "$M/mochi_core/src/materials/batched_arap.cpp" \
    -o "$out" &
  pids+=($!)
done
for p in "${pids[@]}"; do wait "$p"; done
echo "built $HERE/_ref/libsdx_ref.so and $HERE/_ref/libsdx_ref_f32.so"
