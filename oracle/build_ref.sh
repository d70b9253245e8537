#!/usr/bin/env bash
# Builds the reference's own host (CPU/OpenMP) audio path into oracle/_ref/librpp_audio_ref.so.
#
# Test infrastructure only: the library built here is the oracle and the CPU baseline,
# never the product. Sources are compiled where they lie under RPP_REF (read-only);
# nothing from the reference is copied into this repository.  The prebuilt
# third_party/ffts/lib/libffts.a is linked as-is (never inspected).
#
# Flags follow the reference build: src/modules/CMakeLists.txt:105-124 compiles the
# tensor kernels with -mno-fma, which is what makes the outputs bit-exact to the
# shipped goldens under utilities/test_suite/REFERENCE_OUTPUTS_AUDIO/.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# default: the reference checkout beside this repository (../reference)
RPP_REF="${RPP_REF:-$(cd "$(dirname "$0")/../.." && pwd)/reference}"
OUT="$HERE/_ref"
GEN="$OUT/gen"
if [ ! -d "$RPP_REF/src/modules/tensor/cpu/kernel" ]; then
  echo "build_ref.sh: reference sources not found under $RPP_REF" >&2
  exit 2
fi
mkdir -p "$GEN/half"
# generated config headers (the reference's *.h.in, resolved: audio on, HIP/OpenCL/legacy off)
printf '#pragma once\n#define RPP_BACKEND_HIP 0\n#define RPP_BACKEND_OPENCL 0\n' > "$GEN/rpp_backend.h"
printf '#pragma once\n#define RPP_AUDIO_AUGMENTATIONS_SUPPORT 1\n' > "$GEN/rpp_audio_augmentations_support.h"
printf '#pragma once\n#define RPP_LEGACY_SUPPORT 0\n' > "$GEN/rpp_legacy_support.h"
# api/rppdefs.h includes half.hpp unconditionally; the audio path never uses Rpp16f,
# so a minimal stand-in type is enough for it to compile.
cat > "$GEN/half/half.hpp" <<'H'
#pragma once
#include <cstdint>
namespace half_float { struct half { std::uint16_t bits; half() : bits(0) {} explicit half(float) : bits(0) {} half& operator=(float) { bits = 0; return *this; } operator float() const { return 0.f; } }; }
H
INC=(-I"$GEN" -I"$RPP_REF/api" -I"$RPP_REF/src/include/common" -I"$RPP_REF/src/include/common/cpu"
     -I"$RPP_REF/src/include/tensor" -I"$RPP_REF/third_party/ffts/include")
COMMON=(-O3 -DNDEBUG -DAUDIO_SUPPORT -fopenmp -mavx2 -mf16c -std=gnu++17 -fPIC -w)
KERNELS=(non_silent_region_detection to_decibels pre_emphasis_filter down_mixing spectrogram mel_filter_bank resample slice normalize)
OBJS=()
CXX="${CXX:-g++}"
# some gcc installs on PATH lack libgomp.spec; point -B at a gcc lib dir that has it
GCCLIB=""
for d in "$(dirname "$("$CXX" -print-libgcc-file-name)")" /usr/lib/gcc/x86_64-linux-gnu/*; do
  if [ -f "$d/libgomp.spec" ]; then GCCLIB="$d"; break; fi
done
[ -n "$GCCLIB" ] || { echo "build_ref.sh: libgomp.spec not found" >&2; exit 2; }
COMMON+=(-B"$GCCLIB/")
for k in "${KERNELS[@]}"; do
  "$CXX" "${COMMON[@]}" -mno-fma "${INC[@]}" -c "$RPP_REF/src/modules/tensor/cpu/kernel/$k.cpp" -o "$OUT/$k.o" &
  OBJS+=("$OUT/$k.o")
done
"$CXX" "${COMMON[@]}" -mno-fma "${INC[@]}" -c "$RPP_REF/src/modules/tensor/rppt_tensor_audio_augmentations.cpp" -o "$OUT/dispatch.o" &
"$CXX" "${COMMON[@]}" "${INC[@]}" -c "$RPP_REF/src/modules/handle_host.cpp" -o "$OUT/handle_host.o" &
"$CXX" "${COMMON[@]}" "${INC[@]}" -c "$RPP_REF/src/modules/handle_api.cpp" -o "$OUT/handle_api.o" &
"$CXX" "${COMMON[@]}" "${INC[@]}" -c "$HERE/ref_shim.cpp" -o "$OUT/ref_shim.o" &
wait
OBJS+=("$OUT/dispatch.o" "$OUT/handle_host.o" "$OUT/handle_api.o" "$OUT/ref_shim.o")
"$CXX" -shared -fopenmp -B"$GCCLIB/" -o "$OUT/librpp_audio_ref.so" "${OBJS[@]}" "$RPP_REF/third_party/ffts/lib/libffts.a"
rm -f "${OBJS[@]}"
echo "built $OUT/librpp_audio_ref.so"
