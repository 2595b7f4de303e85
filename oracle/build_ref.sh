#!/usr/bin/env bash
# Builds the oracle (test infrastructure only):
#   oracle/_ref/liboracle.so               CPU restatement of the transient solve + CPU Cholesky
#   oracle/_ref/CalcNonstat3DLine_{A2,A3,E2,E3}
#                                          the reference's own 3D transient solver, compiled
#                                          unmodified from its sources with the shim headers in
#                                          oracle/shim and the pardiso_64 stand-in
#   oracle/_ref/CalcNonstat3DLine_{A2,A3,E2,E3}_gpu
#                                          the same objects linked against the product
#                                          library's pardiso_64 (the in-process boundary)
#   oracle/_ref/CalcStat3D_3T_A            the reference's stationary A0 / V solver, same way
#   oracle/_ref/SumNonstat3DOnly           the reference's per-component split of the 3D results
#   oracle/_ref/SummatorEDMN               the reference's line-voltage integration (main.cpp
#                                          only: utils.cpp needs headers absent from the tree)
#   oracle/_ref/TimeDirectSolver           the reference's time-grid regularisation
#   oracle/_ref/CorrectTimeMesh            the reference's short-decade correction
#
# The reference sources are read in place: TDEM_REFERENCE_ROOT, else a checkout
# named "reference" beside the repository (../reference from the repository
# root); nothing is copied into the repository.  When the reference
# tree is absent (for example on a machine that only runs the prebuilt files) the
# reference binaries are skipped and only liboracle.so is built.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
REF="${TDEM_REFERENCE_ROOT:-$HERE/../../reference}"
MOD="$REF/CODE/programs to folder Modules"
JOBS="${JOBS:-$(nproc)}"
CXX="${TDEM_CXX:-g++}"
mkdir -p "$OUT"

OPT="-O2 -g0"
CXXFLAGS_OR="-std=c++17 $OPT -fPIC -pthread -Wall -Wno-unused-function"

# --- oracle library (own code only) -------------------------------------------
build_oracle() {
  local objs=()
  for f in cpu_cholesky pardiso_shim tdem_oracle; do
    if [ -f "$HERE/$f.cpp" ]; then
      if [ ! -f "$OUT/$f.o" ] || [ "$HERE/$f.cpp" -nt "$OUT/$f.o" ] || [ "$HERE/cpu_cholesky.h" -nt "$OUT/$f.o" ]; then
        $CXX $CXXFLAGS_OR -c "$HERE/$f.cpp" -o "$OUT/$f.o"
      fi
      objs+=("$OUT/$f.o")
    fi
  done
  $CXX -shared -pthread -o "$OUT/liboracle.so" "${objs[@]}" -ldl
}
build_oracle

if [ ! -d "$MOD" ]; then
  echo "reference tree not found at $REF: skipping the reference binaries"
  exit 0
fi

# objects are rebuilt when a shim header changes too
SHIM_NEWEST="$(ls -t "$HERE"/shim/*.h | head -1)"

# flags that let the MSVC sources compile with g++ (no source edits)
REFFLAGS="-std=c++17 $OPT -fpermissive -w -D__forceinline=inline -include cmath -include cfloat \
 -include cstring -include ctime -include algorithm -include iterator -include $HERE/shim/llp64_stdio.h \
 -I$HERE/shim"

build_variant() {  # name, source dir, extra compiler flags
  local name="$1" src="$2" extra="${3:-}"
  local obj="$OUT/obj_$name" inc="$OUT/inc_$name"
  mkdir -p "$obj" "$inc"
  # case aliases: the sources include headers with a different capitalisation
  # (forwarding headers, so the real header's own includes resolve next to it)
  rm -f "$inc/Vec_Prep_Data.h" "$inc/Give_out_vec_loop.h"
  [ -f "$src/vec_prep_data.h" ] && printf '#include "%s/vec_prep_data.h"\n' "$src" > "$inc/Vec_Prep_Data.h"
  [ -f "$src/give_out_vec_loop.h" ] && printf '#include "%s/give_out_vec_loop.h"\n' "$src" > "$inc/Give_out_vec_loop.h"
  local objs=()
  local pids=()
  while IFS= read -r -d '' f; do
    local b
    b="$(basename "$f" .cpp)"
    objs+=("$obj/$b.o")
    if [ ! -f "$obj/$b.o" ] || [ "$f" -nt "$obj/$b.o" ] || [ "$SHIM_NEWEST" -nt "$obj/$b.o" ]; then
      $CXX $REFFLAGS $extra -I"$inc" -c "$f" -o "$obj/$b.o" &
      pids+=($!)
      if [ "${#pids[@]}" -ge "$JOBS" ]; then wait "${pids[0]}"; pids=("${pids[@]:1}"); fi
    fi
  done < <(find "$src" -maxdepth 1 -name '*.cpp' -print0 | sort -z)
  for p in "${pids[@]}"; do wait "$p"; done
  $CXX -pthread -o "$OUT/$name" "${objs[@]}" "$OUT/pardiso_shim.o" "$OUT/cpu_cholesky.o" -ldl
  echo "built $OUT/$name"
}

build_variant CalcNonstat3DLine_A2 "$MOD/!programs for 2-point implicit scheme/!programs for A-formulation/CalcNonstat3DLine"
build_variant CalcNonstat3DLine_A3 "$MOD/!programs for 3-point implicit scheme/!programs for A-formulation/CalcNonstat3DLine"
build_variant CalcNonstat3DLine_E2 "$MOD/!programs for 2-point implicit scheme/!programs for E-formulation/CalcNonstat3DLine"
build_variant CalcNonstat3DLine_E3 "$MOD/!programs for 3-point implicit scheme/!programs for E-formulation/CalcNonstat3DLine"
build_variant CalcStat3D_3T_A "$MOD/CalcStat3D_3T_A" "-Dsprintf_s=sprintf"

# The same unmodified reference objects linked against the product library's
# pardiso_64 instead of the CPU stand-in: the in-process solver boundary as a
# maintainer would wire it (oracle/_ref/CalcNonstat3DLine_<V>_gpu, run by the GPU
# tests).  Built when the package library exists (build it first).
PKGLIB="$HERE/../a-e_formulations_3d_timedomain_em_horizontalgroundedwiresource_b200/lib"
if [ -f "$PKGLIB/libtdem_b200.so" ]; then
  for v in A2 A3 E2 E3; do
    $CXX -pthread -o "$OUT/CalcNonstat3DLine_${v}_gpu" "$OUT/obj_CalcNonstat3DLine_$v"/*.o \
      -L"$PKGLIB" -ltdem_b200 -Wl,-rpath,'$ORIGIN/../../a-e_formulations_3d_timedomain_em_horizontalgroundedwiresource_b200/lib'
    echo "built $OUT/CalcNonstat3DLine_${v}_gpu (pardiso_64 from libtdem_b200.so)"
  done
fi

build_plain() {  # name, sources...
  local name="$1"
  shift
  $CXX $REFFLAGS "$@" -o "$OUT/$name"
  echo "built $OUT/$name"
}
build_plain SumNonstat3DOnly "$MOD/SumNonstat3DOnly/main.cpp" "$MOD/SumNonstat3DOnly/openclose.cpp" \
  "$MOD/SumNonstat3DOnly/picket.cpp" "$MOD/SumNonstat3DOnly/utils.cpp" "$MOD/SumNonstat3DOnly/utils_direct_solver.cpp"
build_plain SummatorEDMN "$MOD/SummatorEDMN/main.cpp"
build_plain TimeDirectSolver "$MOD/TimeDirectSolver/main.cpp" "$MOD/TimeDirectSolver/TimeStep.cpp"
build_plain CorrectTimeMesh "$MOD/CorrectTimeMesh/main.cpp"
