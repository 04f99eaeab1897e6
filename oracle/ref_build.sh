#!/usr/bin/env bash
# Builds the reference's own kernels and host routines into oracle/_ref/
# (test infrastructure; outputs never leave oracle/_ref/, which is git-ignored).
#
# Source: old-fun.cu of the reference (same kernels as fun.cu, src/constants.hpp
# material set).  The single-file program is compiled as it lies; a patched copy
# is written under oracle/_ref/src/ with four macro edits the reference's own
# run scripts make by hand (run.sh:75-90, src.sed):
#   ifTFC 1 -> 0            frozen temperature (the synthetic workloads' T model)
#   dx 0.6  -> REF_DX       grid spacing of the workload (0.8 W)
#   i_tip_target (Nx-268) -> REF_ITIP   (Nx-268 is negative on small grids)
#   cinf 0.632514105 -> REF_CINF  nominal melt composition of the workload
#                           (the pull_back fill value, fun.cu:1484)
#   main -> ref_main        so that oracle/ref_harness.cu supplies main()
# and two edits to host-only code off the step path that does not compile as
# shipped (old-fun.cu:2002 uses `step`/`h_para` out of scope in save_parameters;
# old-fun.cu:2205 assigns to a constexpr in AutoBlockSize):
#   drop the "current pulling velocity" fprintf; constexpr int best_metric -> int
# A second copy keeps ifTFC 1 (the reference's production coarse-grid
# temperature) with the other edits, for the TFC harnesses, and writes
# latentHeat and cp as the production sources do (fun.cu:89-97,
# src/constants.hpp:64-71: 22003.0 and 40.0): old-fun.cu writes them as the
# integers (22003) and (40), so its Lcp = latentHeat/cp is the integer
# quotient 550 instead of 550.075.
# Everything else comes in through -D exactly as run.sh passes it.
#
# Usage: ref_build.sh <reference root>   (or REF_ROOT=<reference root>)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${REF_ROOT:-}}"
OUT="$HERE/_ref"
if [ -z "$REF" ]; then
  echo "ref_build: give the reference root as the argument or in REF_ROOT" >&2
  exit 2
fi
if [ ! -f "$REF/old-fun.cu" ]; then
  echo "ref_build: $REF/old-fun.cu not present; keeping prebuilt $OUT" >&2
  exit 0
fi
mkdir -p "$OUT/src"
patch_ref() { # out tfc(0|1)
  local out=$1 tfc=$2
  local tfc_edit='s/^#define[[:space:]]*ifTFC[[:space:]]*1/#define ifTFC 0/'
  [ "$tfc" = 1 ] && tfc_edit='s/^#define[[:space:]]*ifTFC[[:space:]]*1/#define ifTFC 1/'
  local lcp_edit='s/^$//'
  [ "$tfc" = 1 ] && lcp_edit='s/^#define[[:space:]]*latentHeat[[:space:]]*(22003)/#define    latentHeat (22003.0)/; s/^#define[[:space:]]*cp[[:space:]]*(40)/#define    cp (40.0)/'
  sed -e "$tfc_edit" -e "$lcp_edit" \
      -e 's/^\([[:space:]]*\)#define dx 0\.[0-9]*/\1#define dx REF_DX/' \
      -e 's/^#define[[:space:]]*i_tip_target[[:space:]]*(Nx-268)/#define i_tip_target REF_ITIP/' \
      -e 's/^#define[[:space:]]*cinf[[:space:]]*(0\.632514105)/#define cinf REF_CINF/' \
      -e '/current pulling velocity.*Vp_ramp(step/d' \
      -e 's/constexpr int best_metric/int best_metric/' \
      "$REF/old-fun.cu" > "$out"
  grep -q "^#define ifTFC $tfc" "$out"
  grep -q '#define dx REF_DX' "$out"
  grep -q '^#define i_tip_target REF_ITIP' "$out"
  grep -q '^#define cinf REF_CINF' "$out"
  if [ "$tfc" = 1 ]; then
    grep -q '^#define    latentHeat (22003.0)' "$out"
    grep -q '^#define    cp (40.0)' "$out"
  fi
}
PATCHED="$OUT/src/old-fun.fta.cu"
PATCHED_TFC="$OUT/src/old-fun.tfc.cu"
patch_ref "$PATCHED" 0
patch_ref "$PATCHED_TFC" 1

NVCC="${NVCC:-nvcc}"
COMMON=(-std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -ccbin g++
        -Xcompiler -ffp-contract=off -w
        -DREF_DX=0.8 -DREF_CINF=0.90
        -Dtotal_time=1000 -Dif_load=0 '-Dpath_input="./"' -Drun_time=1 -Drandom_seed=0
        -DVp=0.05 -DGG=0.001 -Deps1=0.06 -Deps2=0 -Depk1=0.15 -Dmain=ref_main)

build() { # name nx ny itip extra...   (SRC_COPY: the patched copy, default the FTA one)
  local name=$1 nx=$2 ny=$3 itip=$4; shift 4
  "$NVCC" "${COMMON[@]}" -DREF_PATCHED="\"${SRC_COPY:-$PATCHED}\"" -DNx_all="$nx" -DNy_all="$ny" \
      -DREF_ITIP="$itip" "$@" "$HERE/ref_harness.cu" -o "$OUT/$name"
}
build ref_harness_64 64 64 24
build ref_harness_64_nofma 64 64 24 -fmad=false
build ref_harness_256 256 256 16
build ref_harness_256_nofma 256 256 16 -fmad=false
build ref_harness_2048 2048 2048 16 -UGG -DGG=0.005 -UVp -DVp=0.5
# coarse-grid temperature (TFC): G = 1e7 K/m, V = 0.5 m/s, the reference's own
# TCOLD and 50 um coarse domain; Ny_all - 2 is a multiple of ratio_dxT_dx = 10
# and Ny_all of BLOCK_SIZE_Y = 4, as the reference's TFC grids must be
for tfc_grid in "64 72" "256 252"; do
  set -- $tfc_grid
  SRC_COPY="$PATCHED_TFC" build "ref_harness_tfc_$1x$2" "$1" "$2" 20 -UGG -DGG=0.01 -UVp -DVp=0.5
  SRC_COPY="$PATCHED_TFC" build "ref_harness_tfc_$1x$2_nofma" "$1" "$2" 20 -UGG -DGG=0.01 -UVp -DVp=0.5 -fmad=false
done
# fun.cu as shipped (its own -D list, run.sh:75-90) for the parameter-file
# layout: save_parameters / load_parameters only, host code.
"$NVCC" -std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a -ccbin g++ -w \
    -DREF_SOURCE="\"$REF/fun.cu\"" -Dmain=ref_main \
    -Dtotal_time=120000 -Dif_load=0 '-Dpath_input="./"' -Drun_time=4 -Drandom_seed=3 \
    -DVp=0.6 -DGG=0.002 -Deps1=0.02 -Deps2=0.001 -Depk1=0.1 -DNx_all=768 -DNy_all=832 -DMAX_GPU=1 \
    "$HERE/ref_params_harness.cu" -o "$OUT/ref_params_harness"
# The 3D three-phase model, multi/peritectic_multiGPU/TiAg.cu: a copy with its
# grid macros set to the harness size (the reference edits Nx, Ny, Nz, devNz
# by hand per run), main renamed; oracle/ref3_harness.cu drives the kernels.
TIAG="$REF/multi/peritectic_multiGPU/TiAg.cu"
if [ -f "$TIAG" ]; then
  build3() { # name nx ny devnz
    local name=$1 nx=$2 ny=$3 dnz=$4
    local src="$OUT/src/TiAg.$nx.$ny.$dnz.cu"
    sed -e "s/^#define[[:space:]]*Nx[[:space:]]*512/#define Nx $nx/" \
        -e "s/^#define[[:space:]]*Ny[[:space:]]*512/#define Ny $ny/" \
        -e "s/^#define[[:space:]]*Nz[[:space:]]*506.*/#define Nz (($dnz - 2) * Ngpu + 2)/" \
        -e "s/^#define[[:space:]]*devNz[[:space:]]*128.*/#define devNz $dnz/" "$TIAG" > "$src"
    grep -q "^#define Nx $nx" "$src"
    grep -q "^#define devNz $dnz" "$src"
    "$NVCC" -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -ccbin g++ -w \
        -DREF3_SOURCE="\"$src\"" -Dmain=ref3_main "$HERE/ref3_harness.cu" -o "$OUT/$name"
  }
  build3 ref3_harness_32 32 32 20
  build3 ref3_harness_512 512 512 128
fi
echo "ref_build: built $(ls "$OUT" | grep -c harness) harness binaries in $OUT"
