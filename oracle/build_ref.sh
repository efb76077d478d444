#!/usr/bin/env bash
# Test-infrastructure recipe: compiles the reference's own PairHMM kernels and vector-API scheduler
# from the reference source tree (read in place, never copied) together with oracle/ref_kernels.cpp
# and oracle/ref_shim.cpp into oracle/_ref/libphmm_ref.so.
#
# Layout mirrors src/haplotypecaller/pairhmm/CMakeLists.txt:5-47: the intra and inter kernels are
# compiled twice, once with the AVX2 flags (-mavx -mavx2 -D__AVX2__) and once with the AVX-512 flags
# (-mavx -mavx2 -mavx512f -mavx512dq -mavx512vl -D__AVX512F__), and the scheduler with -mavx -mavx2,
# all with the release flags of the top CMakeLists.txt:32-33 (-O3 -g -fPIC).  The scheduler picks the
# ISA at run time with the reference's CPUID check.  Boost is absent here: oracle/ref_stubs supplies
# the two headers the sources name without using.  The region-API overload of the scheduler
# references ReadRecord methods implemented against libhts (absent); oracle/ref_unreached.cpp binds
# them to aborting stubs, since the vector API used here never reaches them.
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or the REFERENCE_ROOT environment variable)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${REFERENCE_ROOT:?pass the reference source root or set REFERENCE_ROOT}}"
P="$REF/src/haplotypecaller/pairhmm"
OUT="$HERE/_ref"
if [ ! -d "$P" ]; then
    echo "build_ref: reference PairHMM sources not found at $P" >&2
    exit 1
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
INC=(-I"$HERE/ref_stubs" -I"$P" -I"$P/roDV_common" -I"$REF/src/rovaca_logger"
     -I"$REF/third_lib/htslib/include" -I"$REF/third_lib/spdlog/include")
BASE=(-O3 -g -fPIC -std=c++17 -w)
AVX2=(-mavx -mavx2 -D__AVX2__)
AVX512=(-mavx -mavx2 -mavx512f -mavx512dq -mavx512vl -D__AVX512F__)

cc() {  # cc OUT SRC FLAGS...
    local o="$1" s="$2"; shift 2
    g++ "${BASE[@]}" "$@" "${INC[@]}" -c "$s" -o "$TMP/$o" &
}
for isa in avx2 avx512; do
    if [ "$isa" = avx2 ]; then F=("${AVX2[@]}"); else F=("${AVX512[@]}"); fi
    cc "intra_impl_$isa.o" "$P/roDV_intra/pairhmm_impl.cpp" "${F[@]}"
    cc "intra_api_$isa.o" "$P/roDV_intra/pairhmm_api.cpp" "${F[@]}"
    cc "inter_$isa.o" "$P/roDV_inter/pairhmm_inter.cpp" "${F[@]}"
    cc "inter_api_$isa.o" "$P/roDV_inter/pairhmm_inter_api.cpp" "${F[@]}"
    cc "ref_kernels_$isa.o" "$HERE/ref_kernels.cpp" "${F[@]}"
done
cc schedule.o "$P/roDV_schedule.cpp" -mavx -mavx2
cc internal.o "$P/pairhmm_internal.cpp" -mavx -mavx2
cc memory_pool.o "$REF/src/haplotypecaller/common/utils/rovaca_memory_pool.cpp"
cc ref_shim.o "$HERE/ref_shim.cpp" -mavx -mavx2
cc ref_region.o "$HERE/ref_region.cpp" -mavx -mavx2
cc ref_unreached.o "$HERE/ref_unreached.cpp" -mavx -mavx2
wait
g++ -shared -o "$OUT/libphmm_ref.so" "$TMP"/*.o -Wl,--no-undefined -lm
echo "build_ref: wrote $OUT/libphmm_ref.so"
