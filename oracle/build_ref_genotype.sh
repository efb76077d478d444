#!/usr/bin/env bash
# Test-infrastructure recipe: compiles the reference's own genotyping arithmetic -- haplotype-to-
# allele marginalisation (allele_likelihoods.hpp) and the diploid GenotypeLikelihoodCalculator with
# the genotype tables it uses -- from the reference source tree (read in place, never copied)
# together with oracle/ref_genotype_shim.cpp into oracle/_ref/libgenotype_ref.so.
#
# Flags as the reference's release build (CMakeLists.txt:32-33: -O3 -g -fPIC, C++17).  Boost is
# absent: oracle/ref_stubs/boost/math supplies binomial_coefficient (restated; the genotype count
# tables use it) and empty or aborting stand-ins for the digamma and erf_inv headers math_utils.h
# includes, whose functions this path does not call.  The logger is the reference's own
# (src/rovaca_logger, spdlog headers vendored in third_lib).
#
# Usage: oracle/build_ref_genotype.sh REFERENCE_ROOT   (or the REFERENCE_ROOT environment variable)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${REFERENCE_ROOT:?pass the reference source root or set REFERENCE_ROOT}}"
HC="$REF/src/haplotypecaller"
G="$HC/genotype"
OUT="$HERE/_ref"
if [ ! -f "$G/genotype_likelihood_calculator.cpp" ]; then
    echo "build_ref_genotype: reference genotype sources not found under $G" >&2
    exit 1
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
INC=(-I"$HERE/ref_stubs" -I"$G" -I"$G/interface" -I"$G/utils" -I"$HC/common" -I"$HC/common/utils" -I"$HC"
     -I"$REF/src/rovaca_logger" -I"$REF/third_lib/htslib/include" -I"$REF/third_lib/spdlog/include")
BASE=(-O3 -g -fPIC -std=c++17 -w)
cc() {  # cc OUT SRC
    g++ "${BASE[@]}" "${INC[@]}" -c "$2" -o "$TMP/$1" &
}
cc calc.o "$G/genotype_likelihood_calculator.cpp"
cc counts.o "$G/genotype_allele_counts.cpp"
cc likelihoods.o "$G/genotype_likelihoods.cpp"
cc math_utils.o "$HC/common/utils/math_utils.cpp"
cc shim.o "$HERE/ref_genotype_shim.cpp"
wait
g++ -shared -o "$OUT/libgenotype_ref.so" "$TMP"/*.o -Wl,--no-undefined -lm
echo "build_ref_genotype: wrote $OUT/libgenotype_ref.so"
