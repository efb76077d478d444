#!/usr/bin/env bash
# Test-infrastructure recipe: compiles the Rovaca-side binding (integration/pairhmm_engine_b200.cpp)
# with the test driver tests/native/integration_check.cpp against the reference's own headers and
# its RovacaMemoryPool (read in place from the reference tree, never copied), linked to
# rovaca_b200/libphmm_b200.so, into integration/_build/integration_check.  Boost is absent:
# oracle/ref_stubs supplies the headers forward.h names without using.
#
# Usage: integration/build_check.sh REFERENCE_ROOT   (or the REFERENCE_ROOT environment variable)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT="$(dirname "$HERE")"
REF="${1:-${REFERENCE_ROOT:?pass the reference source root or set REFERENCE_ROOT}}"
HC="$REF/src/haplotypecaller"
if [ ! -f "$HC/pairhmm/pairhmm_engine.h" ]; then
    echo "build_check: reference sources not found under $HC" >&2
    exit 1
fi
OUT="$HERE/_build"
mkdir -p "$OUT"
g++ -std=c++17 -O2 -g -w \
    -I"$ROOT/include" -I"$ROOT/oracle/ref_stubs" -I"$HC/pairhmm" -I"$HC/genotype" -I"$HC/common/utils" \
    -I"$REF/src/rovaca_logger" -I"$REF/third_lib/htslib/include" -I"$REF/third_lib/spdlog/include" \
    "$HERE/pairhmm_engine_b200.cpp" "$ROOT/tests/native/integration_check.cpp" "$HC/common/utils/rovaca_memory_pool.cpp" \
    -L"$ROOT/rovaca_b200" -lphmm_b200 -Wl,-rpath,'$ORIGIN/../../rovaca_b200' -o "$OUT/integration_check"
echo "build_check: wrote $OUT/integration_check"
