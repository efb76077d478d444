#!/usr/bin/env bash
# Test-infrastructure recipe: compiles the reference's own Smith-Waterman aligner from the reference
# source tree (read in place, never copied) together with oracle/ref_sw_shim.c into
# oracle/_ref/libsw_ref.so.
#
# Sources and flags follow src/haplotypecaller/common/base/CMakeLists.txt:1-28: sw_avx.c, sw_avx2.c,
# sw_cigar.c and ro_sw.c with -mavx -mavx2 -fgnu89-inline; avx2_sw_core.c with the same; and
# avx512_sw_core.c with -mavx512f -mavx512dq -mavx512bw -mavx512vl added.  htslib's headers (the
# vendored include tree) provide the CIGAR macros.
#
# Usage: oracle/build_ref_sw.sh REFERENCE_ROOT   (or the REFERENCE_ROOT environment variable)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${REFERENCE_ROOT:?pass the reference source root or set REFERENCE_ROOT}}"
B="$REF/src/haplotypecaller/common/base"
OUT="$HERE/_ref"
if [ ! -d "$B/lib/ro_sw" ]; then
    echo "build_ref_sw: reference Smith-Waterman sources not found at $B" >&2
    exit 1
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
INC=(-I"$B/include" -I"$B/lib/ro_sw" -I"$B/lib/sw_avx" -I"$REF/third_lib/htslib/include")
BASE=(-O3 -g -fPIC -w -mavx -mavx2 -fgnu89-inline)
AVX512=(-mavx512f -mavx512dq -mavx512bw -mavx512vl)
cc() {  # cc OUT SRC FLAGS...
    local o="$1" s="$2"; shift 2
    gcc "${BASE[@]}" "$@" "${INC[@]}" -c "$s" -o "$TMP/$o" &
}
cc sw_avx.o "$B/lib/sw_avx/sw_avx.c"
cc sw_avx2.o "$B/lib/sw_avx/sw_avx2.c"
cc sw_cigar.o "$B/lib/ro_sw/sw_cigar.c"
cc ro_sw.o "$B/lib/ro_sw/ro_sw.c"
cc avx2_sw_core.o "$B/lib/ro_sw/avx2_sw_core.c"
cc avx512_sw_core.o "$B/lib/ro_sw/avx512_sw_core.c" "${AVX512[@]}"
cc ref_sw_shim.o "$HERE/ref_sw_shim.c"
wait
gcc -shared -o "$OUT/libsw_ref.so" "$TMP"/*.o -Wl,--no-undefined -lm
echo "build_ref_sw: wrote $OUT/libsw_ref.so"
