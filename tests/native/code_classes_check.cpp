// Exhaustive host check of the haplotype code words and prior classes of phmm_types.h (built and run
// by tests/test_code_classes.py): for every haplotype byte and read byte, in both variants,
//   * the FP64 path's compare of the masked code word equals the match-code compare it replaced,
//   * the packed FP32 path's choice (the class table, plus the byte compare applied to class-4
//     columns of inter reads with bytes outside A/C/G/T) equals that compare,
//   * the class field fits the 5-class table, and guard words (0) read class 0 (the cells computed at
//     guard columns lie outside every haplotype and are discarded, so only the table bound matters).
#include <cstdio>

#include "../../rovaca_b200/csrc/phmm_types.h"

using namespace phmm;

int main()
{
    long bad = 0;
    for (int v = 0; v < 2; ++v) {
        const int V = v == 0 ? kInter : kIntra;
        for (int h = 0; h < 256; ++h) {
            const uint32_t w = hap_code((uint8_t)h, V);
            const uint32_t cls = (w & kTabMask) >> kTabShift;
            if (cls >= (uint32_t)kTabClasses) ++bad;
            for (int r = 0; r < 256; ++r) {
                const uint32_t rc = match_code((uint8_t)r, V);
                const bool want = codes_match(match_code((uint8_t)h, V), rc, V);
                const bool fp64 = codes_match(w & kCodeMatchMask, rc, V);
                bool fp32 = class_matches(cls, rc, V);
                const bool exotic_row = V == kInter && base_class((uint8_t)r) == 4u;
                if (exotic_row && cls == 4u) fp32 = (uint32_t)r == (w & kCodeMatchMask);
                if (fp64 != want || fp32 != want) {
                    if (bad < 10) std::printf("variant %d hap %d read %d: want %d fp64 %d fp32 %d\n", V, h, r, want, fp64, fp32);
                    ++bad;
                }
            }
        }
        if (((0u & kTabMask) >> kTabShift) != 0u) ++bad;  // guard words
    }
    std::printf("%ld mismatches\n", bad);
    return bad == 0 ? 0 : 1;
}
