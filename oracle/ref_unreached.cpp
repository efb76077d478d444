// Test-infrastructure only.  The reference scheduler's region-API overload
// (src/haplotypecaller/pairhmm/roDV_schedule.cpp:364-834) and pairhmm_internal.cpp call ReadRecord /
// Allele accessors whose implementations need libhts, which this image lacks.  The functions that
// oracle/_ref exposes never reach them, so they are defined here as hard failures: the library then
// loads with every symbol bound, and any unexpected call aborts instead of running garbage.
//
// seq_nt16_int is the one libhts data symbol pairhmm_internal.cpp reads: its rolling hash indexes it
// with ASCII bases (pairhmm_internal.cpp:139).  Every hash hit there is confirmed with memcmp and
// equal strings always hash equal, so repeat counts do not depend on the table's values; a
// 256-entry table keeps those reads in bounds.
#include <cstdio>
#include <cstdlib>

#include "../genotype/allele.h"
#include "../genotype/read_record.h"
#include "pairhmm_internal.h"

namespace {
[[noreturn]] void unreached(const char* what)
{
    std::fprintf(stderr, "oracle/_ref: region-API path reached (%s); only the vector API is built\n", what);
    std::abort();
}
}  // namespace

namespace rovaca {
int32_t ReadRecord::seq_length() const { unreached("ReadRecord::seq_length"); }
void ReadRecord::decode_qual(pBases) const { unreached("ReadRecord::decode_qual"); }
pBases ReadRecord::decode_to_str(pMemoryPool) const { unreached("ReadRecord::decode_to_str"); }
uint8_t ReadRecord::mapping_quality() const { unreached("ReadRecord::mapping_quality"); }
uint8_t* ReadRecord::qual() const { unreached("ReadRecord::qual"); }
uint8_t ReadRecord::seq_i(uint32_t) const { unreached("ReadRecord::seq_i"); }
void ReadRecord::ins_gops(pBases) const { unreached("ReadRecord::ins_gops"); }
void ReadRecord::gap_conts(pBases) const { unreached("ReadRecord::gap_conts"); }
pBases Allele::get_bases() const { unreached("Allele::get_bases"); }
}  // namespace rovaca

// A, C, G, T -> 0..3, everything else 4
extern "C" {
extern const int seq_nt16_int[256];
const int seq_nt16_int[256] = {
    4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
    4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
    4, 0, 4, 1, 4, 4, 4, 2, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 3, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
    4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
    4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
    4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
    4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
    4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
};
}
