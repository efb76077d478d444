// Test-infrastructure only.  The reference scheduler's region-API overload
// (src/haplotypecaller/pairhmm/roDV_schedule.cpp:364-834) calls ReadRecord / Allele accessors and
// the PCR model, whose implementations need libhts, which this image lacks.  The vector API that
// oracle/_ref exposes never reaches them, so they are defined here as hard failures: the library
// then loads with every symbol bound, and any unexpected call aborts instead of running garbage.
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
void apply_pcr_error_model_rolling(pBases, pBases, PcrIndelModel) { unreached("apply_pcr_error_model_rolling"); }
}  // namespace rovaca
