// Test-infrastructure only.  C-ABI over the reference's region-path helpers, compiled with the
// reference's pairhmm_internal.cpp into oracle/_ref/libphmm_ref.so by oracle/build_ref.sh.
//   apply_pcr_error_model_rolling / apply_pcr_error_model   src/haplotypecaller/pairhmm/pairhmm_internal.cpp:391-476
//   find_tandem_repeat_units_rolling / find_tandem_repeat_units                                 :260-389
//   normalize_likelihoods                                                                         :248-258
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory_resource>
#include <new>

#include "../genotype/genotype_struct.h"
#include "pairhmm_internal.h"

namespace {
// Bases is a length-prefixed flexible array (genotype/genotype_struct.h:11-15).
rovaca::pBases make_bases(const uint8_t* data, uint32_t n)
{
    void* mem = std::malloc(sizeof(rovaca::Bases) + n + 1);
    rovaca::pBases b = static_cast<rovaca::pBases>(mem);
    b->num = n;
    if (n) std::memcpy(b->data, data, n);
    b->data[n] = 0;
    return b;
}
}  // namespace

extern "C" {

// model: 0 NONE, 1 HOSTILE, 2 AGGRESSIVE, 3 CONSERVATIVE (common/enum.h:8); rolling != 0 selects the
// rolling-hash implementation the scheduler uses, else the plain one.
void ref_pcr_model(const uint8_t* bases, uint32_t n, uint8_t* gap_open, int model, int rolling)
{
    rovaca::pBases b = make_bases(bases, n);
    rovaca::pBases g = make_bases(gap_open, n);
    if (rolling)
        rovaca::apply_pcr_error_model_rolling(b, g, static_cast<PcrIndelModel>(model));
    else
        rovaca::apply_pcr_error_model(b, g, static_cast<PcrIndelModel>(model));
    std::memcpy(gap_open, g->data, n);
    std::free(b);
    std::free(g);
}

int ref_tandem_repeat(const uint8_t* bases, uint32_t n, uint32_t offset, int rolling)
{
    rovaca::pBases b = make_bases(bases, n);
    const int r = rolling ? rovaca::find_tandem_repeat_units_rolling(b, offset) : rovaca::find_tandem_repeat_units(b, offset);
    std::free(b);
    return r;
}

// lk is [n_reads][n_haps], normalised in place.
void ref_normalize(double* lk, uint32_t n_reads, uint32_t n_haps)
{
    rovaca::DoubleVector2D m(std::pmr::new_delete_resource());
    for (uint32_t r = 0; r < n_reads; ++r) m.emplace_back(lk + (size_t)r * n_haps, lk + (size_t)(r + 1) * n_haps);
    rovaca::normalize_likelihoods(m);
    for (uint32_t r = 0; r < n_reads; ++r) std::memcpy(lk + (size_t)r * n_haps, m[r].data(), n_haps * sizeof(double));
}

}  // extern "C"
