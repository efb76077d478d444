// Host-side read preparation and post-processing of the region API (phmm_region.cpp).
#pragma once

#include <cstdint>

namespace phmm {

int tandem_repeat_length(const uint8_t* s, int n, int o);
void apply_pcr_model(const uint8_t* bases, int n, uint8_t* gap_open, int model);
void prepare_read_quals(const uint8_t* q, int n, uint8_t mapq, int32_t min_quality_threshold, uint8_t* out);
void normalize_and_filter(const double* lk_hr, uint32_t n_haps, uint32_t n_reads, const uint64_t* read_len,
                          double* out_hr, uint8_t* keep, uint32_t* n_kept);

}  // namespace phmm
