// Rovaca-side binding of the B200 PairHMM engine: the source a maintainer adds next to
// src/haplotypecaller/pairhmm/pairhmm_engine.cpp.  It compiles against Rovaca's own headers
// (genotype/forward.h, genotype/haplotype.h, genotype/read_record.h, common/utils/rovaca_memory_pool.h)
// and links libphmm_b200.so; nothing in the engine library depends on it.
//
//   init_pairhmm_b200(device)   creates the engine once (call where init_pairhmm_ptr runs,
//                               haplotypecaller.cpp:49) and binds rovaca::call_pairhmm to
//                               call_pairhmm_b200 (the pointer of pairhmm_engine.h:14)
//   call_pairhmm_b200(...)      the drop-in for call_roDV_pairhmm_scheduled
//                               (pairhmm_internal.cpp:576-623): same signature, same result layout
//                               ([hap][n_reads], kept reads first, NaN after), same erasure of the
//                               poorly modelled reads from rs, same all-NaN matrix with every read
//                               kept on any failure, including a pool that is not a RovacaMemoryPool
//   PairHmmRegionRequest        the asynchronous form for a region task that keeps working (e.g. on
//                               the assembly of its next region, haplotypecaller_engine.cpp:107-376)
//                               while the GPU computes this region's likelihoods
#ifndef ROVACA_PAIRHMM_ENGINE_B200_H_
#define ROVACA_PAIRHMM_ENGINE_B200_H_

#include <cstdint>
#include <vector>

#include "../common/enum.h"
#include "../genotype/forward.h"
#include "phmm_b200.h"

namespace rovaca
{

// Creates the process's engine on `device` and binds call_pairhmm; false (call_pairhmm unchanged)
// when no usable GPU is present.
bool init_pairhmm_b200(int32_t device);
void shutdown_pairhmm_b200();
phmm_engine* pairhmm_b200_engine();

DoubleVector2D call_pairhmm_b200(const HaplotypeVector& hs, ReadVector& rs, int32_t min_quality_threshold,
                                 PcrIndelModel pcr_option, pMemoryPool pool);

// One region in flight.  submit() copies the region's haplotype bases, read bases, base qualities
// and MAPQ out of Rovaca's objects and hands them to the serving loop (phmm_submit_region); the
// caller is free to do other work until collect(), which waits, builds the [hap][read] matrix in
// the pool and erases the dropped reads from rs exactly as call_pairhmm does.
class PairHmmRegionRequest
{
public:
    PairHmmRegionRequest() = default;
    PairHmmRegionRequest(const PairHmmRegionRequest&) = delete;
    PairHmmRegionRequest& operator=(const PairHmmRegionRequest&) = delete;
    ~PairHmmRegionRequest();

    // false (with the status in status()) when the request could not be submitted.
    bool submit(phmm_engine* engine, const HaplotypeVector& hs, const ReadVector& rs, int32_t min_quality_threshold,
                PcrIndelModel pcr_option);
    DoubleVector2D collect(ReadVector& rs, pMemoryPool pool);
    phmm_status status() const { return _status; }

private:
    phmm_engine* _engine{nullptr};
    phmm_ticket _ticket{0};
    bool _in_flight{false};
    phmm_status _status{PHMM_OK};
    uint32_t _n_haps{0}, _n_reads{0}, _n_kept{0};
    std::vector<uint8_t> _hap_bases, _read_bases, _read_qual, _mapq, _keep;
    std::vector<uint64_t> _hap_off, _read_off;
    std::vector<double> _lk;
};

}  // namespace rovaca

#endif  // ROVACA_PAIRHMM_ENGINE_B200_H_
