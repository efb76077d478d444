// Rovaca-side binding of the B200 PairHMM engine (see pairhmm_engine_b200.h).
#include "pairhmm_engine_b200.h"

#include <cmath>
#include <mutex>

#include "../common/utils/rovaca_memory_pool.h"
#include "../genotype/haplotype.h"
#include "../genotype/read_record.h"
#include "rovaca_logger.h"

namespace rovaca
{

// the process-wide function pointer of pairhmm_engine.h:14 (defined in pairhmm_engine.cpp)
extern DoubleVector2D (*call_pairhmm)(const HaplotypeVector& hs, ReadVector& rs, int32_t min_quality_threshold,
                                      PcrIndelModel pcr_option, pMemoryPool pool);

namespace
{
std::mutex g_mu;
phmm_engine* g_engine = nullptr;

DoubleVector2D nan_matrix(size_t n_haps, size_t n_reads, pMemoryPool pool)
{
    return DoubleVector2D(n_haps, DoubleVector(n_reads, NAN, pool), pool);
}
}  // namespace

bool init_pairhmm_b200(int32_t device)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_engine) {
        phmm_config cfg{};
        cfg.device = device;
        cfg.use_cuda_graph = 1;
        cfg.autotune = 1;
        if (phmm_engine_create(&cfg, &g_engine) != PHMM_OK) {
            RovacaLogger::error("B200 PairHMM engine unavailable: {}", phmm_last_error());
            g_engine = nullptr;
            return false;
        }
    }
    call_pairhmm = call_pairhmm_b200;
    return true;
}

void shutdown_pairhmm_b200()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_engine) phmm_engine_destroy(g_engine);
    g_engine = nullptr;
}

phmm_engine* pairhmm_b200_engine()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_engine;
}

PairHmmRegionRequest::~PairHmmRegionRequest()
{
    // a request still in flight writes into this object's buffers: wait for it
    if (_in_flight) phmm_wait(_engine, _ticket, -1, nullptr, nullptr);
}

bool PairHmmRegionRequest::submit(phmm_engine* engine, const HaplotypeVector& hs, const ReadVector& rs,
                                  int32_t min_quality_threshold, PcrIndelModel pcr_option)
{
    _engine = engine;
    _n_haps = (uint32_t)hs.size();
    _n_reads = (uint32_t)rs.size();
    _hap_bases.clear();
    _read_bases.clear();
    _read_qual.clear();
    _hap_off.assign(1, 0);
    _read_off.assign(1, 0);
    _mapq.assign(_n_reads, 0);
    for (pHaplotype h : hs) {
        const pBases b = h ? h->get_bases() : nullptr;
        if (b) _hap_bases.insert(_hap_bases.end(), b->data, b->data + b->num);
        _hap_off.push_back(_hap_bases.size());
    }
    for (uint32_t r = 0; r < _n_reads; ++r) {
        const pReadRecord rd = rs[r];
        const int32_t n = rd ? rd->seq_length() : 0;
        for (int32_t i = 0; i < n; ++i) _read_bases.push_back(rd->seq_i((uint32_t)i));  // ASCII, as decode_to_str
        if (n > 0) _read_qual.insert(_read_qual.end(), rd->qual(), rd->qual() + n);
        _mapq[r] = rd ? rd->mapping_quality() : 0;
        _read_off.push_back(_read_bases.size());
    }
    _lk.assign((size_t)_n_haps * _n_reads, NAN);
    _keep.assign(_n_reads, 1);
    _n_kept = _n_reads;
    phmm_region_input in{};
    in.n_haps = _n_haps;
    in.hap_bases = _hap_bases.data();
    in.hap_off = _hap_off.data();
    in.n_reads = _n_reads;
    in.read_bases = _read_bases.data();
    in.read_qual = _read_qual.data();
    in.read_off = _read_off.data();
    in.mapq = _mapq.data();
    in.min_quality_threshold = min_quality_threshold;
    in.pcr_model = (int32_t)pcr_option;
    _status = engine ? phmm_submit_region(engine, &in, nullptr, _lk.data(), _keep.data(), &_n_kept, &_ticket)
                     : PHMM_ERR_NOT_INITIALIZED;
    _in_flight = _status == PHMM_OK;
    return _in_flight;
}

DoubleVector2D PairHmmRegionRequest::collect(ReadVector& rs, pMemoryPool pool)
{
    DoubleVector2D result = nan_matrix(_n_haps, _n_reads, pool);
    if (_in_flight) {
        _status = phmm_wait(_engine, _ticket, -1, nullptr, nullptr);
        _in_flight = false;
    }
    if (_status != PHMM_OK) {
        // the reference's failure result: every likelihood NaN, every read kept
        RovacaLogger::error("B200 PairHMM: {} ({})", phmm_status_string(_status), phmm_last_error());
        return result;
    }
    for (uint32_t h = 0; h < _n_haps; ++h)
        std::copy(_lk.begin() + (size_t)h * _n_reads, _lk.begin() + (size_t)(h + 1) * _n_reads, result[h].begin());
    // erase the dropped reads in order (pairhmm_internal.cpp:614-619)
    for (int64_t r = (int64_t)_n_reads - 1; r >= 0; --r)
        if (!_keep[(size_t)r]) rs.erase(rs.begin() + r);
    return result;
}

DoubleVector2D call_pairhmm_b200(const HaplotypeVector& hs, ReadVector& rs, int32_t min_quality_threshold,
                                 PcrIndelModel pcr_option, pMemoryPool pool)
{
    // the reference insists on its own pool type and returns NaNs otherwise (pairhmm_internal.cpp:581-586)
    if (!dynamic_cast<RovacaMemoryPool*>(pool)) {
        RovacaLogger::error("pool is not RovacaMemoryPool");
        return nan_matrix(hs.size(), rs.size(), pool);
    }
    PairHmmRegionRequest req;
    req.submit(pairhmm_b200_engine(), hs, rs, min_quality_threshold, pcr_option);
    return req.collect(rs, pool);
}

}  // namespace rovaca
