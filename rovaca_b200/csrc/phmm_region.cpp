// Region API: the call_pairhmm path of the reference, around the GPU likelihood engine.
//
// Reference (paths inside the reference project):
//   entry / post-processing      src/haplotypecaller/pairhmm/pairhmm_internal.cpp:576-623
//   read preparation             src/haplotypecaller/pairhmm/roDV_schedule.cpp:522-649
//     quality: min(q, MAPQ); below the threshold -> 6 (MIN_QUALITY, adapter.h:4)      :540-565
//     gap-open 45 ('-'), gap continuation 10 ('+' - 33)                                :510-519,575-604
//       (ReadRecord::ins_gops / gap_conts write the same constants, genotype/read_record.cpp:186-205)
//     PCR model caps gap-open, deletion aliases insertion                             :586-592,607-609
//   PCR tandem-repeat model      src/haplotypecaller/pairhmm/pairhmm_internal.cpp:317-379,431-476
//     caps per repeat length     src/haplotypecaller/pairhmm/adapter.h:13-15
//   normalise (cap at best-4.5)  src/haplotypecaller/pairhmm/pairhmm_internal.cpp:248-258
//   poorly modelled reads        src/haplotypecaller/pairhmm/pairhmm_internal.cpp:23-44,489-497
//   transpose to [hap][read]     src/haplotypecaller/pairhmm/pairhmm_internal.cpp:499-508
// phmm_call_region runs the whole path on the GPU through the serving loop (device read preparation
// and post-processing in phmm_regionk.cu), so concurrent callers (the reference's region thread
// pool) are batched together.  The host functions below compute the same steps; they are exported
// for tests and for callers that prepare reads themselves.
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/phmm_b200.h"
#include "phmm_capi_internal.h"
#include "phmm_region.h"

namespace phmm {

phmm_status server_submit(phmm_engine* engine, const phmm_batch& b, double* out, uint8_t* flags, phmm_ticket* ticket,
                          std::string& err);
phmm_status server_wait(phmm_engine* engine, phmm_ticket ticket, int64_t timeout_us, bool release, double* queued_us,
                        double* total_us, std::string& err);
phmm_status server_submit_region(phmm_engine* engine, const phmm_region_input& in, const phmm_region_events* events,
                                 double* out, uint8_t* keep, uint32_t* n_kept, phmm_ticket* ticket, std::string& err,
                                 const phmm_region_realign* realign = nullptr);

namespace {

constexpr int kMinQuality = 6;
constexpr int kMaxRepeatLength = 20;
constexpr int kMaxStrUnitLength = 8;
constexpr uint8_t kDefaultGapOpen = '-';       // 45
constexpr uint8_t kDefaultGapCont = '+' - 33;  // 10
constexpr double kBestAltDifference = -4.5;
constexpr double kErrorRatePerBase = 0.02;
constexpr double kMaxErrorsPerRead = 2.0;
constexpr double kLog10QualityPerBase = -4.0;

const int kPcrCaps[4][21] = {
    {0},
    {40, 40, 39, 38, 37, 36, 34, 32, 28, 23, 17, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10},  // HOSTILE
    {40, 40, 40, 39, 39, 39, 38, 38, 37, 37, 36, 35, 34, 33, 32, 30, 28, 26, 23, 20, 17},  // AGGRESSIVE
    {40, 40, 40, 40, 39, 39, 39, 39, 39, 38, 38, 38, 37, 37, 37, 36, 36, 35, 34, 33, 33},  // CONSERVATIVE
};

// Consecutive copies of s[u, u+ul) tiling s[t, t+tl): from the front when leading, else from the
// back; stops at the first copy that differs (pairhmm_internal.cpp:146-221, whose rolling hash
// confirms every hash hit with a byte compare, so it counts exactly these copies).
int count_repeats(const uint8_t* s, int n, int u, int ul, int t, int tl, bool leading)
{
    if (tl <= 0 || ul <= 0 || ul > tl || u < 0 || t < 0 || u + ul > n || t + tl > n) return 0;
    int k = 0;
    if (leading) {
        for (int start = 0; start + ul <= tl; start += ul) {
            if (std::memcmp(s + t + start, s + u, ul) != 0) break;
            ++k;
        }
    } else {
        for (int start = tl - ul; start >= 0; start -= ul) {
            if (std::memcmp(s + t + start, s + u, ul) != 0) break;
            ++k;
        }
    }
    return k;
}

}  // namespace

// Tandem-repeat length around position o (find_tandem_repeat_units_rolling_impl,
// pairhmm_internal.cpp:317-379).  The backward search there records its unit at offset
// o - str - 1, which never equals the forward unit at o + 1, so for every position the
// PCR model visits (o < n - 1) the result is: the forward unit (shortest str <= 8 repeating at
// least twice from o+1, else the single base at o+1) counted forwards from o+1 plus its copies
// ending at o, capped at 20.
int tandem_repeat_length(const uint8_t* s, int n, int o)
{
    if (n <= 0) return 0;
    int max_bw = 0;
    if (o >= n - 1) {
        // not reached by the PCR model; kept for completeness: backward search alone
        for (int str = 1; str <= kMaxStrUnitLength; ++str) {
            if (o + 1 - str < 0) break;
            max_bw = count_repeats(s, n, o - str + 1, str, 0, o + 1, false);
            if (max_bw > 1) break;
        }
        return max_bw > kMaxRepeatLength ? kMaxRepeatLength : max_bw;
    }
    int fw_str = 1, max_fw = 0;
    for (int str = 1; str <= kMaxStrUnitLength; ++str) {
        if (o + str + 1 > n) break;
        max_fw = count_repeats(s, n, o + 1, str, o + 1, n - o - 1, true);
        if (max_fw > 1) {
            fw_str = str;
            break;
        }
    }
    max_bw = count_repeats(s, n, o + 1, fw_str, 0, o + 1, false);
    const int rl = max_bw + max_fw;
    return rl > kMaxRepeatLength ? kMaxRepeatLength : rl;
}

// apply_pcr_error_model_rolling (pairhmm_internal.cpp:431-476): every base but the last.
void apply_pcr_model(const uint8_t* bases, int n, uint8_t* gap_open, int model)
{
    if (model <= PHMM_PCR_NONE || model > PHMM_PCR_CONSERVATIVE || n <= 0) return;
    for (int i = 1; i < n; ++i) {
        const int rl = tandem_repeat_length(bases, n, i - 1);
        const int cap = kPcrCaps[model][rl];
        if (gap_open[i - 1] >= cap) gap_open[i - 1] = (uint8_t)cap;
    }
}

void prepare_read_quals(const uint8_t* q, int n, uint8_t mapq, int32_t min_quality_threshold, uint8_t* out)
{
    for (int x = 0; x < n; ++x) {
        uint8_t v = q[x] < mapq ? q[x] : mapq;
        out[x] = (int)v < min_quality_threshold ? (uint8_t)kMinQuality : v;
    }
}

void normalize_and_filter(const double* lk_hr, uint32_t n_haps, uint32_t n_reads, const uint64_t* read_len,
                          double* out_hr, uint8_t* keep, uint32_t* n_kept)
{
    const double nan = std::numeric_limits<double>::quiet_NaN();
    std::vector<double> row(n_haps);
    uint32_t kept = 0;
    for (uint64_t i = 0; i < (uint64_t)n_haps * n_reads; ++i) out_hr[i] = nan;
    for (uint32_t r = 0; r < n_reads; ++r) {
        for (uint32_t h = 0; h < n_haps; ++h) row[h] = lk_hr[(uint64_t)h * n_reads + r];
        // normalize_likelihoods: std::max_element (operator<), so a leading NaN stays the maximum
        if (n_haps > 0) {
            double best = row[0];
            for (uint32_t h = 1; h < n_haps; ++h)
                if (best < row[h]) best = row[h];
            const double cmp = best + kBestAltDifference;
            for (uint32_t h = 0; h < n_haps; ++h) row[h] = row[h] < cmp ? cmp : row[h];
        }
        // collect_poorly_modelled_indices: best over non-NaN values
        double best = -std::numeric_limits<double>::infinity();
        for (uint32_t h = 0; h < n_haps; ++h)
            if (!std::isnan(row[h])) best = std::max(best, row[h]);
        const double min_lk =
            std::min(kMaxErrorsPerRead, std::ceil((double)read_len[r] * kErrorRatePerBase)) * kLog10QualityPerBase;
        const bool drop = best < min_lk;
        keep[r] = drop ? 0 : 1;
        if (!drop) {
            for (uint32_t h = 0; h < n_haps; ++h) out_hr[(uint64_t)h * n_reads + kept] = row[h];
            ++kept;
        }
    }
    *n_kept = kept;
}

}  // namespace phmm

using phmm::set_error;

extern "C" {

phmm_status phmm_call_region(phmm_engine* engine, uint32_t n_haps, const uint8_t* hap_bases, const uint64_t* hap_off,
                             uint32_t n_reads, const uint8_t* read_bases, const uint8_t* read_qual,
                             const uint64_t* read_off, const uint8_t* mapq, int32_t min_quality_threshold,
                             int32_t pcr_model, double* out, uint8_t* keep, uint32_t* n_kept)
{
    try {
        phmm::clear_error();
        if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
        if (!hap_off || !read_off || (n_reads && !mapq) || !keep || !n_kept || (n_haps && n_reads && !out))
            return set_error(PHMM_ERR_INVALID_ARGUMENT, "null argument");
        if (pcr_model < PHMM_PCR_NONE || pcr_model > PHMM_PCR_CONSERVATIVE)
            return set_error(PHMM_ERR_INVALID_ARGUMENT, "pcr_model out of range");
        const uint64_t total = (uint64_t)n_haps * n_reads;
        const double nan = std::numeric_limits<double>::quiet_NaN();
        // On any failure the reference returns an all-NaN matrix and keeps every read
        // (pairhmm_internal.cpp:581,605-610).
        auto fail_matrix = [&]() {
            for (uint64_t i = 0; i < total; ++i) out[i] = nan;
            for (uint32_t r = 0; r < n_reads; ++r) keep[r] = 1;
            *n_kept = n_reads;
        };
        phmm_region_input in{};
        in.n_haps = n_haps;
        in.hap_bases = hap_bases;
        in.hap_off = hap_off;
        in.n_reads = n_reads;
        in.read_bases = read_bases;
        in.read_qual = read_qual;
        in.read_off = read_off;
        in.mapq = mapq;
        in.min_quality_threshold = min_quality_threshold;
        in.pcr_model = pcr_model;
        std::string err;
        phmm_ticket t = 0;
        phmm_status st = phmm::server_submit_region(engine, in, nullptr, out, keep, n_kept, &t, err);
        if (st == PHMM_OK) st = phmm::server_wait(engine, t, -1, true, nullptr, nullptr, err);
        if (st != PHMM_OK) {
            fail_matrix();
            return set_error(st, err);
        }
        return PHMM_OK;
    } catch (const std::bad_alloc&) {
        return set_error(PHMM_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

// Host-only pieces of the region path, exported for tests and for callers that prepare reads
// themselves.  They touch no GPU.
void phmm_host_prepare_quals(const uint8_t* q, uint32_t n, uint8_t mapq, int32_t min_quality_threshold, uint8_t* out)
{
    phmm::prepare_read_quals(q, (int)n, mapq, min_quality_threshold, out);
}

void phmm_host_pcr_model(const uint8_t* bases, uint32_t n, uint8_t* gap_open, int32_t pcr_model)
{
    phmm::apply_pcr_model(bases, (int)n, gap_open, pcr_model);
}

int32_t phmm_host_tandem_repeat_length(const uint8_t* bases, uint32_t n, uint32_t offset)
{
    return phmm::tandem_repeat_length(bases, (int)n, (int)offset);
}

void phmm_host_normalize_filter(const double* lk_hap_read, uint32_t n_haps, uint32_t n_reads, const uint64_t* read_len,
                                double* out, uint8_t* keep, uint32_t* n_kept)
{
    phmm::normalize_and_filter(lk_hap_read, n_haps, n_reads, read_len, out, keep, n_kept);
}

}  // extern "C"
