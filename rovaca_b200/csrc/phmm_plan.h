// Host-side batch planner: validates a phmm_batch, flags reads/haplotypes containing 'N', and cuts
// the batch into wavefront work items grouped by kernel class, longest first inside a class.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/phmm_b200.h"
#include "phmm_types.h"

namespace phmm {

// Descriptor slots: the FP32 classes, then the FP64 classes (numbering in phmm_types.h).
constexpr int kPlanClasses = kClasses32 + kClasses64;

// FP32 tile shape of every (mode, read-length bucket): kh row pairs per lane, single stripe
// (kh >= bucket) or multi-stripe (kMinMultiKH <= kh < bucket, stripes = ceil(R / (32 * kh))).
// Modes as in phmm_types.h: 0 inter with constant gap qualities (insertion = deletion), 1 inter
// per-row, 2 intra.
struct TileTable {
    uint8_t kh[kModes32][kLenBuckets];
    uint8_t multi[kModes32][kLenBuckets];
    // smallest single stripe up to 256 rows, 256-row stripes beyond
    static TileTable defaults();
    bool valid(std::string& err) const;
};

// Region-API parameters of one region (call_pairhmm semantics): reads arrive with raw base
// qualities and are prepared on the device.
struct RegionApiParams {
    int32_t min_quality;  // base qualities below this become 6
    int32_t pcr;          // phmm_pcr_model
};

struct PlanLimits {
    // Reference limits, roDV_schedule.cpp:70-73 (haplotype index <= 4095, read length <= 768,
    // haplotype length <= 1536).
    uint32_t max_haps_per_region = 4096;
    uint32_t max_read_len = 768;
    uint32_t max_hap_len = 1536;
    // Longest haplotype column stream of one work item (single-stripe reads), and of a
    // multi-stripe item (bounded by the per-warp scratch row).
    uint32_t max_stream_single = 8192;
    uint32_t max_stream_multi = 4096;
    // FP32 tile shapes (null: TileTable::defaults())
    const TileTable* tiles = nullptr;
    // Non-null: every region of the batch uses the region API, with these parameters [n_regions];
    // the batch's gap-quality arrays are not read (the device writes them).
    const RegionApiParams* region_api = nullptr;
};

struct Plan {
    uint32_t n_regions = 0, n_reads = 0, n_haps = 0;
    uint64_t read_bases = 0, hap_bases = 0, out_total = 0;
    uint64_t read_base0 = 0, hap_base0 = 0;  // read_off[0], hap_off[0]: the copy starts there
    uint64_t pairs = 0, cells = 0, empty_pairs = 0;
    std::vector<RegionDesc> regions;
    std::vector<uint64_t> read_off, hap_off;  // rebased to start at 0
    std::vector<uint8_t> read_flags, hap_flags;
    std::vector<WorkItem> items;
    std::vector<ClassDesc> classes;  // kPlanClasses: FP32 classes (items), then FP64 (rerun segments)
    uint64_t rerun_slots = 0;
    uint32_t max_multi_stream = 0;   // longest stream among multi-stripe items (0 if none)
    TileTable tiles{};               // the shapes the items were planned with
    bool region_api = false;         // every region uses the region API (device read prep and post)
    // genotyping events of region-API regions (filled by the caller after planning)
    std::vector<EventDesc> events;
    std::vector<int8_t> hap_allele;
    uint64_t allele_lk_total = 0, gl_total = 0;
};

// Sizes of a batch, from one validating pass over its counts and offsets (no copies).
struct BatchScan {
    uint32_t n_haps = 0, n_reads = 0;
    uint64_t hap_base0 = 0, read_base0 = 0;  // hap_off[0], read_off[0]
    uint64_t hap_bases = 0, read_bases = 0, out_total = 0;
    uint64_t pairs = 0, cells = 0;           // pairs with a non-empty read and haplotype, their cells
};

// Validation shared by every entry point: counts, non-decreasing offsets, the reference limits and
// the pointers the batch needs.  Returns PHMM_OK, PHMM_ERR_INVALID_ARGUMENT or
// PHMM_ERR_LIMIT_EXCEEDED (err holds the detail).
phmm_status scan_batch(const phmm_batch& b, const PlanLimits& lim, BatchScan& s, std::string& err);

// scan_batch, then the full plan.  Same return codes.
phmm_status build_plan(const phmm_batch& b, const PlanLimits& lim, Plan& plan, std::string& err);

}  // namespace phmm
