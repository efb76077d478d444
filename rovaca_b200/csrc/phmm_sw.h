// Smith-Waterman realignment of reads to haplotypes on the GPU (kernels and host side in phmm_sw.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/phmm_b200.h"

namespace phmm {

struct SwParams {
    int32_t match, mismatch, gap_open, gap_extend;
};

// One alignment: seq1 = haplotype (rows), seq2 = read (columns); byte offsets into the base buffers.
struct SwItem {
    uint64_t hap_start, read_start;
    uint32_t hap_len, read_len;
};
static_assert(sizeof(SwItem) == 24, "SwItem layout");

// Reference limit: inputs whose longer sequence has kSwMaxSeq bases or more are refused with
// alignment offset 1 (sw_core_template.h:354-361, MAX_SEQ_LEN of sw_avx.c:18).
constexpr int kSwMaxSeq = 2048;
constexpr int kSwBlockWarps = 4;
constexpr int kSwBandWords = 1024;   // trace-back band in shared memory per warp (4 KB)
constexpr int kSwClasses = 14;       // 13 stripe widths (kSwK) + the 16-bit wrap-around class
constexpr int kSwWrapClass = 13;
constexpr int kSwK[kSwClasses] = {1, 2, 3, 4, 5, 6, 7, 8, 10, 12, 16, 20, 24, 24};

// Per-warp scratch layout of one alignment (bytes, 256-aligned sections):
//   bt    [stripes][nrow][32 * nw] u32: per cell a 4-bit code (state 1/2 | extension flags 4/8)
//   bh/be [nrow + 1] i32: H and E of the stripe's right edge column, handed to the next stripe
//   lrow  [ncol + 1] i32: H of the last row; lcol [nrow + 1] i32: H of the last column
//   runs  [nrow + ncol + 4] u32: CIGAR runs in trace-back order
struct SwLayout {
    uint64_t bt, bh, be, lrow, lcol, runs, total;
};

__host__ __device__ inline uint64_t sw_align256(uint64_t x) { return (x + 255) & ~uint64_t(255); }

__host__ __device__ inline SwLayout sw_layout(uint32_t nrow, uint32_t ncol, int K)
{
    const uint64_t nw = (uint64_t)(K + 7) / 8;
    const uint64_t cols = 32ull * K;
    const uint64_t stripes = ncol ? (ncol + cols - 1) / cols : 1;
    SwLayout L;
    L.bt = 0;
    uint64_t o = sw_align256(stripes * nrow * 32ull * nw * 4ull);
    L.bh = o;
    o = sw_align256(o + 4ull * (nrow + 1));
    L.be = o;
    o = sw_align256(o + 4ull * (nrow + 1));
    L.lrow = o;
    o = sw_align256(o + 4ull * (ncol + 1));
    L.lcol = o;
    o = sw_align256(o + 4ull * (nrow + 1));
    L.runs = o;
    o = sw_align256(o + 4ull * (nrow + ncol + 4));
    L.total = o;
    return L;
}

// ro_sw_should_use_int32_avx512 (ro_sw.c:26-40): int32 for reads under 16 bases, match <= 0, or
// min(length) x match above INT16_MAX; int16 otherwise.  variant: 0 as the reference, 1 int32, 2 int16.
__host__ __device__ inline bool sw_uses_int32(int variant, uint32_t nrow, uint32_t ncol, int32_t match)
{
    if (variant == 1) return true;
    if (variant == 2) return false;
    if (ncol < 16 || match <= 0) return true;
    const uint32_t m = nrow < ncol ? nrow : ncol;
    return (long long)m * match > 32767;
}

// True when the 16-bit kernel's adds cannot wrap for these (16-bit) parameters and the shorter
// sequence's length, so that 32-bit arithmetic with the 16-bit constants gives its results: scores
// stay within [cutoff + open + extend, min(length) x match] (checked against [-32768, 32767] with the
// 16-bit low -16384 and cutoff -8192).  The reference's own kernel choice already bounds
// min(length) x match; a forced 16-bit kernel does not.
__host__ __device__ inline bool sw_w16_cannot_wrap(int32_t match, int32_t mismatch, int32_t open, int32_t ext,
                                                   uint32_t min_len)
{
    return mismatch <= match && open <= 0 && ext <= 0 && mismatch >= -24576 && open + ext >= -24576 &&
           ext >= -16384 && (match <= 0 || (long long)min_len * match <= 32767);
}

int sw_class_of(const SwParams& prm, int variant, uint32_t nrow, uint32_t ncol);

// Host plan of one batch of alignments: kernel class of each (by read columns, or the wrap-around
// class), alignments grouped by class most cells first, CIGAR slots, grids and scratch.
struct SwPlan {
    uint32_t n = 0;
    uint32_t cigar_cap = 0;
    std::vector<uint32_t> order;             // item indices grouped by class, most cells first
    std::vector<uint64_t> slot_off;          // per item: its CIGAR slot (ops) in the slot buffer
    uint64_t slots = 0;                      // ops of all slots
    uint32_t begin[kSwClasses + 1] = {};
    uint64_t stride[kSwClasses] = {};        // scratch bytes per warp of each class
    int grid[kSwClasses] = {};
    int gather_blocks = 1;
    uint64_t scratch = 0;                    // bytes for the largest class launch
    uint64_t cells = 0;
};

// Device buffers of one batch (see SwPlan for their sizes: n items, n results, `slots` ops twice,
// `scratch` bytes, kSwClasses claim counters).
struct SwDeviceBufs {
    const SwItem* items = nullptr;
    const uint32_t* order = nullptr;
    const uint64_t* slot_off = nullptr;
    const uint8_t* hap = nullptr;            // base of the items' haplotype offsets
    const uint8_t* read = nullptr;           // base of the items' read offsets
    unsigned int* claim = nullptr;
    unsigned long long* total = nullptr;     // out: CIGAR ops of the batch
    phmm_sw_result* out = nullptr;
    uint32_t* slots = nullptr;
    uint32_t* compact = nullptr;
    uint8_t* scratch = nullptr;
};

// Plans n alignments on `device` from their rows (haplotype lengths, or upper bounds of them) and
// columns (read lengths).
phmm_status sw_plan(int device, const SwParams& prm, int variant, uint32_t n, const uint32_t* nrow,
                    const uint32_t* ncol, uint32_t cigar_cap, SwPlan& p, std::string& err);
// Launches a planned batch on stream st: the class kernels, the CIGAR offset scan and the gather.
// class_ms (optional, kSwClasses): every class timed alone with ev0/ev1 (synchronising).
phmm_status sw_launch(const SwPlan& p, const SwParams& prm, int variant, const SwDeviceBufs& b, cudaStream_t st,
                      cudaEvent_t ev0, cudaEvent_t ev1, float* class_ms, std::string& err);

struct SwArenaLayout;

// ---- realignment of region-API regions' kept reads to their best haplotypes (device side) ----

struct RegionDesc;

// A region-API region of the batch whose kept reads are realigned.
struct RealignRegion {           // 16 bytes
    uint32_t region;             // index in the batch
    uint32_t item_begin;         // its first Smith-Waterman item (one per read, in read order)
    uint64_t prio_off;           // its haplotypes' tie-break priorities
};

struct RealignView {
    const RegionDesc* regions;
    const uint64_t* hap_off;     // batch haplotype offsets into the haplotype bases
    const uint64_t* read_off;    // batch read offsets into the read bases
    const double* norm;          // normalised likelihoods: region blocks at out_off, kept reads first
    const uint8_t* keep;         // [batch reads]
    const RealignRegion* rr;
    uint32_t n_rr;
    const double* prio;
    const uint16_t* clip;        // [items][2]: bases dropped at the read's start and end
    SwItem* items;               // out: the read against its best haplotype
    int32_t* best;               // out: best haplotype (index in the region), -1 for dropped reads
};

// Fills the items and best haplotypes of every realigned region (one block per region).
cudaError_t launch_realign_items(const RealignView& v, int blocks, cudaStream_t st);

// Host side of one batch's realignment: the regions, their inputs, the plan, the device layout in
// the slot's realignment arena, and (after it ran) the results per item.
struct RealignBatch {
    std::vector<RealignRegion> regions;
    std::vector<double> prio;
    std::vector<uint16_t> clip;              // 2 per item
    std::vector<uint32_t> nrow, ncol;        // per item: the region's longest haplotype, the clipped read
    SwPlan plan;
    // device layout (bytes): [rr | prio | clip | order | slot_off] uploaded, then the items,
    // claim counters, [total | results | best] read back, CIGAR slots, compact CIGARs, scratch
    uint64_t o_rr = 0, o_prio = 0, o_clip = 0, o_order = 0, o_slot = 0, o_items = 0, o_claim = 0, o_total = 0,
             o_out = 0, o_best = 0, o_slots = 0, o_compact = 0, o_scratch = 0, bytes = 0;
    uint64_t upload_bytes() const { return o_items; }
    uint64_t head_bytes() const { return o_slots - o_total; }
    void layout();
    // results (realign_finish)
    uint64_t total = 0;
    std::vector<phmm_sw_result> res;
    std::vector<int32_t> best;
    std::vector<uint32_t> cigars;
};

// Device state of the aligner: a stream, a growable arena and pinned staging, owned by an engine.
class SwAligner {
public:
    static phmm_status create(int device, SwAligner** out, std::string& err);
    ~SwAligner();

    // Host buffers in and out (copies inside), synchronous.  out[n]; compact CIGARs (phmm_sw_align).
    phmm_status align(const SwParams& prm, int variant, uint32_t n, const SwItem* items, const uint8_t* hap,
                      uint64_t hap_bytes, const uint8_t* read, uint64_t read_bytes, uint32_t cigar_cap,
                      phmm_sw_result* out, uint32_t* cigars, uint64_t cigar_capacity, uint64_t* cigar_total,
                      float* device_ms, std::string& err);

    // Resident batches: planned and uploaded once, run many times, results read back on demand.
    struct Resident;
    phmm_status resident_create(const SwParams& prm, int variant, uint32_t n, const SwItem* items,
                                const uint8_t* hap, uint64_t hap_bytes, const uint8_t* read, uint64_t read_bytes,
                                uint32_t cigar_cap, Resident** out, std::string& err);
    phmm_status resident_run(Resident* r, int iterations, float* ms_per_run, float* class_ms, std::string& err);
    phmm_status resident_results(Resident* r, phmm_sw_result* out, uint32_t* cigars, uint64_t capacity,
                                 uint64_t* total, std::string& err);
    void resident_destroy(Resident* r);

    int device() const { return dev_; }

private:
    SwAligner() = default;
    phmm_status plan(const SwParams& prm, int variant, uint32_t n, const SwItem* items, uint32_t cigar_cap,
                     SwPlan& p, std::string& err) const;
    phmm_status ensure_pinned(uint64_t bytes, std::string& err);
    phmm_status read_back(uint8_t* d, const SwArenaLayout& L, uint32_t n, phmm_sw_result* out, uint32_t* cigars,
                          uint64_t capacity, uint64_t* total, std::string& err);

    int dev_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev_[2] = {};
    void* arena_ = nullptr;
    size_t arena_bytes_ = 0;
    void* pinned_ = nullptr;
    size_t pinned_bytes_ = 0;
    std::mutex mu_;
};

}  // namespace phmm
