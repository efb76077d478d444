// Plain data types shared by the host planner (g++) and the kernels (nvcc).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define PHMM_HD __host__ __device__
#else
#define PHMM_HD
#endif

namespace phmm {

constexpr int kWarp = 32;
constexpr int kMaxK = 8;          // rows per lane in one stripe (stripe = 256 rows)
#ifndef PHMM_CODE_PAD
#define PHMM_CODE_PAD 64
#endif
constexpr int kCodePad = PHMM_CODE_PAD;  // guard codes before/after the haplotype code stream
// Steps per boundary-free chunk of the packed FP32 sweep (build-time setting).  Measured on B200 with
// the two-value lane state over the 2,000-region benchmark batch: 8 steps 196.8 ms, 10 194.5, 12
// 192.7, 14 191.7, 16 191.3, 20 190.3 (with a 128-word code ring; the per-row gap mode 1.1% slower
// than at 16, the dominant class 0.3%), 24 195.3.  The code ring holds 31 + 2 chunks of words
// (phmm_device2.cuh): beyond 16 steps, or with the prior prefetch, build with PHMM_CODE_RING=128 and
// PHMM_CODE_PAD=128.
#ifndef PHMM_CHUNK_PACKED
#define PHMM_CHUNK_PACKED 16
#endif
constexpr int kChunk = PHMM_CHUNK_PACKED;  // steps per boundary-free fast chunk of the FP32 sweep

enum Variant : int { kInter = 0, kIntra = 1 };

// Read-length buckets: bucket = ceil(R / 32), 1..24 for the reference's R <= 768.
constexpr int kLenBuckets = 24;
PHMM_HD inline int len_bucket(uint64_t R) { return (int)((R + kWarp - 1) / kWarp); }

// FP32 kernel classes (packed path: two reads per warp, one per float2 component).  A class is a mode
//   0: inter, gap qualities constant along the read with insertion = deletion;  1: inter, any other
//   gap qualities (per-row);  2: intra (pairs with 'N')
// and a tile shape: KH row pairs per lane in one stripe of 32*KH rows (KH = 1..8), or stripes of
// 32*KH rows linked through per-warp scratch rows (KH = 4..8).  Which shape a read-length bucket
// runs in is a per-engine table (default: the smallest single stripe, 256-row stripes beyond).
constexpr int kMinMultiKH = 4;
constexpr int kShapes32 = kMaxK + (kMaxK - kMinMultiKH + 1);  // 8 single-stripe + 5 multi-stripe
constexpr int kModes32 = 3;
constexpr int kClasses32 = kModes32 * kShapes32;
PHMM_HD inline int mode32(int variant, int pmode) { return variant == 1 ? 2 : pmode; }
PHMM_HD inline int shape32(int kh, bool multi) { return multi ? kMaxK + kh - kMinMultiKH : kh - 1; }
PHMM_HD inline int class32(int variant, int pmode, int kh, bool multi)
{
    return mode32(variant, pmode) * kShapes32 + shape32(kh, multi);
}
PHMM_HD inline bool class32_multi(int c) { return c % kShapes32 >= kMaxK; }
PHMM_HD inline int class32_kh(int c)
{
    const int s = c % kShapes32;
    return s < kMaxK ? s + 1 : s - kMaxK + kMinMultiKH;
}

// FP64 recompute classes (scalar path, one read per warp): mode * 9 + (multi ? 8 : K - 1) with the
// modes of the FP32 classes (constant gap qualities let a lane hold the gap parameters once) and
// K = ceil(R / 32) rows per lane, multi for R > 256 (stripes of 256 rows).  A pair's FP64 class
// follows the mode of the FP32 class that computed it and its read length, whatever FP32 shape ran.
constexpr int kClasses64 = kModes32 * 9;
PHMM_HD inline int class64(int mode, int k, bool multi) { return mode * 9 + (multi ? 8 : k - 1); }
PHMM_HD inline int class64_for_len(int mode, uint64_t R)
{
    return R > (uint64_t)kWarp * kMaxK ? class64(mode, kMaxK, true) : class64(mode, len_bucket(R), false);
}

struct RegionDesc {               // 32 bytes
    uint64_t out_off;             // first likelihood of this region in the output
    uint32_t hap_begin;           // global index of the region's first haplotype
    uint32_t n_haps;
    uint32_t read_begin;          // global index of the region's first read
    uint32_t n_reads;
    uint32_t api;                 // kRegionApi: reads prepared and results post-processed on device;
                                  // bits 8-15: PCR model
    int32_t min_quality;          // region API: base qualities below this become 6
};
constexpr uint32_t kRegionApi = 1u;

// FP32 work item: two reads of one region (the two float2 components; read[1] may be kNoRead) against a
// run of the region's haplotypes.
constexpr uint32_t kNoRead = 0xffffffffu;
struct WorkItem {                 // 20 bytes
    uint32_t read[2];             // global read indices
    uint32_t region;
    uint16_t hap_lo, hap_hi;      // haplotype range inside the region, [lo, hi)
    uint8_t kh;                   // row pairs per lane: a stripe holds 32 * kh rows
    uint8_t stripes;              // stripes per read (1 for single-stripe shapes)
    uint8_t variant;              // Variant
    uint8_t pmode;                // ParamMode of the FP32 kernel (0: gap parameters constant)
};

// A run of consecutive haplotypes of one work item whose FP32 sums all fell below 1e-28 against
// one read: the FP64 pass streams them through the read like an FP32 work item.
struct RerunEntry {               // 24 bytes
    uint64_t out_idx;             // likelihood of the first pair
    uint32_t read;                // global read index
    uint32_t hap;                 // global index of the first haplotype
    uint32_t n_haps;              // haplotypes in the run
    uint32_t out_stride;          // output index step between consecutive haplotypes
};

template <typename T>
struct ProbTables {               // device copies of the reference's probability tables
    const T* ph2pr;               // [128] 10^(-q/10)
    const T* pmat;                // [128] 1 - ph2pr[q]
    const T* pmis_inter;          // [128] ph2pr[q] * (1/3)
    const T* pmis_intra;          // [128] ph2pr[q] / 3
    const T* gapm;                // [128] 1 - ph2pr[c]
    const T* mm;                  // [128*128] match-to-match, [ins][del]
};

struct BatchView {
    const uint8_t* read_bases;
    const uint8_t* read_q;
    const uint8_t* read_i;
    const uint8_t* read_d;
    const uint8_t* read_c;
    const uint64_t* read_off;     // [n_reads+1]
    const uint8_t* read_flags;    // [n_reads] bit0: contains 'N'
    const uint64_t* hap_off;      // [n_haps+1] offsets into the code streams (without guard)
    const uint32_t* codes_inter;  // [kCodePad + total + kCodePad]
    const uint32_t* codes_intra;
    const uint8_t* hap_flags;     // [n_haps] bit0: contains 'N'
    const RegionDesc* regions;
    double* out;
    uint8_t* pair_flags;          // may be null
};


// Per-class launch descriptor, in device memory so that a captured launch sequence can be
// replayed for any batch that fits the arena (the host rewrites the descriptors, not the graph).
struct ClassDesc {                // 32 bytes
    uint32_t item_off;            // first work item of the class
    uint32_t n_items;
    uint32_t rerun_off;           // first slot of the class's FP64 rerun segment
    uint32_t rerun_cap;           // = pairs of the class (runs <= pairs), so it cannot overflow
    uint32_t claim32;             // FP32 claim counter (zeroed before each batch)
    uint32_t claim64;             // FP64 claim counter
    uint32_t rerun_count;         // runs appended to the rerun segment
    uint32_t rerun_pairs;         // pairs in those runs
};

// Batch-wide sizes, in device memory for the same reason.
struct BatchDesc {
    uint64_t hap_bases_total;     // haplotype bases (length of the code streams without guards)
    uint64_t out_total;           // likelihoods in the output
    uint64_t read_bases_total;
    uint32_t n_regions, n_reads, n_haps, n_items;
    uint32_t region_api;          // regions with kRegionApi (0: the read-prep and post kernels idle)
    uint32_t n_events;            // genotyping events of region-API regions (0: genotype kernel idle)
};

// One genotyping event of a region-API region: a set of alleles, each haplotype mapped to one of
// them or to none.
struct EventDesc {                // 32 bytes
    uint32_t region;
    uint32_t n_alleles;           // 1..kMaxAlleles
    uint64_t hap_allele_off;      // int8 allele of each of the region's haplotypes (-1: none)
    uint64_t gl_off;              // first diploid genotype likelihood, n_alleles*(n_alleles+1)/2 of them
    uint64_t allele_lk_off;       // first allele likelihood: [n_alleles][region's n_reads]
};
constexpr uint32_t kMaxAlleles = 49;  // the reference's genotype tables stop below 50 alleles

// Region-API device arrays (read preparation in, post-processed results out).
struct RegionApiView {
    const BatchDesc* desc;
    const RegionDesc* regions;
    const uint64_t* read_off;
    const uint8_t* read_bases;
    uint8_t* read_q;              // in: raw base qualities; out: capped
    uint8_t* read_i;              // out: gap-open (PCR-capped)
    uint8_t* read_d;              // out: = read_i
    uint8_t* read_c;              // out: gap continuation
    const uint8_t* mapq;          // [n_reads]
    const double* lk;             // likelihoods [hap][read] per region
    double* out;                  // normalised, kept reads first, NaN after
    uint8_t* keep;                // [n_reads]
    uint32_t* n_kept;             // [n_regions]
    // genotyping (events of the regions)
    const EventDesc* events;
    const int8_t* hap_allele;
    double* allele_lk;            // marginal likelihoods, kept reads first, NaN after
    double* gl;                   // diploid genotype log10 likelihoods
    int32_t* best;                // most likely genotype per event
    const double* jacobian;       // log10(1 + 10^(-k/10000)), k = 0..80000
    double log10_two;             // log10(2) as the host's math library gives it
};

// Status bits a kernel raises instead of touching memory it should not.
enum StatusBits : unsigned int {
    kStatusRerunOverflow = 1u,
    kStatusBadItem = 2u,          // read longer than the class's stripe, or scratch too short
};

struct PassControl {
    ClassDesc* cd;                // this class's descriptor
    ClassDesc* cd64;              // FP32 pass: descriptors of the FP64 classes (rerun segments)
    const WorkItem* items;        // all work items (class slice at cd->item_off)
    RerunEntry* rerun;            // all rerun slots (class segment at cd->rerun_off)
    unsigned int* status;         // StatusBits, OR-ed
    void* scratch;                // per-warp stripe rows (multi-stripe reads)
    unsigned int scratch_cols;    // columns per warp scratch row
    unsigned int waves;           // FP32 single-stripe classes: the grid is this many times the
                                  // resident warps and each warp takes an equal share of the items
                                  // (0 or 1: persistent warps that take items until none are left)
};

// Per-byte match codes.
// Inter variant (pairs without 'N'): the code is the byte itself and a pair matches at (i, j) when
// code(read[i]) == code(hap[j]), the raw byte compare of pairhmm_inter.cpp:166-168.
// Intra variant (pairs with an 'N'): the reference's base classes (common.h:42-55, letters other
// than A/C/G/T/N fall in A's class) as one bit each, N matching everything (pairhmm_impl.cpp:26-42);
// a pair matches when code(read[i]) & code(hap[j]) != 0.
PHMM_HD inline uint32_t match_code(uint8_t b, int variant)
{
    if (variant == kInter) return b;
    switch (b) {
    case 'C': return 2u;
    case 'G': return 4u;
    case 'T': return 8u;
    case 'N': return 0xffffffffu;
    default: return 1u;
    }
}

PHMM_HD inline bool codes_match(uint32_t hc, uint32_t rc, int variant)
{
    return variant == kInter ? hc == rc : (hc & rc) != 0u;
}

// Haplotype code words of the code streams: the match code in bits 0-7 (kCodeMatchMask; the intra
// code of N is 0xF there, which matches every read code as 0xffffffff does) and the base's prior
// class in bits 11-13 for the packed FP32 kernels' prior tables: A, C, G, T are classes 0-3; class 4
// is N in the intra variant and every other byte in the inter variant; letters in A's intra class
// are class 0 there.  Guard words (0) are class 0: the cells computed at guard columns lie outside
// every haplotype and are discarded.
constexpr uint32_t kCodeMatchMask = 0xffu;
constexpr int kTabShift = 11;
constexpr uint32_t kTabMask = 7u << kTabShift;
constexpr int kTabClasses = 5;
PHMM_HD inline uint32_t base_class(uint8_t b)
{
    return b == 'A' ? 0u : b == 'C' ? 1u : b == 'G' ? 2u : b == 'T' ? 3u : 4u;
}
PHMM_HD inline uint32_t hap_code(uint8_t b, int variant)
{
    if (variant == kInter) return (uint32_t)b | (base_class(b) << kTabShift);
    const uint32_t c = base_class(b);
    if (c < 4u) return match_code(b, kIntra) | (c << kTabShift);
    return b == 'N' ? (0xfu | (4u << kTabShift)) : 1u;  // other letters: A's class
}
// The match code that a prior class stands for when a read row is tested against it (class 4 of
// the inter variant stands for a byte outside A/C/G/T: it matches no A/C/G/T row).
PHMM_HD inline bool class_matches(uint32_t cls, uint32_t rc, int variant)
{
    if (variant == kInter) return cls < 4u && rc == (cls == 0u ? 'A' : cls == 1u ? 'C' : cls == 2u ? 'G' : 'T');
    return ((cls < 4u ? 1u << cls : 0xfu) & rc) != 0u;
}

}  // namespace phmm
