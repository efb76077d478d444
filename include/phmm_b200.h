/*
 * phmm_b200 — B200-native PairHMM likelihood engine, C ABI.
 *
 * This is the drop-in boundary for the reference's PairHMM entry point
 *   DoubleVector2D (*rovaca::call_pairhmm)(const HaplotypeVector& hs, ReadVector& rs,
 *       int32_t min_quality_threshold, PcrIndelModel pcr_option, pMemoryPool pool)
 *   (src/haplotypecaller/pairhmm/pairhmm_engine.h:14, bound in pairhmm_engine.cpp:19-37,
 *    implemented by call_roDV_pairhmm_scheduled in pairhmm_internal.cpp:576-623)
 * and for the vector API the reference's tests drive
 *   bool pairhmm::schedule::schedule_pairhmm(haplotypes, reads, result, quality, ins, del, gcp, ...)
 *   (src/haplotypecaller/pairhmm/roDV_schedule.h:16-27, roDV_schedule.cpp:154-361).
 *
 * Plain C types only: host pointers and sizes in, host pointers out.  Every call returns a
 * phmm_status; none throws, none aborts the process.  All sequence data is 1 byte per base
 * (ASCII A/C/G/T/N) and all qualities are raw Phred values (not +33), exactly as the reference's
 * TestCase carries them (roDV_common/common.h:27-36).
 *
 * Likelihood layout: for every region, a block of n_haps * n_reads doubles in [hap][read] order,
 * the layout call_pairhmm returns (pairhmm_internal.cpp:499-508,613); blocks follow region order.
 */
#ifndef PHMM_B200_H
#define PHMM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PHMM_API __attribute__((visibility("default")))
#else
#define PHMM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum phmm_status {
    PHMM_OK = 0,
    PHMM_ERR_INVALID_ARGUMENT = 1, /* null pointer, inconsistent sizes, bad enum */
    PHMM_ERR_LIMIT_EXCEEDED = 2,   /* region beyond the reference's limits (roDV_schedule.cpp:70-73):
                                      more than 4096 haplotypes, a read longer than 768 or a
                                      haplotype longer than 1536 */
    PHMM_ERR_OUT_OF_MEMORY = 3,    /* device or pinned-host allocation failed */
    PHMM_ERR_CUDA = 4,             /* a CUDA runtime call failed; see phmm_last_error() */
    PHMM_ERR_NOT_INITIALIZED = 5,  /* engine handle is null or was destroyed */
    PHMM_ERR_TIMEOUT = 6,          /* phmm_wait deadline passed (the request keeps running) */
    PHMM_ERR_CANCELLED = 7,        /* request was cancelled before it was admitted */
    PHMM_ERR_QUEUE_FULL = 8,       /* serving queue at capacity */
    PHMM_ERR_DEVICE_STATUS = 9,    /* a kernel reported an error status word */
    PHMM_ERR_NO_DEVICE = 10,       /* no CUDA device, or the requested ordinal does not exist */
    PHMM_ERR_INTERNAL = 11
} phmm_status;

/* PCR indel error model, same enumerators and meaning as the reference's PcrIndelModel
 * (src/haplotypecaller/common/enum.h:8) and its caps (pairhmm/adapter.h:13-15). */
typedef enum phmm_pcr_model {
    PHMM_PCR_NONE = 0,
    PHMM_PCR_HOSTILE = 1,
    PHMM_PCR_AGGRESSIVE = 2,
    PHMM_PCR_CONSERVATIVE = 3
} phmm_pcr_model;

typedef struct phmm_engine phmm_engine;

typedef struct phmm_config {
    int32_t device;            /* CUDA device ordinal */
    int32_t use_cuda_graph;    /* 1: replay the device-side batch pipeline from a captured CUDA graph */
    int32_t autotune;          /* 1: run the tile-shape autotuner at creation (once per device and
                                  process; later engines reuse its table); 0: default shapes */
    int32_t reserved0;
    uint64_t hbm_budget_bytes; /* serving-loop admission budget for resident region data; 0 = 40 GiB */
    uint64_t chunk_cells;      /* phmm_compute_regions runs a batch of at least this many cells as a
                                  pipeline of region chunks on two device slots, planning and
                                  uploading each chunk while the previous one runs (same results);
                                  0 = 4e10, UINT64_MAX = never */
} phmm_config;

/* A batch of independent active regions in flat, concatenated arrays (host memory). */
typedef struct phmm_batch {
    uint32_t n_regions;
    const uint32_t* n_haps;    /* [n_regions] haplotypes per region */
    const uint32_t* n_reads;   /* [n_regions] reads per region */
    const uint8_t* hap_bases;  /* all haplotypes, region-major */
    const uint64_t* hap_off;   /* [sum(n_haps) + 1] offsets into hap_bases */
    const uint8_t* read_bases; /* all reads, region-major */
    const uint8_t* read_qual;  /* base quality per read base */
    const uint8_t* read_ins;   /* insertion gap-open quality per read base */
    const uint8_t* read_del;   /* deletion gap-open quality per read base */
    const uint8_t* read_gcp;   /* gap-continuation quality per read base */
    const uint64_t* read_off;  /* [sum(n_reads) + 1] offsets into the five read arrays */
} phmm_batch;

typedef struct phmm_stats {
    uint64_t regions;
    uint64_t pairs;         /* read x haplotype pairs computed */
    uint64_t cells;         /* sum over pairs of read_len * hap_len */
    uint64_t pairs_f64;     /* pairs recomputed in FP64 because the FP32 sum fell below 1e-28 */
    uint64_t work_items;    /* wavefront work items of the FP32 pass */
    uint64_t h2d_bytes;
    uint64_t d2h_bytes;
    uint64_t kernel_launches; /* kernels this library launched for the call */
    double device_ms;       /* CUDA-event time of the device pipeline (prep + FP32 + FP64) */
    double fp32_ms;         /* CUDA-event time of the FP32 wavefront pass (prep included) */
    double fp64_ms;         /* CUDA-event time of the FP64 recompute pass */
    double host_ms;         /* wall time of the whole call */
} phmm_stats;

/* ---- engine lifetime ------------------------------------------------------------------- */

/* cfg may be NULL (device 0, graphs on, autotune on, 40 GiB budget). */
PHMM_API phmm_status phmm_engine_create(const phmm_config* cfg, phmm_engine** out_engine);
PHMM_API phmm_status phmm_engine_destroy(phmm_engine* engine);
PHMM_API const char* phmm_status_string(phmm_status status);
/* Detail of the last error raised on the calling thread ("" if none). */
PHMM_API const char* phmm_last_error(void);
/* Library build string (kernel variants, target architecture). */
PHMM_API const char* phmm_version(void);

/* ---- synchronous batch ------------------------------------------------------------------ */

/* Computes every read x haplotype log10 likelihood of every region in the batch.
 *   out        : sum(n_haps[r] * n_reads[r]) doubles; region blocks in order, [hap][read] inside.
 *   pair_flags : optional (may be NULL), same shape; bit 0 set when the pair was recomputed in
 *                FP64 (FP32 sum below 1e-28, roDV_schedule.cpp:35,704).
 *   stats      : optional.
 * Reads are used exactly as given (no quality capping): the semantics of schedule_pairhmm.
 * A pair with an empty read or haplotype gets NaN, as the region API leaves such pairs. */
PHMM_API phmm_status phmm_compute_regions(phmm_engine* engine, const phmm_batch* batch, double* out, uint8_t* pair_flags,
                                 phmm_stats* stats);

/* One region through the full call_pairhmm path (call_roDV_pairhmm_scheduled,
 * pairhmm_internal.cpp:576-623 and the region-API read preparation of roDV_schedule.cpp:522-649):
 *   1. base quality q -> min(q, mapq); below min_quality_threshold -> 6;
 *   2. insertion/deletion gap-open 45 and gap continuation 10 for every base;
 *   3. with a PCR model other than NONE, gap-open capped by tandem-repeat length (deletion uses
 *      the same capped values as insertion);
 *   4. likelihoods, each read's row capped at best - 4.5;
 *   5. reads whose best likelihood is below -4 * min(2, ceil(0.02 * len)) are dropped.
 * out    : [n_haps][n_reads] doubles; column k holds the k-th kept read, trailing columns NaN.
 * keep   : [n_reads] bytes, 1 where the read was kept (the caller erases the others, in order).
 * n_kept : number of kept reads.
 * Steps 1-3 and 4-5 run on the GPU around the likelihood kernels (only bases, raw qualities and
 * MAPQ are uploaded); concurrent calls are batched by the serving loop (phmm_submit_region). */
PHMM_API phmm_status phmm_call_region(phmm_engine* engine, uint32_t n_haps, const uint8_t* hap_bases, const uint64_t* hap_off,
                             uint32_t n_reads, const uint8_t* read_bases, const uint8_t* read_qual,
                             const uint64_t* read_off, const uint8_t* mapq, int32_t min_quality_threshold,
                             int32_t pcr_model, double* out, uint8_t* keep, uint32_t* n_kept);

/* ---- batches without device allocation -------------------------------------------------- */

/* Same computation and result layout as phmm_compute_regions, for callers that cannot call
 * cudaMalloc (a process whose GPU memory belongs to another framework's pool allocator, or a host
 * that forbids allocation on its worker threads): it allocates no device or pinned memory.  All
 * device data of the call lives in a fixed 64 MiB array that is part of this library's device code
 * (every GPU that loads the library holds it until the process exits).  A batch that needs more
 * than that (about 100 regions of the benchmark's shape) is rejected with PHMM_ERR_LIMIT_EXCEEDED.
 * Synchronous; calls on one device are serialised and share the array.  The first call on a device
 * sets that device up (looks up the array's address, uploads the probability tables): make it
 * before any stream capture on the device.  Its copies and kernels run on the device's legacy
 * default stream, so a call waits for, and holds back, work on the caller's blocking streams of
 * that device (streams created with cudaStreamNonBlocking are not affected).  The calling thread's
 * current device is the same after the call as before it.  No counterpart in the reference: an
 * addition of this library. */
PHMM_API phmm_status phmm_compute_regions_noalloc(const phmm_batch* batch, double* out, uint8_t* pair_flags,
                                                  int32_t device);

/* ---- device-resident batches ------------------------------------------------------------ */

typedef struct phmm_resident phmm_resident;

/* Uploads a batch once into a device arena of its own (reads and haplotypes stay in HBM). */
PHMM_API phmm_status phmm_resident_create(phmm_engine* engine, const phmm_batch* batch, int32_t want_flags,
                                          phmm_resident** out_resident);
/* Recomputes the resident batch `iterations` times back to back with no host transfer; stats
 * (optional) report the device time of all iterations together (CUDA events on the engine's
 * stream) and the kernels launched. */
PHMM_API phmm_status phmm_resident_run(phmm_resident* resident, int32_t iterations, phmm_stats* stats);
/* Copies the latest results to the host (layout of phmm_compute_regions; flags may be NULL). */
PHMM_API phmm_status phmm_resident_results(phmm_resident* resident, double* out, uint8_t* pair_flags);
/* Runs the resident batch once with every kernel class alone (one after another on one stream,
 * CUDA events around each launch) for per-kernel timing: class_ms[66] (FP32 classes 0..38, then
 * FP64 classes; 0 for classes without work) and class_cells[66] (cells of the FP32 classes' work
 * items; 0 for FP64 classes, whose work is only known on the device).  The results equal those of
 * phmm_resident_run. */
PHMM_API phmm_status phmm_resident_profile(phmm_resident* resident, float* class_ms, uint64_t* class_cells);
/* Recomputes every pair of the resident batch with the all-FP64 check arithmetic -- FP64 end to
 * end with C = 2^1020, each product rounded and then added (no fused multiply-add), every result
 * below 2^-1022 flushed, the inter prior for pairs without 'N' and the N-aware intra model for the
 * others -- and writes the log10 likelihoods to out (layout of phmm_compute_regions; pairs with an
 * empty read or haplotype NaN).  This is the model every likelihood's error is measured against,
 * computed for the whole batch on the device.  The resident's own results are overwritten: call
 * phmm_resident_run again before phmm_resident_results.  No reference counterpart (the reference's
 * FP64 path, computeLikelihoodsAVX512 with use_double, pairhmm_api.cpp:14-19, is the contracted
 * form of the same model). */
PHMM_API phmm_status phmm_resident_check_fp64(phmm_resident* resident, double* out);
PHMM_API phmm_status phmm_resident_destroy(phmm_resident* resident);

/* Measures the device's FP32 FMA throughput (independent FMA chains on every SM, about 0.1 s),
 * in TFLOP/s counting an FMA as 2 FLOPs, with scalar FFMA and with packed two-wide FFMA2
 * instructions (either pointer may be NULL): the peak the wavefront kernels are compared with. */
PHMM_API phmm_status phmm_fp32_fma_peak(phmm_engine* engine, double* scalar_tflops, double* packed_tflops);

/* ---- host-only pieces of the region path (no GPU involved) ----------------------------- */

/* Base qualities as the region API prepares them: min(q, mapq), below the threshold -> 6
 * (roDV_schedule.cpp:540-565). */
PHMM_API void phmm_host_prepare_quals(const uint8_t* q, uint32_t n, uint8_t mapq, int32_t min_quality_threshold, uint8_t* out);
/* PCR indel model: caps gap_open[i] (i < n-1) by the tandem-repeat length at i
 * (apply_pcr_error_model_rolling, pairhmm_internal.cpp:431-476). */
PHMM_API void phmm_host_pcr_model(const uint8_t* bases, uint32_t n, uint8_t* gap_open, int32_t pcr_model);
/* Tandem-repeat length at offset (find_tandem_repeat_units_rolling, pairhmm_internal.cpp:317-389). */
PHMM_API int32_t phmm_host_tandem_repeat_length(const uint8_t* bases, uint32_t n, uint32_t offset);
/* Post-processing of call_pairhmm on a [hap][read] likelihood matrix: cap each read at best - 4.5,
 * drop poorly modelled reads, compact kept reads into the first columns (NaN after them). */
PHMM_API void phmm_host_normalize_filter(const double* lk_hap_read, uint32_t n_haps, uint32_t n_reads, const uint64_t* read_len,
                                double* out, uint8_t* keep, uint32_t* n_kept);

/* ---- tile shapes and the autotuner (no reference counterpart) ---------------------------------
 *
 * The FP32 pass runs every read in a tile shape chosen by its mode and read-length bucket:
 *   mode 0: pairs without 'N' whose read has constant insertion/deletion/gap qualities and equal
 *           insertion and deletion qualities,
 *   mode 1: other pairs without 'N', mode 2: pairs with 'N';
 *   bucket b = ceil(read length / 32), 1..24;
 *   shape: rows_per_lane KH (32 lanes hold 32 * KH rows of each read) in one stripe (KH >= b), or
 *          multi_stripe with 4 <= KH < b, the read running as ceil(length / (32 * KH)) stripes.
 * FP32 kernel class = mode * 13 + (multi_stripe ? 4 + KH : KH - 1); FP64 recompute class =
 * mode * 9 + (length > 256 ? 8 : b - 1), the mode of the FP32 class that ran the pair.  Results do
 * not depend on the shapes. */
#define PHMM_TILE_MODES 3
#define PHMM_LEN_BUCKETS 24
#define PHMM_FP32_CLASSES 39
#define PHMM_FP64_CLASSES 27

typedef struct phmm_tile_table {
    uint8_t rows_per_lane[PHMM_TILE_MODES][PHMM_LEN_BUCKETS];
    uint8_t multi_stripe[PHMM_TILE_MODES][PHMM_LEN_BUCKETS];
} phmm_tile_table;

/* One candidate shape the autotuner timed. */
typedef struct phmm_tune_entry {
    uint8_t mode, bucket, rows_per_lane, multi_stripe;
    uint8_t chosen;               /* 1: installed for (mode, bucket) */
    uint8_t reserved[3];
    float gcups;                  /* FP32 pass throughput on the calibration batch */
} phmm_tune_entry;

#define PHMM_TUNE_MAX_ENTRIES 512
typedef struct phmm_tune_report {
    uint32_t n_entries;
    uint32_t reserved;
    double seconds;               /* wall time of the tuning run */
    phmm_tune_entry entries[PHMM_TUNE_MAX_ENTRIES];
} phmm_tune_report;

/* Default shapes: the smallest single stripe up to 256 rows, 256-row stripes beyond. */
PHMM_API void phmm_tile_table_default(phmm_tile_table* table);
PHMM_API phmm_status phmm_engine_get_tiles(phmm_engine* engine, phmm_tile_table* table);
/* Installs a table for batches planned from now on (PHMM_ERR_INVALID_ARGUMENT if a shape cannot
 * hold its bucket). */
PHMM_API phmm_status phmm_engine_set_tiles(phmm_engine* engine, const phmm_tile_table* table);
/* Times the candidate shapes of every (mode, bucket) on synthetic calibration batches on the
 * engine's device, installs the fastest and reports every measurement (report may be NULL).
 * An engine created with config.autotune = 1 runs this once per device and process at creation. */
PHMM_API phmm_status phmm_engine_autotune(phmm_engine* engine, phmm_tune_report* report);

/* How a batch is cut into wavefront work, without running it (no GPU involved), under `tiles`
 * (NULL: the default table):
 *   class_items[39]: work items per FP32 kernel class (numbering above); an item is two reads (one
 *     when a region has an odd count) of one shape against a haplotype run;
 *   class_pairs[27]: pairs per FP64 recompute class (the capacity reserved for pairs that
 *     underflow in FP32);
 *   pairs, cells: totals of the batch.
 * Returns the same validation status phmm_compute_regions would. */
PHMM_API phmm_status phmm_host_plan_summary(const phmm_batch* batch, const phmm_tile_table* tiles,
                                            uint32_t class_items[PHMM_FP32_CLASSES],
                                            uint64_t class_pairs[PHMM_FP64_CLASSES], uint64_t* pairs, uint64_t* cells);

/* ---- serving loop ----------------------------------------------------------------------- */

typedef uint64_t phmm_ticket;

/* Submits one region (a phmm_batch with n_regions == 1).  Inputs are copied before the call
 * returns; out / pair_flags (same shape as for phmm_compute_regions) must stay valid until the
 * request completes.  Requests are admitted as device slots and the HBM budget free up, and
 * batched with whatever else is in flight.  Thread-safe. */
PHMM_API phmm_status phmm_submit(phmm_engine* engine, const phmm_batch* region, double* out, uint8_t* pair_flags,
                        phmm_ticket* ticket);
/* One region for the region API (phmm_call_region's inputs). */
typedef struct phmm_region_input {
    uint32_t n_haps;
    const uint8_t* hap_bases;
    const uint64_t* hap_off;    /* [n_haps + 1] */
    uint32_t n_reads;
    const uint8_t* read_bases;
    const uint8_t* read_qual;   /* raw base qualities */
    const uint64_t* read_off;   /* [n_reads + 1] */
    const uint8_t* mapq;        /* [n_reads] */
    int32_t min_quality_threshold;
    int32_t pcr_model;          /* phmm_pcr_model */
} phmm_region_input;

/* Genotyping events of one region: each event is a set of alleles with every haplotype mapped to
 * one of them (or to none), as HaplotypeCaller maps haplotypes to the alleles of a variant site.
 * On the GPU, after the region's reads are normalised and filtered:
 *   allele likelihood (read, allele) = max over the allele's haplotypes (-inf if it has none)
 *     (AlleleLikelihoods::marginal_likelihoods_direct, genotype/allele_likelihoods.hpp:702-730);
 *   diploid genotype likelihoods, genotype (a <= b) at index b(b+1)/2 + a, and the most likely
 *   genotype (first maximum) (GenotypeLikelihoodCalculator, genotype_likelihood_calculator.cpp:59-100).
 * Only these come back to the host when the matrix itself is not asked for. */
typedef struct phmm_region_events {
    uint32_t n_events;
    const uint8_t* n_alleles;    /* [n_events], 1..49 */
    const int8_t* hap_allele;    /* [n_events][n_haps]: allele index of each haplotype, -1 for none */
    double* genotype_lk;         /* out: [sum over events of n_alleles (n_alleles + 1) / 2] log10 */
    int32_t* best_genotype;      /* out: [n_events] */
    double* allele_lk;           /* out, optional: [sum of n_alleles][n_reads], kept reads first, NaN after */
} phmm_region_events;

/* Submits one region with phmm_call_region's semantics; the read preparation (quality cap, gap
 * qualities, PCR model), the post-processing (normalise, drop poorly modelled reads, kept reads
 * first) and, when events is not NULL, the genotyping of its events run on the GPU.  out
 * [n_haps][n_reads] may be NULL when only the genotyping results are wanted.  Output buffers must
 * stay valid until the request completes (phmm_wait); inputs are copied before the call returns.
 * Thread-safe. */
PHMM_API phmm_status phmm_submit_region(phmm_engine* engine, const phmm_region_input* region,
                                        const phmm_region_events* events, double* out, uint8_t* keep,
                                        uint32_t* n_kept, phmm_ticket* ticket);
/* Realignment of a region's kept reads to their best haplotypes on the GPU, on the bases already
 * uploaded for the likelihoods (AssemblyBasedCallerUtils::realign_reads_to_their_best_haplotype,
 * genotype/utils/assembly_based_caller_utils.cpp:146-169):
 *   best haplotype of each kept read = AlleleLikelihoods::search_best_allele over the normalised,
 *     filtered likelihoods, ties among haplotypes within 0.2 log10 of the best broken by hap_priority
 *     (genotype/allele_likelihoods.hpp:589-658; HaplotypeCaller's priority is (is_reference ? 1 : 0)
 *     + 1 - cigar elements, assembly_based_caller_utils.cpp:150-155);
 *   Smith-Waterman of the read without its soft clips (clip_left / clip_right bases removed at each
 *     end, ReadClipper::hard_clip_soft_clipped_bases) against that haplotype with the genotyping
 *     parameters, as AlignmentUtils::create_read_aligned_to_ref calls it (alignment_utils.cpp:571-579).
 * Outputs are per read in the region's read order: best_hap -1 and a zero result for dropped reads;
 * sw[r].cigar_offset indexes `cigars`, which receives the region's CIGAR ops in read order.  When
 * they exceed cigar_capacity the request completes with PHMM_ERR_LIMIT_EXCEEDED, *cigar_total set
 * and everything but cigars filled. */
typedef struct phmm_region_realign {
    const double* hap_priority;  /* [n_haps] */
    const uint16_t* clip_left;   /* [n_reads] or NULL (none) */
    const uint16_t* clip_right;  /* [n_reads] or NULL (none) */
    int32_t* best_hap;           /* out [n_reads] */
    struct phmm_sw_result* sw;   /* out [n_reads] (phmm_sw_result, declared with phmm_sw_align) */
    uint32_t* cigars;            /* out [cigar_capacity] */
    uint64_t cigar_capacity;
    uint64_t* cigar_total;       /* out, optional: ops the region's CIGARs need */
} phmm_region_realign;

/* phmm_submit_region with the realignment of the region's kept reads after the likelihoods (and the
 * genotyping, when events are given), in the same batch on the device (no reference counterpart as
 * one call: it joins call_pairhmm and the realignment that follows it per region). */
PHMM_API phmm_status phmm_submit_region_realign(phmm_engine* engine, const phmm_region_input* region,
                                                const phmm_region_events* events,
                                                const phmm_region_realign* realign, double* out, uint8_t* keep,
                                                uint32_t* n_kept, phmm_ticket* ticket);
/* *done = 1 once the request's results are in out (or it failed / was cancelled). */
PHMM_API phmm_status phmm_poll(phmm_engine* engine, phmm_ticket ticket, int32_t* done);
/* Blocks up to timeout_us (negative = forever).  Once the request is done it returns the request's
 * own status, reports its timing (optional, may be NULL: time queued before admission and time from
 * submit to completion, in microseconds) and releases the ticket.  On PHMM_ERR_TIMEOUT the ticket
 * stays valid. */
PHMM_API phmm_status phmm_wait(phmm_engine* engine, phmm_ticket ticket, int64_t timeout_us, double* queued_us,
                      double* total_us);
/* Cancels a request that has not been admitted to the device yet. */
PHMM_API phmm_status phmm_cancel(phmm_engine* engine, phmm_ticket ticket);

/* Counters of the serving loop since the engine's first submit (no reference counterpart: the
 * reference's region pool keeps no statistics). */
typedef struct phmm_server_stats {
    uint64_t requests_submitted;
    uint64_t requests_done;       /* completed or failed after admission */
    uint64_t batches;             /* device batches formed from the queue */
    uint64_t max_batch_regions;
    uint64_t queue_peak;          /* longest queue seen at submit */
    uint64_t cells_done;
    double batch_ms;              /* summed wall time of the batches, admission to results scattered */
    double device_ms;             /* summed device time of the batches' launch sequences */
    double max_batch_ms;          /* longest batch, admission to results scattered */
    double max_queue_ms;          /* longest wait of a request between submit and admission */
    uint64_t arena_grows;         /* device arena (re)allocations of the serving slots */
    uint64_t graph_captures;      /* CUDA graph captures of the serving slots */
    double max_setup_ms;          /* longest arena growth + graph capture inside one batch */
    double max_host_ms;           /* longest host part of one batch (gather, plan, scatter) */
    /* summed over the batches, in ms: gathering the requests into pinned staging, planning,
     * uploading and launching, waiting for the device (and the results' copy back), and
     * copying the results to the requests */
    double gather_ms, plan_ms, enqueue_ms, wait_ms, scatter_ms;
} phmm_server_stats;

PHMM_API phmm_status phmm_server_stats_get(phmm_engine* engine, phmm_server_stats* stats);

/* ---- several devices --------------------------------------------------------------------
 *
 * The reference runs regions in parallel on a host thread pool (haplotypecaller.cpp:105,
 * haplotypecaller_engine.cpp:119); regions are independent, so several GPUs shard whole regions with
 * nothing exchanged between them. */

/* Splits a batch's regions into n_parts parts balanced by cells (a region's cells: its total read
 * bases times its total haplotype bases): longest-processing-time greedy, regions in decreasing cell
 * order each to the part with the fewest cells so far (ties to the lower part), so that the largest
 * part holds at most the ideal share plus one region.  part_of_region[n_regions] receives each
 * region's part, cells_of_part[n_parts] each part's cells.  Host only; validates the batch like
 * phmm_compute_regions.  No reference counterpart. */
PHMM_API phmm_status phmm_partition_regions(const phmm_batch* batch, uint32_t n_parts, uint32_t* part_of_region,
                                            uint64_t* cells_of_part);

typedef struct phmm_device_set phmm_device_set;

/* One engine per listed device (a device may be listed twice: two engines, each with its own
 * arenas and streams).  cfg as for phmm_engine_create (NULL: defaults); its device field is
 * replaced by each listed device.  No reference counterpart. */
PHMM_API phmm_status phmm_device_set_create(const int32_t* devices, uint32_t n_devices, const phmm_config* cfg,
                                            phmm_device_set** out_set);
PHMM_API phmm_status phmm_device_set_destroy(phmm_device_set* set);
/* The engine of member `index` (owned by the set), for per-device calls. */
PHMM_API phmm_status phmm_device_set_engine(phmm_device_set* set, uint32_t index, phmm_engine** engine);
/* phmm_compute_regions over the set: the regions are partitioned as by phmm_partition_regions, each
 * part is gathered into its device's pinned staging and computed there (one host thread per
 * device, all at once), and every region's likelihoods land in its own range of out (the layout of
 * phmm_compute_regions; results identical to one engine's).  stats: sums over the devices, and the
 * longest device time.  Calls on one set are serialised. */
PHMM_API phmm_status phmm_device_set_compute_regions(phmm_device_set* set, const phmm_batch* batch, double* out,
                                                     uint8_t* pair_flags, phmm_stats* stats);
/* phmm_submit to the member with the fewest cells submitted and not yet waited for. */
PHMM_API phmm_status phmm_device_set_submit(phmm_device_set* set, const phmm_batch* region, double* out,
                                            uint8_t* pair_flags, phmm_ticket* ticket);
/* phmm_wait for a ticket of phmm_device_set_submit; device_index (optional) receives the member
 * that ran it. */
PHMM_API phmm_status phmm_device_set_wait(phmm_device_set* set, phmm_ticket ticket, int64_t timeout_us,
                                          double* queued_us, double* total_us, uint32_t* device_index);

/* ---- Smith-Waterman realignment of reads to their best haplotype ------------------------------
 *
 * Replaces the per-read aligner call of AlignmentUtils::create_read_aligned_to_ref
 * (genotype/utils/alignment_utils.cpp:571-579: seq1 = haplotype, seq2 = read, then
 * sw->avx_function(sw)) and of the assembler (apply/assemble/hc_assemble_cigar_cacl.c:417-428) with
 * one batched call.  Each item's results are the fields that call leaves in the lib_sw_avx context
 * (include/smithwaterman_common.h: score, max_i, max_j, alignment_offset, cigar, cigar_count), equal
 * to the reference's bit for bit: the int16 / int32 kernel choice of ro_sw_avx512_run
 * (lib/ro_sw/ro_sw.c:26-60), its recurrences, tie rules and trace-back (lib/ro_sw/sw_core_template.h,
 * lib/ro_sw/sw_cigar.c).  Inputs whose longer sequence has 2048 bases or more are refused as the
 * reference refuses them: alignment_offset 1, score 0, no CIGAR. */

typedef struct phmm_sw_item {
    uint64_t hap_offset;    /* byte offset of the haplotype (seq1) in hap_bases */
    uint64_t read_offset;   /* byte offset of the read (seq2) in read_bases */
    uint32_t hap_len;
    uint32_t read_len;
} phmm_sw_item;

typedef struct phmm_sw_result {
    int32_t score;
    int32_t alignment_offset;   /* haplotype position of the first aligned read base */
    int32_t max_i, max_j;       /* end cell of the alignment (haplotype, read) */
    uint32_t cigar_count;       /* CIGAR ops of the alignment (at most 2047) */
    uint32_t cigar_offset;      /* its first op in `cigars`; min(cigar_count, cigar_cap) ops stored */
} phmm_sw_result;

/* params = {match, mismatch, gap_open, gap_extend} (NULL: the genotyping parameters 10, -15, -30,
 * -5 of lib/sw_avx/sw_avx.c:15; the assembler uses 200, -150, -260, -11).  variant: 0 = the
 * reference's kernel choice, 1 = its int32 kernel, 2 = its int16 kernel.
 * CIGARs come back compact, in item order: item q's first min(cigar_count, cigar_cap) ops (BAM
 * encoding, length << 4 | op with M 0, I 1, D 2, S 4; read order) at cigars[results[q].cigar_offset].
 * cigar_cap bounds the ops stored per item (0: none; 2047 or more: all).  cigars holds
 * cigar_capacity ops; *cigar_total (optional) receives the ops the batch needs.  If they exceed
 * cigar_capacity the call returns PHMM_ERR_LIMIT_EXCEEDED with results filled and cigars untouched.
 * All pointers are host memory; the call copies in, runs on the engine's device and copies out
 * before it returns. */
PHMM_API phmm_status phmm_sw_align(phmm_engine* engine, const int32_t* params, int32_t variant, uint32_t n,
                                   const phmm_sw_item* items, const uint8_t* hap_bases, uint64_t hap_bytes,
                                   const uint8_t* read_bases, uint64_t read_bytes, uint32_t cigar_cap,
                                   phmm_sw_result* results, uint32_t* cigars, uint64_t cigar_capacity,
                                   uint64_t* cigar_total);

/* Device-resident Smith-Waterman batch (no reference counterpart: it exists to time the kernels with
 * the inputs already in HBM).  Created from host buffers, run `iterations` times back to back
 * (ms_per_run: CUDA-event time per run on the aligner's stream; class_ms[14], optional: time of each
 * kernel class in one more run: stripe widths 1-8, 10, 12, 16, 20, 24 read columns per lane, then the
 * 16-bit wrap-around class), results read back on demand (the layout of phmm_sw_align). */
typedef struct phmm_sw_resident phmm_sw_resident;
PHMM_API phmm_status phmm_sw_resident_create(phmm_engine* engine, const int32_t* params, int32_t variant,
                                             uint32_t n, const phmm_sw_item* items, const uint8_t* hap_bases,
                                             uint64_t hap_bytes, const uint8_t* read_bases, uint64_t read_bytes,
                                             uint32_t cigar_cap, phmm_sw_resident** out);
PHMM_API phmm_status phmm_sw_resident_run(phmm_sw_resident* resident, int32_t iterations, float* ms_per_run,
                                          float* class_ms);
PHMM_API phmm_status phmm_sw_resident_results(phmm_sw_resident* resident, phmm_sw_result* results,
                                              uint32_t* cigars, uint64_t cigar_capacity, uint64_t* cigar_total);
PHMM_API phmm_status phmm_sw_resident_destroy(phmm_sw_resident* resident);

#ifdef __cplusplus
}
#endif

#endif /* PHMM_B200_H */
