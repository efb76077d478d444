// PairHMM engine: one CUDA device, a growable device arena, and the batch pipeline
//   reset/prep -> FP32 class kernels (forked streams) -> FP64 class kernels -> results.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/phmm_b200.h"
#include "phmm_types.h"
#include "phmm_kernels.h"
#include "phmm_plan.h"

namespace phmm {

class SwAligner;
struct RealignBatch;

// Sizes an arena must hold.
struct Capacity {
    uint64_t regions = 0, reads = 0, haps = 0, read_bases = 0, hap_bases = 0, items = 0, rerun = 0, out = 0;
    uint64_t scratch_cols = 0;
    uint64_t events = 0, hap_allele = 0, allele_lk = 0, gl = 0;
    bool covers(const Capacity& o) const;
    Capacity grown_to(const Capacity& need) const;
    static Capacity max_of(const Capacity& a, const Capacity& b);
};

// One device arena with everything a batch needs, plus its streams, events and captured graph.
struct Slot {
    int id = 0;
    char* dev = nullptr;             // device arena
    size_t dev_bytes = 0;
    char* pinned = nullptr;          // pinned host staging for the plan arrays and descriptors
    size_t pinned_bytes = 0;
    Capacity cap;
    Capacity floor;                  // the arena is never sized below this (serving slots pre-size)
    bool overlap = false;            // serving slot: over-subscribed FP32 grids, prioritised streams
    // carved device pointers
    BatchDesc* d_desc = nullptr;
    char* d_desc_pristine = nullptr;  // the batch's descriptor block as uploaded, for replays
    ClassDesc* d_classes = nullptr;
    unsigned int* d_status = nullptr;
    RegionDesc* d_regions = nullptr;
    uint64_t *d_read_off = nullptr, *d_hap_off = nullptr;
    uint8_t *d_read_flags = nullptr, *d_hap_flags = nullptr;
    WorkItem* d_items = nullptr;
    RerunEntry* d_rerun = nullptr;
    double* d_out = nullptr;
    uint8_t* d_pair_flags = nullptr;
    uint8_t *d_rb = nullptr, *d_rq = nullptr, *d_ri = nullptr, *d_rd = nullptr, *d_rc = nullptr;
    uint8_t* d_hb = nullptr;
    uint8_t* d_mapq = nullptr;       // region API: MAPQ per read
    double* d_out2 = nullptr;        // region API: normalised likelihoods, kept reads first
    uint8_t* d_keep = nullptr;       // region API: kept flag per read
    uint32_t* d_nkept = nullptr;     // region API: kept reads per region
    EventDesc* d_events = nullptr;   // genotyping events
    int8_t* d_hap_allele = nullptr;
    double* d_allele_lk = nullptr;
    double* d_gl = nullptr;
    int32_t* d_best = nullptr;
    uint32_t *d_codes_inter = nullptr, *d_codes_intra = nullptr;
    void* d_scratch = nullptr;
    // execution
    cudaStream_t main = nullptr;
    cudaStream_t side[kNumClasses] = {};
    cudaEvent_t ev_fork = nullptr, ev_side[kNumClasses] = {}, ev_t0 = nullptr, ev_t1 = nullptr, ev_t2 = nullptr,
                ev_t3 = nullptr, ev_done = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool graph_flags = false;        // the captured graph writes pair flags
    TileTable graph_tiles{};         // tile table whose FP64 dependencies the graph encodes
    uint64_t launches = 0;           // kernels launched by the last pipeline run
    uint64_t arena_grows = 0;        // arena (re)allocations
    uint64_t graph_captures = 0;
    double setup_ms = 0.0;           // wall time spent growing the arena and capturing graphs
    // realignment of region-API reads to their best haplotypes (grown on demand)
    char* rdev = nullptr;
    size_t rdev_bytes = 0;
    char* rpin = nullptr;
    size_t rpin_bytes = 0;
};

class Engine {
public:
    static phmm_status create(const phmm_config* cfg, Engine** out, std::string& err);
    ~Engine();

    // Synchronous batch (thread-safe; calls are serialised on the engine's default slot).
    phmm_status compute(const phmm_batch& b, double* out, uint8_t* pair_flags, phmm_stats* stats, std::string& err);

    // Pieces used by the serving loop (phmm_serve.cpp), each on a caller-owned slot.
    // overlap: the slot's batches share the GPU with other slots' (serving): over-subscribed FP32
    // grids and prioritised class streams
    phmm_status make_slot(int id, Slot** out, std::string& err, bool overlap = false);
    void free_slot(Slot* s);
    // mapq: MAPQ per read, region-API plans only (their raw qualities are prepared on the device).
    // raw_sent: the batch's bases and qualities were already copied to this arena (upload_raw) and it
    // has not grown since; they are not copied again.
    phmm_status enqueue(Slot& s, const Plan& plan, const phmm_batch& b, bool want_flags, std::string& err,
                        const uint8_t* mapq = nullptr, bool raw_sent = false);
    // Region-API plans: out receives the normalised matrices (kept reads first), keep the kept flag
    // of every read and n_kept the kept reads of every region.
    // Genotyping outputs (plans with events): gl [gl_total], best [events], allele_lk (optional).
    // out may be null to skip the likelihood matrix.
    phmm_status finish(Slot& s, const Plan& plan, double* out, uint8_t* pair_flags, phmm_stats* stats,
                       std::string& err, uint8_t* keep = nullptr, uint32_t* n_kept = nullptr, double* gl = nullptr,
                       int32_t* best = nullptr, double* allele_lk = nullptr);
    // Upload only (descriptor, plan arrays, reads, haplotypes); then run the device pipeline, with
    // restore = true resetting the descriptor from its pristine device copy first (replays).
    phmm_status upload(Slot& s, const Plan& plan, const phmm_batch& b, std::string& err,
                       const uint8_t* mapq = nullptr, bool raw_sent = false);
    // Copies a validated batch's bases and qualities into the slot's arena when it already holds
    // them (returns false, copying nothing, otherwise): the copies then overlap the host planning.
    bool upload_raw(Slot& s, const BatchScan& sc, const phmm_batch& b);
    // Allocates the slot's arena for at least capacity c now (no-op if it already covers it).
    phmm_status reserve(Slot& s, const Capacity& c, std::string& err);
    phmm_status run(Slot& s, const Plan& plan, bool want_flags, bool restore, std::string& err);
    // Captures the slot's pipeline graph again if the graph is missing or was captured for other
    // flags or tiles (no-op without graphs).
    phmm_status ensure_graph(Slot& s, const Plan& plan, bool want_flags, std::string& err);
    phmm_status fp32_fma_peak(double* scalar_tflops, double* packed_tflops, std::string& err);

    // FP32 tile shapes used for new plans (thread-safe copy / replace).
    TileTable tiles() const;
    phmm_status set_tiles(const TileTable& t, std::string& err);
    // Planner limits with a tile table (t must outlive the returned limits).
    static PlanLimits limits_with(const TileTable& t)
    {
        PlanLimits l;
        l.tiles = &t;
        return l;
    }
    // Runs an uploaded plan once with every class alone on the slot's main stream, timing each
    // launch with CUDA events (class_ms[kNumClasses], 0 where a class has no work).
    phmm_status profile_classes(Slot& s, const Plan& plan, float* class_ms, std::string& err);
    // Recomputes every pair of an uploaded plan with the all-FP64 check arithmetic (plain multiply
    // and add, FP64 end to end, every result flushed below 2^-1022) and copies the log10 values to
    // out (the layout of compute(); pairs with an empty read or haplotype NaN).  The slot's results
    // are overwritten; run the plan again to get the engine's own results back.
    phmm_status check_fp64(Slot& s, const Plan& plan, double* out, std::string& err);
    // Measures the FP32 pass of one class alone on an uploaded plan: best of `reps` launches (ms).
    phmm_status time_fp32_class(Slot& s, const Plan& plan, int cls, int reps, float* best_ms, std::string& err);
    // Runs the tile-shape autotuner and installs its table (phmm_tune.cpp).
    phmm_status autotune(phmm_tune_report* report, std::string& err);
    // Realignment of a batch's kept region-API reads to their best haplotypes, on the slot's main
    // stream after the pipeline enqueue() launched (best haplotypes, Smith-Waterman, CIGAR
    // compaction; results and CIGAR sizes copied back before finish() returns); realign_finish()
    // after finish() fetches the CIGARs into rb.
    phmm_status realign_enqueue(Slot& s, RealignBatch& rb, std::string& err);
    phmm_status realign_finish(Slot& s, RealignBatch& rb, std::string& err);
    // The engine's Smith-Waterman aligner (phmm_sw.cu), created on first use.
    phmm_status sw_aligner(SwAligner** out, std::string& err);

    int device() const { return dev_; }
    int num_sms() const { return sms_; }
    const phmm_config& config() const { return cfg_; }
    uint64_t scratch_bytes() const;  // device bytes of the stripe scratch rows (multi-stripe reads)
    uint64_t arena_bytes(const Capacity& c) const;  // device bytes of an arena of capacity c

private:
    Engine() = default;
    phmm_status ensure_capacity(Slot& s, const Plan& plan, std::string& err);
    phmm_status launch_pipeline(Slot& s, bool want_flags, const Plan* plan, const TileTable& tiles, std::string& err);
    phmm_status capture_graph(Slot& s, bool want_flags, const TileTable& tiles, std::string& err);
    int grid_for(int precision, int cls, uint32_t work, unsigned int waves = 1) const;
    uint64_t scratch_warps() const;
    // First warp row of scratch region r (0: FP32 multi-stripe classes, 1 + m: the FP64 multi-stripe
    // class of mode m; 1 + kModes32: the total).
    uint64_t scratch_offset_warps(int region) const;
    // compute() of a batch of at least cfg_.chunk_cells cells: region chunks alternating between the
    // default slot and chunk_slot_, each planned and uploaded while the previous one runs.  *ran is
    // false when the batch does not split (the caller then runs it as one pipeline).
    phmm_status compute_chunked(const phmm_batch& b, const BatchScan& sc, double* out, uint8_t* pair_flags,
                                phmm_stats* stats, std::string& err, bool* ran);

    phmm_config cfg_{};
    int dev_ = 0;
    int sms_ = 0;
    int occ_[2][kNumClasses] = {};
    int full_grid(int precision, int cls, unsigned int waves) const;  // resident blocks (times waves)
    // device probability tables
    void* d_tables_ = nullptr;
    ProbTables<float> tf_{};
    ProbTables<double> td_{};
    const double* d_jacobian_ = nullptr;  // genotyping Jacobian table (inside d_tables_)
    double log10_two_ = 0.0;
    Slot* default_slot_ = nullptr;
    Slot* chunk_slot_ = nullptr;          // second slot of the chunked synchronous path (made on first use)
    cudaEvent_t ev_span_ = nullptr;       // start of a chunked call's device pipeline
    SwAligner* sw_ = nullptr;
    std::mutex sw_mu_;
    std::mutex mu_;
    mutable std::mutex tiles_mu_;
    TileTable tiles_ = TileTable::defaults();
};

// Installs the table tuned for this engine's device earlier in the process, or runs the autotuner
// (phmm_tune.cpp).
phmm_status autotune_once(Engine& e, std::string& err);

}  // namespace phmm
