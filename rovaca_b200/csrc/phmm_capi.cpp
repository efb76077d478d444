// extern "C" entry points of include/phmm_b200.h.  No exception crosses this boundary: every
// entry point catches, records the detail for phmm_last_error() and returns a status.
#include <cstddef>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "../../include/phmm_b200.h"
#include "phmm_capi_internal.h"
#include "phmm_engine.h"
#include "phmm_plan.h"
#include "phmm_sw.h"

static_assert(sizeof(phmm_tile_table) == sizeof(phmm::TileTable), "tile table layouts differ");
static_assert(PHMM_FP32_CLASSES == phmm::kClasses32 && PHMM_FP64_CLASSES == phmm::kClasses64 &&
                  PHMM_TILE_MODES == phmm::kModes32 && PHMM_LEN_BUCKETS == phmm::kLenBuckets,
              "class counts differ between the C ABI and the kernels");

static_assert(sizeof(phmm_sw_item) == sizeof(phmm::SwItem) &&
                  offsetof(phmm_sw_item, hap_len) == offsetof(phmm::SwItem, hap_len) &&
                  offsetof(phmm_sw_item, read_offset) == offsetof(phmm::SwItem, read_start),
              "Smith-Waterman item layouts differ");

namespace phmm {

namespace {
thread_local std::string g_last_error;
}

phmm_status set_error(phmm_status st, const std::string& msg)
{
    g_last_error = msg;
    return st;
}

void clear_error() { g_last_error.clear(); }

Engine* engine_of(phmm_engine* e) { return reinterpret_cast<Engine*>(e); }

}  // namespace phmm

using phmm::set_error;

#define PHMM_GUARD_BEGIN try {
#define PHMM_GUARD_END                                                              \
    }                                                                               \
    catch (const std::bad_alloc&)                                                   \
    {                                                                               \
        return set_error(PHMM_ERR_OUT_OF_MEMORY, "host allocation failed");         \
    }                                                                               \
    catch (const std::exception& ex)                                                \
    {                                                                               \
        return set_error(PHMM_ERR_INTERNAL, ex.what());                             \
    }                                                                               \
    catch (...)                                                                     \
    {                                                                               \
        return set_error(PHMM_ERR_INTERNAL, "unknown exception");                   \
    }

extern "C" {

const char* phmm_status_string(phmm_status status)
{
    switch (status) {
    case PHMM_OK: return "ok";
    case PHMM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case PHMM_ERR_LIMIT_EXCEEDED: return "region exceeds the PairHMM limits";
    case PHMM_ERR_OUT_OF_MEMORY: return "out of memory";
    case PHMM_ERR_CUDA: return "CUDA error";
    case PHMM_ERR_NOT_INITIALIZED: return "engine not initialised";
    case PHMM_ERR_TIMEOUT: return "timed out";
    case PHMM_ERR_CANCELLED: return "cancelled";
    case PHMM_ERR_QUEUE_FULL: return "queue full";
    case PHMM_ERR_DEVICE_STATUS: return "kernel reported an error status";
    case PHMM_ERR_NO_DEVICE: return "no usable CUDA device";
    case PHMM_ERR_INTERNAL: return "internal error";
    }
    return "unknown status";
}

const char* phmm_last_error(void) { return phmm::g_last_error.c_str(); }

const char* phmm_version(void)
{
    return "phmm_b200 1.0 (sm_100a; FP32 wavefront K=1..8 + multi-stripe, inter/intra variants; FP64 recompute)";
}

phmm_status phmm_engine_create(const phmm_config* cfg, phmm_engine** out_engine)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!out_engine) return set_error(PHMM_ERR_INVALID_ARGUMENT, "out_engine is null");
    *out_engine = nullptr;
    phmm::Engine* e = nullptr;
    std::string err;
    phmm_status st = phmm::Engine::create(cfg, &e, err);
    if (st != PHMM_OK) return set_error(st, err);
    *out_engine = reinterpret_cast<phmm_engine*>(e);
    return PHMM_OK;
    PHMM_GUARD_END
}

phmm_status phmm_engine_destroy(phmm_engine* engine)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    phmm::server_release(engine);
    delete phmm::engine_of(engine);
    return PHMM_OK;
    PHMM_GUARD_END
}

phmm_status phmm_compute_regions(phmm_engine* engine, const phmm_batch* batch, double* out, uint8_t* pair_flags,
                                 phmm_stats* stats)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    if (!batch) return set_error(PHMM_ERR_INVALID_ARGUMENT, "batch is null");
    std::string err;
    phmm_status st = phmm::engine_of(engine)->compute(*batch, out, pair_flags, stats, err);
    if (st != PHMM_OK) return set_error(st, err);
    return PHMM_OK;
    PHMM_GUARD_END
}

}  // extern "C"

struct phmm_resident {
    phmm::Engine* eng = nullptr;
    phmm::Slot* slot = nullptr;
    phmm::Plan plan;
    bool flags = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

extern "C" {

phmm_status phmm_resident_destroy(phmm_resident* r)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!r) return set_error(PHMM_ERR_INVALID_ARGUMENT, "resident is null");
    if (r->eng) cudaSetDevice(r->eng->device());
    if (r->e0) cudaEventDestroy(r->e0);
    if (r->e1) cudaEventDestroy(r->e1);
    if (r->slot) r->eng->free_slot(r->slot);
    delete r;
    return PHMM_OK;
    PHMM_GUARD_END
}

phmm_status phmm_resident_create(phmm_engine* engine, const phmm_batch* batch, int32_t want_flags,
                                 phmm_resident** out_resident)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    if (!batch || !out_resident) return set_error(PHMM_ERR_INVALID_ARGUMENT, "batch or out_resident is null");
    *out_resident = nullptr;
    auto* r = new phmm_resident();
    r->eng = phmm::engine_of(engine);
    r->flags = want_flags != 0;
    std::string err;
    const phmm::TileTable tiles = r->eng->tiles();
    phmm_status st = phmm::build_plan(*batch, phmm::Engine::limits_with(tiles), r->plan, err);
    if (st == PHMM_OK) st = r->eng->make_slot(1000, &r->slot, err);
    if (st == PHMM_OK && (cudaEventCreate(&r->e0) != cudaSuccess || cudaEventCreate(&r->e1) != cudaSuccess)) {
        err = "event creation failed";
        st = PHMM_ERR_CUDA;
    }
    if (st == PHMM_OK) st = r->eng->upload(*r->slot, r->plan, *batch, err);
    if (st == PHMM_OK) st = r->eng->run(*r->slot, r->plan, r->flags, false, err);
    if (st == PHMM_OK && cudaStreamSynchronize(r->slot->main) != cudaSuccess) {
        err = std::string("first run failed: ") + cudaGetErrorString(cudaGetLastError());
        st = PHMM_ERR_CUDA;
    }
    if (st != PHMM_OK) {
        phmm_resident_destroy(r);
        return set_error(st, err);
    }
    *out_resident = r;
    return PHMM_OK;
    PHMM_GUARD_END
}

phmm_status phmm_resident_run(phmm_resident* r, int32_t iterations, phmm_stats* stats)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!r || !r->slot) return set_error(PHMM_ERR_INVALID_ARGUMENT, "resident is null");
    if (iterations < 1) return set_error(PHMM_ERR_INVALID_ARGUMENT, "iterations < 1");
    std::string err;
    cudaSetDevice(r->eng->device());
    cudaStream_t m = r->slot->main;
    if (cudaEventRecord(r->e0, m) != cudaSuccess) return set_error(PHMM_ERR_CUDA, "event record failed");
    for (int i = 0; i < iterations; ++i) {
        phmm_status st = r->eng->run(*r->slot, r->plan, r->flags, true, err);
        if (st != PHMM_OK) return set_error(st, err);
    }
    cudaEventRecord(r->e1, m);
    cudaError_t e = cudaEventSynchronize(r->e1);
    if (e != cudaSuccess) return set_error(PHMM_ERR_CUDA, std::string("resident run: ") + cudaGetErrorString(e));
    if (stats) {
        float ms = 0, f32 = 0, f64 = 0;
        cudaEventElapsedTime(&ms, r->e0, r->e1);
        cudaEventElapsedTime(&f32, r->slot->ev_t0, r->slot->ev_t1);
        cudaEventElapsedTime(&f64, r->slot->ev_t1, r->slot->ev_t2);
        *stats = phmm_stats{};
        stats->regions = r->plan.n_regions;
        stats->pairs = r->plan.pairs * (uint64_t)iterations;
        stats->cells = r->plan.cells * (uint64_t)iterations;
        stats->work_items = r->plan.items.size();
        stats->kernel_launches = r->slot->launches * (uint64_t)iterations;
        stats->device_ms = ms;
        stats->fp32_ms = f32;  // last iteration
        stats->fp64_ms = f64;  // last iteration
    }
    return PHMM_OK;
    PHMM_GUARD_END
}

phmm_status phmm_resident_profile(phmm_resident* r, float* class_ms, uint64_t* class_cells)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!r || !r->slot) return set_error(PHMM_ERR_INVALID_ARGUMENT, "resident is null");
    if (!class_ms) return set_error(PHMM_ERR_INVALID_ARGUMENT, "class_ms is null");
    std::string err;
    phmm_status st = r->eng->profile_classes(*r->slot, r->plan, class_ms, err);
    if (st != PHMM_OK) return set_error(st, err);
    if (class_cells) {
        const phmm::Plan& p = r->plan;
        for (int c = 0; c < phmm::kNumClasses; ++c) class_cells[c] = 0;
        for (int c = 0; c < phmm::kClasses32; ++c)
            for (uint32_t i = p.classes[c].item_off; i < p.classes[c].item_off + p.classes[c].n_items; ++i) {
                const phmm::WorkItem& it = p.items[i];
                const phmm::RegionDesc& rg = p.regions[it.region];
                const uint64_t cols = p.hap_off[rg.hap_begin + it.hap_hi] - p.hap_off[rg.hap_begin + it.hap_lo];
                uint64_t rows = 0;
                for (int k = 0; k < 2; ++k)
                    if (it.read[k] != phmm::kNoRead) rows += p.read_off[it.read[k] + 1] - p.read_off[it.read[k]];
                class_cells[c] += rows * cols;
            }
    }
    return PHMM_OK;
    PHMM_GUARD_END
}

phmm_status phmm_resident_results(phmm_resident* r, double* out, uint8_t* pair_flags)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!r || !r->slot) return set_error(PHMM_ERR_INVALID_ARGUMENT, "resident is null");
    if (pair_flags && !r->flags) return set_error(PHMM_ERR_INVALID_ARGUMENT, "resident batch was created without flags");
    if (r->plan.out_total && !out) return set_error(PHMM_ERR_INVALID_ARGUMENT, "out is null");
    std::string err;
    cudaSetDevice(r->eng->device());
    phmm_stats st{};
    phmm_status s = r->eng->finish(*r->slot, r->plan, out, pair_flags, &st, err);
    return s == PHMM_OK ? PHMM_OK : set_error(s, err);
    PHMM_GUARD_END
}

phmm_status phmm_resident_check_fp64(phmm_resident* r, double* out)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!r || !r->slot) return set_error(PHMM_ERR_INVALID_ARGUMENT, "resident is null");
    if (r->plan.out_total && !out) return set_error(PHMM_ERR_INVALID_ARGUMENT, "out is null");
    std::string err;
    phmm_status s = r->eng->check_fp64(*r->slot, r->plan, out, err);
    return s == PHMM_OK ? PHMM_OK : set_error(s, err);
    PHMM_GUARD_END
}

phmm_status phmm_fp32_fma_peak(phmm_engine* engine, double* scalar_tflops, double* packed_tflops)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    std::string err;
    phmm_status st = phmm::engine_of(engine)->fp32_fma_peak(scalar_tflops, packed_tflops, err);
    return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    PHMM_GUARD_END
}

phmm_status phmm_host_plan_summary(const phmm_batch* batch, const phmm_tile_table* tiles,
                                   uint32_t class_items[PHMM_FP32_CLASSES], uint64_t class_pairs[PHMM_FP64_CLASSES],
                                   uint64_t* pairs, uint64_t* cells)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!batch) return set_error(PHMM_ERR_INVALID_ARGUMENT, "batch is null");
    phmm::Plan plan;
    std::string err;
    phmm::TileTable t = phmm::TileTable::defaults();
    if (tiles) std::memcpy(&t, tiles, sizeof(t));
    phmm_status st = phmm::build_plan(*batch, phmm::Engine::limits_with(t), plan, err);
    if (st != PHMM_OK) return set_error(st, err);
    for (int c = 0; c < phmm::kClasses32; ++c)
        if (class_items) class_items[c] = plan.classes[c].n_items;
    for (int c = 0; c < phmm::kClasses64; ++c)
        if (class_pairs) class_pairs[c] = plan.classes[phmm::kClasses32 + c].rerun_cap;
    if (pairs) *pairs = plan.pairs;
    if (cells) *cells = plan.cells;
    return PHMM_OK;
    PHMM_GUARD_END
}

void phmm_tile_table_default(phmm_tile_table* table)
{
    if (!table) return;
    const phmm::TileTable t = phmm::TileTable::defaults();
    std::memcpy(table, &t, sizeof(t));
}

phmm_status phmm_engine_get_tiles(phmm_engine* engine, phmm_tile_table* table)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    if (!table) return set_error(PHMM_ERR_INVALID_ARGUMENT, "table is null");
    const phmm::TileTable t = phmm::engine_of(engine)->tiles();
    std::memcpy(table, &t, sizeof(t));
    return PHMM_OK;
    PHMM_GUARD_END
}

phmm_status phmm_engine_set_tiles(phmm_engine* engine, const phmm_tile_table* table)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    if (!table) return set_error(PHMM_ERR_INVALID_ARGUMENT, "table is null");
    phmm::TileTable t;
    std::memcpy(&t, table, sizeof(t));
    std::string err;
    phmm_status st = phmm::engine_of(engine)->set_tiles(t, err);
    return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    PHMM_GUARD_END
}

phmm_status phmm_engine_autotune(phmm_engine* engine, phmm_tune_report* report)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    std::string err;
    phmm_status st = phmm::engine_of(engine)->autotune(report, err);
    return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    PHMM_GUARD_END
}

static phmm::SwParams sw_params(const int32_t* params)
{
    if (!params) return phmm::SwParams{10, -15, -30, -5};  // sw_parameters_genotype, lib/sw_avx/sw_avx.c:15
    return phmm::SwParams{params[0], params[1], params[2], params[3]};
}

static phmm_status sw_get(phmm_engine* engine, phmm::SwAligner** a)
{
    std::string err;
    phmm_status st = phmm::engine_of(engine)->sw_aligner(a, err);
    return st == PHMM_OK ? PHMM_OK : set_error(st, err);
}

phmm_status phmm_sw_align(phmm_engine* engine, const int32_t* params, int32_t variant, uint32_t n,
                          const phmm_sw_item* items, const uint8_t* hap_bases, uint64_t hap_bytes,
                          const uint8_t* read_bases, uint64_t read_bytes, uint32_t cigar_cap, phmm_sw_result* results,
                          uint32_t* cigars, uint64_t cigar_capacity, uint64_t* cigar_total)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (cigar_total) *cigar_total = 0;
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    if (variant < 0 || variant > 2) return set_error(PHMM_ERR_INVALID_ARGUMENT, "variant must be 0, 1 or 2");
    if (n == 0) return PHMM_OK;
    if (!items || !results || (hap_bytes && !hap_bases) || (read_bytes && !read_bases) || (cigar_capacity && !cigars))
        return set_error(PHMM_ERR_INVALID_ARGUMENT, "null buffer");
    phmm::SwAligner* a = nullptr;
    phmm_status st = sw_get(engine, &a);
    if (st != PHMM_OK) return st;
    std::string err;
    st = a->align(sw_params(params), variant, n, reinterpret_cast<const phmm::SwItem*>(items), hap_bases, hap_bytes,
                  read_bases, read_bytes, cigar_cap, results, cigars, cigar_capacity, cigar_total, nullptr, err);
    return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    PHMM_GUARD_END
}

struct phmm_sw_resident {
    phmm::SwAligner* aligner = nullptr;
    phmm::SwAligner::Resident* res = nullptr;
};

phmm_status phmm_sw_resident_create(phmm_engine* engine, const int32_t* params, int32_t variant, uint32_t n,
                                    const phmm_sw_item* items, const uint8_t* hap_bases, uint64_t hap_bytes,
                                    const uint8_t* read_bases, uint64_t read_bytes, uint32_t cigar_cap,
                                    phmm_sw_resident** out)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!out) return set_error(PHMM_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    if (variant < 0 || variant > 2) return set_error(PHMM_ERR_INVALID_ARGUMENT, "variant must be 0, 1 or 2");
    if ((n && !items) || (hap_bytes && !hap_bases) || (read_bytes && !read_bases))
        return set_error(PHMM_ERR_INVALID_ARGUMENT, "null buffer");
    phmm::SwAligner* a = nullptr;
    phmm_status st = sw_get(engine, &a);
    if (st != PHMM_OK) return st;
    std::string err;
    phmm::SwAligner::Resident* r = nullptr;
    st = a->resident_create(sw_params(params), variant, n, reinterpret_cast<const phmm::SwItem*>(items), hap_bases,
                            hap_bytes, read_bases, read_bytes, cigar_cap, &r, err);
    if (st != PHMM_OK) return set_error(st, err);
    *out = new phmm_sw_resident{a, r};
    return PHMM_OK;
    PHMM_GUARD_END
}

phmm_status phmm_sw_resident_run(phmm_sw_resident* resident, int32_t iterations, float* ms_per_run, float* class_ms)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!resident) return set_error(PHMM_ERR_INVALID_ARGUMENT, "resident is null");
    if (iterations < 0) return set_error(PHMM_ERR_INVALID_ARGUMENT, "iterations must be >= 0");
    std::string err;
    phmm_status st = resident->aligner->resident_run(resident->res, iterations, ms_per_run, class_ms, err);
    return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    PHMM_GUARD_END
}

phmm_status phmm_sw_resident_results(phmm_sw_resident* resident, phmm_sw_result* results, uint32_t* cigars,
                                     uint64_t cigar_capacity, uint64_t* cigar_total)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (cigar_total) *cigar_total = 0;
    if (!resident) return set_error(PHMM_ERR_INVALID_ARGUMENT, "resident is null");
    if (cigar_capacity && !cigars) return set_error(PHMM_ERR_INVALID_ARGUMENT, "null buffer");
    std::string err;
    phmm_status st = resident->aligner->resident_results(resident->res, results, cigars, cigar_capacity, cigar_total,
                                                         err);
    return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    PHMM_GUARD_END
}

phmm_status phmm_sw_resident_destroy(phmm_sw_resident* resident)
{
    PHMM_GUARD_BEGIN
    phmm::clear_error();
    if (!resident) return PHMM_OK;
    resident->aligner->resident_destroy(resident->res);
    delete resident;
    return PHMM_OK;
    PHMM_GUARD_END
}

}  // extern "C"
