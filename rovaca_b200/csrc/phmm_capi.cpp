// extern "C" entry points of include/phmm_b200.h.  No exception crosses this boundary: every
// entry point catches, records the detail for phmm_last_error() and returns a status.
#include <exception>
#include <new>
#include <string>

#include "../../include/phmm_b200.h"
#include "phmm_capi_internal.h"
#include "phmm_engine.h"

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
