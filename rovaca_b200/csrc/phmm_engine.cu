// PairHMM engine runtime (see phmm_engine.h).
//
// Device arena layout (one cudaMalloc per slot, 256-byte aligned sections):
//   descriptor block  BatchDesc | ClassDesc x 18 | status words     (one H2D copy per batch)
//   plan arrays       regions, read_off, hap_off, read/hap N flags, work items
//   read data         bases, q, ins, del, gcp (1 byte per base each)
//   haplotypes        bases, then two u32 match-code streams with guard codes on both ends
//   region API        MAPQ and kept flag per read, kept count per region
//   results           likelihoods (f64), pair flags (u8), normalised likelihoods (f64, region API),
//                     FP64 rerun slots (16 B per pair)
//   scratch           per-warp stripe row for reads longer than 256 (3 values per column)
// The arena only grows; all kernel arguments are arena pointers, so a graph captured for an arena
// replays for every batch that fits it.
#include "phmm_engine.h"
#include "phmm_sw.h"

#include <algorithm>
#include <chrono>
#include <cstring>

#include "phmm_regionk.h"
#include "phmm_tables.h"

// Serving slots share the GPU with the other slots' batches.  Their FP32 single-stripe grids are
// kOverlapWaves times the resident warps, each warp taking an equal share of its class's items and
// exiting, so SMs free up during the pass; their FP32 classes run longest reads first on
// low-priority streams and their FP64 classes on high-priority streams, so an FP64 class whose
// sources have finished takes the SMs that FP32 blocks free, and a batch finishes before the next
// slot's FP32 work has drained.  Measured on B200 (serving loop, 2,000-region pool, 95% of the
// end-to-end batched rate): with 3 slots p50/p99 293/464 ms without, 142/208 ms with; with 5 slots
// 102/183 ms without, 37/57 ms with.  A lone batch (the resident and chunked paths) gains nothing
// from either (1% slower): its FP64 pass is work at full occupancy, not idle SMs.
constexpr unsigned int kOverlapWaves = 4;

namespace phmm {

#define PHMM_CK(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            err = std::string(#call) + " failed: " + cudaGetErrorString(e_);             \
            return PHMM_ERR_CUDA;                                                        \
        }                                                                                \
    } while (0)

namespace {

size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

constexpr size_t kDescBytes = sizeof(BatchDesc) + sizeof(ClassDesc) * kNumClasses + 4 * sizeof(unsigned int);
// Default phmm_config.chunk_cells: a batch of this many cells keeps the device busy for about 17 ms,
// several times what planning and uploading its first chunk take.
constexpr uint64_t kDefaultChunkCells = 40000000000ull;

// Carves the arena for capacity c starting at base (nullptr: only measure).  Returns the size.
size_t carve(const Capacity& c, char* base, Slot* s)
{
    size_t o = 0;
    auto take = [&](size_t bytes) -> char* {
        const size_t at = o;
        o = align_up(o + std::max<size_t>(bytes, 1));
        return base ? base + at : nullptr;
    };
    char* desc = take(kDescBytes);
    char* desc_pristine = take(kDescBytes);
    char* regions = take(c.regions * sizeof(RegionDesc));
    char* read_off = take((c.reads + 1) * sizeof(uint64_t));
    char* hap_off = take((c.haps + 1) * sizeof(uint64_t));
    char* read_flags = take(c.reads);
    char* hap_flags = take(c.haps);
    char* items = take(c.items * sizeof(WorkItem));
    char* rb = take(c.read_bases);
    char* rq = take(c.read_bases);
    char* ri = take(c.read_bases);
    char* rd = take(c.read_bases);
    char* rc = take(c.read_bases);
    char* hb = take(c.hap_bases);
    char* mapq = take(c.reads);
    char* keep = take(c.reads);
    char* nkept = take(c.regions * sizeof(uint32_t));
    char* ci = take((c.hap_bases + 2 * kCodePad) * sizeof(uint32_t));
    char* ca = take((c.hap_bases + 2 * kCodePad) * sizeof(uint32_t));
    char* out = take(c.out * sizeof(double));
    char* pf = take(c.out);
    char* out2 = take(c.out * sizeof(double));
    char* events = take(c.events * sizeof(EventDesc));
    char* hap_allele = take(c.hap_allele);
    char* allele_lk = take(c.allele_lk * sizeof(double));
    char* gl = take(c.gl * sizeof(double));
    char* best = take(c.events * sizeof(int32_t));
    char* rerun = take(c.rerun * sizeof(RerunEntry));
    char* scratch = take(c.scratch_cols * 3 * sizeof(double));  // c.scratch_cols counts all warps' columns
    if (s) {
        s->d_desc = (BatchDesc*)desc;
        s->d_desc_pristine = desc_pristine;
        s->d_classes = (ClassDesc*)(desc + sizeof(BatchDesc));
        s->d_status = (unsigned int*)(desc + sizeof(BatchDesc) + sizeof(ClassDesc) * kNumClasses);
        s->d_regions = (RegionDesc*)regions;
        s->d_read_off = (uint64_t*)read_off;
        s->d_hap_off = (uint64_t*)hap_off;
        s->d_read_flags = (uint8_t*)read_flags;
        s->d_hap_flags = (uint8_t*)hap_flags;
        s->d_items = (WorkItem*)items;
        s->d_rb = (uint8_t*)rb;
        s->d_rq = (uint8_t*)rq;
        s->d_ri = (uint8_t*)ri;
        s->d_rd = (uint8_t*)rd;
        s->d_rc = (uint8_t*)rc;
        s->d_hb = (uint8_t*)hb;
        s->d_mapq = (uint8_t*)mapq;
        s->d_keep = (uint8_t*)keep;
        s->d_nkept = (uint32_t*)nkept;
        s->d_out2 = (double*)out2;
        s->d_events = (EventDesc*)events;
        s->d_hap_allele = (int8_t*)hap_allele;
        s->d_allele_lk = (double*)allele_lk;
        s->d_gl = (double*)gl;
        s->d_best = (int32_t*)best;
        s->d_codes_inter = (uint32_t*)ci;
        s->d_codes_intra = (uint32_t*)ca;
        s->d_out = (double*)out;
        s->d_pair_flags = (uint8_t*)pf;
        s->d_rerun = (RerunEntry*)rerun;
        s->d_scratch = scratch;
    }
    return o;
}

// Pinned staging: descriptor block followed by the plan arrays.
size_t pinned_bytes_for(const Capacity& c)
{
    return align_up(kDescBytes) + align_up(c.regions * sizeof(RegionDesc)) + align_up((c.reads + 1) * 8) +
           align_up((c.haps + 1) * 8) + align_up(c.reads) + align_up(c.haps) + align_up(c.items * sizeof(WorkItem)) +
           align_up(c.events * sizeof(EventDesc)) + align_up(c.hap_allele);
}

Capacity need_of(const Plan& p, uint64_t scratch_warps)
{
    Capacity c;
    c.regions = p.n_regions;
    c.reads = p.n_reads;
    c.haps = p.n_haps;
    c.read_bases = p.read_bases;
    c.hap_bases = p.hap_bases;
    c.items = p.items.size();
    c.rerun = p.rerun_slots;
    c.out = p.out_total;
    c.scratch_cols = p.max_multi_stream ? scratch_warps * (uint64_t)PlanLimits().max_stream_multi : 0;
    c.events = p.events.size();
    c.hap_allele = p.hap_allele.size();
    c.allele_lk = p.allele_lk_total;
    c.gl = p.gl_total;
    return c;
}

}  // namespace

bool Capacity::covers(const Capacity& o) const
{
    return regions >= o.regions && reads >= o.reads && haps >= o.haps && read_bases >= o.read_bases &&
           hap_bases >= o.hap_bases && items >= o.items && rerun >= o.rerun && out >= o.out &&
           scratch_cols >= o.scratch_cols && events >= o.events && hap_allele >= o.hap_allele &&
           allele_lk >= o.allele_lk && gl >= o.gl;
}

Capacity Capacity::max_of(const Capacity& a, const Capacity& b)
{
    Capacity c;
    c.regions = std::max(a.regions, b.regions);
    c.reads = std::max(a.reads, b.reads);
    c.haps = std::max(a.haps, b.haps);
    c.read_bases = std::max(a.read_bases, b.read_bases);
    c.hap_bases = std::max(a.hap_bases, b.hap_bases);
    c.items = std::max(a.items, b.items);
    c.rerun = std::max(a.rerun, b.rerun);
    c.out = std::max(a.out, b.out);
    c.scratch_cols = std::max(a.scratch_cols, b.scratch_cols);
    c.events = std::max(a.events, b.events);
    c.hap_allele = std::max(a.hap_allele, b.hap_allele);
    c.allele_lk = std::max(a.allele_lk, b.allele_lk);
    c.gl = std::max(a.gl, b.gl);
    return c;
}

Capacity Capacity::grown_to(const Capacity& need) const
{
    auto g = [](uint64_t cur, uint64_t want) { return want <= cur ? cur : std::max(want, cur + cur / 2); };
    Capacity c;
    c.regions = g(regions, need.regions);
    c.reads = g(reads, need.reads);
    c.haps = g(haps, need.haps);
    c.read_bases = g(read_bases, need.read_bases);
    c.hap_bases = g(hap_bases, need.hap_bases);
    c.items = g(items, need.items);
    c.rerun = g(rerun, need.rerun);
    c.out = g(out, need.out);
    c.scratch_cols = std::max(scratch_cols, need.scratch_cols);
    c.events = g(events, need.events);
    c.hap_allele = g(hap_allele, need.hap_allele);
    c.allele_lk = g(allele_lk, need.allele_lk);
    c.gl = g(gl, need.gl);
    return c;
}

phmm_status Engine::create(const phmm_config* cfg, Engine** out, std::string& err)
{
    *out = nullptr;
    Engine* e = new Engine();
    if (cfg) {
        e->cfg_ = *cfg;
    } else {
        e->cfg_.device = 0;
        e->cfg_.use_cuda_graph = 1;
        e->cfg_.autotune = 1;
    }
    if (e->cfg_.hbm_budget_bytes == 0) e->cfg_.hbm_budget_bytes = 40ull << 30;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        err = "no CUDA device available";
        delete e;
        return PHMM_ERR_NO_DEVICE;
    }
    if (e->cfg_.device < 0 || e->cfg_.device >= ndev) {
        err = "device ordinal " + std::to_string(e->cfg_.device) + " out of range";
        delete e;
        return PHMM_ERR_NO_DEVICE;
    }
    e->dev_ = e->cfg_.device;
    auto fail = [&](phmm_status st) {
        delete e;
        return st;
    };
#define PHMM_CKE(call)                                                               \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            err = std::string(#call) + " failed: " + cudaGetErrorString(e_);         \
            return fail(PHMM_ERR_CUDA);                                              \
        }                                                                            \
    } while (0)
    PHMM_CKE(cudaSetDevice(e->dev_));
    cudaDeviceProp prop;
    PHMM_CKE(cudaGetDeviceProperties(&prop, e->dev_));
    if (prop.major < 10) {
        err = std::string("device ") + prop.name + " is not sm_100 class; this build targets sm_100a only";
        return fail(PHMM_ERR_NO_DEVICE);
    }
    e->sms_ = prop.multiProcessorCount;
    for (int p = 0; p < 2; ++p)
        for (int c = 0; c < (p == 0 ? kClasses32 : kClasses64); ++c) {
            int b = 0;
            PHMM_CKE(occupancy(p == 0 ? 32 : 64, c, &b));
            e->occ_[p][c] = std::max(b, 1);
        }

    // probability tables
    const HostTables<float>& hf = host_tables_f32();
    const HostTables<double>& hd = host_tables_f64();
    const size_t nf = 5 * 128 + 128 * 128;
    const std::vector<double>& jac = genotype_jacobian();
    const size_t bytes = nf * sizeof(float) + nf * sizeof(double) + jac.size() * sizeof(double);
    PHMM_CKE(cudaMalloc(&e->d_tables_, bytes));
    std::vector<char> host(bytes);
    float* f = (float*)host.data();
    double* d = (double*)(host.data() + nf * sizeof(float));
    auto put = [](auto* dst, const auto& v) {
        std::copy(v.begin(), v.end(), dst);
        return dst + v.size();
    };
    float* fp = f;
    fp = put(fp, hf.ph2pr);
    fp = put(fp, hf.pmat);
    fp = put(fp, hf.pmis_inter);
    fp = put(fp, hf.pmis_intra);
    fp = put(fp, hf.gapm);
    put(fp, hf.mm);
    double* dp = d;
    dp = put(dp, hd.ph2pr);
    dp = put(dp, hd.pmat);
    dp = put(dp, hd.pmis_inter);
    dp = put(dp, hd.pmis_intra);
    dp = put(dp, hd.gapm);
    dp = put(dp, hd.mm);
    put(dp, jac);
    PHMM_CKE(cudaMemcpy(e->d_tables_, host.data(), bytes, cudaMemcpyHostToDevice));
    const float* df = (const float*)e->d_tables_;
    const double* dd = (const double*)((const char*)e->d_tables_ + nf * sizeof(float));
    e->tf_ = ProbTables<float>{df, df + 128, df + 256, df + 384, df + 512, df + 640};
    e->td_ = ProbTables<double>{dd, dd + 128, dd + 256, dd + 384, dd + 512, dd + 640};
    e->d_jacobian_ = dd + nf;
    e->log10_two_ = host_log10_two();
#undef PHMM_CKE
    phmm_status st = e->make_slot(0, &e->default_slot_, err);
    if (st != PHMM_OK) return fail(st);
    if (e->cfg_.autotune) {
        st = autotune_once(*e, err);
        if (st != PHMM_OK) return fail(st);
    }
    *out = e;
    return PHMM_OK;
}

Engine::~Engine()
{
    cudaSetDevice(dev_);
    delete sw_;
    if (default_slot_) free_slot(default_slot_);
    if (chunk_slot_) free_slot(chunk_slot_);
    if (ev_span_) cudaEventDestroy(ev_span_);
    if (d_tables_) cudaFree(d_tables_);
}

namespace {

// Grows a device or pinned buffer of a slot (only between batches of that slot: the slot's stream
// is idle when its serving worker calls these).
phmm_status grow_device(char*& p, size_t& bytes, size_t need, std::string& err)
{
    if (need <= bytes) return PHMM_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    const size_t want = std::max(need, need / 2 * 3);
    if (cudaMalloc(&p, want) != cudaSuccess) {
        cudaGetLastError();
        err = "realignment arena of " + std::to_string(want) + " bytes could not be allocated";
        return PHMM_ERR_OUT_OF_MEMORY;
    }
    bytes = want;
    return PHMM_OK;
}

phmm_status grow_pinned(char*& p, size_t& bytes, size_t need, std::string& err)
{
    if (need <= bytes) return PHMM_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    const size_t want = std::max(need, need / 2 * 3);
    if (cudaMallocHost(&p, want) != cudaSuccess) {
        cudaGetLastError();
        err = "pinned realignment staging of " + std::to_string(want) + " bytes could not be allocated";
        return PHMM_ERR_OUT_OF_MEMORY;
    }
    bytes = want;
    return PHMM_OK;
}

}  // namespace

phmm_status Engine::realign_enqueue(Slot& s, RealignBatch& rb, std::string& err)
{
    if (rb.plan.n == 0) return PHMM_OK;
    rb.layout();
    // growing frees the old buffers, which waits for the device: only this slot's work is queued
    // before the wait, and arenas stop growing once they cover the slot's largest batch
    if (rb.bytes > s.rdev_bytes) PHMM_CK(cudaStreamSynchronize(s.main));
    phmm_status st = grow_device(s.rdev, s.rdev_bytes, rb.bytes, err);
    if (st != PHMM_OK) return st;
    st = grow_pinned(s.rpin, s.rpin_bytes, std::max(rb.upload_bytes(), rb.head_bytes()), err);
    if (st != PHMM_OK) return st;
    char* h = s.rpin;
    char* d = s.rdev;
    std::memcpy(h + rb.o_rr, rb.regions.data(), sizeof(RealignRegion) * rb.regions.size());
    std::memcpy(h + rb.o_prio, rb.prio.data(), 8 * rb.prio.size());
    std::memcpy(h + rb.o_clip, rb.clip.data(), 2 * rb.clip.size());
    std::memcpy(h + rb.o_order, rb.plan.order.data(), 4ull * rb.plan.n);
    std::memcpy(h + rb.o_slot, rb.plan.slot_off.data(), 8ull * rb.plan.n);
    PHMM_CK(cudaMemcpyAsync(d, h, rb.upload_bytes(), cudaMemcpyHostToDevice, s.main));
    RealignView v{};
    v.regions = s.d_regions;
    v.hap_off = s.d_hap_off;
    v.read_off = s.d_read_off;
    v.norm = s.d_out2;
    v.keep = s.d_keep;
    v.rr = (const RealignRegion*)(d + rb.o_rr);
    v.n_rr = (uint32_t)rb.regions.size();
    v.prio = (const double*)(d + rb.o_prio);
    v.clip = (const uint16_t*)(d + rb.o_clip);
    v.items = (SwItem*)(d + rb.o_items);
    v.best = (int32_t*)(d + rb.o_best);
    PHMM_CK(launch_realign_items(v, sms_ * 4, s.main));
    SwDeviceBufs b;
    b.items = v.items;
    b.order = (const uint32_t*)(d + rb.o_order);
    b.slot_off = (const uint64_t*)(d + rb.o_slot);
    b.hap = s.d_hb;
    b.read = s.d_rb;
    b.claim = (unsigned int*)(d + rb.o_claim);
    b.total = (unsigned long long*)(d + rb.o_total);
    b.out = (phmm_sw_result*)(d + rb.o_out);
    b.slots = (uint32_t*)(d + rb.o_slots);
    b.compact = (uint32_t*)(d + rb.o_compact);
    b.scratch = (uint8_t*)(d + rb.o_scratch);
    const SwParams prm{10, -15, -30, -5};  // sw_parameters_genotype, lib/sw_avx/sw_avx.c:15
    st = sw_launch(rb.plan, prm, 0, b, s.main, nullptr, nullptr, nullptr, err);
    if (st != PHMM_OK) return st;
    s.launches += 1 + 2;
    for (int c = 0; c < kSwClasses; ++c) s.launches += rb.plan.grid[c] ? 1 : 0;
    // total, results and best haplotypes come back with the rest of the batch's outputs
    PHMM_CK(cudaMemcpyAsync(h, d + rb.o_total, rb.head_bytes(), cudaMemcpyDeviceToHost, s.main));
    return PHMM_OK;
}

phmm_status Engine::realign_finish(Slot& s, RealignBatch& rb, std::string& err)
{
    const uint32_t n = rb.plan.n;
    rb.res.assign(n, phmm_sw_result{});
    rb.best.assign(n, -1);
    rb.total = 0;
    rb.cigars.clear();
    if (n == 0) return PHMM_OK;
    PHMM_CK(cudaStreamSynchronize(s.main));
    const char* h = s.rpin;
    std::memcpy(&rb.total, h, 8);
    std::memcpy(rb.res.data(), h + (rb.o_out - rb.o_total), sizeof(phmm_sw_result) * n);
    std::memcpy(rb.best.data(), h + (rb.o_best - rb.o_total), 4ull * n);
    rb.cigars.resize(rb.total);
    if (rb.total) {
        phmm_status st = grow_pinned(s.rpin, s.rpin_bytes, 4 * rb.total, err);
        if (st != PHMM_OK) return st;
        PHMM_CK(cudaMemcpyAsync(s.rpin, s.rdev + rb.o_compact, 4 * rb.total, cudaMemcpyDeviceToHost, s.main));
        PHMM_CK(cudaStreamSynchronize(s.main));
        std::memcpy(rb.cigars.data(), s.rpin, 4 * rb.total);
    }
    return PHMM_OK;
}

phmm_status Engine::sw_aligner(SwAligner** out, std::string& err)
{
    std::lock_guard<std::mutex> lk(sw_mu_);
    if (!sw_) {
        phmm_status st = SwAligner::create(dev_, &sw_, err);
        if (st != PHMM_OK) return st;
    }
    *out = sw_;
    return PHMM_OK;
}

phmm_status Engine::make_slot(int id, Slot** out, std::string& err, bool overlap)
{
    *out = nullptr;
    PHMM_CK(cudaSetDevice(dev_));
    Slot* s = new Slot();
    s->id = id;
    auto cleanup = [&]() { free_slot(s); };
    cudaError_t e = cudaStreamCreateWithFlags(&s->main, cudaStreamNonBlocking);
    s->overlap = overlap;
    int least = 0, greatest = 0;
    if (overlap && e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    for (int c = 0; c < kNumClasses && e == cudaSuccess; ++c)
        e = cudaStreamCreateWithPriority(&s->side[c], cudaStreamNonBlocking, c < kClasses32 ? least : greatest);
    for (int c = 0; c < kNumClasses && e == cudaSuccess; ++c) e = cudaEventCreateWithFlags(&s->ev_side[c], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_t0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_t1);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_t2);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_t3);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        err = std::string("stream/event creation failed: ") + cudaGetErrorString(e);
        cleanup();
        return PHMM_ERR_CUDA;
    }
    *out = s;
    return PHMM_OK;
}

void Engine::free_slot(Slot* s)
{
    if (!s) return;
    cudaSetDevice(dev_);
    if (s->main) cudaStreamSynchronize(s->main);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    if (s->dev) cudaFree(s->dev);
    if (s->pinned) cudaFreeHost(s->pinned);
    if (s->rdev) cudaFree(s->rdev);
    if (s->rpin) cudaFreeHost(s->rpin);
    for (int c = 0; c < kNumClasses; ++c) {
        if (s->side[c]) cudaStreamDestroy(s->side[c]);
        if (s->ev_side[c]) cudaEventDestroy(s->ev_side[c]);
    }
    for (cudaEvent_t ev : {s->ev_fork, s->ev_t0, s->ev_t1, s->ev_t2, s->ev_t3, s->ev_done})
        if (ev) cudaEventDestroy(ev);
    if (s->main) cudaStreamDestroy(s->main);
    delete s;
}

uint64_t Engine::scratch_warps() const
{
    // Each resident warp of a multi-stripe class owns a scratch row of 24 bytes per column: two
    // FP32 rows (one per read of the warp) or one FP64 row.  Classes that can run at the same time
    // need disjoint rows: the FP32 multi-stripe classes run one after another on a chained stream
    // and share the first region; each FP64 multi-stripe class (one per mode) has its own, since it
    // overlaps the FP32 pass.
    return scratch_offset_warps(1 + kModes32);
}

uint64_t Engine::scratch_offset_warps(int region) const
{
    // region 0: FP32 multi-stripe classes; 1 + m: the FP64 multi-stripe class of mode m
    int occ32 = 1;
    for (int c = 0; c < kClasses32; ++c)
        if (class32_multi(c)) occ32 = std::max(occ32, occ_[0][c]);
    uint64_t at = (uint64_t)sms_ * occ32 * (kFwdBlock / kWarp);
    if (region == 0) return 0;
    for (int m = 0; m < kModes32; ++m) {
        if (region == 1 + m) return at;
        at += (uint64_t)sms_ * occ_[1][class64(m, kMaxK, true)] * (kFwdBlock / kWarp);
    }
    return at;
}

uint64_t Engine::scratch_bytes() const
{
    return scratch_warps() * (uint64_t)PlanLimits().max_stream_multi * 3 * sizeof(double);
}

uint64_t Engine::arena_bytes(const Capacity& c) const { return carve(c, nullptr, nullptr); }

phmm_status Engine::ensure_capacity(Slot& s, const Plan& plan, std::string& err)
{
    return reserve(s, need_of(plan, scratch_warps()), err);
}

phmm_status Engine::reserve(Slot& s, const Capacity& want, std::string& err)
{
    const Capacity need = Capacity::max_of(want, s.floor);
    if (s.dev && s.cap.covers(need)) return PHMM_OK;
    const Capacity nc = s.dev ? s.cap.grown_to(need) : need;
    const auto t0 = std::chrono::steady_clock::now();
    ++s.arena_grows;
    struct Timer {
        Slot& s;
        std::chrono::steady_clock::time_point t0;
        ~Timer() { s.setup_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); }
    } timer{s, t0};
    PHMM_CK(cudaSetDevice(dev_));
    if (s.main) PHMM_CK(cudaStreamSynchronize(s.main));
    if (s.graph) {
        cudaGraphExecDestroy(s.graph);
        s.graph = nullptr;
    }
    if (s.dev) {
        cudaFree(s.dev);
        s.dev = nullptr;
    }
    if (s.pinned) {
        cudaFreeHost(s.pinned);
        s.pinned = nullptr;
    }
    const size_t bytes = carve(nc, nullptr, nullptr);
    cudaError_t e = cudaMalloc((void**)&s.dev, bytes);
    if (e != cudaSuccess) {
        s.dev = nullptr;
        cudaGetLastError();
        err = "device arena of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e);
        return PHMM_ERR_OUT_OF_MEMORY;
    }
    s.dev_bytes = bytes;
    carve(nc, s.dev, &s);
    const size_t pb = pinned_bytes_for(nc);
    e = cudaMallocHost((void**)&s.pinned, pb);
    if (e != cudaSuccess) {
        s.pinned = nullptr;
        cudaGetLastError();
        err = "pinned staging of " + std::to_string(pb) + " bytes: " + cudaGetErrorString(e);
        return PHMM_ERR_OUT_OF_MEMORY;
    }
    s.pinned_bytes = pb;
    s.cap = nc;
    return PHMM_OK;
}

// Multi-stripe warps index scratch rows by warp and stay persistent.
static unsigned int waves32(int cls, bool overlap)
{
    return overlap && !class32_multi(cls) ? kOverlapWaves : 1u;
}

int Engine::full_grid(int precision, int cls, unsigned int waves) const
{
    return occ_[precision == 32 ? 0 : 1][cls] * sms_ * (precision == 32 ? (int)waves : 1);
}

int Engine::grid_for(int precision, int cls, uint32_t work, unsigned int waves) const
{
    const int full = full_grid(precision, cls, waves);
    const int warps_per_block = kFwdBlock / kWarp;
    const int need = (int)std::min<uint64_t>(((uint64_t)work + warps_per_block - 1) / warps_per_block, (uint64_t)full);
    return std::max(need, 1);
}

namespace {

RegionApiView region_view(const Slot& s, const double* jacobian, double log10_two)
{
    RegionApiView rv;
    rv.events = s.d_events;
    rv.hap_allele = s.d_hap_allele;
    rv.allele_lk = s.d_allele_lk;
    rv.gl = s.d_gl;
    rv.best = s.d_best;
    rv.jacobian = jacobian;
    rv.log10_two = log10_two;
    rv.desc = s.d_desc;
    rv.regions = s.d_regions;
    rv.read_off = s.d_read_off;
    rv.read_bases = s.d_rb;
    rv.read_q = s.d_rq;
    rv.read_i = s.d_ri;
    rv.read_d = s.d_rd;
    rv.read_c = s.d_rc;
    rv.mapq = s.d_mapq;
    rv.lk = s.d_out;
    rv.out = s.d_out2;
    rv.keep = s.d_keep;
    rv.n_kept = s.d_nkept;
    return rv;
}

// FP32 classes that can append reruns to FP64 class c64 under tile table t: the FP32 classes of the
// same mode running the shapes of every read-length bucket whose reads belong to c64.  The intra
// mode takes reads of every mode's table (a read without 'N' runs intra against haplotypes with 'N').
void fp64_sources(const TileTable& t, int c64, bool src[kClasses32])
{
    for (int c = 0; c < kClasses32; ++c) src[c] = false;
    const int mode = c64 / 9;
    for (int b = 1; b <= kLenBuckets; ++b) {
        if (class64_for_len(mode, (uint64_t)b * kWarp) != c64) continue;
        for (int m = 0; m < kModes32; ++m) {
            if (mode != 2 && m != mode) continue;
            const int kh = t.kh[m][b - 1];
            const bool multi = t.multi[m][b - 1] != 0;
            src[mode * kShapes32 + shape32(kh, multi)] = true;
        }
    }
}

}  // namespace

phmm_status Engine::launch_pipeline(Slot& s, bool want_flags, const Plan* plan, const TileTable& tiles, std::string& err)
{
    // plan == nullptr: graph capture (every class launched, persistent full grids).
    BatchView v;
    v.read_bases = s.d_rb;
    v.read_q = s.d_rq;
    v.read_i = s.d_ri;
    v.read_d = s.d_rd;
    v.read_c = s.d_rc;
    v.read_off = s.d_read_off;
    v.read_flags = s.d_read_flags;
    v.hap_off = s.d_hap_off;
    v.codes_inter = s.d_codes_inter;
    v.codes_intra = s.d_codes_intra;
    v.hap_flags = s.d_hap_flags;
    v.regions = s.d_regions;
    v.out = s.d_out;
    v.pair_flags = want_flags ? s.d_pair_flags : nullptr;
    const uint64_t warps = scratch_warps();
    const unsigned int scr_cols = s.cap.scratch_cols ? (unsigned int)(s.cap.scratch_cols / warps) : 0u;
    const unsigned int rec = plan ? cudaEventRecordDefault : cudaEventRecordExternal;

    s.launches = 0;
    PHMM_CK(cudaEventRecordWithFlags(s.ev_t0, s.main, rec));
    PHMM_CK(launch_prep(s.d_desc, s.d_hb, s.d_codes_inter, s.d_codes_intra, s.d_out, v.pair_flags, sms_, s.main));
    s.launches += 2;
    const RegionApiView rv = region_view(s, d_jacobian_, log10_two_);
    if (!plan || plan->region_api) {
        PHMM_CK(launch_read_prep(rv, sms_, s.main));
        ++s.launches;
    }
    PHMM_CK(cudaEventRecord(s.ev_fork, s.main));
    // Each class runs on its own stream.  An FP64 class reads the rerun list that its FP32 source
    // classes append to, so it waits for those classes only and overlaps with the FP32 classes
    // still running.
    bool launched[kNumClasses] = {};
    int prev_multi = -1;
    for (int pass = 0; pass < 2; ++pass) {
        const int precision = pass == 0 ? 32 : 64;
        const int n_cls = pass == 0 ? kClasses32 : kClasses64;
        const int slot0 = pass == 0 ? 0 : kClasses32;  // descriptor slot of the pass's first class
        for (int k = 0; k < n_cls; ++k) {
            // FP32 classes of a mode longest reads first (multi-stripe shapes, then KH = 8 .. 1)
            const int c = pass == 0 && s.overlap ? (k / kShapes32) * kShapes32 + kShapes32 - 1 - k % kShapes32 : k;
            uint32_t work = 0;
            if (plan) {
                work = pass == 0 ? plan->classes[c].n_items : plan->classes[slot0 + c].rerun_cap;
                if (work == 0) continue;
            }
            // FP32 items hold two reads (warps = items); FP64 claims are single pairs
            const unsigned int waves = pass == 0 ? waves32(c, s.overlap) : 1u;
            const int grid = plan ? grid_for(precision, c, work, waves) : full_grid(precision, c, waves);
            PassControl pc{};
            pc.cd = s.d_classes + slot0 + c;
            pc.cd64 = s.d_classes + kClasses32;
            pc.items = s.d_items;
            pc.rerun = s.d_rerun;
            pc.status = s.d_status;
            const bool multi = pass == 0 ? class32_multi(c) : c % 9 == 8;
            const int region = pass == 0 ? 0 : 1 + c / 9;
            pc.scratch = multi ? (void*)((char*)s.d_scratch + scratch_offset_warps(region) * scr_cols * 24) : nullptr;
            pc.scratch_cols = scr_cols;
            pc.waves = waves;
            cudaStream_t st = s.side[slot0 + c];
            PHMM_CK(cudaStreamWaitEvent(st, s.ev_fork, 0));
            // FP32 multi-stripe classes share one scratch region: each waits for the previous one
            if (pass == 0 && multi && prev_multi >= 0) PHMM_CK(cudaStreamWaitEvent(st, s.ev_side[prev_multi], 0));
            if (pass == 1) {
                bool src[kClasses32];
                fp64_sources(tiles, c, src);
                for (int k = 0; k < kClasses32; ++k)
                    if (src[k] && launched[k]) PHMM_CK(cudaStreamWaitEvent(st, s.ev_side[k], 0));
            }
            PHMM_CK(launch_fwd(precision, c, v, tf_, td_, pc, grid, st));
            ++s.launches;
            launched[slot0 + c] = true;
            PHMM_CK(cudaEventRecord(s.ev_side[slot0 + c], st));
            if (pass == 0 && multi) prev_multi = c;
        }
        for (int c = 0; c < n_cls; ++c)
            if (launched[slot0 + c]) PHMM_CK(cudaStreamWaitEvent(s.main, s.ev_side[slot0 + c], 0));
        if (pass == 1 && (!plan || plan->region_api)) {
            PHMM_CK(launch_post_region(rv, sms_, s.main));
            ++s.launches;
            if (!plan || !plan->events.empty()) {
                PHMM_CK(launch_genotype(rv, sms_, s.main));
                ++s.launches;
            }
        }
        PHMM_CK(cudaEventRecordWithFlags(pass == 0 ? s.ev_t1 : s.ev_t2, s.main, rec));
    }
    return PHMM_OK;
}

phmm_status Engine::capture_graph(Slot& s, bool want_flags, const TileTable& tiles, std::string& err)
{
    if (s.graph) {
        cudaGraphExecDestroy(s.graph);
        s.graph = nullptr;
    }
    const auto t0 = std::chrono::steady_clock::now();
    ++s.graph_captures;
    struct Timer {
        Slot& s;
        std::chrono::steady_clock::time_point t0;
        ~Timer() { s.setup_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); }
    } timer{s, t0};
    cudaGraph_t g = nullptr;
    PHMM_CK(cudaStreamBeginCapture(s.main, cudaStreamCaptureModeThreadLocal));
    std::string lerr;
    phmm_status st = launch_pipeline(s, want_flags, nullptr, tiles, lerr);
    cudaError_t e = cudaStreamEndCapture(s.main, &g);
    if (st != PHMM_OK) {
        if (g) cudaGraphDestroy(g);
        err = lerr;
        return st;
    }
    if (e != cudaSuccess) {
        err = std::string("graph capture failed: ") + cudaGetErrorString(e);
        return PHMM_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&s.graph, g, s.overlap ? cudaGraphInstantiateFlagUseNodePriority : 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        s.graph = nullptr;
        err = std::string("graph instantiate failed: ") + cudaGetErrorString(e);
        return PHMM_ERR_CUDA;
    }
    s.graph_flags = want_flags;
    s.graph_tiles = tiles;
    return PHMM_OK;
}

bool Engine::upload_raw(Slot& s, const BatchScan& sc, const phmm_batch& b)
{
    if (!s.dev || sc.read_bases > s.cap.read_bases || sc.hap_bases > s.cap.hap_bases) return false;
    cudaStream_t m = s.main;
    const uint64_t rb = sc.read_bases;
    cudaError_t e = cudaSuccess;
    if (rb) {
        e = cudaMemcpyAsync(s.d_rb, b.read_bases + sc.read_base0, rb, cudaMemcpyHostToDevice, m);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s.d_rq, b.read_qual + sc.read_base0, rb, cudaMemcpyHostToDevice, m);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s.d_ri, b.read_ins + sc.read_base0, rb, cudaMemcpyHostToDevice, m);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s.d_rd, b.read_del + sc.read_base0, rb, cudaMemcpyHostToDevice, m);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s.d_rc, b.read_gcp + sc.read_base0, rb, cudaMemcpyHostToDevice, m);
    }
    if (e == cudaSuccess && sc.hap_bases)
        e = cudaMemcpyAsync(s.d_hb, b.hap_bases + sc.hap_base0, sc.hap_bases, cudaMemcpyHostToDevice, m);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;  // upload() copies them again
    }
    return true;
}

phmm_status Engine::upload(Slot& s, const Plan& plan, const phmm_batch& b, std::string& err, const uint8_t* mapq,
                           bool raw_sent)
{
    if (plan.region_api && plan.n_reads && !mapq) {
        err = "region-API batch without MAPQ";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    const uint64_t grows = s.arena_grows;
    phmm_status st = ensure_capacity(s, plan, err);
    if (st != PHMM_OK) return st;
    if (s.arena_grows != grows) raw_sent = false;  // a new arena: copies into the old one are gone
    PHMM_CK(cudaSetDevice(dev_));
    // stage descriptors + plan arrays in pinned memory, then copy
    char* p = s.pinned;
    size_t o = 0;
    auto stage = [&](const void* src, size_t bytes) -> char* {
        char* at = p + o;
        if (bytes) std::memcpy(at, src, bytes);
        o = align_up(o + std::max<size_t>(bytes, 1));
        return at;
    };
    BatchDesc bd{};
    bd.hap_bases_total = plan.hap_bases;
    bd.out_total = plan.out_total;
    bd.n_regions = plan.n_regions;
    bd.n_reads = plan.n_reads;
    bd.n_haps = plan.n_haps;
    bd.n_items = (uint32_t)plan.items.size();
    bd.read_bases_total = plan.read_bases;
    bd.region_api = plan.region_api ? plan.n_regions : 0;
    bd.n_events = (uint32_t)plan.events.size();
    char* desc = p;
    std::memcpy(desc, &bd, sizeof(bd));
    std::memcpy(desc + sizeof(bd), plan.classes.data(), sizeof(ClassDesc) * kNumClasses);
    std::memset(desc + sizeof(bd) + sizeof(ClassDesc) * kNumClasses, 0, 4 * sizeof(unsigned int));
    o = align_up(kDescBytes);
    char* h_regions = stage(plan.regions.data(), plan.regions.size() * sizeof(RegionDesc));
    char* h_read_off = stage(plan.read_off.data(), plan.read_off.size() * 8);
    char* h_hap_off = stage(plan.hap_off.data(), plan.hap_off.size() * 8);
    char* h_read_flags = stage(plan.read_flags.data(), plan.read_flags.size());
    char* h_hap_flags = stage(plan.hap_flags.data(), plan.hap_flags.size());
    char* h_items = stage(plan.items.data(), plan.items.size() * sizeof(WorkItem));
    char* h_events = stage(plan.events.data(), plan.events.size() * sizeof(EventDesc));
    char* h_hap_allele = stage(plan.hap_allele.data(), plan.hap_allele.size());

    cudaStream_t m = s.main;
    PHMM_CK(cudaMemcpyAsync(s.d_desc, desc, kDescBytes, cudaMemcpyHostToDevice, m));
    PHMM_CK(cudaMemcpyAsync(s.d_regions, h_regions, plan.regions.size() * sizeof(RegionDesc), cudaMemcpyHostToDevice, m));
    PHMM_CK(cudaMemcpyAsync(s.d_read_off, h_read_off, plan.read_off.size() * 8, cudaMemcpyHostToDevice, m));
    PHMM_CK(cudaMemcpyAsync(s.d_hap_off, h_hap_off, plan.hap_off.size() * 8, cudaMemcpyHostToDevice, m));
    if (!plan.read_flags.empty())
        PHMM_CK(cudaMemcpyAsync(s.d_read_flags, h_read_flags, plan.read_flags.size(), cudaMemcpyHostToDevice, m));
    if (!plan.hap_flags.empty())
        PHMM_CK(cudaMemcpyAsync(s.d_hap_flags, h_hap_flags, plan.hap_flags.size(), cudaMemcpyHostToDevice, m));
    if (!plan.items.empty())
        PHMM_CK(cudaMemcpyAsync(s.d_items, h_items, plan.items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, m));
    const uint64_t rb = raw_sent ? 0 : plan.read_bases;
    if (rb) {
        PHMM_CK(cudaMemcpyAsync(s.d_rb, b.read_bases + plan.read_base0, rb, cudaMemcpyHostToDevice, m));
        PHMM_CK(cudaMemcpyAsync(s.d_rq, b.read_qual + plan.read_base0, rb, cudaMemcpyHostToDevice, m));
        if (!plan.region_api) {  // region API: the device writes the gap qualities
            PHMM_CK(cudaMemcpyAsync(s.d_ri, b.read_ins + plan.read_base0, rb, cudaMemcpyHostToDevice, m));
            PHMM_CK(cudaMemcpyAsync(s.d_rd, b.read_del + plan.read_base0, rb, cudaMemcpyHostToDevice, m));
            PHMM_CK(cudaMemcpyAsync(s.d_rc, b.read_gcp + plan.read_base0, rb, cudaMemcpyHostToDevice, m));
        }
    }
    if (plan.hap_bases && !raw_sent)
        PHMM_CK(cudaMemcpyAsync(s.d_hb, b.hap_bases + plan.hap_base0, plan.hap_bases, cudaMemcpyHostToDevice, m));

    if (plan.region_api && plan.n_reads)
        PHMM_CK(cudaMemcpyAsync(s.d_mapq, mapq, plan.n_reads, cudaMemcpyHostToDevice, m));
    if (!plan.events.empty()) {
        PHMM_CK(cudaMemcpyAsync(s.d_events, h_events, plan.events.size() * sizeof(EventDesc), cudaMemcpyHostToDevice, m));
        PHMM_CK(cudaMemcpyAsync(s.d_hap_allele, h_hap_allele, plan.hap_allele.size(), cudaMemcpyHostToDevice, m));
    }
    PHMM_CK(cudaMemcpyAsync(s.d_desc_pristine, s.d_desc, kDescBytes, cudaMemcpyDeviceToDevice, m));
    return PHMM_OK;
}

phmm_status Engine::ensure_graph(Slot& s, const Plan& plan, bool want_flags, std::string& err)
{
    if (cfg_.use_cuda_graph &&
        (!s.graph || s.graph_flags != want_flags || std::memcmp(&s.graph_tiles, &plan.tiles, sizeof(TileTable)) != 0))
        return capture_graph(s, want_flags, plan.tiles, err);
    return PHMM_OK;
}

phmm_status Engine::run(Slot& s, const Plan& plan, bool want_flags, bool restore, std::string& err)
{
    phmm_status st = PHMM_OK;
    cudaStream_t m = s.main;
    if (restore) PHMM_CK(cudaMemcpyAsync(s.d_desc, s.d_desc_pristine, kDescBytes, cudaMemcpyDeviceToDevice, m));
    if (cfg_.use_cuda_graph) {
        st = ensure_graph(s, plan, want_flags, err);
        if (st != PHMM_OK) return st;
        PHMM_CK(cudaGraphLaunch(s.graph, m));
    } else {
        st = launch_pipeline(s, want_flags, &plan, plan.tiles, err);
        if (st != PHMM_OK) return st;
    }
    return PHMM_OK;
}

phmm_status Engine::enqueue(Slot& s, const Plan& plan, const phmm_batch& b, bool want_flags, std::string& err,
                            const uint8_t* mapq, bool raw_sent)
{
    phmm_status st = upload(s, plan, b, err, mapq, raw_sent);
    if (st != PHMM_OK) return st;
    return run(s, plan, want_flags, false, err);
}

phmm_status Engine::finish(Slot& s, const Plan& plan, double* out, uint8_t* pair_flags, phmm_stats* stats,
                           std::string& err, uint8_t* keep, uint32_t* n_kept, double* gl, int32_t* best,
                           double* allele_lk)
{
    cudaStream_t m = s.main;
    char* desc = s.pinned;  // reuse the staged descriptor block for the read-back
    PHMM_CK(cudaMemcpyAsync(desc, s.d_desc, kDescBytes, cudaMemcpyDeviceToHost, m));
    if (plan.region_api) {
        if (plan.n_reads && keep) PHMM_CK(cudaMemcpyAsync(keep, s.d_keep, plan.n_reads, cudaMemcpyDeviceToHost, m));
        if (plan.n_regions && n_kept)
            PHMM_CK(cudaMemcpyAsync(n_kept, s.d_nkept, plan.n_regions * sizeof(uint32_t), cudaMemcpyDeviceToHost, m));
    }
    if (!plan.events.empty()) {
        if (gl) PHMM_CK(cudaMemcpyAsync(gl, s.d_gl, plan.gl_total * sizeof(double), cudaMemcpyDeviceToHost, m));
        if (best) PHMM_CK(cudaMemcpyAsync(best, s.d_best, plan.events.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, m));
        if (allele_lk)
            PHMM_CK(cudaMemcpyAsync(allele_lk, s.d_allele_lk, plan.allele_lk_total * sizeof(double),
                                    cudaMemcpyDeviceToHost, m));
    }
    if (plan.out_total && out) {
        PHMM_CK(cudaMemcpyAsync(out, plan.region_api ? s.d_out2 : s.d_out, plan.out_total * sizeof(double),
                                cudaMemcpyDeviceToHost, m));
        if (pair_flags) PHMM_CK(cudaMemcpyAsync(pair_flags, s.d_pair_flags, plan.out_total, cudaMemcpyDeviceToHost, m));
    }
    PHMM_CK(cudaEventRecord(s.ev_t3, m));
    PHMM_CK(cudaEventSynchronize(s.ev_t3));
    const ClassDesc* cls = (const ClassDesc*)(desc + sizeof(BatchDesc));
    const unsigned int status = *(const unsigned int*)(desc + sizeof(BatchDesc) + sizeof(ClassDesc) * kNumClasses);
    uint64_t f64 = 0;
    for (int c = kClasses32; c < kNumClasses; ++c) f64 += cls[c].rerun_pairs;
    if (stats) {
        stats->regions = plan.n_regions;
        stats->pairs = plan.pairs;
        stats->cells = plan.cells;
        stats->pairs_f64 = f64;
        stats->work_items = plan.items.size();
        stats->kernel_launches = s.launches;
        stats->h2d_bytes = plan.read_bases * 5 + plan.hap_bases;
        stats->d2h_bytes = plan.out_total * (sizeof(double) + (pair_flags ? 1 : 0));
        float a = 0, bms = 0, c2 = 0;
        cudaEventElapsedTime(&a, s.ev_t0, s.ev_t2);
        cudaEventElapsedTime(&bms, s.ev_t0, s.ev_t1);
        cudaEventElapsedTime(&c2, s.ev_t1, s.ev_t2);
        stats->device_ms = a;
        stats->fp32_ms = bms;
        stats->fp64_ms = c2;
    }
    if (status != 0) {
        err = "kernel status word " + std::to_string(status) +
              ((status & kStatusBadItem) ? " (work item does not fit its kernel class)" : "") +
              ((status & kStatusRerunOverflow) ? " (FP64 rerun list overflow)" : "");
        return PHMM_ERR_DEVICE_STATUS;
    }
    return PHMM_OK;
}

phmm_status Engine::fp32_fma_peak(double* scalar_tflops, double* packed_tflops, std::string& err)
{
    std::lock_guard<std::mutex> lk(mu_);
    PHMM_CK(cudaSetDevice(dev_));
    Slot& s = *default_slot_;
    float* sink = nullptr;
    PHMM_CK(cudaMalloc(&sink, sizeof(float) * sms_ * 64));
    const int blocks = sms_ * 8, iters = 1 << 14;
    cudaError_t e = cudaSuccess;
    for (int packed = 0; packed < 2 && e == cudaSuccess; ++packed) {
        launch_fma_peak(sink, blocks, 256, packed != 0, s.main);  // warm-up
        cudaEventRecord(s.ev_t0, s.main);
        launch_fma_peak(sink, blocks, iters, packed != 0, s.main);
        cudaEventRecord(s.ev_t1, s.main);
        e = cudaEventSynchronize(s.ev_t1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, s.ev_t0, s.ev_t1);
        const double flops = 2.0 * 16.0 * (packed ? 2.0 : 1.0) * (double)iters * 256.0 * blocks;
        const double tf = e == cudaSuccess ? flops / (ms * 1e-3) / 1e12 : 0.0;
        if (packed) {
            if (packed_tflops) *packed_tflops = tf;
        } else if (scalar_tflops) {
            *scalar_tflops = tf;
        }
    }
    cudaFree(sink);
    if (e != cudaSuccess) {
        err = std::string("FMA probe failed: ") + cudaGetErrorString(e);
        return PHMM_ERR_CUDA;
    }
    return PHMM_OK;
}

namespace {

// Regions [r0, r1) of a synchronous batch that run as one chunk, with their first haplotype, first
// read and first likelihood in the whole batch.
struct ChunkRange {
    uint32_t r0, r1;
    uint64_t hap0, read0, out0;
};

// Cuts a validated batch at region boundaries near these cumulative shares of its cells: a small
// first chunk gets the device going after little planning and uploading, and the rest is planned
// and uploaded while it runs.  Measured on B200 over the 2,000-region benchmark batch end to end:
// one cut at 15% 2278 GCUPS, one pipeline 2213; cuts at 10% and 55% 2238 and at 12.5%, 42% and 71%
// 2237, their extra chunk tails adding 7-8 ms of device time.  With the current kernels: one cut
// 2713 GCUPS, cuts at 15% and 85% 2682, and either with the serving slots' overlap scheduling on the
// two chunk slots 2712 and 2717 (within noise); later, one cut at 15% 199.3-199.5 ms per batch, at 8%
// 198.2-199.0, at 5% 197.9-198.4, at 3% 201.6-202.1 (the first chunk then ends before the second is
// planned and uploaded) and at 22% 199.8.  The default (build-time setting) is 8%.
std::vector<ChunkRange> split_chunks(const phmm_batch& b, uint64_t total_cells)
{
#ifndef PHMM_CHUNK_FIRST
#define PHMM_CHUNK_FIRST 0.08
#endif
    static const double kEnds[] = {PHMM_CHUNK_FIRST};
    constexpr int kCuts = (int)(sizeof(kEnds) / sizeof(kEnds[0]));
    std::vector<ChunkRange> ch;
    ChunkRange cur{0, 0, 0, 0, 0};
    uint64_t h = 0, r = 0, o = 0, cells = 0;
    int next = 0;
    for (uint32_t g = 0; g < b.n_regions; ++g) {
        const uint32_t nh = b.n_haps[g], nr = b.n_reads[g];
        cells += (b.hap_off[h + nh] - b.hap_off[h]) * (b.read_off[r + nr] - b.read_off[r]);
        h += nh;
        r += nr;
        o += (uint64_t)nh * nr;
        cur.r1 = g + 1;
        if (next < kCuts && (double)cells >= kEnds[next] * (double)total_cells && g + 1 < b.n_regions) {
            ch.push_back(cur);
            cur = ChunkRange{g + 1, g + 1, h, r, o};
            while (next < kCuts && (double)cells >= kEnds[next] * (double)total_cells) ++next;
        }
    }
    if (cur.r1 > cur.r0) ch.push_back(cur);
    return ch;
}

phmm_batch chunk_view(const phmm_batch& b, const ChunkRange& c)
{
    phmm_batch v = b;  // offsets stay absolute: the planner and the uploads start at hap_off[0] / read_off[0]
    v.n_regions = c.r1 - c.r0;
    v.n_haps = b.n_haps + c.r0;
    v.n_reads = b.n_reads + c.r0;
    v.hap_off = b.hap_off + c.hap0;
    v.read_off = b.read_off + c.read0;
    return v;
}

}  // namespace

phmm_status Engine::compute_chunked(const phmm_batch& b, const BatchScan& sc, double* out, uint8_t* pair_flags,
                                    phmm_stats* stats, std::string& err, bool* ran)
{
    *ran = false;
    const std::vector<ChunkRange> ch = split_chunks(b, sc.cells);
    if (ch.size() < 2) return PHMM_OK;
    phmm_status st = PHMM_OK;
    if (!chunk_slot_) {
        // without a second slot (device memory short) the batch runs as one pipeline
        std::string slot_err;
        if (make_slot(1, &chunk_slot_, slot_err) != PHMM_OK) {
            chunk_slot_ = nullptr;
            cudaGetLastError();
            return PHMM_OK;
        }
    }
    if (!ev_span_ && cudaEventCreate(&ev_span_) != cudaSuccess) {
        ev_span_ = nullptr;
        cudaGetLastError();
        return PHMM_OK;
    }
    *ran = true;
    Slot* slots[2] = {default_slot_, chunk_slot_};
    Plan plans[2];
    int pending[2] = {-1, -1};  // chunk in flight on each slot
    const TileTable t = tiles();
    phmm_stats acc{};
    float span_ms = 0.f;
    // Reads a slot's chunk back (waiting for it) and adds its statistics.
    auto retire = [&](int j) -> phmm_status {
        const ChunkRange& c = ch[pending[j]];
        phmm_stats cs{};
        const phmm_status r = finish(*slots[j], plans[j], out ? out + c.out0 : nullptr,
                                     pair_flags ? pair_flags + c.out0 : nullptr, &cs, err);
        pending[j] = -1;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev_span_, slots[j]->ev_t2) == cudaSuccess) span_ms = std::max(span_ms, ms);
        acc.regions += cs.regions;
        acc.pairs += cs.pairs;
        acc.cells += cs.cells;
        acc.pairs_f64 += cs.pairs_f64;
        acc.work_items += cs.work_items;
        acc.kernel_launches += cs.kernel_launches;
        acc.h2d_bytes += cs.h2d_bytes;
        acc.d2h_bytes += cs.d2h_bytes;
        acc.fp32_ms += cs.fp32_ms;
        acc.fp64_ms += cs.fp64_ms;
        return r;
    };
    for (size_t k = 0; k < ch.size() && st == PHMM_OK; ++k) {
        int j = (int)(k & 1);
        if (pending[j] >= 0) {
            st = retire(j);
            if (st != PHMM_OK) break;
        }
        const phmm_batch v = chunk_view(b, ch[k]);
        BatchScan vs;
        st = scan_batch(v, limits_with(t), vs, err);
        if (st != PHMM_OK) break;
        const bool raw_sent = upload_raw(*slots[j], vs, v);
        st = build_plan(v, limits_with(t), plans[j], err);
        if (st == PHMM_OK) st = upload(*slots[j], plans[j], v, err, nullptr, raw_sent);
        if (st == PHMM_ERR_OUT_OF_MEMORY && j == 1) {
            // the second slot cannot grow for this chunk: run it on the first slot once that is free
            cudaStreamSynchronize(slots[1]->main);
            cudaGetLastError();
            err.clear();
            st = PHMM_OK;
            if (pending[0] >= 0) st = retire(0);
            if (st != PHMM_OK) break;
            j = 0;
            plans[0] = std::move(plans[1]);
            st = upload(*slots[0], plans[0], v, err, nullptr, false);
        }
        Slot& s = *slots[j];
        // the span starts where the first chunk's pipeline starts: after a graph capture, which
        // runs on the host while the device waits
        if (st == PHMM_OK && k == 0) st = ensure_graph(s, plans[j], pair_flags != nullptr, err);
        if (st == PHMM_OK && k == 0 && cudaEventRecord(ev_span_, s.main) != cudaSuccess) {
            err = "event record failed";
            st = PHMM_ERR_CUDA;
        }
        if (st == PHMM_OK) st = run(s, plans[j], pair_flags != nullptr, false, err);
        if (st != PHMM_OK) {
            cudaStreamSynchronize(s.main);  // copies already queued read the caller's buffers
            break;
        }
        pending[j] = (int)k;
    }
    // the older chunk first
    const int first = (pending[0] >= 0 && (pending[1] < 0 || pending[0] < pending[1])) ? 0 : 1;
    for (int j : {first, 1 - first}) {
        if (pending[j] < 0) continue;
        if (st == PHMM_OK) {
            st = retire(j);
        } else {
            cudaStreamSynchronize(slots[j]->main);
            pending[j] = -1;
        }
    }
    if (st == PHMM_OK && stats) {
        acc.device_ms = span_ms;
        *stats = acc;
    }
    return st;
}

phmm_status Engine::compute(const phmm_batch& b, double* out, uint8_t* pair_flags, phmm_stats* stats, std::string& err)
{
    const auto t0 = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(mu_);
    Plan plan;
    const TileTable t = tiles();
    // validate, then let the bases and qualities travel while the host plans the batch
    BatchScan sc;
    phmm_status st = scan_batch(b, limits_with(t), sc, err);
    if (st != PHMM_OK) return st;
    PHMM_CK(cudaSetDevice(dev_));
    const uint64_t chunk_cells = cfg_.chunk_cells ? cfg_.chunk_cells : kDefaultChunkCells;
    if (sc.cells >= chunk_cells && b.n_regions >= 2) {
        if (sc.out_total && !out) {
            err = "out is null";
            return PHMM_ERR_INVALID_ARGUMENT;
        }
        bool ran = false;
        st = compute_chunked(b, sc, out, pair_flags, stats, err, &ran);
        if (ran) {
            if (stats) stats->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return st;
        }
        if (st != PHMM_OK) return st;
    }
    const bool raw_sent = b.n_regions > 0 && upload_raw(*default_slot_, sc, b);
    st = build_plan(b, limits_with(t), plan, err);
    if (st == PHMM_OK && plan.out_total && !out) {
        err = "out is null";
        st = PHMM_ERR_INVALID_ARGUMENT;
    }
    if (st != PHMM_OK) {
        if (raw_sent) cudaStreamSynchronize(default_slot_->main);  // the copies read the caller's buffers
        return st;
    }
    st = enqueue(*default_slot_, plan, b, pair_flags != nullptr, err, nullptr, raw_sent);
    if (st != PHMM_OK) return st;
    st = finish(*default_slot_, plan, out, pair_flags, stats, err);
    if (stats) stats->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return st;
}

TileTable Engine::tiles() const
{
    std::lock_guard<std::mutex> lk(tiles_mu_);
    return tiles_;
}

phmm_status Engine::set_tiles(const TileTable& t, std::string& err)
{
    if (!t.valid(err)) return PHMM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(tiles_mu_);
    tiles_ = t;
    return PHMM_OK;
}

phmm_status Engine::time_fp32_class(Slot& s, const Plan& plan, int cls, int reps, float* best_ms, std::string& err)
{
    PHMM_CK(cudaSetDevice(dev_));
    BatchView v{};
    v.read_bases = s.d_rb;
    v.read_q = s.d_rq;
    v.read_i = s.d_ri;
    v.read_d = s.d_rd;
    v.read_c = s.d_rc;
    v.read_off = s.d_read_off;
    v.read_flags = s.d_read_flags;
    v.hap_off = s.d_hap_off;
    v.codes_inter = s.d_codes_inter;
    v.codes_intra = s.d_codes_intra;
    v.hap_flags = s.d_hap_flags;
    v.regions = s.d_regions;
    v.out = s.d_out;
    v.pair_flags = nullptr;
    const uint64_t warps = scratch_warps();
    PassControl pc{};
    pc.cd = s.d_classes + cls;
    pc.cd64 = s.d_classes + kClasses32;
    pc.items = s.d_items;
    pc.rerun = s.d_rerun;
    pc.status = s.d_status;
    pc.scratch = s.d_scratch;  // the FP32 multi-stripe region
    pc.scratch_cols = s.cap.scratch_cols ? (unsigned int)(s.cap.scratch_cols / warps) : 0u;
    const int grid = grid_for(32, cls, plan.classes[cls].n_items);
    cudaStream_t m = s.main;
    float best = 0.f;
    for (int r = 0; r < reps; ++r) {
        // fresh claim counters, rerun segments, codes and outputs for every repetition
        PHMM_CK(cudaMemcpyAsync(s.d_desc, s.d_desc_pristine, kDescBytes, cudaMemcpyDeviceToDevice, m));
        PHMM_CK(launch_prep(s.d_desc, s.d_hb, s.d_codes_inter, s.d_codes_intra, s.d_out, nullptr, sms_, m));
        PHMM_CK(cudaEventRecord(s.ev_t0, m));
        PHMM_CK(launch_fwd(32, cls, v, tf_, td_, pc, grid, m));
        PHMM_CK(cudaEventRecord(s.ev_t1, m));
        PHMM_CK(cudaEventSynchronize(s.ev_t1));
        float ms = 0.f;
        PHMM_CK(cudaEventElapsedTime(&ms, s.ev_t0, s.ev_t1));
        if (r == 0 || ms < best) best = ms;
    }
    unsigned int status = 0;
    PHMM_CK(cudaMemcpy(&status, s.d_status, sizeof(status), cudaMemcpyDeviceToHost));
    if (status != 0) {
        err = "kernel status word " + std::to_string(status) + " while timing class " + std::to_string(cls);
        return PHMM_ERR_DEVICE_STATUS;
    }
    *best_ms = best;
    return PHMM_OK;
}

phmm_status Engine::check_fp64(Slot& s, const Plan& plan, double* out, std::string& err)
{
    PHMM_CK(cudaSetDevice(dev_));
    cudaStream_t m = s.main;
    // Rerun entries covering every pair: per work item and read, the item's run of haplotypes, in
    // the FP64 class of the read's length (modes 1 and 2 only: the check kernels take any read).
    std::vector<std::vector<RerunEntry>> per(kClasses64);
    for (const WorkItem& it : plan.items) {
        const RegionDesc& rg = plan.regions[it.region];
        for (int k = 0; k < 2; ++k) {
            const uint32_t r = it.read[k];
            if (r == kNoRead) continue;
            RerunEntry e;
            e.out_idx = rg.out_off + (uint64_t)it.hap_lo * rg.n_reads + (r - rg.read_begin);
            e.read = r;
            e.hap = rg.hap_begin + it.hap_lo;
            e.n_haps = (uint32_t)(it.hap_hi - it.hap_lo);
            e.out_stride = rg.n_reads;
            const uint64_t R = plan.read_off[r + 1] - plan.read_off[r];
            per[class64_for_len(it.variant == kIntra ? 2 : 1, R)].push_back(e);
        }
    }
    std::vector<RerunEntry> all;
    std::vector<ClassDesc> cd(kClasses64);
    for (int c = 0; c < kClasses64; ++c) {
        cd[c] = ClassDesc{};
        cd[c].rerun_off = (uint32_t)all.size();
        cd[c].rerun_cap = cd[c].rerun_count = (uint32_t)per[c].size();
        all.insert(all.end(), per[c].begin(), per[c].end());
    }
    if (all.size() > s.cap.rerun) {
        err = "check entries exceed the slot's rerun capacity";
        return PHMM_ERR_INTERNAL;
    }
    BatchView v{};
    v.read_bases = s.d_rb;
    v.read_q = s.d_rq;
    v.read_i = s.d_ri;
    v.read_d = s.d_rd;
    v.read_c = s.d_rc;
    v.read_off = s.d_read_off;
    v.read_flags = s.d_read_flags;
    v.hap_off = s.d_hap_off;
    v.codes_inter = s.d_codes_inter;
    v.codes_intra = s.d_codes_intra;
    v.hap_flags = s.d_hap_flags;
    v.regions = s.d_regions;
    v.out = s.d_out;
    v.pair_flags = nullptr;
    // outputs NaN and codes rebuilt (the prep kernels of a run), then the check's own descriptors
    PHMM_CK(cudaMemcpyAsync(s.d_desc, s.d_desc_pristine, kDescBytes, cudaMemcpyDeviceToDevice, m));
    PHMM_CK(launch_prep(s.d_desc, s.d_hb, s.d_codes_inter, s.d_codes_intra, s.d_out, nullptr, sms_, m));
    if (!all.empty())
        PHMM_CK(cudaMemcpyAsync(s.d_rerun, all.data(), all.size() * sizeof(RerunEntry), cudaMemcpyHostToDevice, m));
    PHMM_CK(cudaMemcpyAsync(s.d_classes + kClasses32, cd.data(), kClasses64 * sizeof(ClassDesc), cudaMemcpyHostToDevice,
                            m));
    const uint64_t warps = scratch_warps();
    const unsigned int scr_cols = s.cap.scratch_cols ? (unsigned int)(s.cap.scratch_cols / warps) : 0u;
    for (int c = 9; c < kClasses64; ++c) {
        if (per[c].empty()) continue;
        const bool multi = c % 9 == 8;
        const int region = 1 + c / 9;
        int occ = 0;
        PHMM_CK(occupancy_f64_check(c, &occ));
        uint64_t grid = std::min<uint64_t>(per[c].size(), (uint64_t)std::max(occ, 1) * sms_);
        if (multi) grid = std::min(grid, scratch_offset_warps(region + 1) - scratch_offset_warps(region));
        PassControl pc{};
        pc.cd = s.d_classes + kClasses32 + c;
        pc.cd64 = s.d_classes + kClasses32;
        pc.items = s.d_items;
        pc.rerun = s.d_rerun;
        pc.status = s.d_status;
        pc.scratch = multi ? (void*)((char*)s.d_scratch + scratch_offset_warps(region) * scr_cols * 24) : nullptr;
        pc.scratch_cols = scr_cols;
        PHMM_CK(launch_f64_check(c, v, td_, pc, (int)std::max<uint64_t>(grid, 1), m));
    }
    if (plan.out_total) PHMM_CK(cudaMemcpyAsync(out, s.d_out, plan.out_total * sizeof(double), cudaMemcpyDeviceToHost, m));
    unsigned int status = 0;
    PHMM_CK(cudaMemcpyAsync(&status, s.d_status, sizeof(status), cudaMemcpyDeviceToHost, m));
    PHMM_CK(cudaStreamSynchronize(m));
    if (status != 0) {
        err = "kernel status word " + std::to_string(status) + " in the all-FP64 check";
        return PHMM_ERR_DEVICE_STATUS;
    }
    return PHMM_OK;
}

phmm_status Engine::profile_classes(Slot& s, const Plan& plan, float* class_ms, std::string& err)
{
    PHMM_CK(cudaSetDevice(dev_));
    cudaStream_t m = s.main;
    BatchView v{};
    v.read_bases = s.d_rb;
    v.read_q = s.d_rq;
    v.read_i = s.d_ri;
    v.read_d = s.d_rd;
    v.read_c = s.d_rc;
    v.read_off = s.d_read_off;
    v.read_flags = s.d_read_flags;
    v.hap_off = s.d_hap_off;
    v.codes_inter = s.d_codes_inter;
    v.codes_intra = s.d_codes_intra;
    v.hap_flags = s.d_hap_flags;
    v.regions = s.d_regions;
    v.out = s.d_out;
    v.pair_flags = s.d_pair_flags;
    const uint64_t warps = scratch_warps();
    const unsigned int scr_cols = s.cap.scratch_cols ? (unsigned int)(s.cap.scratch_cols / warps) : 0u;
    std::vector<cudaEvent_t> ev(2 * kNumClasses, nullptr);
    for (auto& e : ev) PHMM_CK(cudaEventCreate(&e));
    struct Cleanup {
        std::vector<cudaEvent_t>& ev;
        ~Cleanup()
        {
            for (auto e : ev)
                if (e) cudaEventDestroy(e);
        }
    } cleanup{ev};
    PHMM_CK(cudaMemcpyAsync(s.d_desc, s.d_desc_pristine, kDescBytes, cudaMemcpyDeviceToDevice, m));
    PHMM_CK(launch_prep(s.d_desc, s.d_hb, s.d_codes_inter, s.d_codes_intra, s.d_out, v.pair_flags, sms_, m));
    const RegionApiView rv = region_view(s, d_jacobian_, log10_two_);
    if (plan.region_api) PHMM_CK(launch_read_prep(rv, sms_, m));
    bool ran[kNumClasses] = {};
    for (int pass = 0; pass < 2; ++pass) {
        const int precision = pass == 0 ? 32 : 64;
        const int n_cls = pass == 0 ? kClasses32 : kClasses64;
        const int slot0 = pass == 0 ? 0 : kClasses32;
        for (int c = 0; c < n_cls; ++c) {
            const uint32_t work = pass == 0 ? plan.classes[c].n_items : plan.classes[slot0 + c].rerun_cap;
            if (work == 0) continue;
            const bool multi = pass == 0 ? class32_multi(c) : c % 9 == 8;
            const int region = pass == 0 ? 0 : 1 + c / 9;
            PassControl pc{};
            pc.cd = s.d_classes + slot0 + c;
            pc.cd64 = s.d_classes + kClasses32;
            pc.items = s.d_items;
            pc.rerun = s.d_rerun;
            pc.status = s.d_status;
            pc.scratch = multi ? (void*)((char*)s.d_scratch + scratch_offset_warps(region) * scr_cols * 24) : nullptr;
            pc.scratch_cols = scr_cols;
            PHMM_CK(cudaEventRecord(ev[2 * (slot0 + c)], m));
            PHMM_CK(launch_fwd(precision, c, v, tf_, td_, pc, grid_for(precision, c, work), m));
            PHMM_CK(cudaEventRecord(ev[2 * (slot0 + c) + 1], m));
            ran[slot0 + c] = true;
        }
    }
    if (plan.region_api) {
        PHMM_CK(launch_post_region(rv, sms_, m));
        if (!plan.events.empty()) PHMM_CK(launch_genotype(rv, sms_, m));
    }
    PHMM_CK(cudaStreamSynchronize(m));
    for (int c = 0; c < kNumClasses; ++c) {
        class_ms[c] = 0.f;
        if (ran[c]) PHMM_CK(cudaEventElapsedTime(&class_ms[c], ev[2 * c], ev[2 * c + 1]));
    }
    return PHMM_OK;
}

}  // namespace phmm
