// Serving loop: continuous batching of single-region requests.
//
// The reference runs one PairHMM call per active region on each of --nthreads pool workers
// (haplotypecaller_engine.cpp:119,254; haplotypecaller.cpp:105).  Here those calls become
// requests: phmm_submit validates and copies the region and queues it; kSlots worker threads each
// own a device slot (arena, streams, captured graph) and pinned staging buffers.  A worker that is
// free takes every queued request that fits the HBM budget and the per-batch cell cap, gathers them
// into its pinned buffer, runs them as one batch, scatters the results and signals the requests.
// While one slot's batch is on the GPU the next worker is already forming and launching the next
// one, so requests that arrive meanwhile are admitted as soon as a slot and budget are free, and
// their kernels overlap with the running ones on the device.  Each pair's
// arithmetic does not depend on what it was batched with, so a region's likelihoods are the same
// alone and in any mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/phmm_b200.h"
#include "phmm_capi_internal.h"
#include "phmm_engine.h"
#include "phmm_sw.h"
#include "phmm_plan.h"

namespace phmm {

namespace {

using Clock = std::chrono::steady_clock;

// Batches in flight at once (build-time setting).  Measured on B200 with the serving slots' overlap
// scheduling (Engine::make_slot), 2,000-region pool at 95% of the end-to-end batched rate: p50/p99
// 37/57 ms with 5 slots, 56/98 ms with 8; without the overlap scheduling, 293/464 ms with 3 slots
// and 102/183 ms with 5.  The loop sustains about 2,730 GCUPS under overload with 5 slots.
#ifndef PHMM_SERVE_SLOTS
#define PHMM_SERVE_SLOTS 5
#endif
constexpr int kSlots = PHMM_SERVE_SLOTS;
// Gathering a batch's requests into pinned staging, and copying the results out to the requests, run
// on up to kGatherThreads threads (the worker and helpers) once a batch moves more than kGatherSplit
// bytes: one thread copies about 5 GB/s to or from page-locked memory, which made the gather a third
// of a large batch's host time.
constexpr int kGatherThreads = 4;
constexpr size_t kGatherSplit = 4u << 20;
// Bound on one batch's work (~40 ms on B200; build-time setting): a burst of requests becomes several
// batches that pipeline through the slots instead of one long batch that every later arrival waits
// behind.  Measured on B200 with 5 slots at 95% of the end-to-end batched rate (2,782 GCUPS): p50/p99
// 81/133 ms at 8e10 cells, 72/117 at 1.2e11, 75/114 at 1.6e11; under overload the loop sustains
// 2,735, 2,787 and 2,812 GCUPS.
#ifndef PHMM_SERVE_MAX_CELLS
#define PHMM_SERVE_MAX_CELLS 120000000000ull
#endif
constexpr uint64_t kMaxBatchCells = PHMM_SERVE_MAX_CELLS;
// Queued requests a forming batch looks through for requests of its kind.
constexpr size_t kAdmitScan = 4096;
constexpr size_t kMaxQueued = 1u << 20;

enum class ReqState { Queued, Running, Done };

struct Request {
    uint64_t id = 0;
    ReqState state = ReqState::Queued;
    phmm_status status = PHMM_OK;
    std::string error;
    // owned copy of the region: haplotype bases, then read bases, quals, ins, del, gcp
    uint32_t n_haps = 0, n_reads = 0;
    uint64_t hap_bases = 0, read_bases = 0;
    std::vector<uint8_t> data;
    std::vector<uint64_t> hap_off, read_off;  // rebased to 0
    double* out = nullptr;
    uint8_t* flags = nullptr;
    // region API (call_pairhmm semantics): data holds haplotype bases, read bases and raw base
    // qualities; the device prepares the reads and post-processes the likelihoods
    bool region_api = false;
    std::vector<uint8_t> mapq;
    RegionApiParams params{};
    uint8_t* keep = nullptr;
    uint32_t* n_kept = nullptr;
    // genotyping events of a region-API request
    std::vector<uint8_t> n_alleles;
    std::vector<int8_t> hap_allele;
    double* gl = nullptr;
    int32_t* best = nullptr;
    double* allele_lk = nullptr;
    uint64_t gl_n = 0, allele_lk_n = 0;
    // realignment of the kept reads to their best haplotypes (region API)
    bool realign = false;
    std::vector<double> prio;            // [n_haps]
    std::vector<uint16_t> clip;          // [n_reads][2]
    uint32_t max_hap = 0;                // longest haplotype
    int32_t* best_hap = nullptr;
    phmm_sw_result* sw = nullptr;
    uint32_t* cigars = nullptr;
    uint64_t cigar_capacity = 0;
    uint64_t* cigar_total = nullptr;
    phmm_status own_status = PHMM_OK;    // a failure of this request alone (its CIGAR buffer)
    std::string own_error;
    uint64_t out_n = 0;
    uint64_t cells = 0;
    uint64_t bytes = 0;  // device footprint estimate for admission
    Clock::time_point t_submit, t_admit, t_done;
};

// Page-locked host buffer that grows on demand (device copies from it are asynchronous DMA).
struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool reserve(size_t n)
    {
        if (n <= bytes) return true;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const size_t want = std::max(n, n / 2 * 3);
        if (cudaMallocHost(&p, want) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return false;
        }
        bytes = want;
        return true;
    }
    ~PinnedBuf()
    {
        if (p) cudaFreeHost(p);
    }
};

struct Server {
    Engine* eng = nullptr;
    std::mutex mu;
    std::condition_variable cv_work;   // workers: queue changed / stop
    std::condition_variable cv_done;   // waiters: a request finished
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> tickets;
    uint64_t next_id = 1;
    uint64_t budget = 0, in_use = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    phmm_server_stats stats{};         // guarded by mu

    void worker(int idx);
};

std::mutex g_reg_mu;
std::map<phmm_engine*, std::unique_ptr<Server>> g_servers;

struct HostCopy {
    uint8_t* dst;
    const uint8_t* src;
    size_t n;
};

// Runs the copies on up to kGatherThreads threads, split into runs of about equal bytes.
void run_copies(const std::vector<HostCopy>& copies, size_t total)
{
    auto run = [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) std::memcpy(copies[i].dst, copies[i].src, copies[i].n);
    };
    const int T = total < kGatherSplit ? 1 : (int)std::min<size_t>(kGatherThreads, copies.size());
    if (T <= 1) {
        run(0, copies.size());
        return;
    }
    std::vector<size_t> cut(T + 1, copies.size());
    cut[0] = 0;
    size_t acc = 0;
    int k = 1;
    for (size_t i = 0; i < copies.size() && k < T; ++i) {
        acc += copies[i].n;
        if (acc * T >= total * k) cut[k++] = i + 1;
    }
    std::vector<std::thread> helpers;
    for (int t = 1; t < T; ++t) helpers.emplace_back(run, cut[t], cut[t + 1]);
    run(cut[0], cut[1]);
    for (auto& h : helpers) h.join();
}

uint64_t footprint(uint64_t read_bases, uint64_t hap_bases, uint64_t pairs, uint64_t n_reads, uint64_t n_haps)
{
    return read_bases * 5 + hap_bases * 9 + pairs * (8 + 1 + 16) + n_reads * 17 + n_haps * 9 + 4096;
}

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// A realigning request's share of the batch's realignment: its reads' best haplotypes and
// alignments (a zero result for dropped reads) and its CIGAR ops, offsets rebased to its buffer.
void scatter_realign(Request& r, const RealignBatch& rb, size_t region)
{
    size_t k = 0;
    while (k < rb.regions.size() && rb.regions[k].region != region) ++k;
    if (k == rb.regions.size()) return;
    const uint32_t i0 = rb.regions[k].item_begin, n = r.n_reads;
    const uint64_t first = n ? rb.res[i0].cigar_offset : 0;
    const uint64_t end = n == 0 ? first : (i0 + n < rb.plan.n) ? rb.res[i0 + n].cigar_offset : rb.total;
    const uint64_t ops = end - first;
    if (r.cigar_total) *r.cigar_total = ops;
    for (uint32_t q = 0; q < n; ++q) {
        r.best_hap[q] = rb.best[i0 + q];
        phmm_sw_result x = rb.res[i0 + q];
        if (rb.best[i0 + q] < 0) x = phmm_sw_result{};
        else x.cigar_offset = (uint32_t)(x.cigar_offset - first);
        r.sw[q] = x;
    }
    if (ops > r.cigar_capacity) {
        r.own_status = PHMM_ERR_LIMIT_EXCEEDED;
        r.own_error = "realign: the region's CIGARs need " + std::to_string(ops) + " ops, the buffer holds " +
                      std::to_string(r.cigar_capacity);
        return;
    }
    if (ops) std::memcpy(r.cigars, rb.cigars.data() + first, 4 * ops);
}

void Server::worker(int idx)
{
    cudaSetDevice(eng->device());
    Slot* slot = nullptr;
    std::string err;
    const phmm_status mk = eng->make_slot(idx + 1, &slot, err, /*overlap=*/true);
    // Pre-size the slot for a full batch (kMaxBatchCells of benchmark-shaped regions, about 700),
    // when the budget allows: an arena that grows while other slots' batches run has to wait for
    // them (freeing device or pinned memory synchronises the device) and capture its graph again.
    Capacity floor;
    floor.regions = 4096;
    floor.reads = 256u << 10;
    floor.haps = 64u << 10;
    floor.read_bases = 48ull << 20;
    floor.hap_bases = 16ull << 20;
    floor.items = 256u << 10;
    floor.rerun = floor.out = 4ull << 20;
    floor.events = 64u << 10;
    floor.hap_allele = 2ull << 20;
    floor.allele_lk = 8ull << 20;
    floor.gl = 1ull << 20;
    const size_t in_floor = floor.hap_bases + 5 * floor.read_bases + floor.reads;
    const size_t out_floor = floor.out * 9 + (floor.gl + floor.allele_lk) * 8 + floor.reads * 2;
    if (slot && eng->arena_bytes(floor) + in_floor <= budget / kSlots) {
        slot->floor = floor;
        std::string rerr;
        if (eng->reserve(*slot, floor, rerr) != PHMM_OK) slot->floor = Capacity();  // grow on demand instead
    }
    std::vector<std::shared_ptr<Request>> batch;
    std::vector<uint32_t> nh, nr;
    std::vector<uint64_t> hoff, roff;
    std::vector<RegionApiParams> params;
    std::vector<HostCopy> copies;
    PinnedBuf in_buf, out_buf;
    if (slot && slot->floor.read_bases) {
        in_buf.reserve(in_floor);
        out_buf.reserve(out_floor);
    }
    for (;;) {
        batch.clear();
        uint64_t batch_bytes = 0, hap_total = 0, read_total = 0, out_total = 0, cells = 0;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || (!queue.empty() && in_use + queue.front()->bytes <= budget); });
            if (stop && queue.empty()) break;
            // Slot arenas only grow, so each batch is held to budget / kSlots: the arenas of all
            // slots together then stay within the budget.  A request alone always fits (checked at
            // submit).
            const uint64_t batch_cap = budget / kSlots;
            const auto now = Clock::now();
            size_t scanned = 0;
            for (auto it = queue.begin(); it != queue.end() && scanned < kAdmitScan; ++scanned) {
                auto& r = *it;
                // A batch holds requests of one kind (region API or plain likelihoods).  A request
                // of the other kind stays queued, in order, and heads the next slot's batch.
                if (!batch.empty() && r->region_api != batch.front()->region_api) {
                    ++it;
                    continue;
                }
                const bool fits = in_use + batch_bytes + r->bytes <= budget &&
                                  (batch.empty() || batch_bytes + r->bytes <= batch_cap);
                if (!fits || (!batch.empty() && cells + r->cells > kMaxBatchCells)) break;
                batch_bytes += r->bytes;
                cells += r->cells;
                hap_total += r->hap_bases;
                read_total += r->read_bases;
                out_total += r->out_n;
                r->state = ReqState::Running;
                r->t_admit = now;
                batch.push_back(r);
                it = queue.erase(it);
            }
            in_use += batch_bytes;
        }
        if (batch.empty()) continue;
        const auto t_start = Clock::now();
        const uint64_t grows0 = slot ? slot->arena_grows : 0, caps0 = slot ? slot->graph_captures : 0;
        const double setup0 = slot ? slot->setup_ms : 0.0;
        double wait_ms = 0.0;  // time blocked on the device in finish()
        // host phases of the batch (ms): gather into pinned staging, planning, upload and launch,
        // results back to the requests
        double gather_ms = 0.0, plan_ms = 0.0, enqueue_ms = 0.0, scatter_ms = 0.0;
        phmm_status st = mk;
        std::string berr = err;
        double device_ms = 0.0;
        bool want_flags = false;
        for (auto& r : batch) want_flags |= r->flags != nullptr;
        const bool api = batch.front()->region_api;
        const int read_arrays = api ? 2 : 5;  // region API: bases and raw qualities only
        uint64_t reads_total = 0;
        for (auto& r : batch) reads_total += r->n_reads;
        // the admitted regions go into the slot's pinned buffers: haplotype bases, then the read
        // arrays (and MAPQ) in; likelihoods (and flags, or kept flags and counts) out
        const size_t in_bytes = hap_total + read_arrays * read_total + (api ? reads_total : 0) + 16;
        uint64_t gl_total = 0, alk_total = 0, n_events = 0;
        bool want_out = false, want_alk = false;
        for (auto& r : batch) {
            gl_total += r->gl_n;
            alk_total += r->allele_lk_n;
            n_events += r->n_alleles.size();
            want_out |= r->out != nullptr;
            want_alk |= r->allele_lk != nullptr;
        }
        const size_t out_bytes = out_total * sizeof(double) + (want_flags ? out_total : 0) +
                                 (api ? reads_total + batch.size() * sizeof(uint32_t) + 16 : 0) +
                                 (gl_total + alk_total) * sizeof(double) + n_events * sizeof(int32_t) + 64;
        if (st == PHMM_OK && !(in_buf.reserve(in_bytes) && out_buf.reserve(out_bytes))) {
            st = PHMM_ERR_OUT_OF_MEMORY;
            berr = "pinned staging for a batch of " + std::to_string(batch.size()) + " regions";
        }
        if (st == PHMM_OK) {
            uint8_t* hb = (uint8_t*)in_buf.p;
            uint8_t* rd[5] = {};
            for (int k = 0; k < read_arrays; ++k) rd[k] = hb + hap_total + (uint64_t)k * read_total;
            uint8_t* mq = hb + hap_total + (uint64_t)read_arrays * read_total;
            uint64_t mo = 0;
            params.clear();
            nh.clear();
            nr.clear();
            hoff.assign(1, 0);
            roff.assign(1, 0);
            uint64_t ho = 0, ro = 0;
            copies.clear();
            size_t copy_bytes = 0;
            auto add = [&](uint8_t* dst, const uint8_t* src, size_t n) {
                if (n) copies.push_back({dst, src, n});
                copy_bytes += n;
            };
            for (auto& r : batch) {
                nh.push_back(r->n_haps);
                nr.push_back(r->n_reads);
                for (uint32_t h = 0; h < r->n_haps; ++h) hoff.push_back(ho + r->hap_off[h + 1]);
                for (uint32_t k = 0; k < r->n_reads; ++k) roff.push_back(ro + r->read_off[k + 1]);
                add(hb + ho, r->data.data(), r->hap_bases);
                for (int k = 0; k < read_arrays && r->read_bases; ++k)
                    add(rd[k] + ro, r->data.data() + r->hap_bases + (uint64_t)k * r->read_bases, r->read_bases);
                if (api) {
                    add(mq + mo, r->mapq.data(), r->n_reads);
                    mo += r->n_reads;
                    params.push_back(r->params);
                }
                ho += r->hap_bases;
                ro += r->read_bases;
            }
            run_copies(copies, copy_bytes);
            phmm_batch b{};
            b.n_regions = (uint32_t)batch.size();
            b.n_haps = nh.data();
            b.n_reads = nr.data();
            b.hap_bases = hb;
            b.hap_off = hoff.data();
            b.read_bases = rd[0];
            b.read_qual = rd[1];
            b.read_ins = rd[2];
            b.read_del = rd[3];
            b.read_gcp = rd[4];
            b.read_off = roff.data();
            const auto t_gathered = Clock::now();
            gather_ms = ms_between(t_start, t_gathered);
            Plan plan;
            const TileTable tiles = eng->tiles();
            PlanLimits lim = Engine::limits_with(tiles);
            if (api) lim.region_api = params.data();
            st = build_plan(b, lim, plan, berr);
            if (st == PHMM_OK && n_events) {
                // events of the batch, in request order
                uint64_t gl_o = 0, alk_o = 0;
                for (size_t i = 0; i < batch.size(); ++i) {
                    auto& r = batch[i];
                    for (size_t e = 0; e < r->n_alleles.size(); ++e) {
                        EventDesc ev{};
                        ev.region = (uint32_t)i;
                        ev.n_alleles = r->n_alleles[e];
                        ev.hap_allele_off = plan.hap_allele.size();
                        ev.gl_off = gl_o;
                        ev.allele_lk_off = alk_o;
                        plan.hap_allele.insert(plan.hap_allele.end(), r->hap_allele.begin() + e * r->n_haps,
                                               r->hap_allele.begin() + (e + 1) * r->n_haps);
                        gl_o += (uint64_t)ev.n_alleles * (ev.n_alleles + 1) / 2;
                        alk_o += (uint64_t)ev.n_alleles * r->n_reads;
                        plan.events.push_back(ev);
                    }
                }
                plan.gl_total = gl_o;
                plan.allele_lk_total = alk_o;
            }
            const auto t_planned = Clock::now();
            plan_ms = ms_between(t_gathered, t_planned);
            if (st == PHMM_OK) st = eng->enqueue(*slot, plan, b, want_flags, berr, api ? mq : nullptr);
            // realignment of the kept reads of the requests that asked for it, after the pipeline
            RealignBatch rb;
            if (st == PHMM_OK && api) {
                uint32_t item = 0;
                for (size_t i = 0; i < batch.size(); ++i) {
                    auto& r = batch[i];
                    if (!r->realign) continue;
                    rb.regions.push_back(RealignRegion{(uint32_t)i, item, (uint64_t)rb.prio.size()});
                    rb.prio.insert(rb.prio.end(), r->prio.begin(), r->prio.end());
                    rb.clip.insert(rb.clip.end(), r->clip.begin(), r->clip.end());
                    for (uint32_t k = 0; k < r->n_reads; ++k) {
                        const uint64_t len = r->read_off[k + 1] - r->read_off[k];
                        rb.nrow.push_back(r->max_hap);
                        rb.ncol.push_back((uint32_t)(len - r->clip[2 * k] - r->clip[2 * k + 1]));
                    }
                    item += r->n_reads;
                }
                if (item) {
                    const SwParams prm{10, -15, -30, -5};  // sw_parameters_genotype, lib/sw_avx/sw_avx.c:15
                    st = sw_plan(eng->device(), prm, 0, item, rb.nrow.data(), rb.ncol.data(), kSwMaxSeq - 1, rb.plan,
                                 berr);
                    if (st == PHMM_OK) st = eng->realign_enqueue(*slot, rb, berr);
                }
            }
            double* out = (double*)out_buf.p;
            uint8_t* flags = want_flags ? (uint8_t*)(out + out_total) : nullptr;
            double* gl = out + out_total;
            double* alk = gl + gl_total;
            int32_t* best = (int32_t*)(alk + alk_total);
            uint32_t* kept_n = api ? (uint32_t*)(best + n_events) : nullptr;
            uint8_t* keep = api ? (uint8_t*)(kept_n + batch.size()) : nullptr;
            if (want_flags) flags = (uint8_t*)(best + n_events);  // plain batches have no events
            phmm_stats ps{};
            const auto t_fin = Clock::now();
            enqueue_ms = ms_between(t_planned, t_fin);
            if (st == PHMM_OK)
                st = eng->finish(*slot, plan, (!api || want_out) ? out : nullptr, flags, &ps, berr, keep, kept_n,
                                 n_events ? gl : nullptr, n_events ? best : nullptr, want_alk ? alk : nullptr);
            if (st == PHMM_OK && rb.plan.n) st = eng->realign_finish(*slot, rb, berr);
            device_ms = ps.device_ms;
            const auto t_back = Clock::now();
            wait_ms = ms_between(t_fin, t_back);
            if (st == PHMM_OK) {
                uint64_t o = 0, ko = 0, go = 0, ao = 0, eo = 0;
                copies.clear();
                size_t copy_bytes = 0;
                auto add = [&](void* dst, const void* src, size_t n) {
                    if (n) copies.push_back({(uint8_t*)dst, (const uint8_t*)src, n});
                    copy_bytes += n;
                };
                for (size_t i = 0; i < batch.size(); ++i) {
                    auto& r = batch[i];
                    if (r->out) add(r->out, out + o, r->out_n * sizeof(double));
                    if (r->flags) add(r->flags, flags + o, r->out_n);
                    if (api) {
                        add(r->keep, keep + ko, r->n_reads);
                        *r->n_kept = kept_n[i];
                    }
                    if (r->realign) scatter_realign(*r, rb, i);
                    if (!r->n_alleles.empty()) {
                        add(r->gl, gl + go, r->gl_n * sizeof(double));
                        add(r->best, best + eo, r->n_alleles.size() * sizeof(int32_t));
                        if (r->allele_lk) add(r->allele_lk, alk + ao, r->allele_lk_n * sizeof(double));
                    }
                    o += r->out_n;
                    ko += r->n_reads;
                    go += r->gl_n;
                    ao += r->allele_lk_n;
                    eo += r->n_alleles.size();
                }
                run_copies(copies, copy_bytes);
            }
            scatter_ms = ms_between(t_back, Clock::now());
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            const auto now = Clock::now();
            for (auto& r : batch) {
                r->status = st != PHMM_OK ? st : r->own_status;
                r->error = st != PHMM_OK ? berr : r->own_error;
                r->state = ReqState::Done;
                r->t_done = now;
                std::vector<uint8_t>().swap(r->data);  // inputs are no longer needed
                stats.max_queue_ms = std::max(stats.max_queue_ms, ms_between(r->t_submit, r->t_admit));
            }
            in_use -= batch_bytes;
            stats.batches += 1;
            stats.requests_done += batch.size();
            stats.cells_done += cells;
            stats.max_batch_regions = std::max<uint64_t>(stats.max_batch_regions, batch.size());
            stats.batch_ms += ms_between(t_start, now);
            stats.device_ms += device_ms;
            stats.max_batch_ms = std::max(stats.max_batch_ms, ms_between(t_start, now));
            stats.gather_ms += gather_ms;
            stats.plan_ms += plan_ms;
            stats.enqueue_ms += enqueue_ms;
            stats.wait_ms += wait_ms;
            stats.scatter_ms += scatter_ms;
            if (slot) {
                stats.arena_grows += slot->arena_grows - grows0;
                stats.graph_captures += slot->graph_captures - caps0;
                stats.max_setup_ms = std::max(stats.max_setup_ms, slot->setup_ms - setup0);
                stats.max_host_ms =
                    std::max(stats.max_host_ms, ms_between(t_start, now) - wait_ms - (slot->setup_ms - setup0));
            }
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
    if (slot) eng->free_slot(slot);
}

Server* server_for(phmm_engine* e, bool create)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    auto it = g_servers.find(e);
    if (it != g_servers.end()) return it->second.get();
    if (!create) return nullptr;
    auto s = std::make_unique<Server>();
    s->eng = engine_of(e);
    s->budget = s->eng->config().hbm_budget_bytes;
    for (int i = 0; i < kSlots; ++i) s->workers.emplace_back(&Server::worker, s.get(), i);
    Server* raw = s.get();
    g_servers[e] = std::move(s);
    return raw;
}

}  // namespace

void server_release(phmm_engine* e)
{
    std::unique_ptr<Server> s;
    {
        std::lock_guard<std::mutex> lk(g_reg_mu);
        auto it = g_servers.find(e);
        if (it == g_servers.end()) return;
        s = std::move(it->second);
        g_servers.erase(it);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        // queued requests will not be served
        for (auto& r : s->queue) {
            r->state = ReqState::Done;
            r->status = PHMM_ERR_CANCELLED;
            r->error = "engine destroyed";
        }
        s->queue.clear();
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    for (auto& t : s->workers) t.join();
}

// Queues a prepared request (admission checks against the HBM budget).
phmm_status enqueue_request(phmm_engine* engine, const std::shared_ptr<Request>& r, phmm_ticket* ticket,
                            std::string& err)
{
    Server* s = server_for(engine, true);
    if (r->bytes > s->budget) {
        err = "region needs about " + std::to_string(r->bytes) + " device bytes, more than the HBM budget of " +
              std::to_string(s->budget);
        return PHMM_ERR_LIMIT_EXCEEDED;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            err = "engine is shutting down";
            return PHMM_ERR_NOT_INITIALIZED;
        }
        if (s->queue.size() >= kMaxQueued) {
            err = "serving queue is full";
            return PHMM_ERR_QUEUE_FULL;
        }
        r->id = s->next_id++;
        r->t_submit = Clock::now();
        s->tickets[r->id] = r;
        s->queue.push_back(r);
        s->stats.requests_submitted += 1;
        s->stats.queue_peak = std::max<uint64_t>(s->stats.queue_peak, s->queue.size());
        *ticket = r->id;
    }
    s->cv_work.notify_one();
    return PHMM_OK;
}

// Submits a copy of one region; used by phmm_submit and the region API.
phmm_status server_submit(phmm_engine* engine, const phmm_batch& b, double* out, uint8_t* flags, phmm_ticket* ticket,
                          std::string& err)
{
    if (b.n_regions != 1) {
        err = "a request holds exactly one region (n_regions == 1)";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    // validate with the planner's rules before queueing (limits, offsets, pointers)
    BatchScan sc;
    phmm_status st = scan_batch(b, PlanLimits(), sc, err);
    if (st != PHMM_OK) return st;
    if (sc.out_total && !out) {
        err = "out is null";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    auto r = std::make_shared<Request>();
    r->n_haps = sc.n_haps;
    r->n_reads = sc.n_reads;
    r->hap_bases = sc.hap_bases;
    r->read_bases = sc.read_bases;
    r->hap_off.resize(sc.n_haps + 1);
    r->read_off.resize(sc.n_reads + 1);
    for (uint32_t h = 0; h <= sc.n_haps; ++h) r->hap_off[h] = b.hap_off[h] - sc.hap_base0;
    for (uint32_t k = 0; k <= sc.n_reads; ++k) r->read_off[k] = b.read_off[k] - sc.read_base0;
    r->data.resize(sc.hap_bases + 5 * sc.read_bases);
    if (sc.hap_bases) std::memcpy(r->data.data(), b.hap_bases + sc.hap_base0, sc.hap_bases);
    const uint8_t* src[5] = {b.read_bases, b.read_qual, b.read_ins, b.read_del, b.read_gcp};
    for (int k = 0; k < 5 && sc.read_bases; ++k)
        std::memcpy(r->data.data() + sc.hap_bases + (uint64_t)k * sc.read_bases, src[k] + sc.read_base0, sc.read_bases);
    r->out = out;
    r->flags = flags;
    r->out_n = sc.out_total;
    r->cells = sc.cells;
    r->bytes = footprint(sc.read_bases, sc.hap_bases, sc.out_total, sc.n_reads, sc.n_haps);
    // a read longer than one stripe needs the per-warp scratch rows
    for (uint32_t k = 0; k < sc.n_reads; ++k)
        if (r->read_off[k + 1] - r->read_off[k] > (uint64_t)kWarp * kMaxK) {
            r->bytes += engine_of(engine)->scratch_bytes();
            break;
        }
    return enqueue_request(engine, r, ticket, err);
}

// Submits one region with call_pairhmm semantics: raw base qualities and MAPQ are copied, the
// device prepares the reads and post-processes the likelihoods.
phmm_status server_submit_region(phmm_engine* engine, const phmm_region_input& in, const phmm_region_events* events,
                                 double* out, uint8_t* keep, uint32_t* n_kept, phmm_ticket* ticket, std::string& err,
                                 const phmm_region_realign* realign)
{
    if (!in.hap_off || !in.read_off || (in.n_reads && (!in.mapq || !keep)) || !n_kept) {
        err = "null argument";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    if (in.pcr_model < PHMM_PCR_NONE || in.pcr_model > PHMM_PCR_CONSERVATIVE) {
        err = "pcr_model out of range";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    phmm_batch b{};
    b.n_regions = 1;
    b.n_haps = &in.n_haps;
    b.n_reads = &in.n_reads;
    b.hap_bases = in.hap_bases;
    b.hap_off = in.hap_off;
    b.read_bases = in.read_bases;
    b.read_qual = in.read_qual;
    b.read_off = in.read_off;
    RegionApiParams params{in.min_quality_threshold, in.pcr_model};
    PlanLimits lim;
    lim.region_api = &params;
    BatchScan sc;
    phmm_status st = scan_batch(b, lim, sc, err);
    if (st != PHMM_OK) return st;
    const uint32_t n_events = events ? events->n_events : 0;
    if (sc.out_total && !out && n_events == 0) {
        err = "out is null";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    if (n_events && (!events->n_alleles || (sc.n_haps && !events->hap_allele) || !events->genotype_lk ||
                     !events->best_genotype)) {
        err = "events: n_alleles, hap_allele, genotype_lk and best_genotype are required";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    auto r = std::make_shared<Request>();
    r->region_api = true;
    for (uint32_t e = 0; e < n_events; ++e) {
        const uint32_t A = events->n_alleles[e];
        if (A < 1 || A > kMaxAlleles) {
            err = "event " + std::to_string(e) + ": " + std::to_string(A) + " alleles (1.." + std::to_string(kMaxAlleles) +
                  " supported)";
            return PHMM_ERR_LIMIT_EXCEEDED;
        }
        for (uint32_t h = 0; h < sc.n_haps; ++h) {
            const int8_t a = events->hap_allele[(uint64_t)e * sc.n_haps + h];
            if (a < -1 || a >= (int)A) {
                err = "event " + std::to_string(e) + ": haplotype " + std::to_string(h) + " mapped to allele " +
                      std::to_string(a) + " of " + std::to_string(A);
                return PHMM_ERR_INVALID_ARGUMENT;
            }
        }
        r->gl_n += (uint64_t)A * (A + 1) / 2;
        r->allele_lk_n += (uint64_t)A * sc.n_reads;
    }
    if (n_events) {
        r->n_alleles.assign(events->n_alleles, events->n_alleles + n_events);
        r->hap_allele.assign(events->hap_allele, events->hap_allele + (uint64_t)n_events * sc.n_haps);
        r->gl = events->genotype_lk;
        r->best = events->best_genotype;
        r->allele_lk = events->allele_lk;
    }
    r->params = params;
    r->n_haps = sc.n_haps;
    r->n_reads = sc.n_reads;
    r->hap_bases = sc.hap_bases;
    r->read_bases = sc.read_bases;
    r->hap_off.resize(sc.n_haps + 1);
    r->read_off.resize(sc.n_reads + 1);
    for (uint32_t h = 0; h <= sc.n_haps; ++h) r->hap_off[h] = in.hap_off[h] - sc.hap_base0;
    for (uint32_t k = 0; k <= sc.n_reads; ++k) r->read_off[k] = in.read_off[k] - sc.read_base0;
    r->data.resize(sc.hap_bases + 2 * sc.read_bases);
    if (sc.hap_bases) std::memcpy(r->data.data(), in.hap_bases + sc.hap_base0, sc.hap_bases);
    if (sc.read_bases) {
        std::memcpy(r->data.data() + sc.hap_bases, in.read_bases + sc.read_base0, sc.read_bases);
        std::memcpy(r->data.data() + sc.hap_bases + sc.read_bases, in.read_qual + sc.read_base0, sc.read_bases);
    }
    r->mapq.assign(in.mapq, in.mapq + sc.n_reads);
    if (realign) {
        if ((sc.n_haps && !realign->hap_priority) || (sc.n_reads && (!realign->best_hap || !realign->sw)) ||
            (realign->cigar_capacity && !realign->cigars)) {
            err = "realign: hap_priority, best_hap and sw are required (cigars when cigar_capacity > 0)";
            return PHMM_ERR_INVALID_ARGUMENT;
        }
        r->realign = true;
        if (sc.n_haps) r->prio.assign(realign->hap_priority, realign->hap_priority + sc.n_haps);
        r->clip.assign(2ull * sc.n_reads, 0);
        for (uint32_t k = 0; k < sc.n_reads; ++k) {
            const uint64_t len = r->read_off[k + 1] - r->read_off[k];
            const uint32_t cl = realign->clip_left ? realign->clip_left[k] : 0;
            const uint32_t cr = realign->clip_right ? realign->clip_right[k] : 0;
            if (cl + cr > len) {
                err = "realign: read " + std::to_string(k) + " clips " + std::to_string(cl) + " + " +
                      std::to_string(cr) + " bases of " + std::to_string(len);
                return PHMM_ERR_INVALID_ARGUMENT;
            }
            r->clip[2 * k] = (uint16_t)cl;
            r->clip[2 * k + 1] = (uint16_t)cr;
        }
        for (uint32_t h = 0; h < sc.n_haps; ++h)
            r->max_hap = std::max<uint32_t>(r->max_hap, (uint32_t)(r->hap_off[h + 1] - r->hap_off[h]));
        r->best_hap = realign->best_hap;
        r->sw = realign->sw;
        r->cigars = realign->cigars;
        r->cigar_capacity = realign->cigar_capacity;
        r->cigar_total = realign->cigar_total;
    }
    r->out = out;
    r->keep = keep;
    r->n_kept = n_kept;
    r->out_n = sc.out_total;
    r->cells = sc.cells;
    r->bytes = footprint(sc.read_bases, sc.hap_bases, sc.out_total, sc.n_reads, sc.n_haps) + sc.out_total * 8 +
               sc.n_reads * 2 + r->hap_allele.size() + (r->gl_n + r->allele_lk_n) * 8 + n_events * 36;
    if (r->realign)  // items, results and two CIGAR slots per read, and its share of the scratch
        r->bytes += sc.n_reads * (96 + 8ull * std::min<uint64_t>(kSwMaxSeq - 1, r->max_hap + (sc.read_bases /
                                                                        std::max<uint32_t>(sc.n_reads, 1) + 1)))
                    + sc.read_bases * (r->max_hap / 2 + 64) + 4096;
    for (uint32_t k = 0; k < sc.n_reads; ++k)
        if (r->read_off[k + 1] - r->read_off[k] > (uint64_t)kWarp * kMaxK) {
            r->bytes += engine_of(engine)->scratch_bytes();
            break;
        }
    return enqueue_request(engine, r, ticket, err);
}

phmm_status server_wait(phmm_engine* engine, phmm_ticket ticket, int64_t timeout_us, bool release, double* queued_us,
                        double* total_us, std::string& err)
{
    Server* s = server_for(engine, false);
    if (!s) {
        err = "no request was ever submitted to this engine";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) {
        err = "unknown ticket " + std::to_string(ticket);
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    std::shared_ptr<Request> r = it->second;
    auto done = [&] { return r->state == ReqState::Done; };
    if (timeout_us < 0)
        s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), done))
        return PHMM_ERR_TIMEOUT;
    using us = std::chrono::duration<double, std::micro>;
    if (queued_us) *queued_us = r->t_admit >= r->t_submit ? us(r->t_admit - r->t_submit).count() : 0.0;
    if (total_us) *total_us = us(r->t_done - r->t_submit).count();
    if (release) s->tickets.erase(ticket);
    if (r->status != PHMM_OK) err = r->error;
    return r->status;
}

}  // namespace phmm

using phmm::set_error;

extern "C" {

phmm_status phmm_submit(phmm_engine* engine, const phmm_batch* region, double* out, uint8_t* pair_flags,
                        phmm_ticket* ticket)
{
    try {
        phmm::clear_error();
        if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
        if (!region || !ticket) return set_error(PHMM_ERR_INVALID_ARGUMENT, "region or ticket is null");
        std::string err;
        phmm_status st = phmm::server_submit(engine, *region, out, pair_flags, ticket, err);
        return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    } catch (const std::bad_alloc&) {
        return set_error(PHMM_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

phmm_status phmm_submit_region(phmm_engine* engine, const phmm_region_input* region, const phmm_region_events* events,
                               double* out, uint8_t* keep, uint32_t* n_kept, phmm_ticket* ticket)
{
    try {
        phmm::clear_error();
        if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
        if (!region || !ticket) return set_error(PHMM_ERR_INVALID_ARGUMENT, "region or ticket is null");
        std::string err;
        phmm_status st = phmm::server_submit_region(engine, *region, events, out, keep, n_kept, ticket, err, nullptr);
        return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    } catch (const std::bad_alloc&) {
        return set_error(PHMM_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

phmm_status phmm_submit_region_realign(phmm_engine* engine, const phmm_region_input* region,
                                       const phmm_region_events* events, const phmm_region_realign* realign,
                                       double* out, uint8_t* keep, uint32_t* n_kept, phmm_ticket* ticket)
{
    try {
        phmm::clear_error();
        if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
        if (!region || !ticket) return set_error(PHMM_ERR_INVALID_ARGUMENT, "region or ticket is null");
        std::string err;
        phmm_status st =
            phmm::server_submit_region(engine, *region, events, out, keep, n_kept, ticket, err, realign);
        return st == PHMM_OK ? PHMM_OK : set_error(st, err);
    } catch (const std::bad_alloc&) {
        return set_error(PHMM_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

phmm_status phmm_poll(phmm_engine* engine, phmm_ticket ticket, int32_t* done)
{
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    if (!done) return set_error(PHMM_ERR_INVALID_ARGUMENT, "done is null");
    std::string err;
    phmm_status st = phmm::server_wait(engine, ticket, 0, false, nullptr, nullptr, err);
    if (st == PHMM_ERR_TIMEOUT) {
        *done = 0;
        return PHMM_OK;
    }
    if (st == PHMM_ERR_INVALID_ARGUMENT) return set_error(st, err);
    *done = 1;
    return PHMM_OK;
}

phmm_status phmm_wait(phmm_engine* engine, phmm_ticket ticket, int64_t timeout_us, double* queued_us, double* total_us)
{
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    std::string err;
    phmm_status st = phmm::server_wait(engine, ticket, timeout_us, true, queued_us, total_us, err);
    return st == PHMM_OK ? PHMM_OK : set_error(st, err);
}

phmm_status phmm_server_stats_get(phmm_engine* engine, phmm_server_stats* stats)
{
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    if (!stats) return set_error(PHMM_ERR_INVALID_ARGUMENT, "stats is null");
    *stats = phmm_server_stats{};
    phmm::Server* s = phmm::server_for(engine, false);
    if (!s) return PHMM_OK;
    std::lock_guard<std::mutex> lk(s->mu);
    *stats = s->stats;
    return PHMM_OK;
}

phmm_status phmm_cancel(phmm_engine* engine, phmm_ticket ticket)
{
    phmm::clear_error();
    if (!engine) return set_error(PHMM_ERR_NOT_INITIALIZED, "engine is null");
    phmm::Server* s = phmm::server_for(engine, false);
    if (!s) return set_error(PHMM_ERR_INVALID_ARGUMENT, "no request was ever submitted to this engine");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) return set_error(PHMM_ERR_INVALID_ARGUMENT, "unknown ticket");
        auto r = it->second;
        if (r->state != phmm::ReqState::Queued)
            return set_error(PHMM_ERR_INVALID_ARGUMENT, "request already admitted; it cannot be cancelled");
        s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), r), s->queue.end());
        r->state = phmm::ReqState::Done;
        r->status = PHMM_ERR_CANCELLED;
        r->error = "cancelled";
        r->t_done = phmm::Clock::now();
    }
    s->cv_done.notify_all();
    return PHMM_OK;
}

}  // extern "C"
