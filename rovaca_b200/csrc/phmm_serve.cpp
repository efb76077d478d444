// Serving loop: continuous batching of single-region requests.
//
// The reference runs one PairHMM call per active region on each of --nthreads pool workers
// (haplotypecaller_engine.cpp:119,254; haplotypecaller.cpp:105).  Here those calls become
// requests: phmm_submit copies the region and queues it; kSlots worker threads each own a device
// slot (arena, streams, captured graph).  A worker that is free takes every queued request that
// fits the HBM budget and the per-batch cell cap, runs them as one batch, scatters the results and
// signals the requests.  While one slot's batch is on the GPU the next worker is already forming
// and launching the next one, so requests that arrive meanwhile are admitted as soon as a slot and
// budget are free, and their kernels overlap with the running ones on the device.  Each pair's
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

namespace phmm {

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kSlots = 3;                           // batches in flight at once
constexpr uint64_t kMaxBatchCells = 200000000000ull;  // bound on one batch's work (~0.1 s on B200)
constexpr size_t kMaxQueued = 1u << 20;

enum class ReqState { Queued, Running, Done };

struct Request {
    uint64_t id = 0;
    ReqState state = ReqState::Queued;
    phmm_status status = PHMM_OK;
    std::string error;
    // owned copy of the region
    uint32_t n_haps = 0, n_reads = 0;
    std::vector<uint8_t> hap_bases, read_bases, q, ins, del, gcp;
    std::vector<uint64_t> hap_off, read_off;
    double* out = nullptr;
    uint8_t* flags = nullptr;
    uint64_t out_n = 0;
    uint64_t cells = 0;
    uint64_t bytes = 0;  // device footprint estimate for admission
    Clock::time_point t_submit, t_admit, t_done;
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

    void worker(int idx);
};

std::mutex g_reg_mu;
std::map<phmm_engine*, std::unique_ptr<Server>> g_servers;

uint64_t footprint(uint64_t read_bases, uint64_t hap_bases, uint64_t pairs, uint64_t n_reads, uint64_t n_haps)
{
    return read_bases * 5 + hap_bases * 9 + pairs * (8 + 1 + 16) + n_reads * 17 + n_haps * 9 + 4096;
}

void Server::worker(int idx)
{
    cudaSetDevice(eng->device());
    Slot* slot = nullptr;
    std::string err;
    const phmm_status mk = eng->make_slot(idx + 1, &slot, err);
    std::vector<std::shared_ptr<Request>> batch;
    std::vector<uint32_t> nh, nr;
    std::vector<uint64_t> hoff, roff;
    std::vector<uint8_t> hb, rb, rq, ri, rd, rc;
    std::vector<double> out;
    std::vector<uint8_t> flags;
    for (;;) {
        batch.clear();
        uint64_t batch_bytes = 0;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || (!queue.empty() && in_use + queue.front()->bytes <= budget); });
            if (stop && queue.empty()) break;
            // Slot arenas only grow, so each batch is held to budget / kSlots: the arenas of all
            // slots together then stay within the budget.  A request alone always fits (checked at
            // submit).
            const uint64_t batch_cap = budget / kSlots;
            uint64_t cells = 0;
            while (!queue.empty()) {
                auto& r = queue.front();
                const bool fits = in_use + batch_bytes + r->bytes <= budget &&
                                  (batch.empty() || batch_bytes + r->bytes <= batch_cap);
                if (!fits || (!batch.empty() && cells + r->cells > kMaxBatchCells)) break;
                batch_bytes += r->bytes;
                cells += r->cells;
                r->state = ReqState::Running;
                r->t_admit = Clock::now();
                batch.push_back(r);
                queue.pop_front();
            }
            in_use += batch_bytes;
        }
        if (batch.empty()) continue;
        phmm_status st = mk;
        std::string berr = err;
        if (st == PHMM_OK) {
            // concatenate the admitted regions into one batch
            nh.clear();
            nr.clear();
            hoff.assign(1, 0);
            roff.assign(1, 0);
            hb.clear();
            rb.clear();
            rq.clear();
            ri.clear();
            rd.clear();
            rc.clear();
            uint64_t out_total = 0;
            bool want_flags = false;
            for (auto& r : batch) {
                nh.push_back(r->n_haps);
                nr.push_back(r->n_reads);
                for (uint32_t h = 0; h < r->n_haps; ++h) hoff.push_back(hb.size() + r->hap_off[h + 1]);
                for (uint32_t k = 0; k < r->n_reads; ++k) roff.push_back(rb.size() + r->read_off[k + 1]);
                hb.insert(hb.end(), r->hap_bases.begin(), r->hap_bases.end());
                rb.insert(rb.end(), r->read_bases.begin(), r->read_bases.end());
                rq.insert(rq.end(), r->q.begin(), r->q.end());
                ri.insert(ri.end(), r->ins.begin(), r->ins.end());
                rd.insert(rd.end(), r->del.begin(), r->del.end());
                rc.insert(rc.end(), r->gcp.begin(), r->gcp.end());
                out_total += r->out_n;
                want_flags |= r->flags != nullptr;
            }
            phmm_batch b{};
            b.n_regions = (uint32_t)batch.size();
            b.n_haps = nh.data();
            b.n_reads = nr.data();
            b.hap_bases = hb.data();
            b.hap_off = hoff.data();
            b.read_bases = rb.data();
            b.read_qual = rq.data();
            b.read_ins = ri.data();
            b.read_del = rd.data();
            b.read_gcp = rc.data();
            b.read_off = roff.data();
            Plan plan;
            st = build_plan(b, PlanLimits(), plan, berr);
            if (st == PHMM_OK) st = eng->enqueue(*slot, plan, b, want_flags, berr);
            if (st == PHMM_OK) {
                out.resize(out_total);
                flags.resize(want_flags ? out_total : 0);
                st = eng->finish(*slot, plan, out.data(), want_flags ? flags.data() : nullptr, nullptr, berr);
            }
            if (st == PHMM_OK) {
                uint64_t o = 0;
                for (auto& r : batch) {
                    if (r->out_n) std::memcpy(r->out, out.data() + o, r->out_n * sizeof(double));
                    if (r->flags && r->out_n) std::memcpy(r->flags, flags.data() + o, r->out_n);
                    o += r->out_n;
                }
            }
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            const auto now = Clock::now();
            for (auto& r : batch) {
                r->status = st;
                r->error = st == PHMM_OK ? std::string() : berr;
                r->state = ReqState::Done;
                r->t_done = now;
                // inputs are no longer needed
                std::vector<uint8_t>().swap(r->hap_bases);
                std::vector<uint8_t>().swap(r->read_bases);
                std::vector<uint8_t>().swap(r->q);
                std::vector<uint8_t>().swap(r->ins);
                std::vector<uint8_t>().swap(r->del);
                std::vector<uint8_t>().swap(r->gcp);
            }
            in_use -= batch_bytes;
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

// Submits a copy of one region; used by phmm_submit and the region API.
phmm_status server_submit(phmm_engine* engine, const phmm_batch& b, double* out, uint8_t* flags, phmm_ticket* ticket,
                          std::string& err)
{
    if (b.n_regions != 1) {
        err = "a request holds exactly one region (n_regions == 1)";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    // validate with the planner's rules before queueing (limits, offsets)
    Plan plan;
    phmm_status st = build_plan(b, PlanLimits(), plan, err);
    if (st != PHMM_OK) return st;
    if (plan.out_total && !out) {
        err = "out is null";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    auto r = std::make_shared<Request>();
    r->n_haps = b.n_haps[0];
    r->n_reads = b.n_reads[0];
    r->hap_off = plan.hap_off;
    r->read_off = plan.read_off;
    r->hap_bases.assign(b.hap_bases ? b.hap_bases + plan.hap_base0 : nullptr,
                        b.hap_bases ? b.hap_bases + plan.hap_base0 + plan.hap_bases : nullptr);
    auto cp = [&](std::vector<uint8_t>& dst, const uint8_t* src) {
        dst.assign(src ? src + plan.read_base0 : nullptr, src ? src + plan.read_base0 + plan.read_bases : nullptr);
    };
    cp(r->read_bases, b.read_bases);
    cp(r->q, b.read_qual);
    cp(r->ins, b.read_ins);
    cp(r->del, b.read_del);
    cp(r->gcp, b.read_gcp);
    r->out = out;
    r->flags = flags;
    r->out_n = plan.out_total;
    r->cells = plan.cells;
    r->bytes = footprint(plan.read_bases, plan.hap_bases, plan.out_total, plan.n_reads, plan.n_haps);
    if (plan.max_multi_stream) r->bytes += engine_of(engine)->arena_bytes_for(plan);
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
        *ticket = r->id;
    }
    s->cv_work.notify_one();
    return PHMM_OK;
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
