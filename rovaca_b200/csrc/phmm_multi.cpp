// Several devices behind one handle: the regions of a batch partitioned across one engine per
// device, and serving requests routed to the least-loaded device.
//
// The reference's only parallelism is its region thread pool (src/haplotypecaller/haplotypecaller.cpp:105,
// haplotypecaller_engine.cpp:119): regions are independent, so the device set shards whole regions,
// with no data exchanged between devices (no peer memory, no collective).  A batch's regions go to
// the devices by longest-processing-time greedy on their cell counts (sum over the region's pairs of
// read length x haplotype length = total read bases x total haplotype bases): regions in decreasing
// cell order, each to the part with the fewest cells so far (ties to the lower index), which bounds
// the largest part by the ideal share plus one region.  Each part's regions are gathered, in batch
// order, into the device's pinned staging buffers, computed on that device's engine (its own host
// thread), and each region's likelihood block is copied back to the region's own range of the
// caller's output.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/phmm_b200.h"
#include "phmm_capi_internal.h"
#include "phmm_plan.h"

namespace phmm {
namespace {

// Cells of every region of a validated batch.
std::vector<uint64_t> region_cells(const phmm_batch& b)
{
    std::vector<uint64_t> cells(b.n_regions);
    uint64_t h = 0, r = 0;
    for (uint32_t g = 0; g < b.n_regions; ++g) {
        const uint64_t hb = b.n_haps[g] ? b.hap_off[h + b.n_haps[g]] - b.hap_off[h] : 0;
        const uint64_t rb = b.n_reads[g] ? b.read_off[r + b.n_reads[g]] - b.read_off[r] : 0;
        cells[g] = hb * rb;
        h += b.n_haps[g];
        r += b.n_reads[g];
    }
    return cells;
}

void lpt(const std::vector<uint64_t>& cells, uint32_t parts, uint32_t* part_of, uint64_t* load)
{
    std::vector<uint32_t> order(cells.size());
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cells[a] > cells[b]; });
    std::fill(load, load + parts, 0);
    for (uint32_t g : order) {
        uint32_t best = 0;
        for (uint32_t p = 1; p < parts; ++p)
            if (load[p] < load[best]) best = p;
        part_of[g] = best;
        load[best] += cells[g];
    }
}

// Growable pinned host buffer (one per device and array).
struct Pinned {
    char* p = nullptr;
    size_t bytes = 0;
    bool ensure(size_t need)
    {
        if (need <= bytes) return true;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const size_t n = std::max<size_t>(need + need / 4, 1 << 20);
        if (cudaHostAlloc((void**)&p, n, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        bytes = n;
        return true;
    }
    ~Pinned()
    {
        if (p) cudaFreeHost(p);
    }
};

struct Member {
    int device = 0;
    phmm_engine* engine = nullptr;
    std::atomic<uint64_t> outstanding_cells{0};
    // staging of a part: counts, offsets, bases/qualities, outputs
    Pinned nh, nr, hoff, roff, hb, rb, rq, ri, rd, rc, out, flags;
};

struct PendingRequest {
    uint32_t member;
    phmm_ticket ticket;
    uint64_t cells;
};

}  // namespace
}  // namespace phmm

struct phmm_device_set {
    std::vector<std::unique_ptr<phmm::Member>> members;
    std::mutex compute_mu;  // one compute_regions at a time (they share the staging buffers)
    std::mutex mu;          // pending requests
    std::unordered_map<phmm_ticket, phmm::PendingRequest> pending;
    phmm_ticket next_ticket = 1;
};

using phmm::set_error;

namespace {

// Gathers the regions of one part (global indices, ascending) into member m's staging buffers and
// returns the sub-batch; false if pinned memory runs out.
bool gather(const phmm_batch& b, const std::vector<uint64_t>& hap_first, const std::vector<uint64_t>& read_first,
            const std::vector<uint32_t>& regs, phmm::Member& m, phmm_batch& sub, uint64_t& out_total)
{
    uint64_t nh = 0, nr = 0, hbytes = 0, rbytes = 0;
    out_total = 0;
    for (uint32_t g : regs) {
        nh += b.n_haps[g];
        nr += b.n_reads[g];
        hbytes += b.hap_off[hap_first[g] + b.n_haps[g]] - b.hap_off[hap_first[g]];
        rbytes += b.read_off[read_first[g] + b.n_reads[g]] - b.read_off[read_first[g]];
        out_total += (uint64_t)b.n_haps[g] * b.n_reads[g];
    }
    if (!m.nh.ensure(regs.size() * 4) || !m.nr.ensure(regs.size() * 4) || !m.hoff.ensure((nh + 1) * 8) ||
        !m.roff.ensure((nr + 1) * 8) || !m.hb.ensure(hbytes) || !m.rb.ensure(rbytes) || !m.rq.ensure(rbytes) ||
        !m.ri.ensure(rbytes) || !m.rd.ensure(rbytes) || !m.rc.ensure(rbytes) || !m.out.ensure(out_total * 8) ||
        !m.flags.ensure(out_total))
        return false;
    uint32_t* snh = (uint32_t*)m.nh.p;
    uint32_t* snr = (uint32_t*)m.nr.p;
    uint64_t* shoff = (uint64_t*)m.hoff.p;
    uint64_t* sroff = (uint64_t*)m.roff.p;
    uint64_t ho = 0, ro = 0, hk = 0, rk = 0;
    shoff[0] = 0;
    sroff[0] = 0;
    for (size_t k = 0; k < regs.size(); ++k) {
        const uint32_t g = regs[k];
        snh[k] = b.n_haps[g];
        snr[k] = b.n_reads[g];
        const uint64_t h0 = b.hap_off[hap_first[g]], h1 = b.hap_off[hap_first[g] + b.n_haps[g]];
        if (h1 > h0) std::memcpy(m.hb.p + ho, b.hap_bases + h0, h1 - h0);
        for (uint32_t h = 0; h < b.n_haps[g]; ++h) shoff[++hk] = ho + (b.hap_off[hap_first[g] + h + 1] - h0);
        ho += h1 - h0;
        const uint64_t r0 = b.read_off[read_first[g]], r1 = b.read_off[read_first[g] + b.n_reads[g]];
        if (r1 > r0) {
            std::memcpy(m.rb.p + ro, b.read_bases + r0, r1 - r0);
            std::memcpy(m.rq.p + ro, b.read_qual + r0, r1 - r0);
            std::memcpy(m.ri.p + ro, b.read_ins + r0, r1 - r0);
            std::memcpy(m.rd.p + ro, b.read_del + r0, r1 - r0);
            std::memcpy(m.rc.p + ro, b.read_gcp + r0, r1 - r0);
        }
        for (uint32_t r = 0; r < b.n_reads[g]; ++r) sroff[++rk] = ro + (b.read_off[read_first[g] + r + 1] - r0);
        ro += r1 - r0;
    }
    sub = phmm_batch{};
    sub.n_regions = (uint32_t)regs.size();
    sub.n_haps = snh;
    sub.n_reads = snr;
    sub.hap_bases = (const uint8_t*)m.hb.p;
    sub.hap_off = shoff;
    sub.read_bases = (const uint8_t*)m.rb.p;
    sub.read_qual = (const uint8_t*)m.rq.p;
    sub.read_ins = (const uint8_t*)m.ri.p;
    sub.read_del = (const uint8_t*)m.rd.p;
    sub.read_gcp = (const uint8_t*)m.rc.p;
    sub.read_off = sroff;
    return true;
}

}  // namespace

extern "C" {

phmm_status phmm_partition_regions(const phmm_batch* batch, uint32_t n_parts, uint32_t* part_of_region,
                                   uint64_t* cells_of_part)
{
    try {
        phmm::clear_error();
        if (!batch || !part_of_region || !cells_of_part)
            return set_error(PHMM_ERR_INVALID_ARGUMENT, "batch, part_of_region or cells_of_part is null");
        if (n_parts == 0) return set_error(PHMM_ERR_INVALID_ARGUMENT, "n_parts is 0");
        phmm::BatchScan sc;
        std::string err;
        const phmm_status st = phmm::scan_batch(*batch, phmm::PlanLimits(), sc, err);
        if (st != PHMM_OK) return set_error(st, err);
        phmm::lpt(phmm::region_cells(*batch), n_parts, part_of_region, cells_of_part);
        return PHMM_OK;
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

phmm_status phmm_device_set_destroy(phmm_device_set* set)
{
    phmm::clear_error();
    if (!set) return set_error(PHMM_ERR_NOT_INITIALIZED, "device set is null");
    for (auto& m : set->members)
        if (m->engine) phmm_engine_destroy(m->engine);
    delete set;
    return PHMM_OK;
}

phmm_status phmm_device_set_create(const int32_t* devices, uint32_t n_devices, const phmm_config* cfg,
                                   phmm_device_set** out_set)
{
    try {
        phmm::clear_error();
        if (!devices || !out_set || n_devices == 0)
            return set_error(PHMM_ERR_INVALID_ARGUMENT, "devices or out_set is null, or no device given");
        *out_set = nullptr;
        auto* set = new phmm_device_set();
        for (uint32_t k = 0; k < n_devices; ++k) {
            phmm_config c{};
            if (cfg) {
                c = *cfg;
            } else {
                c.use_cuda_graph = 1;
                c.autotune = 1;
            }
            c.device = devices[k];
            auto m = std::make_unique<phmm::Member>();
            m->device = devices[k];
            const phmm_status st = phmm_engine_create(&c, &m->engine);
            if (st != PHMM_OK) {
                const std::string detail = phmm_last_error();
                phmm_device_set_destroy(set);
                return set_error(st, "device " + std::to_string(devices[k]) + ": " + detail);
            }
            set->members.push_back(std::move(m));
        }
        *out_set = set;
        return PHMM_OK;
    } catch (const std::bad_alloc&) {
        return set_error(PHMM_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

phmm_status phmm_device_set_engine(phmm_device_set* set, uint32_t index, phmm_engine** engine)
{
    phmm::clear_error();
    if (!set) return set_error(PHMM_ERR_NOT_INITIALIZED, "device set is null");
    if (!engine || index >= set->members.size()) return set_error(PHMM_ERR_INVALID_ARGUMENT, "bad index or engine");
    *engine = set->members[index]->engine;
    return PHMM_OK;
}

phmm_status phmm_device_set_compute_regions(phmm_device_set* set, const phmm_batch* batch, double* out,
                                            uint8_t* pair_flags, phmm_stats* stats)
{
    try {
        phmm::clear_error();
        if (!set) return set_error(PHMM_ERR_NOT_INITIALIZED, "device set is null");
        if (!batch) return set_error(PHMM_ERR_INVALID_ARGUMENT, "batch is null");
        const auto t_start = std::chrono::steady_clock::now();
        phmm::BatchScan sc;
        std::string err;
        phmm_status st = phmm::scan_batch(*batch, phmm::PlanLimits(), sc, err);
        if (st != PHMM_OK) return set_error(st, err);
        if (sc.out_total && !out) return set_error(PHMM_ERR_INVALID_ARGUMENT, "out is null");
        const uint32_t P = (uint32_t)set->members.size();
        if (P == 1) return phmm_compute_regions(set->members[0]->engine, batch, out, pair_flags, stats);
        std::lock_guard<std::mutex> lk(set->compute_mu);
        const phmm_batch& b = *batch;
        std::vector<uint32_t> part(b.n_regions);
        std::vector<uint64_t> load(P);
        phmm::lpt(phmm::region_cells(b), P, part.data(), load.data());
        std::vector<std::vector<uint32_t>> regs(P);
        std::vector<uint64_t> hap_first(b.n_regions), read_first(b.n_regions), out_first(b.n_regions);
        uint64_t h = 0, r = 0, o = 0;
        for (uint32_t g = 0; g < b.n_regions; ++g) {
            regs[part[g]].push_back(g);
            hap_first[g] = h;
            read_first[g] = r;
            out_first[g] = o;
            h += b.n_haps[g];
            r += b.n_reads[g];
            o += (uint64_t)b.n_haps[g] * b.n_reads[g];
        }
        std::vector<phmm_status> status(P, PHMM_OK);
        std::vector<std::string> errs(P);
        std::vector<phmm_stats> pst(P);
        auto work = [&](uint32_t p) {
            if (regs[p].empty()) return;
            phmm::Member& m = *set->members[p];
            phmm_batch sub;
            uint64_t sub_out = 0;
            if (!gather(b, hap_first, read_first, regs[p], m, sub, sub_out)) {
                status[p] = PHMM_ERR_OUT_OF_MEMORY;
                errs[p] = "pinned staging for device " + std::to_string(m.device);
                return;
            }
            double* so = (double*)m.out.p;
            uint8_t* sf = pair_flags ? (uint8_t*)m.flags.p : nullptr;
            status[p] = phmm_compute_regions(m.engine, &sub, so, sf, &pst[p]);
            if (status[p] != PHMM_OK) {
                errs[p] = phmm_last_error();
                return;
            }
            uint64_t at = 0;
            for (uint32_t g : regs[p]) {
                const uint64_t n = (uint64_t)b.n_haps[g] * b.n_reads[g];
                if (n) {
                    std::memcpy(out + out_first[g], so + at, n * sizeof(double));
                    if (pair_flags) std::memcpy(pair_flags + out_first[g], sf + at, n);
                }
                at += n;
            }
        };
        std::vector<std::thread> pool;
        for (uint32_t p = 1; p < P; ++p) pool.emplace_back(work, p);
        work(0);
        for (auto& t : pool) t.join();
        for (uint32_t p = 0; p < P; ++p)
            if (status[p] != PHMM_OK)
                return set_error(status[p], "device " + std::to_string(set->members[p]->device) + ": " + errs[p]);
        if (stats) {
            *stats = phmm_stats{};
            for (uint32_t p = 0; p < P; ++p) {
                if (regs[p].empty()) continue;
                stats->regions += pst[p].regions;
                stats->pairs += pst[p].pairs;
                stats->cells += pst[p].cells;
                stats->pairs_f64 += pst[p].pairs_f64;
                stats->work_items += pst[p].work_items;
                stats->h2d_bytes += pst[p].h2d_bytes;
                stats->d2h_bytes += pst[p].d2h_bytes;
                stats->kernel_launches += pst[p].kernel_launches;
                stats->device_ms = std::max(stats->device_ms, pst[p].device_ms);
                stats->fp32_ms = std::max(stats->fp32_ms, pst[p].fp32_ms);
                stats->fp64_ms = std::max(stats->fp64_ms, pst[p].fp64_ms);
            }
            stats->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        }
        return PHMM_OK;
    } catch (const std::bad_alloc&) {
        return set_error(PHMM_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

phmm_status phmm_device_set_submit(phmm_device_set* set, const phmm_batch* region, double* out, uint8_t* pair_flags,
                                   phmm_ticket* ticket)
{
    try {
        phmm::clear_error();
        if (!set) return set_error(PHMM_ERR_NOT_INITIALIZED, "device set is null");
        if (!region || !ticket) return set_error(PHMM_ERR_INVALID_ARGUMENT, "region or ticket is null");
        phmm::BatchScan sc;
        std::string err;
        const phmm_status vst = phmm::scan_batch(*region, phmm::PlanLimits(), sc, err);
        if (vst != PHMM_OK) return set_error(vst, err);
        // the device with the fewest cells submitted and not yet waited for
        uint32_t best = 0;
        for (uint32_t k = 1; k < set->members.size(); ++k)
            if (set->members[k]->outstanding_cells.load() < set->members[best]->outstanding_cells.load()) best = k;
        phmm::Member& m = *set->members[best];
        phmm_ticket t = 0;
        const phmm_status st = phmm_submit(m.engine, region, out, pair_flags, &t);
        if (st != PHMM_OK) return st;  // phmm_submit recorded the detail
        m.outstanding_cells += sc.cells;
        std::lock_guard<std::mutex> lk(set->mu);
        const phmm_ticket mine = set->next_ticket++;
        set->pending[mine] = phmm::PendingRequest{best, t, sc.cells};
        *ticket = mine;
        return PHMM_OK;
    } catch (const std::bad_alloc&) {
        return set_error(PHMM_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

phmm_status phmm_device_set_wait(phmm_device_set* set, phmm_ticket ticket, int64_t timeout_us, double* queued_us,
                                 double* total_us, uint32_t* device_index)
{
    try {
        phmm::clear_error();
        if (!set) return set_error(PHMM_ERR_NOT_INITIALIZED, "device set is null");
        phmm::PendingRequest pr;
        {
            std::lock_guard<std::mutex> lk(set->mu);
            auto it = set->pending.find(ticket);
            if (it == set->pending.end()) return set_error(PHMM_ERR_INVALID_ARGUMENT, "unknown ticket");
            pr = it->second;
        }
        if (device_index) *device_index = pr.member;
        phmm::Member& m = *set->members[pr.member];
        const phmm_status st = phmm_wait(m.engine, pr.ticket, timeout_us, queued_us, total_us);
        if (st == PHMM_ERR_TIMEOUT) return st;
        {
            std::lock_guard<std::mutex> lk(set->mu);
            set->pending.erase(ticket);
        }
        m.outstanding_cells -= pr.cells;
        return st;
    } catch (const std::exception& ex) {
        return set_error(PHMM_ERR_INTERNAL, ex.what());
    }
}

}  // extern "C"
