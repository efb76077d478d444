// Tile-shape autotuner.
//
// For every FP32 mode (inter with constant gap qualities, inter per-row, intra) and read-length
// bucket (ceil(R / 32)), the candidate shapes are the single stripe that holds the bucket and the
// multi-stripe shapes (4..8 row pairs per lane) whose padded rows stay within 25% of the tightest
// candidate, plus the default shape.  Each candidate runs the FP32 class kernel alone, persistent
// grid, on a synthetic calibration batch of that bucket (reads of the bucket's middle length
// against 8 haplotypes of 300 bases, about four waves of resident warps) and is timed with CUDA
// events (best of 3).  A candidate replaces the default only when it is more than 3% faster.  The
// chosen table is kept per device for the process, so engines created later reuse it without
// tuning again.  Shapes change only the speed: every cell runs the same operations on the same
// operands whatever the shape, so results are bit-identical under any table.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/phmm_b200.h"
#include "phmm_engine.h"
#include "phmm_plan.h"

namespace phmm {

namespace {

struct Shape {
    int kh;
    bool multi;
};

uint64_t padded_rows(int kh, bool multi, uint64_t R)
{
    const uint64_t stripe = (uint64_t)kWarp * kh;
    return multi ? (R + stripe - 1) / stripe * stripe : stripe;
}

std::vector<Shape> candidates(int bucket, Shape def)
{
    std::vector<Shape> c;
    const uint64_t R = (uint64_t)kWarp * bucket;  // longest read of the bucket
    if (bucket <= kMaxK) c.push_back({bucket, false});
    uint64_t tight = bucket <= kMaxK ? R : ~0ull;
    for (int kh = kMinMultiKH; kh <= kMaxK && kh < bucket; ++kh) tight = std::min(tight, padded_rows(kh, true, R));
    for (int kh = kMinMultiKH; kh <= kMaxK && kh < bucket; ++kh)
        if (padded_rows(kh, true, R) * 4 <= tight * 5) c.push_back({kh, true});
    bool has_def = false;
    for (const Shape& s : c) has_def |= s.kh == def.kh && s.multi == def.multi;
    if (!has_def) c.insert(c.begin(), def);
    return c;
}

uint64_t splitmix(uint64_t& s)
{
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Calibration batch of one bucket: `regions` regions of 8 haplotypes (300 bases) and 64 reads.
struct Calibration {
    std::vector<uint32_t> nh, nr;
    std::vector<uint8_t> hb, rb, rq, ri, rd, rc;
    std::vector<uint64_t> hoff, roff;

    void make(int mode, uint64_t R, uint32_t regions, uint64_t seed)
    {
        constexpr uint32_t kHaps = 8, kHapLen = 300, kReads = 64;
        static const uint8_t acgt[4] = {'A', 'C', 'G', 'T'};
        uint64_t s = seed;
        nh.assign(regions, kHaps);
        nr.assign(regions, kReads);
        for (auto* v : {&hb, &rb, &rq, &ri, &rd, &rc}) v->clear();
        hoff.assign(1, 0);
        roff.assign(1, 0);
        for (uint32_t g = 0; g < regions; ++g) {
            for (uint32_t h = 0; h < kHaps; ++h) {
                for (uint32_t j = 0; j < kHapLen; ++j) hb.push_back(acgt[splitmix(s) & 3]);
                hoff.push_back(hb.size());
            }
            for (uint32_t r = 0; r < kReads; ++r) {
                for (uint64_t i = 0; i < R; ++i) {
                    const uint64_t x = splitmix(s);
                    rb.push_back(mode == 2 && i == R / 2 ? 'N' : acgt[x & 3]);
                    rq.push_back((uint8_t)(10 + (x >> 8) % 31));
                    ri.push_back(45);
                    rd.push_back(45);
                    rc.push_back(mode == 1 ? (uint8_t)(8 + (x >> 16) % 5) : 10);
                }
                roff.push_back(rb.size());
            }
        }
    }

    phmm_batch view() const
    {
        phmm_batch b{};
        b.n_regions = (uint32_t)nh.size();
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
        return b;
    }
};

std::mutex g_tuned_mu;
std::map<int, TileTable> g_tuned;  // device -> table chosen by the first tuning run

}  // namespace

phmm_status Engine::autotune(phmm_tune_report* report, std::string& err)
{
    const auto t0 = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(mu_);  // the default slot is ours while tuning
    if (report) std::memset(report, 0, sizeof(*report));
    const TileTable def = TileTable::defaults();
    TileTable best = def;
    Calibration cal;
    for (int mode = 0; mode < kModes32; ++mode) {
        const int variant = mode == 2 ? kIntra : kInter;
        const int pmode = mode == 0 ? 0 : 1;
        for (int bucket = 1; bucket <= kLenBuckets; ++bucket) {
            const Shape d{def.kh[mode][bucket - 1], def.multi[mode][bucket - 1] != 0};
            const std::vector<Shape> cand = candidates(bucket, d);
            if (cand.size() < 2) continue;
            const uint64_t R = (uint64_t)kWarp * bucket - kWarp / 2;
            // about four waves of the largest candidate grid, two reads per work item
            int occ = 1;
            for (const Shape& c : cand) occ = std::max(occ, occ_[0][class32(variant, pmode, c.kh, c.multi)]);
            const uint64_t items = 4ull * occ * sms_ * (kFwdBlock / kWarp);
            const uint32_t regions = (uint32_t)std::max<uint64_t>(1, (items + 31) / 32);
            cal.make(mode, R, regions, 0x5eed0000ull + (uint64_t)mode * 64 + bucket);
            const phmm_batch b = cal.view();
            double base_gcups = 0.0, best_gcups = 0.0;
            Shape pick = d;
            for (const Shape& c : cand) {
                TileTable t = def;
                t.kh[mode][bucket - 1] = (uint8_t)c.kh;
                t.multi[mode][bucket - 1] = c.multi ? 1 : 0;
                Plan plan;
                phmm_status st = build_plan(b, limits_with(t), plan, err);
                if (st != PHMM_OK) return st;
                st = upload(*default_slot_, plan, b, err);
                if (st != PHMM_OK) return st;
                const int cls = class32(variant, pmode, c.kh, c.multi);
                float ms = 0.f;
                st = time_fp32_class(*default_slot_, plan, cls, 3, &ms, err);
                if (st != PHMM_OK) return st;
                const double gcups = ms > 0.f ? (double)plan.cells / (ms * 1e-3) / 1e9 : 0.0;
                if (c.kh == d.kh && c.multi == d.multi) base_gcups = gcups;
                if (gcups > best_gcups) {
                    best_gcups = gcups;
                    pick = c;
                }
                if (report && report->n_entries < PHMM_TUNE_MAX_ENTRIES) {
                    phmm_tune_entry& e = report->entries[report->n_entries++];
                    e.mode = (uint8_t)mode;
                    e.bucket = (uint8_t)bucket;
                    e.rows_per_lane = (uint8_t)c.kh;
                    e.multi_stripe = c.multi ? 1 : 0;
                    e.gcups = (float)gcups;
                }
            }
            // keep the default unless the winner is clearly faster
            if (!(pick.kh == d.kh && pick.multi == d.multi) && best_gcups > base_gcups * 1.03) {
                best.kh[mode][bucket - 1] = (uint8_t)pick.kh;
                best.multi[mode][bucket - 1] = pick.multi ? 1 : 0;
            }
        }
    }
    if (!best.valid(err)) return PHMM_ERR_INTERNAL;
    if (report) {
        for (uint32_t i = 0; i < report->n_entries; ++i) {
            phmm_tune_entry& e = report->entries[i];
            e.chosen = best.kh[e.mode][e.bucket - 1] == e.rows_per_lane &&
                       (best.multi[e.mode][e.bucket - 1] != 0) == (e.multi_stripe != 0);
        }
        report->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    {
        std::lock_guard<std::mutex> lt(tiles_mu_);
        tiles_ = best;
    }
    {
        std::lock_guard<std::mutex> lg(g_tuned_mu);
        g_tuned[dev_] = best;
    }
    return PHMM_OK;
}

phmm_status autotune_once(Engine& e, std::string& err)
{
    {
        std::lock_guard<std::mutex> lg(g_tuned_mu);
        auto it = g_tuned.find(e.device());
        if (it != g_tuned.end()) return e.set_tiles(it->second, err);
    }
    return e.autotune(nullptr, err);
}

}  // namespace phmm
