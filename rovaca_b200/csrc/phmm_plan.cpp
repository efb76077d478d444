// Batch planner (see phmm_plan.h).
//
// Reference behaviour mirrored here:
//   limits                      src/haplotypecaller/pairhmm/roDV_schedule.cpp:70-73,374-381,445-459
//   pairs with an N go to the   src/haplotypecaller/pairhmm/roDV_schedule.cpp:96,105,417-441
//   intra kernel (N wildcard)   (region API tests 'N' only, :422,:435)
//   empty read or haplotype     src/haplotypecaller/pairhmm/roDV_schedule.cpp:460 (pair skipped,
//                               its likelihood stays NaN, pairhmm_internal.cpp:593)
// Instead of the reference's greedy SIMD grouping (roDV_schedule.cpp:87-142), reads of a region are
// paired (two reads per warp, equal kernel class) and each pair becomes one work item per run of
// the region's haplotypes: the warp streams all of them through both reads.
#include "phmm_plan.h"

#include <algorithm>
#include <cstring>
#include <thread>

namespace phmm {

namespace {

bool has_n(const uint8_t* p, uint64_t n) { return n > 0 && std::memchr(p, 'N', (size_t)n) != nullptr; }

// True when every byte equals the first: the array equals itself shifted by one.
bool constant_run(const uint8_t* p, uint64_t n) { return n < 2 || std::memcmp(p, p + 1, (size_t)(n - 1)) == 0; }

struct Run {
    uint16_t lo, hi;
    uint32_t cols;
    uint8_t variant;
};

// Splits haplotypes [0, n) of a region into runs of non-empty haplotypes whose column stream
// stays within max_cols; with split_on_n, a run also never mixes N and non-N haplotypes.
void make_runs(const uint64_t* hoff, const uint8_t* hflags, uint32_t n, uint32_t max_cols, bool split_on_n,
               std::vector<Run>& runs)
{
    runs.clear();
    uint32_t h = 0;
    while (h < n) {
        const uint64_t H = hoff[h + 1] - hoff[h];
        if (H == 0) {
            ++h;
            continue;
        }
        Run r;
        r.lo = (uint16_t)h;
        r.cols = 0;
        r.variant = split_on_n ? (hflags[h] & 1) : kIntra;
        while (h < n) {
            const uint64_t Hh = hoff[h + 1] - hoff[h];
            if (Hh == 0) break;
            if (split_on_n && (hflags[h] & 1) != r.variant) break;
            if (r.cols > 0 && r.cols + Hh > max_cols) break;
            r.cols += (uint32_t)Hh;
            ++h;
        }
        r.hi = (uint16_t)h;
        runs.push_back(r);
    }
}

}  // namespace

TileTable TileTable::defaults()
{
    TileTable t{};
    for (int m = 0; m < kModes32; ++m)
        for (int b = 1; b <= kLenBuckets; ++b) {
            t.kh[m][b - 1] = (uint8_t)std::min(b, kMaxK);
            t.multi[m][b - 1] = b > kMaxK ? 1 : 0;
        }
    return t;
}

bool TileTable::valid(std::string& err) const
{
    for (int m = 0; m < kModes32; ++m)
        for (int b = 1; b <= kLenBuckets; ++b) {
            const int k = kh[m][b - 1];
            const bool mu = multi[m][b - 1] != 0;
            const bool ok = mu ? (k >= kMinMultiKH && k <= kMaxK && k < b) : (k >= b && k <= kMaxK);
            if (!ok) {
                err = "tile shape of mode " + std::to_string(m) + ", bucket " + std::to_string(b) + " (reads of " +
                      std::to_string(32 * (b - 1) + 1) + "-" + std::to_string(32 * b) + " bases): " +
                      (mu ? "multi-stripe" : "single-stripe") + " with " + std::to_string(k) +
                      " row pairs per lane cannot hold it";
                return false;
            }
        }
    return true;
}

phmm_status scan_batch(const phmm_batch& b, const PlanLimits& lim, BatchScan& s, std::string& err)
{
    s = BatchScan();
    if (b.n_regions == 0) return PHMM_OK;
    if (!b.n_haps || !b.n_reads || !b.hap_off || !b.read_off) {
        err = "batch: n_haps, n_reads, hap_off and read_off are required";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    uint64_t nh = 0, nr = 0;
    for (uint32_t r = 0; r < b.n_regions; ++r) {
        nh += b.n_haps[r];
        nr += b.n_reads[r];
        if (b.n_haps[r] > lim.max_haps_per_region) {
            err = "region " + std::to_string(r) + ": " + std::to_string(b.n_haps[r]) + " haplotypes exceeds the limit of " +
                  std::to_string(lim.max_haps_per_region);
            return PHMM_ERR_LIMIT_EXCEEDED;
        }
    }
    if (nh > 0xffffffffull || nr > 0xffffffffull) {
        err = "batch: more than 2^32 haplotypes or reads";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    s.n_haps = (uint32_t)nh;
    s.n_reads = (uint32_t)nr;
    s.hap_base0 = b.hap_off[0];
    s.read_base0 = b.read_off[0];
    // offsets non-decreasing, lengths within the limits; per region the non-empty pairs and cells
    uint64_t h = 0, r = 0;
    for (uint32_t g = 0; g < b.n_regions; ++g) {
        uint64_t hcols = 0, hnon = 0, rrows = 0, rnon = 0;
        for (uint32_t k = 0; k < b.n_haps[g]; ++k, ++h) {
            if (b.hap_off[h + 1] < b.hap_off[h]) {
                err = "hap_off is not non-decreasing at " + std::to_string(h + 1);
                return PHMM_ERR_INVALID_ARGUMENT;
            }
            const uint64_t H = b.hap_off[h + 1] - b.hap_off[h];
            if (H > lim.max_hap_len) {
                err = "haplotype " + std::to_string(h) + " longer than " + std::to_string(lim.max_hap_len);
                return PHMM_ERR_LIMIT_EXCEEDED;
            }
            hcols += H;
            hnon += H > 0;
        }
        for (uint32_t k = 0; k < b.n_reads[g]; ++k, ++r) {
            if (b.read_off[r + 1] < b.read_off[r]) {
                err = "read_off is not non-decreasing at " + std::to_string(r + 1);
                return PHMM_ERR_INVALID_ARGUMENT;
            }
            const uint64_t R = b.read_off[r + 1] - b.read_off[r];
            if (R > lim.max_read_len) {
                err = "read " + std::to_string(r) + " longer than " + std::to_string(lim.max_read_len);
                return PHMM_ERR_LIMIT_EXCEEDED;
            }
            rrows += R;
            rnon += R > 0;
        }
        s.out_total += (uint64_t)b.n_haps[g] * b.n_reads[g];
        s.pairs += hnon * rnon;
        s.cells += hcols * rrows;
    }
    s.hap_bases = b.hap_off[nh] - s.hap_base0;
    s.read_bases = b.read_off[nr] - s.read_base0;
    const bool gaps_needed = lim.region_api == nullptr;
    if ((s.hap_bases > 0 && !b.hap_bases) ||
        (s.read_bases > 0 && (!b.read_bases || !b.read_qual ||
                              (gaps_needed && (!b.read_ins || !b.read_del || !b.read_gcp))))) {
        err = "batch: sequence or quality pointer is null";
        return PHMM_ERR_INVALID_ARGUMENT;
    }
    return PHMM_OK;
}

phmm_status build_plan(const phmm_batch& b, const PlanLimits& lim, Plan& plan, std::string& err)
{
    plan = Plan();
    plan.classes.assign(kPlanClasses, ClassDesc{});
    plan.tiles = lim.tiles ? *lim.tiles : TileTable::defaults();
    plan.region_api = lim.region_api != nullptr;
    if (lim.tiles && !plan.tiles.valid(err)) return PHMM_ERR_INVALID_ARGUMENT;
    const TileTable& tiles = plan.tiles;
    BatchScan sc;
    const phmm_status st = scan_batch(b, lim, sc, err);
    if (st != PHMM_OK || b.n_regions == 0) return st;
    const uint64_t nh = sc.n_haps, nr = sc.n_reads;
    plan.n_regions = b.n_regions;
    plan.n_haps = sc.n_haps;
    plan.n_reads = sc.n_reads;
    plan.hap_base0 = sc.hap_base0;
    plan.read_base0 = sc.read_base0;
    plan.hap_off.resize(nh + 1);
    plan.read_off.resize(nr + 1);
    for (uint64_t h = 0; h <= nh; ++h) plan.hap_off[h] = b.hap_off[h] - plan.hap_base0;
    for (uint64_t r = 0; r <= nr; ++r) plan.read_off[r] = b.read_off[r] - plan.read_base0;
    plan.hap_bases = sc.hap_bases;
    plan.read_bases = sc.read_bases;
    const uint8_t* hb = b.hap_bases + plan.hap_base0;
    const uint8_t* rb = b.read_bases + plan.read_base0;

    plan.hap_flags.resize(nh);
    plan.read_flags.resize(nr);
    plan.regions.resize(b.n_regions);
    {
        uint64_t out_off = 0;
        uint32_t hap_begin = 0, read_begin = 0;
        for (uint32_t g = 0; g < b.n_regions; ++g) {
            RegionDesc& rd = plan.regions[g];
            rd = RegionDesc{};
            rd.out_off = out_off;
            rd.hap_begin = hap_begin;
            rd.n_haps = b.n_haps[g];
            rd.read_begin = read_begin;
            rd.n_reads = b.n_reads[g];
            if (lim.region_api) {
                rd.api = kRegionApi | ((uint32_t)(lim.region_api[g].pcr & 0xff) << 8);
                rd.min_quality = lim.region_api[g].min_quality;
            }
            out_off += (uint64_t)b.n_haps[g] * b.n_reads[g];
            hap_begin += b.n_haps[g];
            read_begin += b.n_reads[g];
        }
        plan.out_total = out_off;
    }

    // Regions are planned independently on host threads: N flags, gap modes, read pairing,
    // haplotype runs and work items, each counted per (FP32 class, stream-length bucket).
    constexpr int kBuckets = 64;
    constexpr uint32_t kBucketCols = 128;
    struct Part {
        std::vector<WorkItem> raw;
        std::vector<uint32_t> key;
        std::vector<uint32_t> count;
        uint64_t rerun_cap[kClasses64] = {};
        uint64_t pairs = 0, cells = 0;
        uint32_t max_multi = 0;
    };
    auto plan_range = [&](uint32_t g0, uint32_t g1, Part& part) {
        part.count.assign((size_t)kClasses32 * kBuckets, 0);
        std::vector<Run> runs_split, runs_all, runs_split_m, runs_all_m;
        struct ReadKey {
            uint32_t key;  // (N, gap mode, multi, stripes, kh) packed; reads with equal keys share an item
            uint32_t read;
        };
        std::vector<ReadKey> rk;
        for (uint32_t g = g0; g < g1; ++g) {
            const RegionDesc& rd = plan.regions[g];
            const uint32_t M = rd.n_haps, N = rd.n_reads, hap_begin = rd.hap_begin, read_begin = rd.read_begin;
            for (uint32_t h = hap_begin; h < hap_begin + M; ++h)
                plan.hap_flags[h] = has_n(hb + plan.hap_off[h], plan.hap_off[h + 1] - plan.hap_off[h]);
            const uint64_t* hoff = plan.hap_off.data() + hap_begin;
            const uint8_t* hfl = plan.hap_flags.data() + hap_begin;
            rk.clear();
            for (uint32_t r = 0; r < N; ++r) {
                const uint32_t gr = read_begin + r;
                const uint64_t a = plan.read_off[gr], R = plan.read_off[gr + 1] - a;
                plan.read_flags[gr] = has_n(rb + a, R);
                if (R == 0) continue;
                // Mode 0 (the FP32 kernels' PM_EQ): gap qualities constant along the read, insertion
                // and deletion qualities equal (as qualities & 127, which is what the tables read).
                // Region API: gap-open = insertion = deletion, constant unless a PCR model caps them.
                bool uniform;
                if (lim.region_api) {
                    uniform = lim.region_api[g].pcr == PHMM_PCR_NONE;
                } else {
                    const uint8_t* ib = b.read_ins + plan.read_base0 + a;
                    const uint8_t* db = b.read_del + plan.read_base0 + a;
                    const uint8_t* cb = b.read_gcp + plan.read_base0 + a;
                    uniform = constant_run(ib, R) && constant_run(db, R) && constant_run(cb, R) &&
                              (ib[0] & 127) == (db[0] & 127);
                }
                const uint32_t n_flag = plan.read_flags[gr] & 1;
                const int mode = n_flag ? 2 : (uniform ? 0 : 1);
                const int bucket = len_bucket(R);
                const uint32_t kh = tiles.kh[mode][bucket - 1];
                const bool multi = tiles.multi[mode][bucket - 1] != 0;
                const uint32_t stripes = multi ? (uint32_t)((R + kWarp * kh - 1) / (kWarp * kh)) : 1;
                rk.push_back({(n_flag << 22) | ((uniform ? 0u : 1u) << 21) | ((multi ? 1u : 0u) << 20) | (stripes << 4) | kh,
                              gr});
            }
            std::stable_sort(rk.begin(), rk.end(), [](const ReadKey& x, const ReadKey& y) { return x.key < y.key; });
            bool runs_ready = false, runs_m_ready = false;
            for (size_t k = 0; k < rk.size();) {
                const uint32_t key = rk[k].key;
                const uint32_t r0 = rk[k].read;
                const uint32_t r1 = (k + 1 < rk.size() && rk[k + 1].key == key) ? rk[k + 1].read : kNoRead;
                k += (r1 == kNoRead) ? 1 : 2;
                const uint32_t kh = key & 0xf, stripes = (key >> 4) & 0xffff;
                const bool uniform = ((key >> 21) & 1) == 0, read_n = ((key >> 22) & 1) != 0;
                const bool multi = ((key >> 20) & 1) != 0;
                const std::vector<Run>* runs;
                if (!multi) {
                    if (!runs_ready) {
                        make_runs(hoff, hfl, M, lim.max_stream_single, true, runs_split);
                        make_runs(hoff, hfl, M, lim.max_stream_single, false, runs_all);
                        runs_ready = true;
                    }
                    runs = read_n ? &runs_all : &runs_split;
                } else {
                    if (!runs_m_ready) {
                        make_runs(hoff, hfl, M, lim.max_stream_multi, true, runs_split_m);
                        make_runs(hoff, hfl, M, lim.max_stream_multi, false, runs_all_m);
                        runs_m_ready = true;
                    }
                    runs = read_n ? &runs_all_m : &runs_split_m;
                }
                const uint64_t R0 = plan.read_off[r0 + 1] - plan.read_off[r0];
                const uint64_t R1 = r1 == kNoRead ? 0 : plan.read_off[r1 + 1] - plan.read_off[r1];
                const uint64_t rows = R0 + R1;
                const uint32_t nreads = r1 == kNoRead ? 1 : 2;
                for (const Run& run : *runs) {
                    WorkItem it{};
                    it.read[0] = r0;
                    it.read[1] = r1;
                    it.region = g;
                    it.hap_lo = run.lo;
                    it.hap_hi = run.hi;
                    it.kh = (uint8_t)kh;
                    it.stripes = (uint8_t)stripes;
                    it.variant = read_n ? (uint8_t)kIntra : run.variant;
                    it.pmode = (it.variant == kInter && uniform) ? 0 : 1;
                    const int c32 = class32(it.variant, it.pmode, (int)kh, multi);
                    const uint32_t bucket = std::min<uint32_t>(run.cols / kBucketCols, kBuckets - 1);
                    const uint32_t skey = (uint32_t)c32 * kBuckets + (kBuckets - 1 - bucket);  // longest first
                    part.raw.push_back(it);
                    part.key.push_back(skey);
                    ++part.count[skey];
                    const uint32_t npairs = nreads * (uint32_t)(run.hi - run.lo);
                    // each read's pairs may go to the FP64 class of its own length
                    const int m = mode32(it.variant, it.pmode);
                    part.rerun_cap[class64_for_len(m, R0)] += run.hi - run.lo;
                    if (r1 != kNoRead) part.rerun_cap[class64_for_len(m, R1)] += run.hi - run.lo;
                    part.pairs += npairs;
                    part.cells += (uint64_t)run.cols * rows;
                    if (multi) part.max_multi = std::max(part.max_multi, run.cols);
                }
            }
        }
    };
    const uint64_t work = plan.read_bases + plan.hap_bases;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nthreads = (unsigned)std::min<uint64_t>({hw, 32u, b.n_regions, work / (1u << 20) + 1});
    std::vector<Part> parts(nthreads);
    {
        // contiguous region ranges with about equal bases each
        std::vector<uint32_t> cut(nthreads + 1, b.n_regions);
        cut[0] = 0;
        uint64_t acc = 0;
        unsigned t = 1;
        for (uint32_t g = 0; g < b.n_regions && t < nthreads; ++g) {
            const RegionDesc& rd = plan.regions[g];
            acc += plan.read_off[rd.read_begin + rd.n_reads] - plan.read_off[rd.read_begin] +
                   plan.hap_off[rd.hap_begin + rd.n_haps] - plan.hap_off[rd.hap_begin];
            if (acc * nthreads >= work * t) cut[t++] = g + 1;
        }
        std::vector<std::thread> pool;
        for (unsigned t2 = 1; t2 < nthreads; ++t2) pool.emplace_back(plan_range, cut[t2], cut[t2 + 1], std::ref(parts[t2]));
        plan_range(cut[0], cut[1], parts[0]);
        for (auto& th : pool) th.join();
    }
    std::vector<uint32_t> count((size_t)kClasses32 * kBuckets, 0);
    size_t n_items = 0;
    for (const Part& p : parts) {
        for (size_t i = 0; i < count.size(); ++i) count[i] += p.count[i];
        for (int c = 0; c < kClasses64; ++c) plan.classes[kClasses32 + c].rerun_cap += (uint32_t)p.rerun_cap[c];
        plan.pairs += p.pairs;
        plan.cells += p.cells;
        plan.max_multi_stream = std::max(plan.max_multi_stream, p.max_multi);
        n_items += p.raw.size();
    }
    plan.empty_pairs = plan.out_total - plan.pairs;

    // stable counting sort by key (parts in region order)
    std::vector<uint32_t> start(count.size() + 1, 0);
    for (size_t i = 0; i < count.size(); ++i) start[i + 1] = start[i] + count[i];
    plan.items.resize(n_items);
    {
        std::vector<uint32_t> pos(start.begin(), start.end() - 1);
        for (const Part& p : parts)
            for (size_t i = 0; i < p.raw.size(); ++i) plan.items[pos[p.key[i]]++] = p.raw[i];
    }
    for (int c = 0; c < kClasses32; ++c) {
        ClassDesc& cd = plan.classes[c];
        cd.item_off = start[(size_t)c * kBuckets];
        cd.n_items = start[(size_t)(c + 1) * kBuckets] - cd.item_off;
    }
    uint32_t rerun_off = 0;
    for (int c = kClasses32; c < kPlanClasses; ++c) {
        ClassDesc& cd = plan.classes[c];
        cd.rerun_off = rerun_off;
        rerun_off += cd.rerun_cap;
    }
    for (ClassDesc& cd : plan.classes) cd.claim32 = cd.claim64 = cd.rerun_count = cd.rerun_pairs = 0;
    plan.rerun_slots = rerun_off;
    return PHMM_OK;
}

}  // namespace phmm
