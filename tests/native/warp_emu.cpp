// CPU emulation of the engine's wavefront kernels: the device code of rovaca_b200/csrc
// (phmm_warp32.cuh: the FP32 class loop and two-reads-per-warp sweep; phmm_warp64.cuh: the FP64
// recompute loop, also in its all-FP64 check form) compiled with g++ and run on 32 host threads,
// one per lane (tests/native/warp_emu_shim.h), over a batch planned by the engine's own planner
// (phmm_plan.cpp) with its own tables (phmm_tables.cpp).  Every class runs on one emulated warp,
// which claims all of its work items; the launch order is the engine's (FP32 classes, then FP64).
//
// It checks the kernels' index arithmetic and recurrences on the CPU, before any GPU run: the
// results must equal the oracle's pair for pair (tests/test_warp_emulator.py).  Every memory access
// of the device code goes to host vectors sized as the engine sizes its arena, with the same guard
// words around the code streams.
//
// Usage: warp_emu IN OUT MODE TILES
//   IN     batch: "PHMMEMU1", u32 n_regions, u64 haps, u64 reads, u64 hap bytes, u64 read bytes, then
//          n_haps[u32], n_reads[u32], hap_off[u64, haps+1], read_off[u64, reads+1], hap bases,
//          read bases, qualities, insertion, deletion and gap-continuation qualities
//   OUT    likelihoods [f64, out_total], pair flags [u8, out_total], status word [u32]
//   MODE   engine (FP32 pass, then the FP64 recompute) | check64 (every pair, all-FP64 model)
//   TILES  default | multi<KH> (read-length buckets above KH run in stripes of 32 KH rows)
#include "warp_emu_shim.h"

#include <cstdio>
#include <functional>
#include <string>
#include <thread>
#include <vector>

#include "../../rovaca_b200/csrc/phmm_plan.h"
#include "../../rovaca_b200/csrc/phmm_tables.h"
#include "../../rovaca_b200/csrc/phmm_warp32.cuh"
#include "../../rovaca_b200/csrc/phmm_warp64.cuh"

using namespace phmm;

namespace {

template <typename T>
bool read_vec(FILE* f, std::vector<T>& v, size_t n)
{
    v.resize(n);
    return n == 0 || fread(v.data(), sizeof(T), n, f) == n;
}

// one warp: 32 threads run fn(lane) in lockstep at every collective
void run_warp(const std::function<void(int)>& fn)
{
    warp_emu::Warp w;
    std::vector<std::thread> lanes;
    for (int l = 0; l < 32; ++l)
        lanes.emplace_back([&, l] {
            warp_emu::enter_lane(&w, l);
            fn(l);
        });
    for (auto& t : lanes) t.join();
}

template <int KH, int V, int PM, bool MULTI>
void f32_class(const BatchView& b, const ProbTables<float>& t, const PassControl& pc)
{
    std::vector<float4> tab(tab_floats4<KH>() + kRingFloat4);
    run_warp([&](int lane) { warp_items32<KH, V, PM, MULTI>(b, t, pc, tab.data(), lane, 0, 0xffffffffu); });
}

template <int V, int PM>
void f32_mode(int shape, const BatchView& b, const ProbTables<float>& t, const PassControl& pc)
{
    switch (shape) {
    case 0: f32_class<1, V, PM, false>(b, t, pc); break;
    case 1: f32_class<2, V, PM, false>(b, t, pc); break;
    case 2: f32_class<3, V, PM, false>(b, t, pc); break;
    case 3: f32_class<4, V, PM, false>(b, t, pc); break;
    case 4: f32_class<5, V, PM, false>(b, t, pc); break;
    case 5: f32_class<6, V, PM, false>(b, t, pc); break;
    case 6: f32_class<7, V, PM, false>(b, t, pc); break;
    case 7: f32_class<8, V, PM, false>(b, t, pc); break;
    case 8: f32_class<4, V, PM, true>(b, t, pc); break;
    case 9: f32_class<5, V, PM, true>(b, t, pc); break;
    case 10: f32_class<6, V, PM, true>(b, t, pc); break;
    case 11: f32_class<7, V, PM, true>(b, t, pc); break;
    case 12: f32_class<8, V, PM, true>(b, t, pc); break;
    }
}

template <int K, int V, int PM, bool MULTI, bool UNF>
void f64_class(const BatchView& b, const ProbTables<double>& t, const PassControl& pc)
{
    std::vector<double> tab(prior_table_size<K>());
    run_warp([&](int lane) { warp_reruns64<K, V, PM, MULTI, UNF>(b, t, pc, tab.data(), lane, 0); });
}

template <int V, int PM, bool UNF>
void f64_mode(int shape, const BatchView& b, const ProbTables<double>& t, const PassControl& pc)
{
    switch (shape) {
    case 0: f64_class<1, V, PM, false, UNF>(b, t, pc); break;
    case 1: f64_class<2, V, PM, false, UNF>(b, t, pc); break;
    case 2: f64_class<3, V, PM, false, UNF>(b, t, pc); break;
    case 3: f64_class<4, V, PM, false, UNF>(b, t, pc); break;
    case 4: f64_class<5, V, PM, false, UNF>(b, t, pc); break;
    case 5: f64_class<6, V, PM, false, UNF>(b, t, pc); break;
    case 6: f64_class<7, V, PM, false, UNF>(b, t, pc); break;
    case 7: f64_class<8, V, PM, false, UNF>(b, t, pc); break;
    case 8: f64_class<8, V, PM, true, UNF>(b, t, pc); break;
    }
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: warp_emu IN OUT engine|check64|eq64|row64 default|multi<KH>\n");
        return 2;
    }
    const std::string mode = argv[3], tiles_arg = argv[4];
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    char magic[8];
    uint32_t n_regions = 0;
    uint64_t n_haps = 0, n_reads = 0, hap_bytes = 0, read_bytes = 0;
    if (fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "PHMMEMU1", 8) != 0 || fread(&n_regions, 4, 1, f) != 1 ||
        fread(&n_haps, 8, 1, f) != 1 || fread(&n_reads, 8, 1, f) != 1 || fread(&hap_bytes, 8, 1, f) != 1 ||
        fread(&read_bytes, 8, 1, f) != 1)
        return 2;
    std::vector<uint32_t> nh, nr;
    std::vector<uint64_t> hoff, roff;
    std::vector<uint8_t> hb, rb, rq, ri, rd, rc;
    if (!read_vec(f, nh, n_regions) || !read_vec(f, nr, n_regions) || !read_vec(f, hoff, n_haps + 1) ||
        !read_vec(f, roff, n_reads + 1) || !read_vec(f, hb, hap_bytes) || !read_vec(f, rb, read_bytes) ||
        !read_vec(f, rq, read_bytes) || !read_vec(f, ri, read_bytes) || !read_vec(f, rd, read_bytes) ||
        !read_vec(f, rc, read_bytes))
        return 2;
    std::fclose(f);
    phmm_batch batch{n_regions, nh.data(), nr.data(), hb.data(), hoff.data(), rb.data(), rq.data(), ri.data(),
                     rd.data(), rc.data(), roff.data()};

    TileTable tiles = TileTable::defaults();
    if (tiles_arg.rfind("multi", 0) == 0) {
        const int kh = std::stoi(tiles_arg.substr(5));
        for (int m = 0; m < kModes32; ++m)
            for (int bk = 1; bk <= kLenBuckets; ++bk)
                if (kh < bk) {
                    tiles.kh[m][bk - 1] = (uint8_t)kh;
                    tiles.multi[m][bk - 1] = 1;
                }
    }
    PlanLimits lim;
    lim.tiles = &tiles;
    Plan plan;
    std::string err;
    if (build_plan(batch, lim, plan, err) != PHMM_OK) {
        std::fprintf(stderr, "plan: %s\n", err.c_str());
        return 3;
    }

    // the device arrays, as the engine's arena holds them (reads rebased to the plan's offsets)
    const uint8_t* r0 = rb.data() + plan.read_base0;
    std::vector<uint8_t> d_rb(r0, r0 + plan.read_bases), d_rq(rq.data() + plan.read_base0, rq.data() + plan.read_base0 + plan.read_bases),
        d_ri(ri.data() + plan.read_base0, ri.data() + plan.read_base0 + plan.read_bases),
        d_rd(rd.data() + plan.read_base0, rd.data() + plan.read_base0 + plan.read_bases),
        d_rc(rc.data() + plan.read_base0, rc.data() + plan.read_base0 + plan.read_bases);
    std::vector<uint32_t> ci(plan.hap_bases + 2 * kCodePad, 0u), ca(plan.hap_bases + 2 * kCodePad, 0u);
    for (uint64_t k = 0; k < plan.hap_bases; ++k) {
        ci[kCodePad + k] = hap_code(hb[plan.hap_base0 + k], kInter);
        ca[kCodePad + k] = hap_code(hb[plan.hap_base0 + k], kIntra);
    }
    std::vector<double> out(plan.out_total, std::nan(""));
    std::vector<uint8_t> flags(plan.out_total, 0);
    std::vector<ClassDesc> classes(plan.classes);
    std::vector<RerunEntry> rerun(std::max<uint64_t>(plan.rerun_slots, 1));
    unsigned int status = 0;
    const unsigned int scratch_cols = PlanLimits().max_stream_multi;
    std::vector<double> scratch((size_t)scratch_cols * 3);  // one warp's row: 3 float2 or 3 double per column

    BatchView v{};
    v.read_bases = d_rb.data();
    v.read_q = d_rq.data();
    v.read_i = d_ri.data();
    v.read_d = d_rd.data();
    v.read_c = d_rc.data();
    v.read_off = plan.read_off.data();
    v.read_flags = plan.read_flags.data();
    v.hap_off = plan.hap_off.data();
    v.codes_inter = ci.data();
    v.codes_intra = ca.data();
    v.hap_flags = plan.hap_flags.data();
    v.regions = plan.regions.data();
    v.out = out.data();
    v.pair_flags = flags.data();
    const HostTables<float>& hf = host_tables_f32();
    const HostTables<double>& hd = host_tables_f64();
    const ProbTables<float> tf{hf.ph2pr.data(), hf.pmat.data(), hf.pmis_inter.data(), hf.pmis_intra.data(),
                               hf.gapm.data(), hf.mm.data()};
    const ProbTables<double> td{hd.ph2pr.data(), hd.pmat.data(), hd.pmis_inter.data(), hd.pmis_intra.data(),
                                hd.gapm.data(), hd.mm.data()};
    PassControl pc{};
    pc.cd64 = classes.data() + kClasses32;
    pc.items = plan.items.data();
    pc.rerun = rerun.data();
    pc.status = &status;
    pc.scratch = scratch.data();
    pc.scratch_cols = scratch_cols;

    if (mode == "engine") {
        for (int c = 0; c < kClasses32; ++c) {
            if (!classes[c].n_items) continue;
            pc.cd = classes.data() + c;
            const int m = c / kShapes32, s = c % kShapes32;
            if (m == 0) f32_mode<kInter, PM_EQ>(s, v, tf, pc);
            else if (m == 1) f32_mode<kInter, PM_ROW>(s, v, tf, pc);
            else f32_mode<kIntra, PM_ROW>(s, v, tf, pc);
        }
        for (int c = 0; c < kClasses64; ++c) {
            if (!classes[kClasses32 + c].rerun_count) continue;
            pc.cd = classes.data() + kClasses32 + c;
            const int m = c / 9, s = c % 9;
            if (m == 0) f64_mode<kInter, PM_EQ, false>(s, v, td, pc);
            else if (m == 1) f64_mode<kInter, PM_ROW, false>(s, v, td, pc);
            else f64_mode<kIntra, PM_ROW, false>(s, v, td, pc);
        }
    } else if (mode == "check64" || mode == "eq64" || mode == "row64") {
        // every pair: per work item and read, the item's haplotype run, in the FP64 class of the
        // read's length (modes 1 and 2), as Engine::check_fp64 lays them out.  eq64: every pair of the
        // FP32 classes of mode 0 through the FP64 recompute classes of mode 0 instead (the
        // reference's FP64 kernel for each of them, not only for the underflowed ones)
        const bool eq = mode == "eq64", row = mode == "row64";
        std::vector<std::vector<RerunEntry>> per(kClasses64);
        for (const WorkItem& it : plan.items) {
            if (eq && mode32(it.variant, it.pmode) != 0) continue;
            if (row && mode32(it.variant, it.pmode) == 0) continue;
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
                const int m64 = eq ? 0 : it.variant == kIntra ? 2 : 1;
                per[class64_for_len(m64, plan.read_off[r + 1] - plan.read_off[r])].push_back(e);
            }
        }
        rerun.clear();
        for (int c = 0; c < kClasses64; ++c) {
            ClassDesc& cd = classes[kClasses32 + c];
            cd = ClassDesc{};
            cd.rerun_off = (uint32_t)rerun.size();
            cd.rerun_cap = cd.rerun_count = (uint32_t)per[c].size();
            rerun.insert(rerun.end(), per[c].begin(), per[c].end());
        }
        rerun.resize(std::max<size_t>(rerun.size(), 1));
        pc.rerun = rerun.data();
        for (int c = eq ? 0 : 9; c < (eq ? 9 : kClasses64); ++c) {
            if (!classes[kClasses32 + c].rerun_count) continue;
            pc.cd = classes.data() + kClasses32 + c;
            const int s = c % 9;
            const bool unf = !row;  // check64: the all-FP64 check arithmetic
            if (eq) f64_mode<kInter, PM_EQ, false>(s, v, td, pc);
            else if (c / 9 == 1 && unf) f64_mode<kInter, PM_ROW, true>(s, v, td, pc);
            else if (c / 9 == 1) f64_mode<kInter, PM_ROW, false>(s, v, td, pc);
            else if (unf) f64_mode<kIntra, PM_ROW, true>(s, v, td, pc);
            else f64_mode<kIntra, PM_ROW, false>(s, v, td, pc);
        }
    } else {
        return 2;
    }

    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    fwrite(out.data(), 8, out.size(), o);
    fwrite(flags.data(), 1, flags.size(), o);
    fwrite(&status, 4, 1, o);
    std::fclose(o);
    return 0;
}
