// Test driver for integration/pairhmm_engine_b200.cpp, the Rovaca-side binding of the engine,
// compiled against the reference's own headers (genotype/forward.h, haplotype.h, read_record.h,
// common/utils/rovaca_memory_pool.h) and its RovacaMemoryPool.
//
// The reference's ReadRecord and Allele accessors are implemented against libhts, which is not in
// this image; this driver defines the four the binding reads (seq_length, seq_i, qual,
// mapping_quality) and Allele::get_bases over fake records kept in side tables, keyed by the
// record's address.  The records are never constructed: only their addresses are used.
//
// Input (stdin): lines "H <bases>" (haplotype, the first is the reference), "R <bases> <mapq>
// <q,q,...>" (read), "E" (end of a region); mode from argv[1]:
//   foreign-pool   call_pairhmm_b200 with a pool that is not a RovacaMemoryPool
//   no-engine      call_pairhmm_b200 before any engine exists
//   sync           init_pairhmm_b200(0), then every region through the bound rovaca::call_pairhmm
//   pipeline       init_pairhmm_b200(0), then region k+1 submitted before region k is collected
//                  (PairHmmRegionRequest), a stand-in for the assembly of the next region between
// Output per region: "region <k> reads <n_left> kept <i...>" then "row <h> <v...>" (%.17g, nan).
// argv[2], argv[3]: min_quality_threshold, PCR model (0-3).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <iostream>
#include <memory>
#include <memory_resource>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../integration/pairhmm_engine_b200.h"
#include "../genotype/haplotype.h"
#include "../genotype/read_record.h"
#include "../common/utils/rovaca_memory_pool.h"

namespace {
struct FakeRead {
    std::string bases;
    std::vector<uint8_t> qual;
    uint8_t mapq;
};
std::unordered_map<const void*, FakeRead> g_reads;
std::unordered_map<const void*, rovaca::pBases> g_haps;
}  // namespace

namespace rovaca {
DoubleVector2D (*call_pairhmm)(const HaplotypeVector& hs, ReadVector& rs, int32_t min_quality_threshold,
                               PcrIndelModel pcr_option, pMemoryPool pool) = nullptr;
int32_t ReadRecord::seq_length() const { return (int32_t)g_reads.at(this).bases.size(); }
uint8_t ReadRecord::seq_i(uint32_t i) const { return (uint8_t)g_reads.at(this).bases.at(i); }
uint8_t* ReadRecord::qual() const { return const_cast<uint8_t*>(g_reads.at(this).qual.data()); }
uint8_t ReadRecord::mapping_quality() const { return g_reads.at(this).mapq; }
pBases Allele::get_bases() const { return g_haps.at(this); }
}  // namespace rovaca

namespace {
struct Region {
    rovaca::HaplotypeVector hs;
    rovaca::ReadVector rs;
    std::vector<rovaca::pReadRecord> original;
};

std::deque<std::vector<char>> g_storage;  // addresses of the fake objects

void* fake_object(size_t bytes)
{
    g_storage.emplace_back(bytes + 16);
    return g_storage.back().data();
}

void print(size_t k, const Region& g, const rovaca::DoubleVector2D& m)
{
    std::printf("region %zu reads %zu kept", k, g.rs.size());
    for (size_t i = 0, j = 0; i < g.original.size() && j < g.rs.size(); ++i)
        if (g.original[i] == g.rs[j]) {
            std::printf(" %zu", i);
            ++j;
        }
    std::printf("\n");
    for (size_t h = 0; h < m.size(); ++h) {
        std::printf("row %zu", h);
        for (double v : m[h]) std::printf(" %.17g", v);
        std::printf("\n");
    }
}
}  // namespace

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: integration_check MODE THRESHOLD PCR < regions\n");
        return 2;
    }
    const std::string mode = argv[1];
    const int32_t thr = std::atoi(argv[2]);
    const auto pcr = (PcrIndelModel)std::atoi(argv[3]);
    std::vector<uint8_t> cache(64u << 20);
    rovaca::RovacaMemoryPool pool(cache.data(), cache.size());
    std::vector<Region> regions(1, Region{rovaca::HaplotypeVector(&pool), rovaca::ReadVector(&pool), {}});
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        std::string tag;
        in >> tag;
        if (tag == "H") {
            std::string b;
            in >> b;
            auto* bases = (rovaca::pBases)fake_object(sizeof(rovaca::Bases) + b.size());
            bases->num = (uint32_t)b.size();
            std::copy(b.begin(), b.end(), bases->data);
            auto* h = (rovaca::pHaplotype)fake_object(sizeof(rovaca::Haplotype));
            g_haps[h] = bases;
            regions.back().hs.push_back(h);
        } else if (tag == "R") {
            FakeRead fr;
            int mq = 0;
            std::string qs;
            in >> fr.bases >> mq >> qs;
            fr.mapq = (uint8_t)mq;
            std::stringstream qss(qs);
            for (std::string q; std::getline(qss, q, ',');)
                if (!q.empty()) fr.qual.push_back((uint8_t)std::atoi(q.c_str()));
            auto* r = (rovaca::pReadRecord)fake_object(sizeof(rovaca::ReadRecord));
            g_reads[r] = fr;
            regions.back().rs.push_back(r);
            regions.back().original.push_back(r);
        } else if (tag == "E") {
            regions.push_back(Region{rovaca::HaplotypeVector(&pool), rovaca::ReadVector(&pool), {}});
        }
    }
    if (regions.back().hs.empty() && regions.back().rs.empty()) regions.pop_back();

    if (mode == "foreign-pool") {
        for (size_t k = 0; k < regions.size(); ++k)
            print(k, regions[k],
                  rovaca::call_pairhmm_b200(regions[k].hs, regions[k].rs, thr, pcr, std::pmr::new_delete_resource()));
        return 0;
    }
    if (mode == "no-engine") {
        for (size_t k = 0; k < regions.size(); ++k)
            print(k, regions[k], rovaca::call_pairhmm_b200(regions[k].hs, regions[k].rs, thr, pcr, &pool));
        return 0;
    }
    if (!rovaca::init_pairhmm_b200(0) || rovaca::call_pairhmm != rovaca::call_pairhmm_b200) {
        std::fprintf(stderr, "init_pairhmm_b200 failed: %s\n", phmm_last_error());
        return 3;
    }
    if (mode == "sync") {
        for (size_t k = 0; k < regions.size(); ++k)
            print(k, regions[k], rovaca::call_pairhmm(regions[k].hs, regions[k].rs, thr, pcr, &pool));
    } else if (mode == "pipeline") {
        std::vector<std::unique_ptr<rovaca::PairHmmRegionRequest>> req;
        std::vector<rovaca::DoubleVector2D> res;
        for (size_t k = 0; k < regions.size(); ++k) {
            req.push_back(std::make_unique<rovaca::PairHmmRegionRequest>());
            req.back()->submit(rovaca::pairhmm_b200_engine(), regions[k].hs, regions[k].rs, thr, pcr);
            if (k > 0) res.push_back(req[k - 1]->collect(regions[k - 1].rs, &pool));
        }
        if (!regions.empty()) res.push_back(req.back()->collect(regions.back().rs, &pool));
        for (size_t k = 0; k < regions.size(); ++k) print(k, regions[k], res[k]);
    } else {
        std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
        return 2;
    }
    rovaca::shutdown_pairhmm_b200();
    return 0;
}
