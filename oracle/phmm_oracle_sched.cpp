// PairHMM oracle, part 2: the reference's vector-API scheduler, restated so the oracle reproduces
// schedule_pairhmm pair for pair, including which kernel variant and precision each pair got.
//
// TEST INFRASTRUCTURE ONLY (see phmm_oracle.c).  Restates src/haplotypecaller/pairhmm/
// roDV_schedule.cpp:37-68 (pair record), :87-142 (greedy_grouping), :144-152 (containsN),
// :169-361 (schedule_pairhmm_with_allocator, vector API), and the result conversions of
// roDV_inter/pairhmm_inter_api.h:10-15 and roDV_intra/pairhmm_api.cpp:14-23.
//
// std::sort is not stable, so the order of equal-length pairs, and with it the grouping, depends on
// the sort's exact sequence of moves.  The pair record and comparator below are the reference's, so
// libstdc++'s std::sort produces the same permutation from the same initial order.
#include <cmath>
#include <cstdint>
#include <vector>
#include <algorithm>

extern "C" {
float oracle_raw_f32(const uint8_t* hap, uint32_t hl, const uint8_t* rd, uint32_t rl, const uint8_t* q,
                     const uint8_t* iq, const uint8_t* dq, const uint8_t* cq, int kernel, int fused);
double oracle_raw_f64(const uint8_t* hap, uint32_t hl, const uint8_t* rd, uint32_t rl, const uint8_t* q,
                      const uint8_t* iq, const uint8_t* dq, const uint8_t* cq, int kernel, int fused);
}

namespace {

constexpr int kInter = 0, kIntra = 1, kFused = 1;
constexpr float kMinAccepted = 1e-28f;
constexpr float kLog10CF = 36.1236000061f;
constexpr double kLog10CD = 307.050595577260822;

struct Pair {  // roDV_schedule.cpp:37-68
    static constexpr uint8_t kN = 0x1, kUsed = 0x2;
    uint32_t read_idx;
    uint16_t hap_idx, hap_len, read_len;
    uint8_t flags;
    bool n() const { return flags & kN; }
    bool used() const { return flags & kUsed; }
    void set_used(bool v) { flags = v ? (flags | kUsed) : (flags & ~kUsed); }
};

struct Group {
    std::vector<size_t> idx;
};

std::vector<Group> greedy_grouping(std::vector<Pair>& pairs, double max_idle, uint32_t w)
{
    std::vector<Group> groups;
    if (w == 0) return groups;
    const size_t total = pairs.size();
    for (size_t i = 0; i < total; ++i) {
        if (pairs[i].used() || pairs[i].n()) continue;
        Group g;
        size_t k = i;
        while (k < total && g.idx.size() < w) {
            if (!pairs[k].used() && !pairs[k].n()) g.idx.push_back(k);
            ++k;
        }
        if (g.idx.size() < w) break;
        uint32_t mh = 0, mr = 0;
        uint64_t sum = 0;
        for (size_t p : g.idx) {
            mh = std::max<uint32_t>(mh, pairs[p].hap_len);
            mr = std::max<uint32_t>(mr, pairs[p].read_len);
            sum += (uint64_t)pairs[p].hap_len * pairs[p].read_len;
        }
        const uint64_t cap = (uint64_t)mh * mr * w;
        const uint64_t idle = cap > sum ? cap - sum : 0;
        const double ratio = cap == 0 ? 0.0 : (double)idle / (double)cap;
        if (ratio <= max_idle) {
            for (size_t p : g.idx) pairs[p].set_used(true);
            groups.push_back(std::move(g));
        }
    }
    return groups;
}

bool contains_n(const uint8_t* s, uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i)
        if (s[i] == 'N' || s[i] == 'n') return true;
    return false;
}

}  // namespace

extern "C" {

// Route codes written per pair ([hap][read]):
//   0 inter FP32            1 inter FP32 underflow -> inter FP64
//   2 intra FP32            3 intra FP32 underflow -> intra FP64
//   4 inter FP32 underflow -> intra FP64 (left over by the FP64 grouping)
// out is [hap][read] log10 like the engine (the reference's own result is [read][hap]).
int oracle_schedule(uint32_t n_haps, const uint8_t* hap_bases, const uint64_t* hap_off, uint32_t n_reads,
                    const uint8_t* rb, const uint8_t* q, const uint8_t* iq, const uint8_t* dq, const uint8_t* cq,
                    const uint64_t* read_off, double idle_f, double idle_d, uint32_t width_f, uint32_t width_d,
                    double* out, uint8_t* route)
{
    const size_t M = n_haps, N = n_reads;
    if (M == 0 || N == 0) return -1;
    auto hap = [&](size_t h) { return hap_bases + hap_off[h]; };
    auto hl = [&](size_t h) { return (uint32_t)(hap_off[h + 1] - hap_off[h]); };
    auto rd = [&](size_t r) { return rb + read_off[r]; };
    auto rl = [&](size_t r) { return (uint32_t)(read_off[r + 1] - read_off[r]); };
    auto raw32 = [&](size_t h, size_t r, int kernel) {
        const uint64_t a = read_off[r];
        return oracle_raw_f32(hap(h), hl(h), rd(r), rl(r), q + a, iq + a, dq + a, cq + a, kernel, kFused);
    };
    auto raw64 = [&](size_t h, size_t r, int kernel) {
        const uint64_t a = read_off[r];
        return oracle_raw_f64(hap(h), hl(h), rd(r), rl(r), q + a, iq + a, dq + a, cq + a, kernel, kFused);
    };
    auto put = [&](size_t h, size_t r, double v, uint8_t code) {
        out[h * N + r] = v;
        route[h * N + r] = code;
    };

    std::vector<bool> hn(M), rn(N);
    for (size_t h = 0; h < M; ++h) hn[h] = contains_n(hap(h), hl(h));
    for (size_t r = 0; r < N; ++r) rn[r] = contains_n(rd(r), rl(r));
    std::vector<Pair> pairs;
    pairs.reserve(M * N);
    for (size_t h = 0; h < M; ++h)
        for (size_t r = 0; r < N; ++r) {
            Pair p;
            p.read_idx = (uint32_t)r;
            p.hap_idx = (uint16_t)h;
            p.hap_len = (uint16_t)hl(h);
            p.read_len = (uint16_t)rl(r);
            p.flags = (hn[h] || rn[r]) ? Pair::kN : 0;
            pairs.push_back(p);
        }
    std::sort(pairs.begin(), pairs.end(), [](const Pair& a, const Pair& b) {
        if (a.hap_len == b.hap_len) return a.read_len > b.read_len;
        return a.hap_len > b.hap_len;
    });
    std::vector<bool> done_f(M * N, false), done_d(M * N, false);
    // step 1: FP32 inter groups
    for (const Group& g : greedy_grouping(pairs, idle_f, width_f)) {
        for (size_t p : g.idx) {
            Pair& pr = pairs[p];
            const float v = raw32(pr.hap_idx, pr.read_idx, kInter);
            if ((double)v < (double)kMinAccepted) {
                pr.set_used(false);
            } else {
                pr.set_used(true);
                put(pr.hap_idx, pr.read_idx, std::log10((double)v) - (double)kLog10CF, 0);
                done_d[pr.hap_idx * N + pr.read_idx] = true;
            }
            done_f[pr.hap_idx * N + pr.read_idx] = true;
        }
    }
    // step 2: FP64 inter groups over the FP32 underflows
    for (Pair& pr : pairs)
        if (!done_f[pr.hap_idx * N + pr.read_idx]) pr.set_used(true);
    for (const Group& g : greedy_grouping(pairs, idle_d, width_d)) {
        for (size_t p : g.idx) {
            const Pair& pr = pairs[p];
            const double v = raw64(pr.hap_idx, pr.read_idx, kInter);
            put(pr.hap_idx, pr.read_idx, std::log10(v) - kLog10CD, 1);
            done_d[pr.hap_idx * N + pr.read_idx] = true;
        }
    }
    // step 3: the rest through the intra kernel
    for (size_t h = 0; h < M; ++h)
        for (size_t r = 0; r < N; ++r) {
            if (done_d[h * N + r]) continue;
            const bool use_double = done_f[h * N + r];
            const float vf = use_double ? 0.0f : raw32(h, r, kIntra);
            if (vf < kMinAccepted) {
                const double vd = raw64(h, r, kIntra);
                put(h, r, std::log10(vd) - kLog10CD, use_double ? 4 : 3);
            } else {
                put(h, r, (double)(log10f(vf) - kLog10CF), 2);
            }
        }
    return 0;
}

}  // extern "C"
