// Test-infrastructure only.  ISA-specific half of the C-ABI over the reference's own PairHMM
// kernels: oracle/build_ref.sh compiles this file twice, once with the reference's AVX-512 flags
// (REF_TAG=avx512) and once with its AVX2 flags (REF_TAG=avx2), mirroring how the reference's
// CMake builds each kernel per ISA (src/haplotypecaller/pairhmm/CMakeLists.txt:10-47).
// oracle/ref_shim.cpp picks one at run time with the reference's own CPUID check.
//
// Wrapped reference functions (paths inside the reference project):
//   intra single-pair kernel      src/haplotypecaller/pairhmm/roDV_intra/pairhmm_impl.cpp:286
//   intra FP32->FP64 switch       src/haplotypecaller/pairhmm/roDV_intra/pairhmm_api.cpp:14-35
//   inter lock-step kernel        src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter.cpp:141
//   inter API (raw/log10 results) src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter_api.cpp:61,85,109,133
#include <cstdint>
#include <cstring>
#include <vector>

#include "roDV_adapter/rovaca_pool_allocator.h"
#include "roDV_common/common.h"
#include "roDV_intra/pairhmm_api.h"
#include "roDV_intra/pairhmm_impl.h"
#include "roDV_inter/pairhmm_inter_api.h"

#if defined(__AVX512F__)
using IntraF = pairhmm::intra::PairHMMComputer<pairhmm::intra::AVX512FloatTraits>;
using IntraD = pairhmm::intra::PairHMMComputer<pairhmm::intra::AVX512DoubleTraits>;
#define REF_INTER_F pairhmm::inter::compute_inter_pairhmm_AVX512_float
#define REF_INTER_D pairhmm::inter::compute_inter_pairhmm_AVX512_double
#define REF_INTRA_LOG pairhmm::intra::computeLikelihoodsAVX512
static constexpr uint32_t kWF = 16, kWD = 8;
#define REF_FN(name) ref_avx512_##name
#else
using IntraF = pairhmm::intra::PairHMMComputer<pairhmm::intra::AVX2FloatTraits>;
using IntraD = pairhmm::intra::PairHMMComputer<pairhmm::intra::AVX2DoubleTraits>;
#define REF_INTER_F pairhmm::inter::compute_inter_pairhmm_AVX2_float
#define REF_INTER_D pairhmm::inter::compute_inter_pairhmm_AVX2_double
#define REF_INTRA_LOG pairhmm::intra::computeLikelihoodsAVX2
static constexpr uint32_t kWF = 8, kWD = 4;
#define REF_FN(name) ref_avx2_##name
#endif

namespace {

// Every array handed to a reference kernel is copied into an owned, zero-padded buffer (the
// reference's own tests over-allocate the same way), so callers may pass views into larger
// concatenated arrays.
struct Padded {
    std::vector<uint8_t> hap, rs, q, i, d, c;
    pairhmm::common::TestCase tc{};
    Padded(const uint8_t* h, uint32_t hl, const uint8_t* r, uint32_t rl, const uint8_t* q_, const uint8_t* i_,
           const uint8_t* d_, const uint8_t* c_)
    {
        auto cp = [](std::vector<uint8_t>& dst, const uint8_t* src, uint32_t n) {
            dst.assign(n + 128, 0);
            if (n) std::memcpy(dst.data(), src, n);
        };
        cp(hap, h, hl);
        cp(rs, r, rl);
        cp(q, q_, rl);
        cp(i, i_, rl);
        cp(d, d_, rl);
        cp(c, c_, rl);
        tc.rslen = rl;
        tc.haplen = hl;
        tc.hap = hap.data();
        tc.rs = rs.data();
        tc.q = q.data();
        tc.i = i.data();
        tc.d = d.data();
        tc.c = c.data();
    }
};

}  // namespace

extern "C" {

int REF_FN(inter_width_f32)(void) { return (int)kWF; }
int REF_FN(inter_width_f64)(void) { return (int)kWD; }

float REF_FN(intra_raw_f32)(const uint8_t* hap, uint32_t hl, const uint8_t* rs, uint32_t rl, const uint8_t* q,
                            const uint8_t* i, const uint8_t* d, const uint8_t* c)
{
    Padded p(hap, hl, rs, rl, q, i, d, c);
    return IntraF::compute(p.tc);
}

double REF_FN(intra_raw_f64)(const uint8_t* hap, uint32_t hl, const uint8_t* rs, uint32_t rl, const uint8_t* q,
                             const uint8_t* i, const uint8_t* d, const uint8_t* c)
{
    Padded p(hap, hl, rs, rl, q, i, d, c);
    return IntraD::compute(p.tc);
}

double REF_FN(intra_log10)(const uint8_t* hap, uint32_t hl, const uint8_t* rs, uint32_t rl, const uint8_t* q,
                           const uint8_t* i, const uint8_t* d, const uint8_t* c, int use_double)
{
    Padded p(hap, hl, rs, rl, q, i, d, c);
    return REF_INTRA_LOG(p.tc, use_double != 0);
}

int REF_FN(inter)(int dbl, uint32_t n, const uint8_t* const* hap, const uint32_t* hl, const uint8_t* const* rs,
                  const uint32_t* rl, const uint8_t* const* q, const uint8_t* const* i, const uint8_t* const* d,
                  const uint8_t* const* c, int raw, double* out)
{
    const uint32_t w = dbl ? kWD : kWF;
    if (n != w) return -1;
    std::vector<Padded> pads;
    pads.reserve(n);
    std::vector<pairhmm::common::TestCase> tcs(n);
    for (uint32_t k = 0; k < n; ++k) {
        pads.emplace_back(hap[k], hl[k], rs[k], rl[k], q[k], i[k], d[k], c[k]);
        tcs[k] = pads.back().tc;
    }
    rovaca::roDV_adapter::DefaultAllocator alloc;
    bool ok = dbl ? REF_INTER_D(tcs.data(), n, out, alloc, raw == 0) : REF_INTER_F(tcs.data(), n, out, alloc, raw == 0);
    return ok ? 0 : -2;
}

}  // extern "C"
