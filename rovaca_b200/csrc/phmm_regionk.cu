// Device-side read preparation and post-processing of the region API (call_pairhmm semantics), so
// that a region's reads go up as bases + raw qualities + MAPQ and come back as the consumer's
// normalised matrix, with no per-base host pass either side.
//
// Reference (paths inside the reference project):
//   quality: min(q, MAPQ); below the threshold -> 6       src/haplotypecaller/pairhmm/roDV_schedule.cpp:540-565
//   gap-open 45, gap continuation 10                      src/haplotypecaller/pairhmm/roDV_schedule.cpp:510-519,575-604
//   PCR model: gap-open capped by tandem-repeat length    src/haplotypecaller/pairhmm/pairhmm_internal.cpp:431-476
//     repeat finder                                       src/haplotypecaller/pairhmm/pairhmm_internal.cpp:146-221,317-379
//     caps per repeat length                              src/haplotypecaller/pairhmm/adapter.h:13-15
//     deletion gap-open aliases the capped insertion one  src/haplotypecaller/pairhmm/roDV_schedule.cpp:607-609
//   normalise: cap each read at best - 4.5                src/haplotypecaller/pairhmm/pairhmm_internal.cpp:248-258
//   drop poorly modelled reads                            src/haplotypecaller/pairhmm/pairhmm_internal.cpp:23-44
//   [hap][read], kept reads first                         src/haplotypecaller/pairhmm/pairhmm_internal.cpp:489-508
//   haplotype -> allele marginalisation (max)             src/haplotypecaller/genotype/allele_likelihoods.hpp:702-730
//   diploid genotype likelihoods                          src/haplotypecaller/genotype/genotype_likelihood_calculator.cpp:59-100
// The host functions of phmm_region.cpp compute the same values and are what the tests compare to.
#include <cuda_runtime.h>

#include <cstdint>

#include "phmm_regionk.h"

namespace phmm {

namespace {

constexpr int kMaxReadLen = 768;
constexpr int kPrepWarps = 8;  // warps per block of the read-preparation kernel
constexpr int kPostThreads = 256;

__constant__ uint8_t c_pcr_caps[4][21] = {
    {0},
    {40, 40, 39, 38, 37, 36, 34, 32, 28, 23, 17, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10},  // HOSTILE
    {40, 40, 40, 39, 39, 39, 38, 38, 37, 37, 36, 35, 34, 33, 32, 30, 28, 26, 23, 20, 17},  // AGGRESSIVE
    {40, 40, 40, 40, 39, 39, 39, 39, 39, 38, 38, 38, 37, 37, 37, 36, 36, 35, 34, 33, 33},  // CONSERVATIVE
};

// Copies of s[u, u+ul) tiling s[t, t+tl) from its front (leading) or back, stopping at the first
// copy that differs; counting stops at 21, which is enough because the repeat length is capped at 20
// and the search only asks whether a count exceeds 1.
__device__ int count_repeats(const uint8_t* s, int n, int u, int ul, int t, int tl, bool leading)
{
    if (tl <= 0 || ul <= 0 || ul > tl || u < 0 || t < 0 || u + ul > n || t + tl > n) return 0;
    int k = 0;
    for (int c = 0; c < tl / ul && k < 21; ++c) {
        const int start = leading ? c * ul : tl - (c + 1) * ul;
        bool same = true;
        for (int x = 0; x < ul; ++x) same &= s[t + start + x] == s[u + x];
        if (!same) break;
        ++k;
    }
    return k;
}

// Tandem-repeat length around position o < n - 1: the shortest unit (<= 8) starting at o + 1 that
// repeats at least twice forwards (else the single base at o + 1), its forward copies from o + 1
// plus its copies ending at o, capped at 20.
__device__ int repeat_length(const uint8_t* s, int n, int o)
{
    int fw_str = 1, max_fw = 0;
    for (int str = 1; str <= 8; ++str) {
        if (o + str + 1 > n) break;
        max_fw = count_repeats(s, n, o + 1, str, o + 1, n - o - 1, true);
        if (max_fw > 1) {
            fw_str = str;
            break;
        }
    }
    const int max_bw = count_repeats(s, n, o + 1, fw_str, 0, o + 1, false);
    const int rl = max_bw + max_fw;
    return rl > 20 ? 20 : rl;
}

// One warp per read of a region-API region: the read's bases are staged in shared memory and each
// lane prepares positions lane, lane + 32, ...
__global__ void __launch_bounds__(kPrepWarps * 32) read_prep_kernel(RegionApiView v)
{
    __shared__ uint8_t bases[kPrepWarps][kMaxReadLen];
    const BatchDesc* d = v.desc;
    if (d->region_api == 0) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n_regions = d->n_regions;
    for (uint32_t g = blockIdx.x; g < n_regions; g += gridDim.x) {
        const RegionDesc rg = v.regions[g];
        if (!(rg.api & kRegionApi)) continue;
        const int pcr = (rg.api >> 8) & 0xff;
        for (uint32_t k = w; k < rg.n_reads; k += kPrepWarps) {
            const uint32_t r = rg.read_begin + k;
            const uint64_t a = v.read_off[r];
            const int n = (int)(v.read_off[r + 1] - a);
            if (n <= 0 || n > kMaxReadLen) continue;  // lengths are validated on the host
            for (int i = lane; i < n; i += 32) bases[w][i] = v.read_bases[a + i];
            __syncwarp();
            const uint8_t mq = v.mapq[r];
            for (int i = lane; i < n; i += 32) {
                const uint8_t q0 = v.read_q[a + i];
                const uint8_t q = q0 < mq ? q0 : mq;
                v.read_q[a + i] = (int)q < rg.min_quality ? (uint8_t)6 : q;
                uint8_t gop = 45;
                if (pcr >= 1 && pcr <= 3 && i < n - 1) {
                    const uint8_t cap = c_pcr_caps[pcr][repeat_length(bases[w], n, i)];
                    if (gop >= cap) gop = cap;
                }
                v.read_i[a + i] = gop;
                v.read_d[a + i] = gop;
                v.read_c[a + i] = 10;
            }
            __syncwarp();
        }
    }
}

// One block per region-API region: each read's row is capped at best - 4.5 (best by the `<` scan
// the reference's max_element makes, so a leading NaN stays the best), poorly modelled reads are
// dropped, and kept reads are written first in [hap][read] order with NaN after them.
__global__ void __launch_bounds__(kPostThreads) post_region_kernel(RegionApiView v)
{
    __shared__ uint32_t warp_sums[kPostThreads / 32];
    __shared__ uint32_t base_kept;
    const BatchDesc* d = v.desc;
    if (d->region_api == 0) return;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    const uint32_t n_regions = d->n_regions;
    for (uint32_t g = blockIdx.x; g < n_regions; g += gridDim.x) {
        const RegionDesc rg = v.regions[g];
        if (!(rg.api & kRegionApi)) continue;
        const uint32_t M = rg.n_haps, N = rg.n_reads;
        const double* lk = v.lk + rg.out_off;
        double* out = v.out + rg.out_off;
        for (uint64_t i = threadIdx.x; i < (uint64_t)M * N; i += blockDim.x) out[i] = nan;
        if (threadIdx.x == 0) base_kept = 0;
        __syncthreads();
        for (uint32_t r0 = 0; r0 < N; r0 += blockDim.x) {
            const uint32_t r = r0 + threadIdx.x;
            bool keep = false;
            double cmp = 0.0;
            if (r < N) {
                double best = M ? lk[r] : 0.0;
                for (uint32_t h = 1; h < M; ++h) {
                    const double x = lk[(uint64_t)h * N + r];
                    if (best < x) best = x;
                }
                cmp = best - 4.5;
                double best2 = -__longlong_as_double(0x7ff0000000000000ll);
                for (uint32_t h = 0; h < M; ++h) {
                    double x = lk[(uint64_t)h * N + r];
                    x = x < cmp ? cmp : x;
                    if (!(x != x)) best2 = best2 < x ? x : best2;
                }
                const uint64_t len = v.read_off[rg.read_begin + r + 1] - v.read_off[rg.read_begin + r];
                const double per = ceil((double)len * 0.02);
                const double min_lk = (2.0 < per ? 2.0 : per) * -4.0;
                keep = !(best2 < min_lk);
                v.keep[rg.read_begin + r] = keep ? 1 : 0;
            }
            // kept index: exclusive scan of keep over the block, after the previous chunks
            const unsigned int ballot = __ballot_sync(0xffffffffu, keep);
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            if (lane == 0) warp_sums[w] = __popc(ballot);
            __syncthreads();
            uint32_t before = base_kept;
            for (int k = 0; k < w; ++k) before += warp_sums[k];
            before += __popc(ballot & ((1u << lane) - 1u));
            if (keep)
                for (uint32_t h = 0; h < M; ++h) {
                    const double x = lk[(uint64_t)h * N + r];
                    out[(uint64_t)h * N + before] = x < cmp ? cmp : x;
                }
            __syncthreads();
            if (threadIdx.x == blockDim.x - 1) {
                uint32_t total = 0;
                for (int k = 0; k < (int)(blockDim.x >> 5); ++k) total += warp_sums[k];
                base_kept += total;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) v.n_kept[g] = base_kept;
        __syncthreads();
    }
}

// MathUtils::approximate_log10sum_log10(a, b) (common/utils/math_utils.cpp:280-290) with the
// Jacobian table of math_utils.h:209-242: the larger value plus the tabulated correction at the
// rounded difference, none beyond a difference of 8.
__device__ __forceinline__ double approx_log10sum(double a, double b, const double* jac)
{
    if (a > b) {
        const double t = a;
        a = b;
        b = t;
    }
    if (a == -__longlong_as_double(0x7ff0000000000000ll)) return b;
    const double diff = __dsub_rn(b, a);
    constexpr double kInvStep = 1.0 / 0.0001;
    return __dadd_rn(b, diff < 8.0 ? jac[(size_t)round(__dmul_rn(diff, kInvStep))] : 0.0);
}

// One block per event: allele likelihoods are the maximum over the event's haplotypes of each
// allele (AlleleLikelihoods::marginal_likelihoods_direct, genotype/allele_likelihoods.hpp:702-730;
// -inf when an allele has no haplotype, NaN never wins), over the region's kept reads.  Diploid
// genotype g = (a <= b), g = b(b+1)/2 + a, gets
//   GL = sum_r v_r - K log10(2),  v_r = lk(r,a) + log10(2) if a == b else log10sum(lk(r,a), lk(r,b)),
// summed from 0 in read order (GenotypeLikelihoodCalculator, genotype_likelihood_calculator.cpp:
// 59-100 and .h:90-142).  The most likely genotype is the first maximum.
__global__ void __launch_bounds__(kPostThreads) genotype_kernel(RegionApiView v)
{
    const BatchDesc* d = v.desc;
    const uint32_t n_events = d->n_events;
    if (n_events == 0) return;
    const double ninf = -__longlong_as_double(0x7ff0000000000000ll);
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    for (uint32_t e = blockIdx.x; e < n_events; e += gridDim.x) {
        const EventDesc ev = v.events[e];
        const RegionDesc rg = v.regions[ev.region];
        const uint32_t M = rg.n_haps, N = rg.n_reads, A = ev.n_alleles;
        const uint32_t K = v.n_kept[ev.region];
        const double* lk = v.out + rg.out_off;  // normalised, kept reads first
        const int8_t* map = v.hap_allele + ev.hap_allele_off;
        double* alk = v.allele_lk + ev.allele_lk_off;
        for (uint64_t i = threadIdx.x; i < (uint64_t)A * N; i += blockDim.x) {
            const uint32_t a = (uint32_t)(i / N), r = (uint32_t)(i % N);
            double best = ninf;
            if (r < K) {
                for (uint32_t h = 0; h < M; ++h)
                    if (map[h] == (int8_t)a) {
                        const double x = lk[(uint64_t)h * N + r];
                        if (x > best) best = x;
                    }
            } else {
                best = nan;
            }
            alk[i] = best;
        }
        __syncthreads();
        const uint32_t G = A * (A + 1) / 2;
        double* gl = v.gl + ev.gl_off;
        for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) {
            uint32_t b = 0;
            while ((b + 1) * (b + 2) / 2 <= g) ++b;
            const uint32_t a = g - b * (b + 1) / 2;
            const double* la = alk + (uint64_t)a * N;
            const double* lb = alk + (uint64_t)b * N;
            double sum = 0.0;
            for (uint32_t r = 0; r < K; ++r)
                sum = __dadd_rn(sum, a == b ? __dadd_rn(la[r], v.log10_two) : approx_log10sum(la[r], lb[r], v.jacobian));
            // explicit roundings: no fused multiply-add, as the host computes it
            gl[g] = __dsub_rn(sum, __dmul_rn((double)K, v.log10_two));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int32_t arg = 0;
            for (uint32_t g = 1; g < G; ++g)
                if (gl[g] > gl[arg]) arg = (int32_t)g;
            v.best[e] = arg;
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_genotype(const RegionApiView& v, int num_sms, cudaStream_t st)
{
    genotype_kernel<<<num_sms * 2, kPostThreads, 0, st>>>(v);
    return cudaGetLastError();
}

cudaError_t launch_read_prep(const RegionApiView& v, int num_sms, cudaStream_t st)
{
    read_prep_kernel<<<num_sms * 4, kPrepWarps * 32, 0, st>>>(v);
    return cudaGetLastError();
}

cudaError_t launch_post_region(const RegionApiView& v, int num_sms, cudaStream_t st)
{
    post_region_kernel<<<num_sms * 2, kPostThreads, 0, st>>>(v);
    return cudaGetLastError();
}

}  // namespace phmm
