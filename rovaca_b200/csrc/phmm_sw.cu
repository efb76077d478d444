// Smith-Waterman realignment of reads to haplotypes on the GPU: the aligner HaplotypeCaller runs for
// every read against its best haplotype (AssemblyBasedCallerUtils::realign_reads_to_their_best_haplotype,
// genotype/utils/assembly_based_caller_utils.cpp:146-169 -> AlignmentUtils::create_read_aligned_to_ref,
// alignment_utils.cpp:571-579, seq1 = haplotype, seq2 = read).
//
// Reference arithmetic (common/base/lib/ro_sw/sw_core_template.h:111-352, sw_cigar.c:22-171, ro_sw.c):
//   E(i,j) = max(H(i,j-1) + open, E(i,j-1) + extend)   insertion; extension flag 4 unless open > ext
//   F(i,j) = max(F(i-1,j) + extend, H(i-1,j) + open)   deletion;  extension flag 8 likewise
//   H(i,j) = max(cutoff, H(i-1,j-1) + (s1[i] == s2[j] ? match : mismatch)), then E if E > H
//            (state insertion 1), then F if F > H (state deletion 2)
//   H(0,j) = H(i,0) = 0, E(i,0) = F(0,j) = low
// in int16 with wrap-around adds (low -16384, cutoff -8192) or int32 (low INT32_MIN/2, cutoff -1e8) as
// ro_sw_avx512_run chooses.  The best end cell is scanned over the last row and the last column in
// the reference's anti-diagonal order with its two tie rules; the path is traced back through the
// per-cell codes (soft clips at both ends, extension states), merged into runs and emitted as BAM
// CIGAR ops in read order.  Results equal the reference build's bit for bit.
//
// Mapping: one warp per alignment.  A stripe of 32 x K read columns is spread over the lanes, K
// consecutive columns per lane; the warp streams the haplotype rows as a wavefront (lane l works on
// row t + 1 - l at step t), so that the left neighbour's H and E of the same row, and its H of the row
// above (the diagonal), arrive by one shuffle each.  Reads longer than a stripe run stripe after
// stripe, the right edge column of one stripe (H, E per row) feeding the next.  Each lane packs the
// 4-bit codes of its K cells into ceil(K/8) words per row, stored to a per-warp scratch area in
// HBM; the trace-back walks that area through bands of rows staged in shared memory.  The 16-bit
// kernel is run in 32-bit arithmetic with the 16-bit constants whenever its adds cannot wrap
// (sw_w16_cannot_wrap); otherwise one class emulates the wrap-around on every add.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "phmm_sw.h"
#include "phmm_types.h"

namespace phmm {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kStIns = 1, kStDel = 2, kStInsExt = 4, kStDelExt = 8, kStClip = 9;

struct SwView {
    const SwItem* items;
    const uint32_t* order;       // this class's item indices, most cells first
    uint32_t n;
    const uint8_t* hap;
    const uint8_t* read;
    SwParams prm;
    int variant;
    uint8_t* scratch;
    uint64_t stride;             // scratch bytes per warp
    unsigned int* claim;
    phmm_sw_result* out;
    const uint64_t* slot_off;    // per item: its CIGAR slot in `ops` (min(cap, nrow + ncol) ops)
    uint32_t* ops;
    uint32_t cigar_cap;
};

// Score add: two's-complement 32-bit, wrapped to 16 bits in the wrap-around class when the
// alignment runs the int16 kernel (w16; an int32 alignment in that class adds in 32 bits).
template <bool WRAP>
__device__ __forceinline__ int sadd(int a, int b, bool w16)
{
    const int s = (int)((unsigned)a + (unsigned)b);
    return (WRAP && w16) ? (int)(short)s : s;
}

__device__ __forceinline__ uint32_t op_of(uint32_t run)
{
    const uint32_t st = run >> 16, len = run & 0xffffu;
    const uint32_t op = st == 0 ? 0u : st == kStIns ? 1u : st == kStDel ? 2u : 4u;
    return (len << 4) | op;
}

// Forward pass, end-cell selection and trace-back of one alignment.
// Whether max(cutoff, H(i-1,j-1) + s) can change any cell of an alignment.  E(i,j) >= open + (j-1) x
// min(extend, 0) for every cell (E(i,1) >= H(i,0) + open, then each step adds at most -extend), and
// wherever E > cutoff the cutoff changes neither H nor the state (E then wins over a diagonal term
// below the cutoff with or without it).  So an alignment whose read is short enough for
// open + (ncol - 1) x min(extend, 0) > cutoff runs without it.  Only for classes without 16-bit
// wrap-around, where these bounds are exact integer bounds.
__device__ __forceinline__ bool sw_cutoff_can_bind(const SwView& v, const SwItem& it)
{
    const bool i32 = sw_uses_int32(v.variant, it.hap_len, it.read_len, v.prm.match);
    const long long open = i32 ? v.prm.gap_open : (short)v.prm.gap_open;
    const long long ext = i32 ? v.prm.gap_extend : (short)v.prm.gap_extend;
    const long long cutoff = i32 ? -100000000 : -8192;
    const long long ncol = it.read_len;
    return !(open + (ncol > 0 ? ncol - 1 : 0) * (ext < 0 ? ext : 0) > cutoff);
}

template <int K, bool WRAP, bool CUT>
__device__ void sw_one(const SwView& v, uint32_t idx, int lane, uint8_t* scr, uint32_t* band)
{
    constexpr int NW = (K + 7) / 8;
    constexpr int ROW = 32 * NW;                 // u32 words per stripe row
    constexpr int BAND_ROWS = kSwBandWords / ROW;
    constexpr int S = 32 * K;
    const SwItem it = v.items[idx];
    const int nrow = (int)it.hap_len, ncol = (int)it.read_len;
    phmm_sw_result res{0, 0, 0, 0, 0, 0};
    if (max(nrow, ncol) >= kSwMaxSeq) {
        res.alignment_offset = 1;
        if (lane == 0) v.out[idx] = res;
        return;
    }
    const bool i32 = sw_uses_int32(v.variant, it.hap_len, it.read_len, v.prm.match);
    const bool w16 = !i32;
    const int match = i32 ? v.prm.match : (int)(short)v.prm.match;
    const int mismatch = i32 ? v.prm.mismatch : (int)(short)v.prm.mismatch;
    const int open = i32 ? v.prm.gap_open : (int)(short)v.prm.gap_open;
    const int ext = i32 ? v.prm.gap_extend : (int)(short)v.prm.gap_extend;
    const int low = i32 ? INT_MIN / 2 : -16384;
    const int cutoff = i32 ? -100000000 : -8192;
    int best = i32 ? INT_MIN : -32768;
    int mi = 0, mj = 0;

    const SwLayout L = sw_layout(it.hap_len, it.read_len, K);
    uint32_t* bt = (uint32_t*)(scr + L.bt);
    int* bh = (int*)(scr + L.bh);
    int* be = (int*)(scr + L.be);
    int* lrow = (int*)(scr + L.lrow);
    int* lcol = (int*)(scr + L.lcol);
    uint32_t* runs = (uint32_t*)(scr + L.runs);
    const uint8_t* hap = v.hap + it.hap_start;
    const uint8_t* rd = v.read + it.read_start;

    if (nrow == 0 || ncol == 0) {
        // only boundary cells: H = 0 on the last row (empty haplotype) or column (empty read); with
        // both empty there is no candidate at all
        if (nrow == 0 && ncol > 0) { best = 0; mj = 1; }
        if (ncol == 0 && nrow > 0) { best = 0; mi = nrow; }
    } else {
        const int stripes = (ncol + S - 1) / S;
        for (int s = 0; s < stripes; ++s) {
            const int j0 = s * S;
            const bool last = s == stripes - 1;
            int rb[K], Hp[K], Fp[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int j = j0 + lane * K + k + 1;
                rb[k] = j <= ncol ? (int)rd[j - 1] : -1;
                Hp[k] = 0;
                Fp[k] = low;
            }
            const int jc = ncol - j0 - 1;          // stripe slot of column ncol (last stripe)
            const bool holds_last_col = last && lane == jc / K;
            const int kc = jc - (jc / K) * K;
            int hb = 0, hnext = (int)hap[0];
            int bnh = 0, bne = low;                // lane 0: left edge of the next row
            if (s > 0 && lane == 0) { bnh = bh[1]; bne = be[1]; }
            int hprev = 0;                         // H(i-1, left column) of this lane
            int hout = 0, eout = low;              // H, E of this lane's last column, previous step
            uint32_t* bts = bt + (uint64_t)s * nrow * ROW;
            const int steps = nrow + 31;
            // one wavefront step; FULL: every lane is on a real row (steps 31 .. nrow - 1), so the
            // activity tests drop out of the cell loop
            auto step = [&](int t, auto full) {
                constexpr bool FULL = decltype(full)::value;
                const int i = t + 1 - lane;
                const bool act = FULL || (i >= 1 && i <= nrow);
                hb = __shfl_up_sync(kFull, hb, 1);
                int hl = __shfl_up_sync(kFull, hout, 1);
                int el = __shfl_up_sync(kFull, eout, 1);
                if (lane == 0) {
                    hb = hnext;
                    hnext = t + 1 < nrow ? (int)hap[t + 1] : 0;
                    hl = bnh;
                    el = bne;
                    if (s > 0 && t + 2 <= nrow) { bnh = bh[t + 2]; bne = be[t + 2]; }
                }
                int diag = hprev;
                hprev = hl;
                uint32_t code[NW];
#pragma unroll
                for (int w = 0; w < NW; ++w) code[w] = 0;
                int hc = 0;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const int eo = sadd<WRAP>(hl, open, w16), ee = sadd<WRAP>(el, ext, w16);
                    const int e = max(eo, ee);
                    const int fe = sadd<WRAP>(Fp[k], ext, w16), fo = sadd<WRAP>(Hp[k], open, w16);
                    const int f = max(fe, fo);
                    int h = sadd<WRAP>(diag, hb == rb[k] ? match : mismatch, w16);
                    if (CUT) h = max(h, cutoff);
                    uint32_t c = (eo > ee ? 0u : (uint32_t)kStInsExt) | (fo > fe ? 0u : (uint32_t)kStDelExt);
                    if (e > h) { c |= kStIns; h = e; }
                    if (f > h) { c = (c & ~3u) | kStDel; h = f; }
                    diag = Hp[k];
                    if (act) { Hp[k] = h; Fp[k] = f; }
                    hl = h;
                    el = e;
                    code[k / 8] |= c << (4 * (k % 8));
                    if (k == kc) hc = h;
                }
                hout = act ? hl : 0;               // a lane before its first row stands for row 0
                eout = act ? el : low;
                if (act) {
                    uint32_t* row = bts + (uint64_t)(i - 1) * ROW + lane;
#pragma unroll
                    for (int w = 0; w < NW; ++w) row[w * 32] = code[w];
                    if (i == nrow) {
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const int j = j0 + lane * K + k + 1;
                            if (j <= ncol) lrow[j] = Hp[k];
                        }
                    }
                    if (holds_last_col) lcol[i] = hc;
                    if (!last && lane == 31) { bh[i] = hl; be[i] = el; }
                }
            };
            int t = 0;
            for (; t < min(31, steps); ++t) step(t, std::false_type{});
            for (; t < nrow; ++t) step(t, std::true_type{});
            for (; t < steps; ++t) step(t, std::false_type{});
            __syncwarp();
        }

        // end cell: only candidates equal to the maximum matter, visited in the reference's order
        // (anti-diagonal a ascending; the last-row cell (nrow, a - nrow) before the last-column cell
        // (a - ncol, ncol)), sw_core_template.h:332-347
        int smax = INT_MIN;
        for (int j = 1 + lane; j <= ncol; j += 32) smax = max(smax, lrow[j]);
        for (int i = 1 + lane; i <= nrow; i += 32) smax = max(smax, lcol[i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) smax = max(smax, __shfl_xor_sync(kFull, smax, o));
        const int alo = min(nrow, ncol) + 1, ahi = nrow + ncol;
        for (int a0 = alo; a0 <= ahi; a0 += 32) {
            const int a = a0 + lane;
            const bool rc = a <= ahi && a >= nrow + 1 && lrow[a - nrow] == smax;
            const bool cc = a <= ahi && a >= ncol + 1 && lcol[a - ncol] == smax;
            uint32_t mr = __ballot_sync(kFull, rc), mc = __ballot_sync(kFull, cc);
            while (mr | mc) {
                const int l = __ffs(mr | mc) - 1;
                const int aa = a0 + l;
                if ((mr >> l) & 1u) {
                    const int ci = nrow, cj = aa - nrow;
                    if (best < smax || abs(ci - cj) < abs(mi - mj)) { best = smax; mi = ci; mj = cj; }
                }
                if ((mc >> l) & 1u) {
                    const int ci = aa - ncol, cj = ncol;
                    if (best < smax || mj == ncol || abs(ci - cj) <= abs(mi - mj)) { best = smax; mi = ci; mj = cj; }
                }
                mr &= ~(1u << l);
                mc &= ~(1u << l);
            }
        }
    }

    // trace-back (sw_cigar.c:36-146), uniform across the warp; runs merged as they come
    int i = mi, j = mj;
    int nr = 0, cst = -1, clen = 0;
    auto push = [&](int st, int len) {
        if (nr > 0 && cst == st) {
            clen += len;
        } else {
            if (nr > 0 && lane == 0) runs[nr - 1] = ((uint32_t)cst << 16) | (uint32_t)clen;
            cst = st;
            clen = len;
            ++nr;
        }
    };
    if (j < ncol) push(kStClip, ncol - j);
    int state = 0;
    int bs = -1, br0 = 0, br1 = -1;
    while (i > 0 && j > 0) {
        const int s = (j - 1) / S, jj = (j - 1) - s * S, ln = jj / K, k = jj - ln * K;
        if (s != bs || i - 1 < br0 || i - 1 > br1) {
            bs = s;
            br1 = i - 1;
            br0 = max(0, br1 - BAND_ROWS + 1);
            const uint32_t* src = bt + ((uint64_t)s * nrow + br0) * ROW;
            const int words = (br1 - br0 + 1) * ROW;
            __syncwarp();
            for (int q = lane; q < words; q += 32) band[q] = src[q];
            __syncwarp();
        }
        const uint32_t w = band[(i - 1 - br0) * ROW + (k >> 3) * 32 + ln];
        const int b = (int)((w >> (4 * (k & 7))) & 15u);
        if (state == kStInsExt) {
            --j;
            ++clen;
            state = b & kStInsExt;
        } else if (state == kStDelExt) {
            --i;
            ++clen;
            state = b & kStDelExt;
        } else if ((b & 3) == 0) {
            --i;
            --j;
            push(0, 1);
            state = 0;
        } else if ((b & 3) == kStIns) {
            --j;
            push(kStIns, 1);
            state = b & kStInsExt;
        } else {
            --i;
            push(kStDel, 1);
            state = b & kStDelExt;
        }
    }
    if (j > 0) push(kStClip, j);
    if (nr > 0 && lane == 0) runs[nr - 1] = ((uint32_t)cst << 16) | (uint32_t)clen;
    __syncwarp();

    // read order, at most kSwMaxSeq - 1 ops (sw_cigar.c:162-170)
    const int count = min(nr, kSwMaxSeq - 1);
    const int wr = min(count, (int)v.cigar_cap);
    uint32_t* dst = v.ops + v.slot_off[idx];
    for (int q = lane; q < wr; q += 32) dst[q] = op_of(runs[nr - 1 - q]);
    res.score = best;
    res.alignment_offset = i;
    res.max_i = mi;
    res.max_j = mj;
    res.cigar_count = (uint32_t)count;
    if (lane == 0) v.out[idx] = res;
    __syncwarp();
}

// Resident blocks per SM the register allocation must allow: 5 for up to 6 columns per lane (102
// registers), 4 up to 12 (128), 3 beyond (170).
template <int K>
constexpr int sw_min_blocks()
{
    return K <= 6 ? 5 : K <= 12 ? 4 : 3;
}

template <int K, bool WRAP>
__global__ void __launch_bounds__(32 * kSwBlockWarps, sw_min_blocks<K>()) sw_kernel(SwView v)
{
    __shared__ uint32_t band[kSwBlockWarps][kSwBandWords];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint8_t* scr = v.scratch + ((uint64_t)blockIdx.x * kSwBlockWarps + wib) * v.stride;
    for (;;) {
        unsigned int q = 0;
        if (lane == 0) q = atomicAdd(v.claim, 1u);
        q = __shfl_sync(kFull, q, 0);
        if (q >= v.n) break;
        const uint32_t idx = v.order[q];
        if (WRAP || sw_cutoff_can_bind(v, v.items[idx]))
            sw_one<K, WRAP, true>(v, idx, lane, scr, band[wib]);
        else
            sw_one<K, WRAP, false>(v, idx, lane, scr, band[wib]);
    }
}

// Exclusive scan of min(cigar_count, cap) over the items in order: each item's offset in the compact
// CIGAR buffer, and the total.  One block; 4 items per thread per round.
constexpr int kScanThreads = 1024, kScanItems = 4;

__global__ void __launch_bounds__(kScanThreads) sw_scan_kernel(phmm_sw_result* out, uint32_t n, uint32_t cap,
                                                               unsigned long long* total)
{
    __shared__ unsigned long long wsum[kScanThreads / 32];
    __shared__ unsigned long long carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < n; base += (uint64_t)kScanThreads * kScanItems) {
        unsigned long long c[kScanItems], own = 0;
#pragma unroll
        for (int u = 0; u < kScanItems; ++u) {
            const uint64_t q = base + (uint64_t)tid * kScanItems + u;
            c[u] = q < n ? (unsigned long long)min(out[q].cigar_count, cap) : 0ull;
            own += c[u];
        }
        unsigned long long x = own;  // inclusive scan over the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            unsigned long long w = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(kFull, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        const unsigned long long chunk = wsum[kScanThreads / 32 - 1];
        unsigned long long before = carry + (wid ? wsum[wid - 1] : 0ull) + (x - own);
#pragma unroll
        for (int u = 0; u < kScanItems; ++u) {
            const uint64_t q = base + (uint64_t)tid * kScanItems + u;
            if (q < n) out[q].cigar_offset = (uint32_t)before;
            before += c[u];
        }
        __syncthreads();
        if (tid == 0) carry += chunk;
        __syncthreads();
    }
    if (tid == 0) *total = carry;
}

// Copies every item's CIGAR from its slot to its place in the compact buffer (one warp per item).
__global__ void __launch_bounds__(256) sw_gather_kernel(const phmm_sw_result* __restrict__ out,
                                                         const uint64_t* __restrict__ slot_off,
                                                         const uint32_t* __restrict__ ops, uint32_t* __restrict__ compact,
                                                         uint32_t n, uint32_t cap)
{
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t q = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); q < n; q += nwarps) {
        const uint32_t cnt = min(out[q].cigar_count, cap);
        const uint32_t* src = ops + slot_off[q];
        uint32_t* dst = compact + out[q].cigar_offset;
        for (uint32_t k = lane; k < cnt; k += 32) dst[k] = src[k];
    }
}

// AlleleLikelihoods::search_best_allele with can_be_reference and priorities
// (genotype/allele_likelihoods.hpp:589-658): the most likely haplotype of one read (column `col` of
// a [hap][read] block with row stride `stride`); when the runner-up is within the log10 informative
// threshold (0.2, allele_likelihoods.hpp:27), the haplotypes within that threshold of the best are
// ranked by priority instead.
__device__ int search_best_haplotype(const double* v, uint64_t stride, uint32_t col, uint32_t M, const double* pr)
{
    const double thr = 0.2;
    int best = 0, second = 0;
    double lb = v[col], sl = -__longlong_as_double(0x7ff0000000000000ll);
    for (uint32_t a = 1; a < M; ++a) {
        const double c = v[(uint64_t)a * stride + col];
        if (c > lb) {
            second = best;
            best = (int)a;
            sl = lb;
            lb = c;
        } else if (c > sl) {
            second = (int)a;
            sl = c;
        }
    }
    if (lb - sl < thr) {
        double bp = pr[best], sp = pr[second];
        for (uint32_t a = 0; a < M; ++a) {
            const double c = v[(uint64_t)a * stride + col];
            if ((int)a == best || lb - c > thr) continue;
            const double cp = pr[a];
            if (cp > bp) {
                second = best;
                best = (int)a;
                sp = bp;
                bp = cp;
            } else if (cp > sp) {
                second = (int)a;
                sp = cp;
            }
        }
    }
    return best;
}

constexpr int kRealignThreads = 256;

// One block per realigned region: each kept read's column in the normalised block (a block scan of
// the kept flags, as the post-processing placed them), its best haplotype and its alignment item.
__global__ void __launch_bounds__(kRealignThreads) realign_items_kernel(RealignView v)
{
    __shared__ uint32_t warp_sums[kRealignThreads / 32];
    __shared__ uint32_t base_kept;
    for (uint32_t k = blockIdx.x; k < v.n_rr; k += gridDim.x) {
        const RealignRegion rr = v.rr[k];
        const RegionDesc rg = v.regions[rr.region];
        const uint32_t M = rg.n_haps, N = rg.n_reads;
        const double* norm = v.norm + rg.out_off;
        if (threadIdx.x == 0) base_kept = 0;
        __syncthreads();
        for (uint32_t r0 = 0; r0 < N; r0 += blockDim.x) {
            const uint32_t r = r0 + threadIdx.x;
            const bool keep = r < N && v.keep[rg.read_begin + r] != 0;
            const unsigned int ballot = __ballot_sync(kFull, keep);
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            if (lane == 0) warp_sums[w] = __popc(ballot);
            __syncthreads();
            uint32_t col = base_kept;
            for (int q = 0; q < w; ++q) col += warp_sums[q];
            col += __popc(ballot & ((1u << lane) - 1u));
            if (r < N) {
                SwItem it{};
                int b = -1;
                if (keep && M > 0) {
                    b = search_best_haplotype(norm, N, col, M, v.prio + rr.prio_off);
                    const uint64_t h0 = v.hap_off[rg.hap_begin + b], h1 = v.hap_off[rg.hap_begin + b + 1];
                    const uint64_t q0 = v.read_off[rg.read_begin + r], q1 = v.read_off[rg.read_begin + r + 1];
                    const uint32_t cl = v.clip[2ull * (rr.item_begin + r)], cr = v.clip[2ull * (rr.item_begin + r) + 1];
                    it.hap_start = h0;
                    it.hap_len = (uint32_t)(h1 - h0);
                    it.read_start = q0 + cl;
                    it.read_len = (uint32_t)(q1 - q0) - cl - cr;  // clips checked against the length at submit
                }
                v.items[rr.item_begin + r] = it;
                v.best[rr.item_begin + r] = b;
            }
            __syncthreads();
            if (threadIdx.x == blockDim.x - 1) {
                uint32_t total = 0;
                for (int q = 0; q < (int)(blockDim.x >> 5); ++q) total += warp_sums[q];
                base_kept += total;
            }
            __syncthreads();
        }
    }
}

using SwKernel = void (*)(SwView);

const SwKernel kSwKernels[kSwClasses] = {
    sw_kernel<1, false>,  sw_kernel<2, false>,  sw_kernel<3, false>,  sw_kernel<4, false>,  sw_kernel<5, false>,
    sw_kernel<6, false>,  sw_kernel<7, false>,  sw_kernel<8, false>,  sw_kernel<10, false>, sw_kernel<12, false>,
    sw_kernel<16, false>, sw_kernel<20, false>, sw_kernel<24, false>, sw_kernel<24, true>,
};

}  // namespace

int sw_class_of(const SwParams& prm, int variant, uint32_t nrow, uint32_t ncol)
{
    if (!sw_uses_int32(variant, nrow, ncol, prm.match) && ncol > 0 && nrow > 0 &&
        std::max(nrow, ncol) < (uint32_t)kSwMaxSeq &&
        !sw_w16_cannot_wrap((short)prm.match, (short)prm.mismatch, (short)prm.gap_open, (short)prm.gap_extend,
                            std::min(nrow, ncol)))
        return kSwWrapClass;
    const uint32_t k = std::max<uint32_t>(1, (ncol + 31) / 32);
    for (int c = 0; c < kSwWrapClass; ++c)
        if ((uint32_t)kSwK[c] >= k) return c;
    return kSwWrapClass - 1;  // K = 24 stripes
}

// Device arena of one aligner batch: inputs (items, order, slot offsets, bases), then the outputs
// (total, results), the CIGAR slots, the compact CIGAR buffer and the per-warp scratch.
struct SwArenaLayout {
    uint64_t items, order, slot_off, hap, read, claim, total, out, slots, compact, scratch, bytes;
    uint64_t in_bytes() const { return claim; }                 // [0, claim): uploaded together
    uint64_t head_bytes() const { return slots - total; }       // [total, slots): total + results

    SwArenaLayout(uint32_t n, uint64_t hap_bytes, uint64_t read_bytes, uint64_t nslots, uint64_t scratch_bytes)
    {
        auto a = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
        items = 0;
        order = a(items + sizeof(SwItem) * (uint64_t)n);
        slot_off = a(order + 4ull * n);
        hap = a(slot_off + 8ull * n);
        read = a(hap + std::max<uint64_t>(hap_bytes, 1));
        claim = a(read + std::max<uint64_t>(read_bytes, 1));
        total = a(claim + 4ull * kSwClasses);
        out = total + 8;
        slots = a(out + sizeof(phmm_sw_result) * (uint64_t)n);
        compact = a(slots + 4ull * std::max<uint64_t>(nslots, 1));
        scratch = a(compact + 4ull * std::max<uint64_t>(nslots, 1));
        bytes = scratch + scratch_bytes;
    }

    SwDeviceBufs bufs(uint8_t* d) const
    {
        SwDeviceBufs b;
        b.items = (const SwItem*)(d + items);
        b.order = (const uint32_t*)(d + order);
        b.slot_off = (const uint64_t*)(d + slot_off);
        b.hap = d + hap;
        b.read = d + read;
        b.claim = (unsigned int*)(d + claim);
        b.total = (unsigned long long*)(d + total);
        b.out = (phmm_sw_result*)(d + out);
        b.slots = (uint32_t*)(d + slots);
        b.compact = (uint32_t*)(d + compact);
        b.scratch = d + scratch;
        return b;
    }
};

struct SwAligner::Resident {
    SwParams prm{};
    int variant = 0;
    SwPlan plan;
    void* arena = nullptr;
    uint8_t* d = nullptr;
    SwArenaLayout lay{0, 0, 0, 0, 0};
};

namespace {

#define SW_CK(call)                                                                   \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            err = std::string(#call) + " failed: " + cudaGetErrorString(e_);          \
            return PHMM_ERR_CUDA;                                                     \
        }                                                                             \
    } while (0)

// Scratch of one class launch is held under this bound by launching fewer resident warps.
constexpr uint64_t kSwScratchCap = 6ull << 30;

// Copy into the pinned staging buffer; large copies are split over host threads (one thread copies
// at a fraction of the memory bandwidth, and the bases of a genome-scale batch are ~100 MB).
void staged_copy(void* dst, const void* src, size_t bytes)
{
    constexpr size_t kPerThread = 8u << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = (unsigned)std::min<size_t>({hw, 8u, bytes / kPerThread});
    if (nt <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t part = (bytes + nt - 1) / nt;
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) {
        const size_t o = (size_t)t * part;
        if (o < bytes) pool.emplace_back([=] { std::memcpy((char*)dst + o, (const char*)src + o, std::min(part, bytes - o)); });
    }
    std::memcpy(dst, src, std::min(part, bytes));
    for (auto& th : pool) th.join();
}

phmm_status check_items(uint32_t n, const SwItem* items, uint64_t hap_bytes, uint64_t read_bytes, std::string& err)
{
    for (uint32_t q = 0; q < n; ++q) {
        const SwItem& it = items[q];
        if (it.hap_start > hap_bytes || it.hap_len > hap_bytes - it.hap_start || it.read_start > read_bytes ||
            it.read_len > read_bytes - it.read_start) {
            err = "Smith-Waterman item " + std::to_string(q) + " lies outside its base buffers";
            return PHMM_ERR_INVALID_ARGUMENT;
        }
    }
    return PHMM_OK;
}

// Multiprocessors and resident blocks per multiprocessor of each kernel class, per device (once).
struct SwDeviceInfo {
    bool ready = false;
    int sms = 0;
    int occ[kSwClasses] = {};
};
std::mutex g_info_mu;
SwDeviceInfo g_info[64];

phmm_status device_info(int device, SwDeviceInfo& out, std::string& err)
{
    if (device < 0 || device >= 64) {
        err = "device ordinal out of range";
        return PHMM_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lk(g_info_mu);
    SwDeviceInfo& di = g_info[device];
    if (!di.ready) {
        int cur = 0;
        SW_CK(cudaGetDevice(&cur));
        SW_CK(cudaSetDevice(device));
        SW_CK(cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, device));
        for (int c = 0; c < kSwClasses; ++c) {
            int b = 0;
            SW_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kSwKernels[c], 32 * kSwBlockWarps, 0));
            di.occ[c] = std::max(b, 1);
        }
        SW_CK(cudaSetDevice(cur));
        di.ready = true;
    }
    out = di;
    return PHMM_OK;
}

}  // namespace

phmm_status sw_plan(int device, const SwParams& prm, int variant, uint32_t n, const uint32_t* nrow,
                    const uint32_t* ncol, uint32_t cigar_cap, SwPlan& p, std::string& err)
{
    SwDeviceInfo di;
    phmm_status st = device_info(device, di, err);
    if (st != PHMM_OK) return st;
    p = SwPlan();
    p.n = n;
    p.cigar_cap = std::min<uint32_t>(cigar_cap, kSwMaxSeq - 1);
    std::vector<uint8_t> cls(n);
    uint32_t counts[kSwClasses] = {};
    p.slot_off.resize(n);
    for (uint32_t q = 0; q < n; ++q) {
        cls[q] = (uint8_t)sw_class_of(prm, variant, nrow[q], ncol[q]);
        ++counts[cls[q]];
        p.cells += (uint64_t)nrow[q] * ncol[q];
        p.slot_off[q] = p.slots;
        if (std::max(nrow[q], ncol[q]) < (uint32_t)kSwMaxSeq)  // runs <= rows + columns consumed
            p.slots += std::min<uint64_t>(p.cigar_cap, (uint64_t)nrow[q] + ncol[q]);
    }
    if (p.slots > 0xffffffffull) {
        err = "Smith-Waterman batch needs more than 2^32 CIGAR ops of room: split it";
        return PHMM_ERR_LIMIT_EXCEEDED;
    }
    p.begin[0] = 0;
    for (int c = 0; c < kSwClasses; ++c) p.begin[c + 1] = p.begin[c] + counts[c];
    // one counting sort: by class, then most cells first in buckets of 4096 cells (the claim order
    // only balances the persistent warps' load, so buckets are as good as an exact order)
    constexpr uint32_t kBuckets = 1024;
    auto key = [&](uint32_t q) {
        const uint64_t b = std::min<uint64_t>(kBuckets - 1, ((uint64_t)nrow[q] * ncol[q]) >> 12);
        return (uint32_t)cls[q] * kBuckets + (kBuckets - 1 - (uint32_t)b);
    };
    std::vector<uint32_t> start((size_t)kSwClasses * kBuckets + 1, 0);
    for (uint32_t q = 0; q < n; ++q) ++start[key(q) + 1];
    for (size_t k = 1; k < start.size(); ++k) start[k] += start[k - 1];
    p.order.assign(n, 0);
    for (uint32_t q = 0; q < n; ++q) p.order[start[key(q)]++] = q;
    p.scratch = 0;
    for (int c = 0; c < kSwClasses; ++c) {
        auto first = p.order.begin() + p.begin[c], lastp = p.order.begin() + p.begin[c + 1];
        uint64_t stride = 256;
        for (auto it = first; it != lastp; ++it) {
            if (std::max(nrow[*it], ncol[*it]) >= (uint32_t)kSwMaxSeq) continue;  // refused: no scratch
            stride = std::max(stride, sw_layout(nrow[*it], ncol[*it], kSwK[c]).total);
        }
        p.stride[c] = stride;
        const uint32_t m = counts[c];
        uint64_t g = std::min<uint64_t>((m + kSwBlockWarps - 1) / kSwBlockWarps, (uint64_t)di.occ[c] * di.sms);
        g = std::min<uint64_t>(g, std::max<uint64_t>(1, kSwScratchCap / (kSwBlockWarps * stride)));
        p.grid[c] = m == 0 ? 0 : (int)g;
        p.scratch = std::max(p.scratch, (uint64_t)p.grid[c] * kSwBlockWarps * stride);
    }
    p.gather_blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 7) / 8, (uint64_t)di.sms * 8));
    return PHMM_OK;
}

phmm_status sw_launch(const SwPlan& p, const SwParams& prm, int variant, const SwDeviceBufs& b, cudaStream_t st,
                      cudaEvent_t ev0, cudaEvent_t ev1, float* class_ms, std::string& err)
{
    if (p.n == 0) return PHMM_OK;
    SW_CK(cudaMemsetAsync(b.claim, 0, sizeof(unsigned int) * kSwClasses, st));
    for (int c = 0; c < kSwClasses; ++c) {
        if (class_ms) class_ms[c] = 0.f;
        if (p.grid[c] == 0) continue;
        SwView v{};
        v.items = b.items;
        v.order = b.order + p.begin[c];
        v.n = p.begin[c + 1] - p.begin[c];
        v.hap = b.hap;
        v.read = b.read;
        v.prm = prm;
        v.variant = variant;
        v.scratch = b.scratch;
        v.stride = p.stride[c];
        v.claim = b.claim + c;
        v.out = b.out;
        v.slot_off = b.slot_off;
        v.ops = b.slots;
        v.cigar_cap = p.cigar_cap;
        if (class_ms) SW_CK(cudaEventRecord(ev0, st));
        kSwKernels[c]<<<p.grid[c], 32 * kSwBlockWarps, 0, st>>>(v);
        SW_CK(cudaGetLastError());
        if (class_ms) {
            SW_CK(cudaEventRecord(ev1, st));
            SW_CK(cudaEventSynchronize(ev1));
            SW_CK(cudaEventElapsedTime(&class_ms[c], ev0, ev1));
        }
    }
    sw_scan_kernel<<<1, kScanThreads, 0, st>>>(b.out, p.n, p.cigar_cap, b.total);
    SW_CK(cudaGetLastError());
    sw_gather_kernel<<<p.gather_blocks, 256, 0, st>>>(b.out, b.slot_off, b.slots, b.compact, p.n, p.cigar_cap);
    SW_CK(cudaGetLastError());
    return PHMM_OK;
}

cudaError_t launch_realign_items(const RealignView& v, int blocks, cudaStream_t st)
{
    if (v.n_rr == 0) return cudaSuccess;
    realign_items_kernel<<<std::max(1, std::min<int>(blocks, (int)v.n_rr)), kRealignThreads, 0, st>>>(v);
    return cudaGetLastError();
}

void RealignBatch::layout()
{
    auto a = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
    const uint64_t n = plan.n;
    o_rr = 0;
    o_prio = a(o_rr + sizeof(RealignRegion) * regions.size());
    o_clip = a(o_prio + 8ull * prio.size());
    o_order = a(o_clip + 2ull * clip.size());
    o_slot = a(o_order + 4ull * n);
    o_items = a(o_slot + 8ull * n);
    o_claim = a(o_items + sizeof(SwItem) * n);
    o_total = a(o_claim + 4ull * kSwClasses);
    o_out = o_total + 8;
    o_best = o_out + sizeof(phmm_sw_result) * n;
    o_slots = a(o_best + 4ull * n);
    o_compact = a(o_slots + 4ull * std::max<uint64_t>(plan.slots, 1));
    o_scratch = a(o_compact + 4ull * std::max<uint64_t>(plan.slots, 1));
    bytes = o_scratch + plan.scratch;
}

phmm_status SwAligner::create(int device, SwAligner** out, std::string& err)
{
    *out = nullptr;
    SwAligner* a = new SwAligner();
    a->dev_ = device;
    auto fail = [&](phmm_status st) {
        delete a;
        return st;
    };
#define SW_CKC(call)                                                                  \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            err = std::string(#call) + " failed: " + cudaGetErrorString(e_);          \
            return fail(PHMM_ERR_CUDA);                                               \
        }                                                                             \
    } while (0)
    SW_CKC(cudaSetDevice(device));
    SW_CKC(cudaStreamCreateWithFlags(&a->stream_, cudaStreamNonBlocking));
    SW_CKC(cudaEventCreate(&a->ev_[0]));
    SW_CKC(cudaEventCreate(&a->ev_[1]));
#undef SW_CKC
    *out = a;
    return PHMM_OK;
}

SwAligner::~SwAligner()
{
    cudaSetDevice(dev_);
    if (arena_) cudaFree(arena_);
    if (pinned_) cudaFreeHost(pinned_);
    for (auto& e : ev_)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
}

phmm_status SwAligner::plan(const SwParams& prm, int variant, uint32_t n, const SwItem* items, uint32_t cigar_cap,
                            SwPlan& p, std::string& err) const
{
    std::vector<uint32_t> nrow(n), ncol(n);
    for (uint32_t q = 0; q < n; ++q) {
        nrow[q] = items[q].hap_len;
        ncol[q] = items[q].read_len;
    }
    return sw_plan(dev_, prm, variant, n, nrow.data(), ncol.data(), cigar_cap, p, err);
}

phmm_status SwAligner::ensure_pinned(uint64_t bytes, std::string& err)
{
    if (bytes <= pinned_bytes_) return PHMM_OK;
    if (pinned_) {
        SW_CK(cudaStreamSynchronize(stream_));
        cudaFreeHost(pinned_);
    }
    pinned_ = nullptr;
    pinned_bytes_ = 0;
    SW_CK(cudaMallocHost(&pinned_, bytes + bytes / 4));
    pinned_bytes_ = bytes + bytes / 4;
    return PHMM_OK;
}

// Results and the compact CIGARs of an arena that has run, to host memory (synchronous).
phmm_status SwAligner::read_back(uint8_t* d, const SwArenaLayout& L, uint32_t n, phmm_sw_result* out,
                                 uint32_t* cigars, uint64_t capacity, uint64_t* total, std::string& err)
{
    phmm_status st = ensure_pinned(L.head_bytes(), err);
    if (st != PHMM_OK) return st;
    uint8_t* h = (uint8_t*)pinned_;
    SW_CK(cudaMemcpyAsync(h, d + L.total, L.head_bytes(), cudaMemcpyDeviceToHost, stream_));
    SW_CK(cudaStreamSynchronize(stream_));
    uint64_t tot = 0;
    std::memcpy(&tot, h, 8);
    if (out) std::memcpy(out, h + (L.out - L.total), sizeof(phmm_sw_result) * (size_t)n);
    if (total) *total = tot;
    if (!cigars || tot == 0) return PHMM_OK;
    if (tot > capacity) {
        err = "the batch's CIGARs need " + std::to_string(tot) + " ops, the buffer holds " + std::to_string(capacity);
        return PHMM_ERR_LIMIT_EXCEEDED;
    }
    st = ensure_pinned(4 * tot, err);
    if (st != PHMM_OK) return st;
    h = (uint8_t*)pinned_;
    SW_CK(cudaMemcpyAsync(h, d + L.compact, 4 * tot, cudaMemcpyDeviceToHost, stream_));
    SW_CK(cudaStreamSynchronize(stream_));
    std::memcpy(cigars, h, 4 * tot);
    return PHMM_OK;
}

phmm_status SwAligner::align(const SwParams& prm, int variant, uint32_t n, const SwItem* items, const uint8_t* hap,
                             uint64_t hap_bytes, const uint8_t* read, uint64_t read_bytes, uint32_t cigar_cap,
                             phmm_sw_result* out, uint32_t* cigars, uint64_t cigar_capacity, uint64_t* cigar_total,
                             float* device_ms, std::string& err)
{
    if (device_ms) *device_ms = 0.f;
    if (cigar_total) *cigar_total = 0;
    if (n == 0) return PHMM_OK;
    phmm_status st = check_items(n, items, hap_bytes, read_bytes, err);
    if (st != PHMM_OK) return st;
    std::lock_guard<std::mutex> lk(mu_);
    SW_CK(cudaSetDevice(dev_));
    SwPlan p;
    st = plan(prm, variant, n, items, cigar_cap, p, err);
    if (st != PHMM_OK) return st;
    const SwArenaLayout L(n, hap_bytes, read_bytes, p.slots, p.scratch);
    if (L.bytes > arena_bytes_) {
        if (arena_) {
            SW_CK(cudaStreamSynchronize(stream_));
            cudaFree(arena_);
            arena_ = nullptr;
            arena_bytes_ = 0;
        }
        const uint64_t sz = L.bytes + L.bytes / 4;
        if (cudaMalloc(&arena_, sz) != cudaSuccess) {
            cudaGetLastError();
            err = "Smith-Waterman arena of " + std::to_string(sz) + " bytes could not be allocated";
            return PHMM_ERR_OUT_OF_MEMORY;
        }
        arena_bytes_ = sz;
    }
    // inputs through pinned staging in one copy: items | order | slot offsets | haplotypes | reads
    st = ensure_pinned(L.in_bytes(), err);
    if (st != PHMM_OK) return st;
    uint8_t* h = (uint8_t*)pinned_;
    uint8_t* d = (uint8_t*)arena_;
    staged_copy(h + L.items, items, sizeof(SwItem) * (size_t)n);
    std::memcpy(h + L.order, p.order.data(), 4ull * n);
    std::memcpy(h + L.slot_off, p.slot_off.data(), 8ull * n);
    if (hap_bytes) staged_copy(h + L.hap, hap, hap_bytes);
    if (read_bytes) staged_copy(h + L.read, read, read_bytes);
    SW_CK(cudaMemcpyAsync(d, h, L.in_bytes(), cudaMemcpyHostToDevice, stream_));
    SW_CK(cudaEventRecord(ev_[0], stream_));
    st = sw_launch(p, prm, variant, L.bufs(d), stream_, ev_[0], ev_[1], nullptr, err);
    if (st != PHMM_OK) return st;
    SW_CK(cudaEventRecord(ev_[1], stream_));
    st = read_back(d, L, n, out, cigars, cigar_capacity, cigar_total, err);
    if (device_ms) cudaEventElapsedTime(device_ms, ev_[0], ev_[1]);
    return st;
}

phmm_status SwAligner::resident_create(const SwParams& prm, int variant, uint32_t n, const SwItem* items,
                                       const uint8_t* hap, uint64_t hap_bytes, const uint8_t* read,
                                       uint64_t read_bytes, uint32_t cigar_cap, Resident** out, std::string& err)
{
    *out = nullptr;
    phmm_status st = check_items(n, items, hap_bytes, read_bytes, err);
    if (st != PHMM_OK) return st;
    std::lock_guard<std::mutex> lk(mu_);
    SW_CK(cudaSetDevice(dev_));
    Resident* r = new Resident();
    r->prm = prm;
    r->variant = variant;
    st = plan(prm, variant, n, items, cigar_cap, r->plan, err);
    if (st != PHMM_OK) {
        delete r;
        return st;
    }
    r->lay = SwArenaLayout(n, hap_bytes, read_bytes, r->plan.slots, r->plan.scratch);
    if (cudaMalloc(&r->arena, r->lay.bytes) != cudaSuccess) {
        cudaGetLastError();
        err = "Smith-Waterman resident arena of " + std::to_string(r->lay.bytes) + " bytes could not be allocated";
        delete r;
        return PHMM_ERR_OUT_OF_MEMORY;
    }
    r->d = (uint8_t*)r->arena;
    auto up = [&](uint64_t off, const void* src, uint64_t bytes) {
        return bytes ? cudaMemcpyAsync(r->d + off, src, bytes, cudaMemcpyHostToDevice, stream_) : cudaSuccess;
    };
    const SwArenaLayout& L = r->lay;
    cudaError_t e = up(L.items, items, sizeof(SwItem) * (uint64_t)n);
    if (e == cudaSuccess) e = up(L.order, r->plan.order.data(), 4ull * n);
    if (e == cudaSuccess) e = up(L.slot_off, r->plan.slot_off.data(), 8ull * n);
    if (e == cudaSuccess) e = up(L.hap, hap, hap_bytes);
    if (e == cudaSuccess) e = up(L.read, read, read_bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(r->d + L.total, 0, L.head_bytes(), stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) {
        err = std::string("Smith-Waterman resident upload failed: ") + cudaGetErrorString(e);
        cudaFree(r->arena);
        delete r;
        return PHMM_ERR_CUDA;
    }
    *out = r;
    return PHMM_OK;
}

phmm_status SwAligner::resident_run(Resident* r, int iterations, float* ms_per_run, float* class_ms, std::string& err)
{
    std::lock_guard<std::mutex> lk(mu_);
    SW_CK(cudaSetDevice(dev_));
    if (ms_per_run) *ms_per_run = 0.f;
    if (r->plan.n == 0) return PHMM_OK;
    const SwDeviceBufs b = r->lay.bufs(r->d);
    if (iterations > 0) {
        SW_CK(cudaEventRecord(ev_[0], stream_));
        for (int it = 0; it < iterations; ++it) {
            phmm_status st = sw_launch(r->plan, r->prm, r->variant, b, stream_, nullptr, nullptr, nullptr, err);
            if (st != PHMM_OK) return st;
        }
        SW_CK(cudaEventRecord(ev_[1], stream_));
        SW_CK(cudaEventSynchronize(ev_[1]));
        float ms = 0.f;
        SW_CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
        if (ms_per_run) *ms_per_run = ms / iterations;
    }
    if (class_ms) {
        phmm_status st = sw_launch(r->plan, r->prm, r->variant, b, stream_, ev_[0], ev_[1], class_ms, err);
        if (st != PHMM_OK) return st;
        SW_CK(cudaStreamSynchronize(stream_));
    }
    return PHMM_OK;
}

phmm_status SwAligner::resident_results(Resident* r, phmm_sw_result* out, uint32_t* cigars, uint64_t capacity,
                                        uint64_t* total, std::string& err)
{
    std::lock_guard<std::mutex> lk(mu_);
    SW_CK(cudaSetDevice(dev_));
    if (total) *total = 0;
    if (r->plan.n == 0) return PHMM_OK;
    return read_back(r->d, r->lay, r->plan.n, out, cigars, capacity, total, err);
}

void SwAligner::resident_destroy(Resident* r)
{
    if (!r) return;
    {
        std::lock_guard<std::mutex> lk(mu_);
        cudaSetDevice(dev_);
        cudaStreamSynchronize(stream_);
        if (r->arena) cudaFree(r->arena);
    }
    delete r;
}

}  // namespace phmm
