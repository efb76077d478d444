// Device-side PairHMM forward wavefront for sm_100a.
//
// Reference arithmetic reproduced here (paths inside the reference project):
//   per-row tables    src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter.cpp:59-101
//                     src/haplotypecaller/pairhmm/roDV_intra/pairhmm_impl.cpp:88-112,149-156
//   cell update       src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter.cpp:165-195 (inter)
//                     src/haplotypecaller/pairhmm/roDV_intra/pairhmm_impl.cpp:235-280 (intra)
//   boundary, sum     src/haplotypecaller/pairhmm/roDV_inter/pairhmm_inter.cpp:230-273
//   N as wildcard     src/haplotypecaller/pairhmm/roDV_intra/pairhmm_impl.cpp:13-44
//   FP32 -> FP64      src/haplotypecaller/pairhmm/roDV_schedule.cpp:35,269-279
//
// The reference's AVX-512 objects are built by GCC with FMA available, and GCC contracts the
// cell update into this order (checked bit for bit against the reference build):
//   inter  s = fma(Ddiag, gapm, fma(Mdiag, mm, Idiag*gapm))
//   intra  s = fma(Ddiag, gapm, fma(Idiag, gapm, Mdiag*mm))
//   both   M = s * prior,  I = fma(Iup, xx, Mup*mx),  D = fma(Dleft, yy, Mleft*my)
// The kernels below issue exactly these operations with explicit round-to-nearest intrinsics
// (never re-contracted), with flush-to-zero like the reference's MXCSR setting, so each pair's
// raw FP32 (and FP64) sum is bit-identical to the reference kernel of the same variant.
//
// Mapping.  One warp owns one read (one "stripe" of 32*K padded rows: lane l holds rows
// l*K .. l*K+K-1) and streams a run of the region's haplotypes through it as one concatenated
// column stream.  At step t lane l works on stream column p = t - l; the three values of its
// bottom row go to lane l+1 by warp shuffle, and lane 31's bottom row is the read's last row,
// whose M and I are summed per haplotype.  Rows are padded at the top, and a pad row carries
// coefficients (prior 0, mx = my = 0, xx = 1) that make it reproduce the boundary row exactly
// (M = I = 0, D = C/H), so the read's last row is always lane 31's last slot.  Crossing from one
// haplotype to the next only resets a lane's left-hand state, so the fill/drain of the wavefront
// is paid once per work item instead of once per pair.  Reads longer than 32*8 rows run as
// several stripes, the bottom row of one stripe feeding the next through a per-warp scratch row.
#pragma once

#include <cstdint>

#include "phmm_types.h"

namespace phmm {

// Steps per boundary-free chunk of the scalar sweep (the FP64 recompute), a build-time setting:
// the double-precision cell update is about twice the code of the FP32 one, so the unrolled chunk
// decides how much of the hot loop the instruction cache has to hold.  Measured on B200 over the
// 2,000-region benchmark batch: chunks of 2 or 4 steps cut the FP64 tail from 54 to 39 ms against
// 8 steps (instruction-fetch stalls), 4 being marginally the best.
#ifndef PHMM_CHUNK_SCALAR
#define PHMM_CHUNK_SCALAR 4
#endif
constexpr int kChunkScalar = PHMM_CHUNK_SCALAR;

// Explicitly rounded arithmetic: these are never contracted or reassociated by the compiler.
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }

// FP64 has no hardware flush-to-zero; the reference's MXCSR.FTZ flushes tiny double results, so
// the FP64 path flushes explicitly.  Results below 2^-1022 only arise far below any likelihood
// that survives the FP32 -> FP64 switch, so this only keeps the two paths identical.  Every value
// of the recurrence is >= 0 (probabilities times a positive scale), so a double is subnormal or
// zero exactly when its high word is below 0x00100000 (biased exponent 0): an integer compare and
// two selects, with no FP64-pipe instruction (a DSETP would take one of the pipe's slots per flush,
// eight per cell).
__device__ __forceinline__ float ftz(float x) { return x; }  // FP32: hardware FTZ (-ftz=true)
__device__ __forceinline__ double ftz(double x) { return __double2hiint(x) < 0x00100000 ? 0.0 : x; }

template <typename T>
struct Scale;
template <>
struct Scale<float> {
    // 2^120, log10(2^120) as the float constant of adapter.h:25, threshold of roDV_schedule.cpp:35
    __device__ static float initial() { return 1.329227995784916e36f; }
    __device__ static double log10_initial() { return (double)36.1236000061f; }
};
template <>
struct Scale<double> {
    __device__ static double initial() { return 1.1235582092889474e307; }  // 2^1020
    __device__ static double log10_initial() { return 307.050595577260822; }
};

// Lane 0 claims the warp's next work index from a per-class counter.
__device__ __forceinline__ unsigned int claim(unsigned int* counter, int lane)
{
    unsigned int idx = 0;
    if (lane == 0) idx = atomicAdd(counter, 1u);
    return __shfl_sync(0xffffffffu, idx, 0);
}

template <typename T>
__device__ __forceinline__ T shfl_up1(T v)
{
    return __shfl_up_sync(0xffffffffu, v, 1);
}

// Gap parameters: PM_ALL when a read's insertion, deletion and gap-continuation qualities are each
// constant along it, PM_ROW otherwise.  In PM_ALL, mm, gapm, mx and my are held once per lane
// instead of once per row (xx stays per row: pad rows need xx = 1), which frees registers.  PM_EQ
// (the FP32 kernels of mode 0 and the FP64 classes of mode 0, phmm_device64.cuh) is PM_ALL with
// equal insertion and deletion qualities, mx == my: the product M[i][j] * mx that feeds I[i+1][j] is
// the product M[i][j] * my that feeds D[i][j+1], so it is formed once (the two reference operations
// have the same operands, hence the same bits).  The sweep below serves PM_ALL and PM_ROW.
enum ParamMode : int { PM_ALL = 0, PM_ROW = 1, PM_EQ = 2 };

// One lane's rows of the current stripe.  The match priors are not held here: each lane tabulates
// its rows' priors for the five haplotype base classes in shared memory (prior_slot), so a cell
// takes its prior with a load at its column's class instead of a compare and a select.
template <typename T, int K, int PM>
struct LaneRows {
    static constexpr int NR = PM == PM_ROW ? K : 1;
    T Mp[K], Ip[K], Dp[K];        // values at the previous column
    T xx[K];
    T mm[NR], gm[NR], mx[NR], my[NR];
    uint32_t padmask;             // bit k: slot k is a pad row
};

// A warp's prior table: [class][row slot][lane], kTabClasses * K * kWarp values.
template <int K>
__host__ __device__ constexpr int prior_table_size()
{
    return kTabClasses * K * kWarp;
}
template <int K>
__device__ __forceinline__ int prior_slot(uint32_t cls, int k, int lane)
{
    return ((int)cls * K + k) * kWarp + lane;
}

// Loads this lane's rows of the stripe and writes their priors to the warp's table.  Returns true
// when one of the lane's rows is an inter row with a byte outside A/C/G/T: such a byte can equal a
// haplotype byte of class 4, whose table entry holds the mismatch prior (sweep corrects it).
template <typename T, int K, int V, int PM>
__device__ __forceinline__ bool load_rows(LaneRows<T, K, PM>& L, T* tab, const BatchView& b, const ProbTables<T>& tb,
                                          uint64_t roff, int R, int first_padded_row, int pad, int lane)
{
    bool exotic = false;
    L.padmask = 0;
    if (PM == PM_ALL) {
        // constant along the read: its first row gives them (pad rows ignore them)
        const uint64_t o = roff;
        const int iq = R > 0 ? b.read_i[o] & 127 : 0, dq = R > 0 ? b.read_d[o] & 127 : 0;
        const int c = R > 0 ? b.read_c[o] & 127 : 0;
        L.mm[0] = tb.mm[iq * 128 + dq];
        L.gm[0] = tb.gapm[c];
        L.mx[0] = tb.ph2pr[iq];
        L.my[0] = tb.ph2pr[dq];
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int i = first_padded_row + lane * K + k - pad;  // 0-based read position
        const int r = PM == PM_ROW ? k : 0;
        T pa = T(0), pb = T(0);  // pad rows: prior 0 for every class
        uint32_t rc = 0u;
        if (i >= 0 && i < R) {
            const uint64_t o = roff + (uint64_t)i;
            const int q = b.read_q[o] & 127, c = b.read_c[o] & 127;
            pa = tb.pmat[q];
            pb = (V == kInter) ? tb.pmis_inter[q] : tb.pmis_intra[q];
            L.xx[k] = tb.ph2pr[c];
            if (PM == PM_ROW) {
                const int iq = b.read_i[o] & 127, dq = b.read_d[o] & 127;
                L.mm[r] = tb.mm[iq * 128 + dq];
                L.gm[r] = tb.gapm[c];
                L.mx[r] = tb.ph2pr[iq];
                L.my[r] = tb.ph2pr[dq];
            }
            const uint8_t base = b.read_bases[o];
            rc = match_code(base, V);
            if (V == kInter) exotic |= base_class(base) == 4u;
        } else {
            L.xx[k] = T(1);
            if (PM == PM_ROW) {
                L.mm[r] = T(0);
                L.gm[r] = T(0);
                L.mx[r] = T(0);
                L.my[r] = T(0);
            }
            L.padmask |= 1u << k;
        }
#pragma unroll
        for (int c = 0; c < kTabClasses; ++c) tab[prior_slot<K>((uint32_t)c, k, lane)] = class_matches((uint32_t)c, rc, V) ? pa : pb;
    }
    return exotic;
}

// Compute column p for all K rows of this lane.  (sM, sI, sD): the row above this lane's first
// row at column p; (dM, dI, dD): the same row at column p-1.  In PM_ALL pad rows share the lane's
// gap parameters: their prior 0 keeps M = 0, their I stays 0 (the rows above are pad or boundary
// rows with M = I = 0) and xx = 1 keeps D, so they still reproduce the boundary row.
// FLUSH: flush every result below 2^-1022 to zero (FP64 steps whose inputs may be that small); the
// FP32 path flushes in hardware either way.
// UNF: the all-FP64 check arithmetic instead of the reference's contracted one: every product
// rounded, then summed left to right (s = (M mm + I gapm) + D gapm, I = M mx + I xx,
// D = M my + D yy), each result flushed -- the plain-arithmetic FP64 model every likelihood's error
// is measured against.
template <typename T, int K, int V, int PM, bool FLUSH = true, bool UNF = false>
__device__ __forceinline__ void cells(LaneRows<T, K, PM>& L, const T (&pr)[K], T sM, T sI, T dM, T dI, T dD)
{
    auto fz = [](T x) { return FLUSH ? ftz(x) : x; };
    T diM = dM, diI = dI, diD = dD, upM = sM, upI = sI;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int r = PM == PM_ROW ? k : 0;
        const T oM = L.Mp[k], oI = L.Ip[k], oD = L.Dp[k];
        const T prior = pr[k];
        T s, nI, nD;
        if (UNF) {
            s = fz(radd(fz(radd(fz(rmul(diM, L.mm[r])), fz(rmul(diI, L.gm[r])))), fz(rmul(diD, L.gm[r]))));
            nI = fz(radd(fz(rmul(upM, L.mx[r])), fz(rmul(upI, L.xx[k]))));
            nD = fz(radd(fz(rmul(oM, L.my[r])), fz(rmul(oD, L.xx[k]))));
        } else {
            if (V == kInter)
                s = fz(rfma(diD, L.gm[r], fz(rfma(diM, L.mm[r], fz(rmul(diI, L.gm[r]))))));
            else
                s = fz(rfma(diD, L.gm[r], fz(rfma(diI, L.gm[r], fz(rmul(diM, L.mm[r]))))));
            nI = fz(rfma(upI, L.xx[k], fz(rmul(upM, L.mx[r]))));
            nD = fz(rfma(oD, L.xx[k], fz(rmul(oM, L.my[r]))));
        }
        const T nM = fz(rmul(s, prior));
        L.Mp[k] = nM;
        L.Ip[k] = nI;
        L.Dp[k] = nD;
        diM = oM;
        diI = oI;
        diD = oD;
        upM = nM;
        upI = nI;
    }
}

// Smallest value every nonzero input of an FP64 step must reach for no result of that step to fall
// below 2^-1022, so that the step may skip the flushes and still give the flushed results.  Every
// nonzero probability of the tables is at least 2^-44 (the smallest, ph2pr(127) / 3, is 6.6e-14), all
// values are >= 0, and a sum of non-negative terms is at least its largest term; the longest chain
// of products in one step is the insertion recurrence down the lane's K rows (I(a) >= I(a-1) xx,
// after M(a-1) = s prior and the product M mx), so every nonzero result is >= input x 2^(-44 (K+1)).
// Expressed as the high word of that double (biased exponent 1023 - 1022 + 44 (K + 1)).
#ifndef PHMM_F64_VOTE
#define PHMM_F64_VOTE 1  // 0: every FP64 step flushes (no vote)
#endif

// Steps per vote: the bound then covers that many steps (an input of the second step is at least
// the first step's inputs x 2^(-44 (K+1))).  Measured on B200: 2 cut the FP64 pass of the
// underflow-stress shape from 56 to 50 ms against 1; 3 gained nothing more, and at 4 the bound
// (2^562 for K = 8) is above most values, so nearly every step flushes.
#ifndef PHMM_F64_VOTE_EVERY
#define PHMM_F64_VOTE_EVERY 2
#endif

template <int K, int STEPS = PHMM_F64_VOTE_EVERY>
__device__ __forceinline__ uint32_t flush_free_hi()
{
    return (uint32_t)(1 + 44 * STEPS * (K + 1)) << 20;
}

// Whether every nonzero input of the lane's next step reaches flush_free_hi<K>(): its rows and the
// diagonal values (dM, dI, dD) it holds; the values from the row above are the neighbour lane's rows,
// checked by that lane.  Flushed values are 0 or normal, so a zero high word means the value is 0.
template <int K, int PM>
__device__ __forceinline__ bool rows_flush_free(const LaneRows<double, K, PM>& L, double dM, double dI, double dD)
{
    uint32_t m = min(min((uint32_t)__double2hiint(dM) - 1u, (uint32_t)__double2hiint(dI) - 1u),
                     (uint32_t)__double2hiint(dD) - 1u);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        m = min(m, (uint32_t)__double2hiint(L.Mp[k]) - 1u);
        m = min(m, (uint32_t)__double2hiint(L.Ip[k]) - 1u);
        m = min(m, (uint32_t)__double2hiint(L.Dp[k]) - 1u);
    }
    return m >= flush_free_hi<K>() - 1u;
}

struct SweepOut {
    double* out;
    uint8_t* pair_flags;
    uint64_t out_base;            // output index of the stream's first haplotype
    uint32_t out_stride;          // output index step between consecutive haplotypes
    uint32_t read;                // global read index (for the rerun list)
};

// Sweep one stripe over the column stream of haplotypes [g_lo, g_hi) (global indices).
//   FROM_SCR: the row above the stripe comes from scratch (stripe > 0), else the boundary row.
//   TO_SCR:   the stripe's bottom row goes to scratch (not the last stripe), else it is summed.
//   above_row0: the row above this lane's first slot is the boundary row 0 or a pad row.
//   tab: the warp's prior table (load_rows); exotic: this lane holds an inter row with a byte
//   outside A/C/G/T, read position row0 + lane * K + k in slot k (roff, R: the read).
template <typename T, int K, int V, int PM, bool FROM_SCR, bool TO_SCR, bool UNF = false>
__device__ void sweep(LaneRows<T, K, PM>& L, const T* tab, const BatchView& b, const ProbTables<T>& tb,
                      const PassControl& pc, const SweepOut& so, uint32_t g_lo, uint32_t g_hi, T* scr, int lane,
                      bool above_row0, bool exotic, uint64_t roff, int R, int row0)
{
    const uint64_t s0 = b.hap_off[g_lo];
    const int Tcols = (int)(b.hap_off[g_hi] - s0);
    const uint32_t* codes = (V == kInter ? b.codes_inter : b.codes_intra) + kCodePad + s0;
    const T C = Scale<T>::initial();

    // Per-lane stream cursor: cur = haplotype being processed, nb = stream column of the next
    // boundary (first column of the next haplotype, or the end of the stream).
    uint32_t cur = g_lo;
    int nb = 0;
    bool started = false;
    T D0 = T(0);
    T sumM = T(0), sumI = T(0);
    T dM = T(0), dI = T(0), dD = T(0);
    bool flush_free = false;  // FP64: the current step's inputs are all 0 or above the bound

    const int steps = Tcols + kWarp;  // lane 31 reaches column Tcols (the end) at step Tcols + 31

    // Run by a lane whose column p has reached nb, after the step's shuffles.
    auto boundary = [&]() {
        if (started) {
            if (!TO_SCR && lane == kWarp - 1) {
                // sums of flushed non-negative values are 0 or normal: no flush needed
                const T tot = radd(sumM, sumI);
                const uint64_t oi = so.out_base + (uint64_t)(cur - g_lo) * so.out_stride;
                so.out[oi] = log10((double)tot) - Scale<T>::log10_initial();
            }
            ++cur;
        }
        started = true;
        if (cur < g_hi) {
            const int H = (int)(b.hap_off[cur + 1] - b.hap_off[cur]);
            nb += H;
            D0 = C / (T)H;
            // Left edge of the new haplotype: column 0 is zero in every real row; pad rows stand
            // for the boundary row 0, whose D is C/H in every column.
#pragma unroll
            for (int k = 0; k < K; ++k) {
                L.Mp[k] = T(0);
                L.Ip[k] = T(0);
                L.Dp[k] = ((L.padmask >> k) & 1u) ? D0 : T(0);
            }
            dM = T(0);
            dI = T(0);
            dD = above_row0 ? D0 : T(0);
            sumM = T(0);
            sumI = T(0);
        } else {
            nb = 0x7fffffff;
        }
    };

    auto step = [&](int t, bool check) {
        const int p = t - lane;
        T sM = shfl_up1(L.Mp[K - 1]);
        T sI = shfl_up1(L.Ip[K - 1]);
        T sD = shfl_up1(L.Dp[K - 1]);
        if (check && p == nb) boundary();
        if (lane == 0) {
            if (FROM_SCR) {
                const bool ok = p >= 0 && p < Tcols;
                sM = ok ? scr[3 * p + 0] : T(0);
                sI = ok ? scr[3 * p + 1] : T(0);
                sD = ok ? scr[3 * p + 2] : T(0);
            } else {
                sM = T(0);
                sI = T(0);
                sD = D0;
            }
        }
        // the column's priors: its code word's class selects the row slots of the lane's table
        const uint32_t w = codes[p];
        const uint32_t cls = (w & kTabMask) >> kTabShift;
        T pr[K];
#pragma unroll
        for (int k = 0; k < K; ++k) pr[k] = tab[prior_slot<K>(cls, k, lane)];
        if (V == kInter && exotic && cls == 4u) {
            // class 4 holds the mismatch prior for every row; a row whose byte equals this
            // haplotype byte takes the match prior (the raw byte compare of the inter variant)
            const uint32_t hb = w & kCodeMatchMask;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int i = row0 + lane * K + k;
                if (i >= 0 && i < R && b.read_bases[roff + i] == hb) pr[k] = tb.pmat[b.read_q[roff + i] & 127];
            }
        }
        // FP64: the flushes can only change a step whose inputs hold a value below the bound; the
        // warp votes every PHMM_F64_VOTE_EVERY steps (the scratch row read by stripes after the first
        // is not checked)
        constexpr bool kVote = PHMM_F64_VOTE && sizeof(T) == 8 && !FROM_SCR;
        if (kVote && flush_free)
            cells<T, K, V, PM, false, UNF>(L, pr, sM, sI, dM, dI, dD);
        else
            cells<T, K, V, PM, true, UNF>(L, pr, sM, sI, dM, dI, dD);
        dM = sM;
        dI = sI;
        dD = sD;
        if (TO_SCR) {
            if (lane == kWarp - 1 && p >= 0 && p < Tcols) {
                scr[3 * p + 0] = L.Mp[K - 1];
                scr[3 * p + 1] = L.Ip[K - 1];
                scr[3 * p + 2] = L.Dp[K - 1];
            }
        } else {
            sumM = radd(sumM, L.Mp[K - 1]);
            sumI = radd(sumI, L.Ip[K - 1]);
        }
        if constexpr (kVote)
            if (PHMM_F64_VOTE_EVERY == 1 || t % PHMM_F64_VOTE_EVERY == PHMM_F64_VOTE_EVERY - 1)
                flush_free = __all_sync(0xffffffffu, rows_flush_free(L, dM, dI, dD));
    };

    for (int t0 = 0; t0 < steps; t0 += kChunkScalar) {
        // Lanes cover stream columns [t0-31, t0+kChunkScalar-1] in this chunk.  Lane 31 trails, so
        // its next boundary is the first boundary at or after t0-31: past the chunk means no lane
        // meets a boundary and the chunk needs no per-step check.
        const int nb31 = __shfl_sync(0xffffffffu, nb, kWarp - 1);
        if (nb31 >= t0 + kChunkScalar && t0 + kChunkScalar <= steps) {
#pragma unroll
            for (int u = 0; u < kChunkScalar; ++u) step(t0 + u, false);
        } else {
            for (int u = 0; u < kChunkScalar; ++u)
                if (t0 + u < steps) step(t0 + u, true);
        }
    }
}

}  // namespace phmm
