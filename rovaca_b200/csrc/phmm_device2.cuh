// FP32 wavefront with packed FP32 arithmetic (sm_100a __ffma2_rn / __fmul2_rn).
//
// Arithmetic per cell is exactly the reference's (see phmm_device.cuh for the operation order and
// the reference lines); a packed instruction applies it to two cells with the same per-component
// rounding as the scalar intrinsics, so results stay bit-identical.
//
// Mapping.  16 lanes per read, two reads per warp (lanes 0-15 and 16-31), both streaming the same
// run of haplotype columns.  Lane l of a group holds 2*KH rows of its read as two halves of KH rows
// that behave as two "virtual lanes" v = 2l (half A) and v = 2l + 1 (half B): virtual lane v works
// on stream column p = t - v at step t, so half B runs one column behind half A.  Row a of half A and
// row a of half B are then independent within a step (half B's top row reads half A's bottom row of
// the previous step), so each pair of rows is one float2: the M, I and D updates of both halves are
// single packed instructions and the I recurrence down the rows runs for both halves at once.
// Virtual lane 31 (lane 15, half B) holds the read's last row; rows are padded at the top and pad
// rows reproduce the boundary row exactly (prior 0 keeps M = 0, I stays 0 because the rows above
// have M = I = 0, and xx = 1 keeps D = C/H).  Reads longer than 256 rows run as stripes linked
// through a per-group scratch row, as in the scalar path.
//
// Gap parameters: PM_ALL when a read's insertion, deletion and gap-continuation qualities are each
// constant along it (the region API without a PCR model, and the benchmark data), PM_ROW otherwise.
// In PM_ALL, mm, gapm, mx and my are held once per lane instead of once per row (xx stays per row:
// pad rows need xx = 1), which leaves registers for more rows per lane.
#pragma once

#include <cstdint>

#include "phmm_device.cuh"

namespace phmm {

constexpr int kLanesPerRead = 16;

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 rmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 rfma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ float shfl_up16(float v) { return __shfl_up_sync(0xffffffffu, v, 1, kLanesPerRead); }
__device__ __forceinline__ int shfl_idx(int v, int src) { return __shfl_sync(0xffffffffu, v, src); }

template <int KH, int PM>
struct LaneRows2 {
    static constexpr int NR = PM == PM_ROW ? KH : 1;
    float2 Mp[KH], Ip[KH], Dp[KH];  // (half A, half B) values at each half's previous column
    float2 pa[KH], pb[KH], xx[KH];
    uint32_t rcA[KH], rcB[KH];
    float2 mm[NR], gm[NR], mx[NR], my[NR];
    uint32_t padA, padB;            // bit a: row a of the half is a pad row
};

struct RowParams {
    float pa, pb, mm, gm, mx, xx, my;
    uint32_t rc;
    bool pad;
};

template <int V>
__device__ __forceinline__ RowParams row_params(const BatchView& b, const ProbTables<float>& tb, uint64_t roff, int R,
                                                int i)
{
    RowParams r;
    if (i >= 0 && i < R) {
        const uint64_t o = roff + (uint64_t)i;
        const int q = b.read_q[o] & 127, iq = b.read_i[o] & 127, dq = b.read_d[o] & 127, c = b.read_c[o] & 127;
        r.pa = tb.pmat[q];
        r.pb = (V == kInter) ? tb.pmis_inter[q] : tb.pmis_intra[q];
        r.mm = tb.mm[iq * 128 + dq];
        r.gm = tb.gapm[c];
        r.mx = tb.ph2pr[iq];
        r.xx = tb.ph2pr[c];
        r.my = tb.ph2pr[dq];
        r.rc = match_code(b.read_bases[o], V);
        r.pad = false;
    } else {
        r.pa = r.pb = r.mm = r.gm = r.mx = r.my = 0.f;
        r.xx = 1.f;
        r.rc = 0u;
        r.pad = true;
    }
    return r;
}

// Loads this lane's rows of the stripe starting at padded row `first` (`pad` rows precede row 1).
template <int KH, int V, int PM>
__device__ __forceinline__ void load_rows2(LaneRows2<KH, PM>& L, const BatchView& b, const ProbTables<float>& tb,
                                           uint64_t roff, int R, int first, int pad, int l)
{
    L.padA = 0;
    L.padB = 0;
    if (PM == PM_ALL) {
        // constant along the read: any real row gives them (pad rows ignore them)
        const RowParams r0 = row_params<V>(b, tb, roff, R, R > 0 ? 0 : -1);
        L.mm[0] = f2(r0.mm, r0.mm);
        L.gm[0] = f2(r0.gm, r0.gm);
        L.mx[0] = f2(r0.mx, r0.mx);
        L.my[0] = f2(r0.my, r0.my);
    }
#pragma unroll
    for (int a = 0; a < KH; ++a) {
        const RowParams A = row_params<V>(b, tb, roff, R, first + (2 * l) * KH + a - pad);
        const RowParams B = row_params<V>(b, tb, roff, R, first + (2 * l + 1) * KH + a - pad);
        L.pa[a] = f2(A.pa, B.pa);
        L.pb[a] = f2(A.pb, B.pb);
        L.xx[a] = f2(A.xx, B.xx);
        L.rcA[a] = A.rc;
        L.rcB[a] = B.rc;
        if (PM == PM_ROW) {
            L.mm[a] = f2(A.mm, B.mm);
            L.gm[a] = f2(A.gm, B.gm);
            L.mx[a] = f2(A.mx, B.mx);
            L.my[a] = f2(A.my, B.my);
        }
        L.padA |= (A.pad ? 1u : 0u) << a;
        L.padB |= (B.pad ? 1u : 0u) << a;
    }
}

// All 2*KH rows of the lane for one step.  (upM, upI): row above each half's first row at that
// half's column; (dgM, dgI, dgD): the same rows one column to the left.
template <int KH, int V, int PM>
__device__ __forceinline__ void cells2(LaneRows2<KH, PM>& L, uint32_t hcA, uint32_t hcB, float2 upM, float2 upI,
                                       float2 dgM, float2 dgI, float2 dgD)
{
#pragma unroll
    for (int a = 0; a < KH; ++a) {
        const int r = PM == PM_ROW ? a : 0;
        const float2 oM = L.Mp[a], oI = L.Ip[a], oD = L.Dp[a];
        const float2 prior = f2(codes_match(hcA, L.rcA[a], V) ? L.pa[a].x : L.pb[a].x,
                                codes_match(hcB, L.rcB[a], V) ? L.pa[a].y : L.pb[a].y);
        float2 s;
        if (V == kInter)
            s = rfma2(dgD, L.gm[r], rfma2(dgM, L.mm[r], rmul2(dgI, L.gm[r])));
        else
            s = rfma2(dgD, L.gm[r], rfma2(dgI, L.gm[r], rmul2(dgM, L.mm[r])));
        const float2 nM = rmul2(s, prior);
        const float2 nI = rfma2(upI, L.xx[a], rmul2(upM, L.mx[r]));
        const float2 nD = rfma2(oD, L.xx[a], rmul2(oM, L.my[r]));
        L.Mp[a] = nM;
        L.Ip[a] = nI;
        L.Dp[a] = nD;
        dgM = oM;
        dgI = oI;
        dgD = oD;
        upM = nM;
        upI = nI;
    }
}

// Sweep one stripe of both reads of the warp over the column stream of haplotypes [g_lo, g_hi).
//   FROM_SCR: the row above virtual lane 0 comes from the group's scratch row (stripe > 0).
//   TO_SCR:   virtual lane 31's bottom row goes to the scratch row (not the last stripe).
// so.read is this group's read (UINT32_MAX: no read; the group computes pad rows only and writes
// nothing).  aboveA / aboveB: the row above half A's / half B's first row is row 0 or a pad row.
template <int KH, int V, int PM, bool FROM_SCR, bool TO_SCR>
__device__ void sweep2(LaneRows2<KH, PM>& L, const BatchView& b, const PassControl& pc, const SweepOut& so,
                       uint32_t g_lo, uint32_t g_hi, float* scr, int lane, bool aboveA)
{
    const int l = lane & (kLanesPerRead - 1);
    const bool writer = (l == kLanesPerRead - 1) && so.read != 0xffffffffu;
    const uint64_t s0 = b.hap_off[g_lo];
    const int Tcols = (int)(b.hap_off[g_hi] - s0);
    const uint32_t* codes = (V == kInter ? b.codes_inter : b.codes_intra) + kCodePad + s0;
    const float C = Scale<float>::initial();

    // cursors of the two virtual lanes (B trails A by one column)
    uint32_t curA = g_lo, curB = g_lo;
    int nbA = 0, nbB = 0;
    bool startedB = false;
    float D0A = 0.f, D0B = 0.f;
    float sumM = 0.f, sumI = 0.f;
    float dM = 0.f, dI = 0.f, dD = 0.f;  // row above half A's top row, one column left (from the shuffle)
    float eM = 0.f, eI = 0.f, eD = 0.f;  // half A's bottom row two columns left: half B's diagonal
    uint32_t hcPrev = 0u;

    const int steps = Tcols + 2 * kLanesPerRead;

    auto boundaryA = [&]() {
        if (curA < g_hi) {
            const int H = (int)(b.hap_off[curA + 1] - b.hap_off[curA]);
            nbA += H;
            D0A = C / (float)H;
#pragma unroll
            for (int a = 0; a < KH; ++a) {
                L.Mp[a].x = 0.f;
                L.Ip[a].x = 0.f;
                L.Dp[a].x = ((L.padA >> a) & 1u) ? D0A : 0.f;
            }
            dM = 0.f;
            dI = 0.f;
            dD = aboveA ? D0A : 0.f;
            ++curA;
        } else {
            nbA = 0x7fffffff;
        }
    };
    // Writer lane: the open run of consecutive underflowed haplotypes (first haplotype, its output).
    uint32_t run_lo = 0xffffffffu;
    uint64_t run_oi = 0;
    auto close_run = [&](uint32_t end) {
        if (run_lo == 0xffffffffu) return;
        const unsigned int slot = atomicAdd(&pc.cd->rerun_count, 1u);
        if (slot < pc.cd->rerun_cap) {
            RerunEntry e;
            e.out_idx = run_oi;
            e.read = so.read;
            e.hap = run_lo;
            e.n_haps = end - run_lo;
            e.out_stride = so.out_stride;
            pc.rerun[pc.cd->rerun_off + slot] = e;
            atomicAdd(&pc.cd->rerun_pairs, end - run_lo);
        } else {
            atomicOr(pc.status, kStatusRerunOverflow);
        }
        run_lo = 0xffffffffu;
    };
    auto boundaryB = [&]() {
        if (startedB) {
            if (writer && !TO_SCR) {
                const float tot = radd(sumM, sumI);
                const uint64_t oi = so.out_base + (uint64_t)(curB - g_lo) * so.out_stride;
                so.out[oi] = log10((double)tot) - Scale<float>::log10_initial();
                const bool under = (double)tot < (double)1e-28f;
                if (under) {
                    if (run_lo == 0xffffffffu) {
                        run_lo = curB;
                        run_oi = oi;
                    }
                } else {
                    close_run(curB);
                }
                if (curB + 1 == g_hi) close_run(g_hi);
                if (so.pair_flags) so.pair_flags[oi] = under ? 1 : 0;
            }
            ++curB;
        }
        startedB = true;
        if (curB < g_hi) {
            const int H = (int)(b.hap_off[curB + 1] - b.hap_off[curB]);
            nbB += H;
            D0B = C / (float)H;
#pragma unroll
            for (int a = 0; a < KH; ++a) {
                L.Mp[a].y = 0.f;
                L.Ip[a].y = 0.f;
                L.Dp[a].y = ((L.padB >> a) & 1u) ? D0B : 0.f;
            }
            // half B's diagonal at its first column is half A's bottom row at column -1: half A
            // reset it one step earlier, so eM/eI/eD already hold the boundary values.
            sumM = 0.f;
            sumI = 0.f;
        } else {
            nbB = 0x7fffffff;
        }
    };

    auto step = [&](int t, bool check) {
        const int pA = t - 2 * l;
        const int pB = pA - 1;
        // Half B's up input is half A's bottom row at B's column, computed in the previous step.
        // It is read before half A's boundary reset: when A starts a new haplotype at this step,
        // B is still on the last column of the previous one.
        const float aM = L.Mp[KH - 1].x, aI = L.Ip[KH - 1].x;
        float sM = shfl_up16(L.Mp[KH - 1].y);
        float sI = shfl_up16(L.Ip[KH - 1].y);
        float sD = shfl_up16(L.Dp[KH - 1].y);
        if (check) {
            if (pA == nbA) boundaryA();
            if (pB == nbB) boundaryB();
        }
        if (l == 0) {
            if (FROM_SCR) {
                const bool ok = pA >= 0 && pA < Tcols;
                sM = ok ? scr[3 * pA + 0] : 0.f;
                sI = ok ? scr[3 * pA + 1] : 0.f;
                sD = ok ? scr[3 * pA + 2] : 0.f;
            } else {
                sM = 0.f;
                sI = 0.f;
                sD = D0A;
            }
        }
        const uint32_t hcA = codes[pA];
        const uint32_t hcB = hcPrev;
        hcPrev = hcA;
        // half B's inputs: half A's bottom row at B's column and one column to the left.  The value
        // kept for B's next diagonal is taken after A's reset: if A started a haplotype here, B
        // starts it one step later and its diagonal there is the boundary value.
        const float2 upM = f2(sM, aM);
        const float2 upI = f2(sI, aI);
        const float2 dgM = f2(dM, eM), dgI = f2(dI, eI), dgD = f2(dD, eD);
        eM = L.Mp[KH - 1].x;
        eI = L.Ip[KH - 1].x;
        eD = L.Dp[KH - 1].x;
        dM = sM;
        dI = sI;
        dD = sD;
        cells2<KH, V, PM>(L, hcA, hcB, upM, upI, dgM, dgI, dgD);
        if (TO_SCR) {
            if (l == kLanesPerRead - 1 && pB >= 0 && pB < Tcols) {
                scr[3 * pB + 0] = L.Mp[KH - 1].y;
                scr[3 * pB + 1] = L.Ip[KH - 1].y;
                scr[3 * pB + 2] = L.Dp[KH - 1].y;
            }
        } else {
            sumM = radd(sumM, L.Mp[KH - 1].y);
            sumI = radd(sumI, L.Ip[KH - 1].y);
        }
    };

    for (int t0 = 0; t0 < steps; t0 += kChunk) {
        // Virtual lanes cover columns [t0-31, t0+kChunk-1] in this chunk; virtual lane 31 (lane 15,
        // half B) trails, so its next boundary is the first one at or after t0-31.
        const int nbLast = shfl_idx(nbB, kLanesPerRead - 1);
        if (nbLast >= t0 + kChunk && t0 + kChunk <= steps) {
#pragma unroll
            for (int u = 0; u < kChunk; ++u) step(t0 + u, false);
        } else {
            for (int u = 0; u < kChunk; ++u)
                if (t0 + u < steps) step(t0 + u, true);
        }
    }
}

}  // namespace phmm
