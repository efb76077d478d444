// One warp's share of an FP32 class: the persistent claim loop over the class's work items and the
// two-reads-per-warp sweep of each (phmm_device2.cuh).  Device code only: the class kernels
// (phmm_fwd32.cuh) call it with their shared prior table, and it compiles for the host as well,
// where tests/native/warp_emu.cpp runs it on 32 threads standing for the lanes.
#pragma once

#include "phmm_device2.cuh"

namespace phmm {

// Two reads per warp (X and Y, the two components of every float2) against a run of haplotypes.
// The stripe holds 32 * KH rows; MULTI runs `stripes` of them top to bottom, linked through the
// warp's scratch row.
template <int KH, int V, int PM, bool MULTI>
__device__ __forceinline__ void run_pair2(const BatchView& b, const ProbTables<float>& tb, const PassControl& pc,
                                          const SweepOut2& so, uint32_t g_lo, uint32_t g_hi, int lane, int stripes,
                                          float2* scr, float4* tab)
{
    constexpr int SR = kWarp * KH;  // rows per stripe
    LaneRows2<KH, PM> L;
    ReadPair rp;
    bool bad = false;
    const int S = MULTI ? stripes : 1;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        rp.roff[k] = 0;
        rp.R[k] = 0;
        if (so.read[k] != kNoRead) {
            rp.roff[k] = b.read_off[so.read[k]];
            rp.R[k] = (int)(b.read_off[so.read[k] + 1] - rp.roff[k]);
            bad |= rp.R[k] <= 0;
        }
        bad |= rp.R[k] > SR * S;
        rp.pad[k] = SR * S - rp.R[k];
    }
    const int Tcols = (int)(b.hap_off[g_hi] - b.hap_off[g_lo]);
    // A planning error skips the item; its pairs stay NaN and the status word reports it.
    bad |= so.read[0] == kNoRead || (MULTI && (S < 2 || Tcols > (int)pc.scratch_cols));
    if (bad) {
        if (lane == 0) atomicOr(pc.status, kStatusBadItem);
        return;
    }
    const bool aboveX = lane * KH <= rp.pad[0], aboveY = lane * KH <= rp.pad[1];
    if (!MULTI) {
        const bool exotic = __any_sync(0xffffffffu, load_rows2<KH, V, PM>(L, tab, b, tb, rp, 0, lane));
        sweep2<KH, V, PM, false, false>(L, tab, b, tb, pc, so, rp, 0, g_lo, g_hi, scr, lane, aboveX, aboveY, exotic);
    } else {
        for (int s = 0; s < S; ++s) {
            const bool exotic = __any_sync(0xffffffffu, load_rows2<KH, V, PM>(L, tab, b, tb, rp, s * SR, lane));
            const bool aX = s == 0 && aboveX, aY = s == 0 && aboveY;
            if (s == 0)
                sweep2<KH, V, PM, false, true>(L, tab, b, tb, pc, so, rp, 0, g_lo, g_hi, scr, lane, aX, aY, exotic);
            else if (s == S - 1)
                sweep2<KH, V, PM, true, false>(L, tab, b, tb, pc, so, rp, s * SR, g_lo, g_hi, scr, lane, aX, aY,
                                               exotic);
            else
                sweep2<KH, V, PM, true, true>(L, tab, b, tb, pc, so, rp, s * SR, g_lo, g_hi, scr, lane, aX, aY,
                                              exotic);
            __syncwarp();  // lane 31's scratch row is read by lane 0 in the next stripe
        }
    }
}

// The claim loop of one warp: work items of the class (pc.cd) until its counter runs out or the warp
// has taken `cap` of them.  tab: the warp's shared prior table (and code ring); warp_id: the warp's
// index in the grid (its scratch row).
template <int KH, int V, int PM, bool MULTI>
__device__ __forceinline__ void warp_items32(const BatchView& b, const ProbTables<float>& tb, const PassControl& pc,
                                             float4* tab, int lane, unsigned int warp_id, unsigned int cap)
{
    float2* scr = MULTI ? (float2*)pc.scratch + (size_t)warp_id * pc.scratch_cols * 3 : nullptr;
    const unsigned int n = pc.cd->n_items;
    const WorkItem* items = pc.items + pc.cd->item_off;
    // the kernel's class mode (0 constant gaps with insertion = deletion, 1 per-row, 2 intra); its
    // underflowed pairs go to the FP64 classes of that mode
    const int mode = mode32(V, PM == PM_ROW ? 1 : 0);
    for (unsigned int taken = 0; taken < cap; ++taken) {
        const unsigned int idx = claim(&pc.cd->claim32, lane);
        if (idx >= n) break;
        const WorkItem it = items[idx];
        const RegionDesc rg = b.regions[it.region];
        SweepOut2 so;
        so.out = b.out;
        so.pair_flags = b.pair_flags;
        so.out_stride = rg.n_reads;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            so.read[k] = it.read[k];
            const uint32_t r = it.read[k] == kNoRead ? rg.read_begin : it.read[k];
            so.out_base[k] = rg.out_off + (uint64_t)it.hap_lo * rg.n_reads + (r - rg.read_begin);
            // underflowed pairs go to the FP64 class of this mode and the read's length
            const uint64_t R = it.read[k] == kNoRead ? 1 : b.read_off[r + 1] - b.read_off[r];
            so.cd64[k] = pc.cd64 + class64_for_len(mode, R);
        }
        run_pair2<KH, V, PM, MULTI>(b, tb, pc, so, rg.hap_begin + it.hap_lo, rg.hap_begin + it.hap_hi, lane,
                                    it.stripes, scr, tab);
    }
}

}  // namespace phmm
