// One warp's share of an FP64 recompute class: the persistent claim loop over the class's runs of
// underflowed pairs, each streamed through its read (phmm_device.cuh).  Device code only: the class
// kernels (phmm_kernels.cu) call it, and it compiles for the host as well, where
// tests/native/warp_emu.cpp runs it on 32 threads standing for the lanes.
#pragma once

#include <type_traits>

#include "phmm_device.cuh"
#include "phmm_device64.cuh"

namespace phmm {

// ------------------------------------------------------------------------------------------
// One read against a run of haplotypes [g_lo, g_hi).
// ------------------------------------------------------------------------------------------
template <typename T, int K, int V, int PM, bool MULTI, bool UNF = false>
__device__ __forceinline__ void run_read(const BatchView& b, const ProbTables<T>& tb, const PassControl& pc,
                                         const SweepOut& so, uint32_t g_lo, uint32_t g_hi, int lane, T* scr, T* tab)
{
    const uint64_t roff = b.read_off[so.read];
    const int R = (int)(b.read_off[so.read + 1] - roff);
    const int Tcols = (int)(b.hap_off[g_hi] - b.hap_off[g_lo]);
    // A read that does not fit the class's stripe, or a multi-stripe stream longer than the
    // scratch row, means a planning bug: report it and leave the pairs as NaN.
    if (R <= 0 || (!MULTI && R > kWarp * K) || (MULTI && (R <= kWarp * K || Tcols > (int)pc.scratch_cols))) {
        if (lane == 0) atomicOr(pc.status, kStatusBadItem);
        return;
    }
    if constexpr (PM == PM_EQ || (PM == PM_ROW && !UNF)) {
        // the recompute pass: the two-value lane state (phmm_device64.cuh), one value per read for
        // constant gaps with insertion = deletion, per row otherwise
        static_assert(sizeof(T) == 8 && !UNF, "the two-value lane state is the FP64 recompute");
        using LR = typename std::conditional<PM == PM_EQ, LaneRowsEq<K>, LaneRowsRow<K>>::type;
        LR L;
        constexpr int SR = kWarp * K;  // rows per stripe
        const int stripes = MULTI ? (R + SR - 1) / SR : 1;
        const int pad = SR * stripes - R;
        for (int s = 0; s < stripes; ++s) {
            bool exotic;
            if constexpr (PM == PM_EQ)
                exotic = load_rows_eq<K, V>(L, tab, b, tb, roff, R, s * SR, pad, lane);
            else
                exotic = load_rows_row<K, V>(L, tab, b, tb, roff, R, s * SR, pad, lane);
            const bool above_row0 = (s == 0) && (lane * K <= pad);
            const int row0 = s * SR - pad;  // read position of slot 0 of lane 0
            if (!MULTI)
                sweep_eq<K, V, false, false>(L, tab, b, tb, so, g_lo, g_hi, scr, lane, above_row0, exotic, roff, R, row0);
            else if (s == 0)
                sweep_eq<K, V, false, true>(L, tab, b, tb, so, g_lo, g_hi, scr, lane, above_row0, exotic, roff, R, row0);
            else if (s == stripes - 1)
                sweep_eq<K, V, true, false>(L, tab, b, tb, so, g_lo, g_hi, scr, lane, above_row0, exotic, roff, R, row0);
            else
                sweep_eq<K, V, true, true>(L, tab, b, tb, so, g_lo, g_hi, scr, lane, above_row0, exotic, roff, R, row0);
            if (MULTI) __syncwarp();  // lane 31's scratch row is read by lane 0 in the next stripe
        }
    } else {
        LaneRows<T, K, PM> L;
        if (!MULTI) {
            const int pad = kWarp * K - R;
            const bool exotic = load_rows<T, K, V, PM>(L, tab, b, tb, roff, R, 0, pad, lane);
            sweep<T, K, V, PM, false, false, UNF>(L, tab, b, tb, pc, so, g_lo, g_hi, scr, lane, lane * K <= pad, exotic,
                                                  roff, R, -pad);
        } else {
            constexpr int SR = kWarp * K;  // rows per stripe
            const int stripes = (R + SR - 1) / SR;
            const int pad = SR * stripes - R;
            for (int s = 0; s < stripes; ++s) {
                const bool exotic = load_rows<T, K, V, PM>(L, tab, b, tb, roff, R, s * SR, pad, lane);
                const bool above_row0 = (s == 0) && (lane * K <= pad);
                const int row0 = s * SR - pad;  // read position of slot 0 of lane 0
                if (s == 0)
                    sweep<T, K, V, PM, false, true, UNF>(L, tab, b, tb, pc, so, g_lo, g_hi, scr, lane, above_row0, exotic,
                                                         roff, R, row0);
                else if (s == stripes - 1)
                    sweep<T, K, V, PM, true, false, UNF>(L, tab, b, tb, pc, so, g_lo, g_hi, scr, lane, above_row0, exotic,
                                                         roff, R, row0);
                else
                    sweep<T, K, V, PM, true, true, UNF>(L, tab, b, tb, pc, so, g_lo, g_hi, scr, lane, above_row0, exotic,
                                                        roff, R, row0);
                __syncwarp();  // lane 31's scratch row is read by lane 0 in the next stripe
            }
        }
    }
}

// The claim loop of one warp over the class's rerun segment (pc.cd).  UNF: the all-FP64 check
// arithmetic (plain multiply and add); the recompute pass proper uses the reference's contracted
// arithmetic.  tab: the warp's shared prior table (prior_table_size<K>() values); warp_id: the
// warp's index in the grid (its scratch row).
template <int K, int V, int PM, bool MULTI, bool UNF = false>
__device__ __forceinline__ void warp_reruns64(const BatchView& b, const ProbTables<double>& tb, const PassControl& pc,
                                              double* tab, int lane, unsigned int warp_id)
{
    double* scr = MULTI ? (double*)pc.scratch + (size_t)warp_id * pc.scratch_cols * 3 : nullptr;
    const unsigned int n = min(pc.cd->rerun_count, pc.cd->rerun_cap);
    const RerunEntry* rerun = pc.rerun + pc.cd->rerun_off;
    for (;;) {
        const unsigned int idx = claim(&pc.cd->claim64, lane);
        if (idx >= n) break;
        const RerunEntry e = rerun[idx];
        SweepOut so;
        so.out = b.out;
        so.pair_flags = nullptr;
        so.out_base = e.out_idx;
        so.out_stride = e.out_stride;
        so.read = e.read;
        run_read<double, K, V, PM, MULTI, UNF>(b, tb, pc, so, e.hap, e.hap + e.n_haps, lane, scr, tab);
    }
}

}  // namespace phmm
