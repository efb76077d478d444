// Persistent FP32 wavefront kernels (packed path of phmm_device2.cuh), one kernel per class:
// mode (variant and gap-parameter mode) x tile shape (row pairs per lane, single or multi-stripe).
// The three modes are instantiated in three translation units (phmm_fwd32_m0/m1/m2.cu) so that
// they compile in parallel; each exports a launcher and an occupancy query over its 13 shapes.
#pragma once

#include <cuda_runtime.h>

#include "phmm_device2.cuh"
#include "phmm_kernels.h"

namespace phmm {

// Two reads per warp (one per 16-lane group) against a run of haplotypes.  The stripe holds
// 32 * KH rows; MULTI runs `stripes` of them top to bottom, linked through the group's scratch row.
template <int KH, int V, int PM, bool MULTI>
__device__ __forceinline__ void run_pair2(const BatchView& b, const ProbTables<float>& tb, const PassControl& pc,
                                          const SweepOut& so, uint32_t g_lo, uint32_t g_hi, int lane, int stripes,
                                          float* scr)
{
    constexpr int SR = 2 * kLanesPerRead * KH;  // rows per stripe (32 virtual lanes x KH)
    const int l = lane & (kLanesPerRead - 1);
    LaneRows2<KH, PM> L;
    uint64_t roff = 0;
    int R = 0;
    if (so.read != kNoRead) {
        roff = b.read_off[so.read];
        R = (int)(b.read_off[so.read + 1] - roff);
    }
    const int S = MULTI ? stripes : 1;
    const int Tcols = (int)(b.hap_off[g_hi] - b.hap_off[g_lo]);
    // Both groups run the sweep together (full-warp shuffles), so a planning error in either skips
    // the item for both; its pairs stay NaN and the status word reports it.
    const bool bad = (so.read != kNoRead && R <= 0) || R > SR * S || (MULTI && (S < 2 || Tcols > (int)pc.scratch_cols));
    if (__any_sync(0xffffffffu, bad)) {
        if (lane == 0) atomicOr(pc.status, kStatusBadItem);
        return;
    }
    // underflowed pairs go to the FP64 class of this mode and this read's length
    PassControl pr = pc;
    pr.cd = pc.cd64 + class64_for_len(mode32(V, PM), (uint64_t)R);
    const int pad = SR * S - R;
    if (!MULTI) {
        load_rows2<KH, V, PM>(L, b, tb, roff, R, 0, pad, l);
        sweep2<KH, V, PM, false, false>(L, b, pr, so, g_lo, g_hi, scr, lane, 2 * l * KH <= pad);
    } else {
        for (int s = 0; s < S; ++s) {
            load_rows2<KH, V, PM>(L, b, tb, roff, R, s * SR, pad, l);
            const bool aboveA = (s == 0) && (2 * l * KH <= pad);
            if (s == 0)
                sweep2<KH, V, PM, false, true>(L, b, pr, so, g_lo, g_hi, scr, lane, aboveA);
            else if (s == S - 1)
                sweep2<KH, V, PM, true, false>(L, b, pr, so, g_lo, g_hi, scr, lane, aboveA);
            else
                sweep2<KH, V, PM, true, true>(L, b, pr, so, g_lo, g_hi, scr, lane, aboveA);
            __syncwarp();  // lane 15's scratch row is read by lane 0 of the group in the next stripe
        }
    }
}

// Resident warps per SM the compiler is asked to allow for the wide shapes (KH >= 6), whose natural
// register count (170-230 per thread) leaves two warps per scheduler: each scheduler's sub-partition
// holds 16K registers, so 168 registers per thread are the most that fit three warps.  Measured on
// B200 over the 2,000-region batch: 12 warps per SM (a few bytes of spills at KH 7-8) take the FP32
// pass from 242 to 235 ms.  A build-time setting (1 leaves the compiler free).
#ifndef PHMM_WIDE_MIN_WARPS
#define PHMM_WIDE_MIN_WARPS 12
#endif
template <int KH>
constexpr int min_blocks32()
{
    return KH >= 6 ? PHMM_WIDE_MIN_WARPS : 1;
}

template <int KH, int V, int PM, bool MULTI>
__global__ void __launch_bounds__(kFwdBlock, min_blocks32<KH>()) fwd_f32_kernel(BatchView b, ProbTables<float> tb,
                                                                                 PassControl pc)
{
    const int lane = threadIdx.x & (kWarp - 1);
    const int group = lane / kLanesPerRead;
    const unsigned int warp_id = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    float* scr = MULTI ? (float*)pc.scratch + ((size_t)warp_id * 2 + group) * pc.scratch_cols * 3 : nullptr;
    const unsigned int n = pc.cd->n_items;
    const WorkItem* items = pc.items + pc.cd->item_off;
    for (;;) {
        const unsigned int idx = claim(&pc.cd->claim32, lane);
        if (idx >= n) break;
        const WorkItem it = items[idx];
        const RegionDesc rg = b.regions[it.region];
        SweepOut so;
        so.out = b.out;
        so.pair_flags = b.pair_flags;
        so.read = it.read[group];
        so.out_base = rg.out_off + (uint64_t)it.hap_lo * rg.n_reads + (so.read - rg.read_begin);
        so.out_stride = rg.n_reads;
        run_pair2<KH, V, PM, MULTI>(b, tb, pc, so, rg.hap_begin + it.hap_lo, rg.hap_begin + it.hap_hi, lane,
                                    it.stripes, scr);
    }
}

typedef void (*F32Kernel)(BatchView, ProbTables<float>, PassControl);

// The 13 shapes of one mode, in shape32 order: single stripe KH = 1..8, multi-stripe KH = 4..8.
#define PHMM_SHAPES32(V, PM)                                                                              \
    fwd_f32_kernel<1, V, PM, false>, fwd_f32_kernel<2, V, PM, false>, fwd_f32_kernel<3, V, PM, false>,    \
        fwd_f32_kernel<4, V, PM, false>, fwd_f32_kernel<5, V, PM, false>, fwd_f32_kernel<6, V, PM, false>, \
        fwd_f32_kernel<7, V, PM, false>, fwd_f32_kernel<8, V, PM, false>, fwd_f32_kernel<4, V, PM, true>,  \
        fwd_f32_kernel<5, V, PM, true>, fwd_f32_kernel<6, V, PM, true>, fwd_f32_kernel<7, V, PM, true>,    \
        fwd_f32_kernel<8, V, PM, true>

#define PHMM_DEFINE_MODE32(MODE, V, PM)                                                                    \
    static const F32Kernel kF32Mode##MODE[kShapes32] = {PHMM_SHAPES32(V, PM)};                             \
    cudaError_t launch_f32_mode##MODE(int shape, const BatchView& b, const ProbTables<float>& tf,          \
                                      const PassControl& pc, int grid, cudaStream_t st)                     \
    {                                                                                                      \
        kF32Mode##MODE[shape]<<<grid, kFwdBlock, 0, st>>>(b, tf, pc);                                      \
        return cudaGetLastError();                                                                         \
    }                                                                                                      \
    cudaError_t occupancy_f32_mode##MODE(int shape, int* blocks_per_sm)                                    \
    {                                                                                                      \
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kF32Mode##MODE[shape], kFwdBlock, 0); \
    }

cudaError_t launch_f32_mode0(int shape, const BatchView& b, const ProbTables<float>& tf, const PassControl& pc,
                             int grid, cudaStream_t st);
cudaError_t launch_f32_mode1(int shape, const BatchView& b, const ProbTables<float>& tf, const PassControl& pc,
                             int grid, cudaStream_t st);
cudaError_t launch_f32_mode2(int shape, const BatchView& b, const ProbTables<float>& tf, const PassControl& pc,
                             int grid, cudaStream_t st);
cudaError_t occupancy_f32_mode0(int shape, int* blocks_per_sm);
cudaError_t occupancy_f32_mode1(int shape, int* blocks_per_sm);
cudaError_t occupancy_f32_mode2(int shape, int* blocks_per_sm);

}  // namespace phmm
