// Persistent FP32 wavefront kernels (packed path of phmm_device2.cuh), one kernel per class:
// mode (variant and gap-parameter mode) x tile shape (row pairs per lane, single or multi-stripe).
// The three modes are instantiated in three translation units (phmm_fwd32_m0/m1/m2.cu) so that
// they compile in parallel; each exports a launcher and an occupancy query over its 13 shapes.
#pragma once

#include <cuda_runtime.h>

#include "phmm_device2.cuh"
#include "phmm_kernels.h"

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

// Resident warps per SM the compiler is asked to allow, one byte per KH (KH = 1 in the low byte):
// PHMM_F32_MIN_WARPS for mode 0 (inter, constant gap qualities), PHMM_F32_MIN_WARPS_OTHER for modes 1
// and 2, whose per-row gap parameters or intra arithmetic need more registers.  Each scheduler's
// sub-partition holds 16K registers: 168 registers per thread fit three warps, 128 fit four; left
// free, the compiler spends registers on loading the priors of a whole chunk of steps early.  Build-
// time settings (1 leaves the compiler free).  Measured on B200: mode 0 runs the 2,000-region batch
// 1.5% faster with 16 warps per SM than with 12 for KH >= 4; modes 1 and 2 spill at 128 registers
// and run a batch of per-row gap qualities and N reads (300 regions) at 2090 GCUPS with 12 warps per
// SM against 1614 with 16.
#ifndef PHMM_F32_MIN_WARPS
#define PHMM_F32_MIN_WARPS 0x10101010100c0101ull
#endif
#ifndef PHMM_F32_MIN_WARPS_OTHER
#define PHMM_F32_MIN_WARPS_OTHER 0x0c0c0c0c0c0c0101ull
#endif
template <int KH, int V, int PM>
__host__ __device__ constexpr int min_blocks32()
{
    return (int)((((V == kInter && PM != PM_ROW) ? (unsigned long long)(PHMM_F32_MIN_WARPS)
                                                 : (unsigned long long)(PHMM_F32_MIN_WARPS_OTHER)) >>
                  (8 * (KH - 1))) &
                 0xffu);
}

template <int KH, int V, int PM, bool MULTI>
__global__ void __launch_bounds__(kFwdBlock, min_blocks32<KH, V, PM>()) fwd_f32_kernel(BatchView b, ProbTables<float> tb,
                                                                                 PassControl pc)
{
    __shared__ float4 tab[tab_floats4<KH>() + kRingFloat4];
    const int lane = threadIdx.x & (kWarp - 1);
    const unsigned int warp_id = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    float2* scr = MULTI ? (float2*)pc.scratch + (size_t)warp_id * pc.scratch_cols * 3 : nullptr;
    const unsigned int n = pc.cd->n_items;
    const WorkItem* items = pc.items + pc.cd->item_off;
    // the kernel's class mode (0 constant gaps with insertion = deletion, 1 per-row, 2 intra); its
    // underflowed pairs go to the FP64 classes of that mode
    const int mode = mode32(V, PM == PM_ROW ? 1 : 0);
    for (;;) {
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
