// Persistent FP32 wavefront kernels (packed path of phmm_device2.cuh), one kernel per class:
// mode (variant and gap-parameter mode) x tile shape (row pairs per lane, single or multi-stripe).
// The three modes are instantiated in three translation units (phmm_fwd32_m0/m1/m2.cu) so that
// they compile in parallel; each exports a launcher and an occupancy query over its 13 shapes.
#pragma once

#include <cuda_runtime.h>

#include "phmm_warp32.cuh"
#include "phmm_kernels.h"

namespace phmm {

// Resident warps per SM the compiler is asked to allow, one byte per KH (KH = 1 in the low byte):
// PHMM_F32_MIN_WARPS for mode 0 (inter, constant gap qualities), PHMM_F32_MIN_WARPS_OTHER for modes 1
// and 2, whose per-row gap parameters or intra arithmetic need more registers.  Each scheduler's
// sub-partition holds 16K registers: 168 registers per thread fit three warps, 128 fit four; left
// free, the compiler spends registers on loading the priors of a whole chunk of steps early.  Build-
// time settings (1 leaves the compiler free).  Measured on B200: mode 0 runs the 2,000-region batch
// 1.5% faster with 16 warps per SM than with 12 for KH >= 4; modes 1 and 2 spill at 128 registers
// and run a batch of per-row gap qualities and N reads (300 regions) at 2090 GCUPS with 12 warps per
// SM against 1614 with 16.  KH 4 and 5 in mode 0 run 24 warps per SM (80 registers, spills in the
// boundary code): their classes 1.4% and 0.8% faster than at 16 on the 2,000-region batch.
#ifndef PHMM_F32_MIN_WARPS
#define PHMM_F32_MIN_WARPS 0x10101018180c0101ull
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
    // Over-subscribed grid (waves > 1): warps that exit after their share leave room on the SMs for
    // blocks of higher-priority kernels.  Multi-stripe warps index scratch rows by warp and stay
    // persistent.
    const unsigned int n_warps = gridDim.x * (blockDim.x / kWarp);
    const unsigned int cap = (!MULTI && pc.waves > 1) ? (pc.cd->n_items + n_warps - 1) / n_warps : 0xffffffffu;
    warp_items32<KH, V, PM, MULTI>(b, tb, pc, tab, lane, warp_id, cap);
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
