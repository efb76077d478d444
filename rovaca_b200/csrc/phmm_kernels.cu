// PairHMM kernels for sm_100a: haplotype code preparation, the persistent FP64 recompute pass, the
// FMA throughput probes and the launch wrappers of every class.  Device arithmetic lives in
// phmm_device.cuh (scalar) and phmm_device2.cuh (packed FP32); the FP32 class kernels are in
// phmm_fwd32.cuh, instantiated per mode in phmm_fwd32_m0/m1/m2.cu.
//
// Every kernel class (precision, rows per lane, variant, FP32 gap-parameter mode, stripe mode) is
// its own kernel, so each gets the register allocation its own live state needs instead of the
// union of all paths.  Work items are grouped by class on the host.
#include <cuda_runtime.h>

#include "phmm_fwd32.cuh"
#include "phmm_warp64.cuh"
#include "phmm_kernels.h"

namespace phmm {

// ------------------------------------------------------------------------------------------
// Haplotype bytes -> per-variant match codes (grid-stride).
// ------------------------------------------------------------------------------------------
__global__ void prep_codes_kernel(const BatchDesc* __restrict__ desc, const uint8_t* __restrict__ hap_bases,
                                  uint32_t* __restrict__ codes_inter, uint32_t* __restrict__ codes_intra)
{
    const uint64_t total = desc->hap_bases_total;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const uint8_t b = hap_bases[i];
        codes_inter[kCodePad + i] = hap_code(b, kInter);
        codes_intra[kCodePad + i] = hap_code(b, kIntra);
    }
    // guard codes on both sides of the stream: match nothing
    if (blockIdx.x == 0) {
        for (int k = threadIdx.x; k < kCodePad; k += blockDim.x) {
            codes_inter[k] = 0u;
            codes_intra[k] = 0u;
            codes_inter[kCodePad + total + k] = 0u;
            codes_intra[kCodePad + total + k] = 0u;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Output reset: every likelihood NaN (pairs with an empty read or haplotype stay NaN), flags 0.
// ------------------------------------------------------------------------------------------
__global__ void reset_outputs_kernel(const BatchDesc* __restrict__ desc, double* __restrict__ out,
                                     uint8_t* __restrict__ flags)
{
    const uint64_t total = desc->out_total;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        out[i] = nan;
        if (flags) flags[i] = 0;
    }
}

// ------------------------------------------------------------------------------------------
// FP64 pass for one class over the runs of underflowed pairs the FP32 pass appended, one run per
// claim, streamed through the read like an FP32 work item.
// ------------------------------------------------------------------------------------------
// Resident warps per SM of the FP64 classes of mode 0 (constant gaps, insertion = deletion), the
// compiler's register bound: 8 rows per lane at 12 warps (168 registers, no spills), 7 rows at 16
// (128 registers, 48 bytes of spill loads).  Measured on B200 with the two-value lane state: 8 rows
// at 12 warps ran the underflow-stress shape's FP64 pass in 43.7 ms against 44.9 at 16, and the
// benchmark batch's 8-row class in 8.8 against 9.1 ms; 7 rows ran 5.1 ms at 16 against 5.3 at 12.
// The other classes keep what they need.  Build-time settings.
#ifndef PHMM_F64_MIN_WARPS_K8
#define PHMM_F64_MIN_WARPS_K8 12
#endif
#ifndef PHMM_F64_MIN_WARPS_K7
#define PHMM_F64_MIN_WARPS_K7 16
#endif
template <int K, int PM>
constexpr int min_blocks64()
{
    return PM != PM_EQ ? 1 : K == 8 ? PHMM_F64_MIN_WARPS_K8 : K == 7 ? PHMM_F64_MIN_WARPS_K7 : 1;
}

// UNF: the all-FP64 check arithmetic (plain multiply and add), used to measure the error of every
// likelihood; the recompute pass proper uses the reference's contracted arithmetic.
template <int K, int V, int PM, bool MULTI, bool UNF = false>
__global__ void __launch_bounds__(kFwdBlock, min_blocks64<K, PM>()) fwd_f64_kernel(BatchView b, ProbTables<double> tb, PassControl pc)
{
    __shared__ double tab[prior_table_size<K>()];
    const int lane = threadIdx.x & (kWarp - 1);
    const unsigned int warp_id = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    warp_reruns64<K, V, PM, MULTI, UNF>(b, tb, pc, tab, lane, warp_id);
}

// ------------------------------------------------------------------------------------------
// FP32 FMA throughput probe: 16 independent FMA chains per thread on every SM.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) fma_peak_kernel(float* sink, int iters, float a, float b)
{
    float x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = (float)(threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = __fmaf_rn(x[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += x[k];
    if (s == -1.0f) sink[blockIdx.x] = s;  // never true; keeps the chains alive
}

// Same with packed FFMA2: 16 independent float2 chains (32 FMAs per thread per iteration).
__global__ void __launch_bounds__(256) fma2_peak_kernel(float* sink, int iters, float a, float b)
{
    float2 x[16];
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = make_float2((float)(threadIdx.x + k) * 1e-3f, (float)(threadIdx.x - k) * 1e-3f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = __ffma2_rn(x[k], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += x[k].x + x[k].y;
    if (s == -1.0f) sink[blockIdx.x] = s;
}

cudaError_t launch_fma_peak(float* sink, int blocks, int iters, bool packed, cudaStream_t st)
{
    if (packed)
        fma2_peak_kernel<<<blocks, 256, 0, st>>>(sink, iters, 0.999f, 1e-4f);
    else
        fma_peak_kernel<<<blocks, 256, 0, st>>>(sink, iters, 0.999f, 1e-4f);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// Class tables and host-side launch wrappers.
// ------------------------------------------------------------------------------------------
typedef void (*F64Kernel)(BatchView, ProbTables<double>, PassControl);

#define PHMM_ROW64(V, PM)                                                                                 \
    fwd_f64_kernel<1, V, PM, false>, fwd_f64_kernel<2, V, PM, false>, fwd_f64_kernel<3, V, PM, false>,    \
        fwd_f64_kernel<4, V, PM, false>, fwd_f64_kernel<5, V, PM, false>, fwd_f64_kernel<6, V, PM, false>, \
        fwd_f64_kernel<7, V, PM, false>, fwd_f64_kernel<8, V, PM, false>, fwd_f64_kernel<8, V, PM, true>

static const F64Kernel kF64[kClasses64] = {PHMM_ROW64(kInter, PM_EQ), PHMM_ROW64(kInter, PM_ROW),
                                           PHMM_ROW64(kIntra, PM_ROW)};

// All-FP64 check kernels: the same shapes with plain multiply/add, per-row gap parameters (any
// read), inter and intra variants (FP64 classes of modes 1 and 2).
#define PHMM_ROW64_CHECK(V)                                                                               \
    fwd_f64_kernel<1, V, PM_ROW, false, true>, fwd_f64_kernel<2, V, PM_ROW, false, true>,                 \
        fwd_f64_kernel<3, V, PM_ROW, false, true>, fwd_f64_kernel<4, V, PM_ROW, false, true>,             \
        fwd_f64_kernel<5, V, PM_ROW, false, true>, fwd_f64_kernel<6, V, PM_ROW, false, true>,             \
        fwd_f64_kernel<7, V, PM_ROW, false, true>, fwd_f64_kernel<8, V, PM_ROW, false, true>,             \
        fwd_f64_kernel<8, V, PM_ROW, true, true>
static const F64Kernel kF64Check[2 * 9] = {PHMM_ROW64_CHECK(kInter), PHMM_ROW64_CHECK(kIntra)};

cudaError_t launch_prep(const BatchDesc* desc, const uint8_t* hap_bases, uint32_t* codes_inter, uint32_t* codes_intra,
                        double* out, uint8_t* flags, int num_sms, cudaStream_t st)
{
    const int threads = 256;
    reset_outputs_kernel<<<num_sms * 4, threads, 0, st>>>(desc, out, flags);
    prep_codes_kernel<<<num_sms * 4, threads, 0, st>>>(desc, hap_bases, codes_inter, codes_intra);
    return cudaGetLastError();
}

cudaError_t launch_fwd(int precision, int cls, const BatchView& b, const ProbTables<float>& tf,
                       const ProbTables<double>& td, const PassControl& pc, int grid, cudaStream_t st)
{
    if (cls < 0 || cls >= (precision == 32 ? kClasses32 : kClasses64) || grid <= 0) return cudaErrorInvalidValue;
    if (precision == 32) {
        const int mode = cls / kShapes32, shape = cls % kShapes32;
        if (mode == 0) return launch_f32_mode0(shape, b, tf, pc, grid, st);
        if (mode == 1) return launch_f32_mode1(shape, b, tf, pc, grid, st);
        return launch_f32_mode2(shape, b, tf, pc, grid, st);
    }
    kF64[cls]<<<grid, kFwdBlock, 0, st>>>(b, td, pc);
    return cudaGetLastError();
}

cudaError_t launch_f64_check(int cls, const BatchView& b, const ProbTables<double>& td, const PassControl& pc, int grid,
                             cudaStream_t st)
{
    if (cls < 9 || cls >= kClasses64 || grid <= 0) return cudaErrorInvalidValue;
    kF64Check[cls - 9]<<<grid, kFwdBlock, 0, st>>>(b, td, pc);
    return cudaGetLastError();
}

cudaError_t occupancy_f64_check(int cls, int* blocks_per_sm)
{
    if (cls < 9 || cls >= kClasses64) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kF64Check[cls - 9], kFwdBlock, 0);
}

cudaError_t occupancy(int precision, int cls, int* blocks_per_sm)
{
    if (cls < 0 || cls >= (precision == 32 ? kClasses32 : kClasses64)) return cudaErrorInvalidValue;
    if (precision == 32) {
        const int mode = cls / kShapes32, shape = cls % kShapes32;
        if (mode == 0) return occupancy_f32_mode0(shape, blocks_per_sm);
        if (mode == 1) return occupancy_f32_mode1(shape, blocks_per_sm);
        return occupancy_f32_mode2(shape, blocks_per_sm);
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kF64[cls], kFwdBlock, 0);
}

}  // namespace phmm
