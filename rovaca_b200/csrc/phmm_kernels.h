// Launch wrappers for the PairHMM kernels (definitions in phmm_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "phmm_types.h"

namespace phmm {

// Threads per block of the persistent wavefront kernels: one warp, so that resident warps are
// limited by the register file at warp granularity (kernels with 170-250 registers per thread fit
// 10-11 warps per SM instead of the 8 that four-warp blocks allow).
constexpr int kFwdBlock = 32;

// Kernel classes: see class32 / class64 in phmm_types.h.
constexpr int kNumClasses = kClasses32 + kClasses64;  // descriptor slots: FP32 classes, then FP64

// NaN-fills the output, zeroes the pair flags and builds the per-variant haplotype match codes,
// with every size read from the device-side batch descriptor.
cudaError_t launch_prep(const BatchDesc* desc, const uint8_t* hap_bases, uint32_t* codes_inter, uint32_t* codes_intra,
                        double* out, uint8_t* flags, int num_sms, cudaStream_t st);
// precision 32: FP32 pass of class `cls` (0..kClasses32-1) over its work items; precision 64: FP64
// pass of class `cls` (0..kClasses64-1) over its rerun segment.
cudaError_t launch_fwd(int precision, int cls, const BatchView& b, const ProbTables<float>& tf,
                       const ProbTables<double>& td, const PassControl& pc, int grid, cudaStream_t st);
cudaError_t occupancy(int precision, int cls, int* blocks_per_sm);
// All-FP64 check pass of FP64 class `cls` (9..kClasses64-1: modes 1 and 2, any read) over its rerun
// segment, with plain multiply/add instead of the reference's contracted arithmetic.
cudaError_t launch_f64_check(int cls, const BatchView& b, const ProbTables<double>& td, const PassControl& pc, int grid,
                             cudaStream_t st);
cudaError_t occupancy_f64_check(int cls, int* blocks_per_sm);
// 256-thread blocks, each thread running 16 independent FMA chains (scalar FFMA, or packed FFMA2
// with two FMAs per instruction) for iters steps.
cudaError_t launch_fma_peak(float* sink, int blocks, int iters, bool packed, cudaStream_t st);

}  // namespace phmm
