// Launch wrappers for the PairHMM kernels (definitions in phmm_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "phmm_types.h"

namespace phmm {

constexpr int kFwdBlock = 128;  // threads per block of the persistent wavefront kernels

// Kernel classes: index = variant * 9 + (multi-stripe ? 8 : K - 1), K = rows per lane.
constexpr int kClassesPerVariant = 9;
constexpr int kNumClasses = 2 * kClassesPerVariant;
inline int class_index(int variant, int k, bool multi) { return variant * kClassesPerVariant + (multi ? 8 : k - 1); }
inline int class_k(int cls) { return (cls % kClassesPerVariant) == 8 ? kMaxK : (cls % kClassesPerVariant) + 1; }
inline bool class_multi(int cls) { return (cls % kClassesPerVariant) == 8; }
inline int class_variant(int cls) { return cls / kClassesPerVariant; }

// NaN-fills the output, zeroes the pair flags and builds the per-variant haplotype match codes,
// with every size read from the device-side batch descriptor.
cudaError_t launch_prep(const BatchDesc* desc, const uint8_t* hap_bases, uint32_t* codes_inter, uint32_t* codes_intra,
                        double* out, uint8_t* flags, int num_sms, cudaStream_t st);
// precision 32: FP32 pass over pc.items; precision 64: FP64 pass over pc.rerun.
cudaError_t launch_fwd(int precision, int cls, const BatchView& b, const ProbTables<float>& tf,
                       const ProbTables<double>& td, const PassControl& pc, int grid, cudaStream_t st);
cudaError_t occupancy(int precision, int cls, int* blocks_per_sm);
// 256-thread blocks, each thread running 16 independent FMA chains for iters steps.
cudaError_t launch_fma_peak(float* sink, int blocks, int iters, cudaStream_t st);

}  // namespace phmm
