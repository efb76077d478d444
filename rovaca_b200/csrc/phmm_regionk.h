// Region-API device kernels (definitions in phmm_regionk.cu): read preparation before the FP32 pass
// and post-processing after the FP64 pass, both idle when no region of the batch uses the region API.
#pragma once

#include <cuda_runtime.h>

#include "phmm_types.h"

namespace phmm {

cudaError_t launch_read_prep(const RegionApiView& v, int num_sms, cudaStream_t st);
cudaError_t launch_post_region(const RegionApiView& v, int num_sms, cudaStream_t st);
// After launch_post_region: allele likelihoods, diploid genotype likelihoods and calls per event.
cudaError_t launch_genotype(const RegionApiView& v, int num_sms, cudaStream_t st);

}  // namespace phmm
