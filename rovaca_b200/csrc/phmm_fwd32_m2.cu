// FP32 wavefront kernels of mode 2: intra pairs (read or haplotype with 'N').
#include "phmm_fwd32.cuh"

namespace phmm {

PHMM_DEFINE_MODE32(2, kIntra, PM_ROW)

}  // namespace phmm
