// FP32 wavefront kernels of mode 1: inter pairs with per-row gap qualities.
#include "phmm_fwd32.cuh"

namespace phmm {

PHMM_DEFINE_MODE32(1, kInter, PM_ROW)

}  // namespace phmm
