// FP32 wavefront kernels of mode 0: inter pairs whose read has constant gap qualities with equal
// insertion and deletion qualities.
#include "phmm_fwd32.cuh"

namespace phmm {

PHMM_DEFINE_MODE32(0, kInter, PM_EQ)

}  // namespace phmm
