// Split-BF16 tcgen05 engine of the global repetition map (under construction).
#include "common.cuh"

namespace sred {

cudaError_t launch_gram_tc(const __nv_bfloat16*, const __nv_bfloat16*, int, int, const BlockParams*, const float*,
                           EpiConsts, double*, double*, int, int*, cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace sred
