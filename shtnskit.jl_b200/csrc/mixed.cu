// mixed.cu — mixed-precision (tensor core) Legendre path.
#include "kernels.cuh"

namespace shtb {

int mixed_synthesis(const shtb_plan*, const void*, void*, int, int, void*, cudaStream_t) {
  return set_error(SHTB_ERR_UNSUPPORTED, "mixed precision path not built yet");
}
int mixed_analysis(const shtb_plan*, const void*, void*, int, int, void*, cudaStream_t) {
  return set_error(SHTB_ERR_UNSUPPORTED, "mixed precision path not built yet");
}

}  // namespace shtb
