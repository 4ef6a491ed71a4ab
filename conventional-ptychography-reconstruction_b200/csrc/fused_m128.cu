// fused_m128.cu -- instantiations of the fused kernel for 128 x 128 probes.
#include "fused.cuh"

namespace pty {
int launch_fused_128(int mode, int loss, const FusedArgs& a, cudaStream_t s) {
  return launch_fused_m<128>(mode, loss, a, s);
}
}  // namespace pty
