// fused_m64.cu -- instantiations of the fused kernel for 64 x 64 probes.
#include "fused.cuh"

namespace pty {
int launch_fused_64(int mode, int loss, const FusedArgs& a, cudaStream_t s) {
  return launch_fused_m<64>(mode, loss, a, s);
}
}  // namespace pty
