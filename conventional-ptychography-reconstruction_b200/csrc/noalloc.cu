// noalloc.cu -- ptycho_fwd_adj for callers that cannot allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc at the point where they
// run the forward/adjoint: an FFI runtime (Go, Java, a real-time control
// loop) that owns no CUDA allocator, a process whose device memory is handed
// out by another framework's pool that it cannot reach, or a step that must
// not trigger the implicit device synchronisation of a fresh allocation.
// ptycho_fwd_adj_noalloc gives them the same computation with its scratch in
// a fixed array that lives in the library itself:
//
//   * the array is a file-scope static __device__ buffer of kNoAllocScratchBytes
//     (48 MiB); every GPU that loads this library holds it until the process
//     exits;
//   * a call whose scratch need (ptycho_fwd_adj_workspace_size) exceeds it is
//     rejected with PTYCHO_ERR_WORKSPACE before any device work;
//   * the array's device address is looked up with cudaGetSymbolAddress on
//     every call, in the caller's current context: a __device__ symbol's
//     address belongs to a CUDA context, so a cached address could point into
//     memory of a context that was reset or is not current.  The first call in
//     a context may load the library's module there; make that first call
//     before any stream capture;
//   * arguments the workspace entry point would refuse (sizes, probe shape)
//     are refused with the same status before the address is looked up;
//   * all calls share the one array and it keeps the last call's contents:
//     the arrival counters that must start at zero are cleared by the fused
//     kernel of each call, everything else is written before it is read.
//     Calls that overlap on the GPU (different streams, or other host threads)
//     race on the array; order them on one stream.
// The entry point allocates nothing itself and calls no allocating routine.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ptycho_b200.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(48) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// device address of the scratch array in the current context
int scratch_for_current_context(void** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PTYCHO_ERR_LAUNCH;
  *out = p;
  return PTYCHO_OK;
}

}  // namespace

extern "C" int ptycho_fwd_adj_noalloc(const float* O, int H, int W, const float* P, int M, int N,
                                      const int32_t* tl, const float* Imeas, int F,
                                      const int32_t* batch, int B, int loss_type,
                                      double* loss_per_pattern, double* loss_total, float* dO,
                                      float* dP, unsigned flags, int32_t* status_out,
                                      ptycho_stream_t stream) {
  const size_t need = ptycho_fwd_adj_workspace_size(H, W, M, N, B);
  if (need == 0)  // sizes or probe shape the workspace entry point refuses: its own status, no device work
    return ptycho_fwd_adj(O, H, W, P, M, N, tl, Imeas, F, batch, B, loss_type, loss_per_pattern,
                          loss_total, dO, dP, flags, nullptr, 0, status_out, stream);
  if (need > kNoAllocScratchBytes) return PTYCHO_ERR_WORKSPACE;
  void* scratch = nullptr;
  const int st = scratch_for_current_context(&scratch);
  if (st) return st;
  return ptycho_fwd_adj(O, H, W, P, M, N, tl, Imeas, F, batch, B, loss_type, loss_per_pattern,
                        loss_total, dO, dP, flags, scratch, kNoAllocScratchBytes, status_out, stream);
}
