// api.cu -- extern "C" entry points of libptycho_b200 (see include/ptycho_b200.h).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "assemble.cuh"
#include "fused.cuh"
#include "general.cuh"

namespace pty {

struct WsLayout {
  size_t E, scr, part, loss, tlb, done, lpart, total;
};

// square 64, 128, 256: the fused kernels; every other M x N: the general path
static bool fused_probe(int M, int N) { return M == N && (M == 64 || M == 128 || M == 256); }

static WsLayout ws_layout(int M, int N, int B) {
  const size_t G = (size_t(B) + kGroup - 1) / kGroup;
  const size_t MN = size_t(M) * N;
  WsLayout L;
  size_t off = 0;
  L.E = off;
  off += pty_align_up(size_t(B) * MN * sizeof(float2), 256);
  L.scr = off;  // the general path's FD planes
  if (!fused_probe(M, N)) off += pty_align_up(size_t(B) * MN * 3 * sizeof(float), 256);
  L.part = off;  // dP group partials: the assembly's groups of kGroup, or the M = 256 path's of kDpGroup
  const size_t GP = (M == 256 && N == 256) ? std::max(G, (size_t(B) + kDpGroup - 1) / kDpGroup) : G;
  off += pty_align_up(GP * MN * sizeof(float2), 256);
  L.loss = off;
  off += pty_align_up(size_t(B) * sizeof(double), 256);
  L.tlb = off;
  off += pty_align_up(size_t(B) * sizeof(int2), 256);
  L.done = off;  // arrival counters of the dP reduction (self-resetting)
  off += pty_align_up(size_t(dp_counters(M, N)) * sizeof(unsigned), 256);
  L.lpart = off;  // M = 256 line-DFT path: FP64 loss partial per (pattern, column block)
  if (M == 256 && N == 256) off += pty_align_up(size_t(B) * kSplit256Blocks * sizeof(double), 256);
  L.total = off;
  return L;
}

static bool supported_probe(int M, int N) { return fused_probe(M, N) || general_supported(M, N); }

static int check_common(const float* O, int H, int W, const float* P, int M, int N, const int32_t* tl,
                        int F, const int32_t* batch, int B) {
  if (!O || !P || (B > 0 && !tl) || H <= 0 || W <= 0 || B < 0 || F < 0) return PTYCHO_ERR_INVALID_ARG;
  if (!batch && B > F) return PTYCHO_ERR_INVALID_ARG;
  if (!supported_probe(M, N)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (H < M || W < N) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(O, 8) || !pty_aligned(P, 8) || !pty_aligned(tl, 8) || !pty_aligned(batch, 4))
    return PTYCHO_ERR_MISALIGNED;
  return PTYCHO_OK;
}

static int launch_fused(int M, int mode, int loss, const FusedArgs& a, cudaStream_t s) {
  if (M == 64) return launch_fused_64(mode, loss, a, s);
  if (M == 128) return launch_fused_128(mode, loss, a, s);
  return launch_fused_256(mode, loss, a, s);
}

static FusedArgs make_args(const float* O, int H, int W, const float* P, const int32_t* tl,
                           const float* Imeas, int F, const int32_t* batch, int B, int32_t* status) {
  FusedArgs a{};
  a.O = reinterpret_cast<const float2*>(O);
  a.H = H;
  a.W = W;
  a.P = reinterpret_cast<const float2*>(P);
  a.tl = reinterpret_cast<const int2*>(tl);
  a.Imeas = Imeas;
  a.F = F;
  a.batch = batch;
  a.B = B;
  a.status = status;
  return a;
}

}  // namespace pty

using namespace pty;

extern "C" {

const char* ptycho_status_string(int status) {
  switch (status) {
    case PTYCHO_OK: return "ok";
    case PTYCHO_ERR_INVALID_ARG: return "invalid argument";
    case PTYCHO_ERR_UNSUPPORTED_SIZE: return "unsupported size";
    case PTYCHO_ERR_MISALIGNED: return "misaligned pointer";
    case PTYCHO_ERR_WORKSPACE: return "workspace too small";
    case PTYCHO_ERR_LAUNCH: return "CUDA launch failed";
    case PTYCHO_ERR_WINDOW: return "scan window outside the canvas";
    case PTYCHO_ERR_TIMEOUT: return "bounded wait timed out";
    default: return "unknown status";
  }
}

int ptycho_version(void) { return 200; }

int ptycho_forward_intensity(const float* O, int H, int W, const float* P, int M, int N,
                             const int32_t* tl, int F, const int32_t* batch, int B, float* I_out,
                             int32_t* status_out, ptycho_stream_t stream) {
  int st = check_common(O, H, W, P, M, N, tl, F, batch, B);
  if (st) return st;
  if (B == 0) return PTYCHO_OK;
  if (!I_out) return PTYCHO_ERR_INVALID_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  FusedArgs a = make_args(O, H, W, P, tl, nullptr, F, batch, B, status_out);
  a.I_out = I_out;
  if (fused_probe(M, N)) return launch_fused(M, MODE_INTENSITY, 0, a, s);
  return PTYCHO_ERR_UNSUPPORTED_SIZE;  // other shapes need scratch: ptycho_forward_intensity_ws
}

size_t ptycho_forward_intensity_workspace_size(int M, int N, int B) {
  if (B < 0 || !supported_probe(M, N)) return 0;
  if (fused_probe(M, N)) return 256;  // the fused kernels need none
  return pty_align_up(size_t(B) * M * N * sizeof(float2), 256);
}

int ptycho_forward_intensity_ws(const float* O, int H, int W, const float* P, int M, int N,
                                const int32_t* tl, int F, const int32_t* batch, int B, float* I_out,
                                void* workspace, size_t workspace_bytes, int32_t* status_out,
                                ptycho_stream_t stream) {
  int st = check_common(O, H, W, P, M, N, tl, F, batch, B);
  if (st) return st;
  if (B == 0) return PTYCHO_OK;
  if (!I_out) return PTYCHO_ERR_INVALID_ARG;
  if (fused_probe(M, N))
    return ptycho_forward_intensity(O, H, W, P, M, N, tl, F, batch, B, I_out, status_out, stream);
  if (!workspace || workspace_bytes < ptycho_forward_intensity_workspace_size(M, N, B)) return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(workspace, 256)) return PTYCHO_ERR_MISALIGNED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  FusedArgs a = make_args(O, H, W, P, tl, nullptr, F, batch, B, status_out);
  a.I_out = I_out;
  return general_forward_intensity(a, M, N, static_cast<float2*>(workspace), s);
}

size_t ptycho_fwd_adj_workspace_size(int H, int W, int M, int N, int B) {
  if (H <= 0 || W <= 0 || B < 0 || !supported_probe(M, N)) return 0;
  return ws_layout(M, N, B).total;
}

int ptycho_fwd_adj(const float* O, int H, int W, const float* P, int M, int N, const int32_t* tl,
                   const float* Imeas, int F, const int32_t* batch, int B, int loss_type,
                   double* loss_per_pattern, double* loss_total, float* dO, float* dP, unsigned flags,
                   void* workspace, size_t workspace_bytes, int32_t* status_out,
                   ptycho_stream_t stream) {
  int st = check_common(O, H, W, P, M, N, tl, F, batch, B);
  if (st) return st;
  if (loss_type < 0 || loss_type > 3) return PTYCHO_ERR_INVALID_ARG;
  if (B > 0 && !Imeas) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(Imeas, 16)) return PTYCHO_ERR_MISALIGNED;
  if ((dO && !pty_aligned(dO, 8)) || (dP && !pty_aligned(dP, 8))) return PTYCHO_ERR_MISALIGNED;
  const WsLayout L = ws_layout(M, N, B);
  if (!workspace || workspace_bytes < L.total) return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(workspace, 256)) return PTYCHO_ERR_MISALIGNED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const bool acc = (flags & PTYCHO_FLAG_ACCUMULATE) != 0;
  char* ws = static_cast<char*>(workspace);
  float2* Ews = reinterpret_cast<float2*>(ws + L.E);
  float2* part = reinterpret_cast<float2*>(ws + L.part);
  double* lp = loss_per_pattern ? loss_per_pattern : reinterpret_cast<double*>(ws + L.loss);
  int2* tlb = reinterpret_cast<int2*>(ws + L.tlb);
  unsigned* done = reinterpret_cast<unsigned*>(ws + L.done);

  if (B == 0) {  // empty batch: zero gradients and loss
    if (!acc) {
      if (dO) cudaMemsetAsync(dO, 0, size_t(H) * W * sizeof(float2), s);
      if (dP) cudaMemsetAsync(dP, 0, size_t(M) * N * sizeof(float2), s);
    }
    if (loss_total) cudaMemsetAsync(loss_total, 0, sizeof(double), s);
    return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
  }
  FusedArgs a = make_args(O, H, W, P, tl, Imeas, F, batch, B, status_out);
  a.loss_pat = lp;
  const bool adj = dO || dP;
  const bool fused = fused_probe(M, N);
  const int mode = adj ? MODE_ADJ : MODE_LOSS;
  if (fused && M == 256 && split256_supported(mode, loss_type)) {
    // the line-DFT kernels use E' as their scratch in both modes; on large
    // batches the probe gradient comes out of the inverse-row kernel
    a.Eout = Ews;
    a.tlb = tlb;
    if (adj) {
      a.done = done;
      a.ndone = dp_counters(M, N);
    }
    const bool dp_fused = adj && dP && B >= kDpFuseMinB;
    st = launch_split256(mode, loss_type, a, reinterpret_cast<double*>(ws + L.lpart), dp_fused ? part : nullptr, s);
    if (st) return st;
    if (dp_fused) {
      st = launch_assemble(Ews, reinterpret_cast<const float2*>(O), reinterpret_cast<const float2*>(P), tlb, B, H,
                           W, M, N, true, reinterpret_cast<float2*>(dO), nullptr, part, done, lp, nullptr, acc, s);
      if (st) return st;
      return split256_dp_sum(part, B, reinterpret_cast<float2*>(dP), acc, lp, loss_total, s);
    }
  } else if (fused) {
    if (adj) {
      a.Eout = Ews;
      a.tlb = tlb;
      a.done = done;
      a.ndone = dp_counters(M, N);
    }
    st = launch_fused(M, mode, loss_type, a, s);
  } else {
    // the arrival counters start at zero: the fused kernel zeroes them, here a memset
    if (adj && cudaMemsetAsync(done, 0, size_t(dp_counters(M, N)) * sizeof(unsigned), s) != cudaSuccess)
      return PTYCHO_ERR_LAUNCH;
    st = general_fwd_adj(a, M, N, loss_type, adj, Ews, reinterpret_cast<float*>(ws + L.scr), tlb, s);
  }
  if (st) return st;
  return launch_assemble(Ews, reinterpret_cast<const float2*>(O), reinterpret_cast<const float2*>(P), tlb, B, H,
                         W, M, N, fused, reinterpret_cast<float2*>(dO), reinterpret_cast<float2*>(dP), part, done,
                         lp, loss_total, acc, s);
}

}  // extern "C"
