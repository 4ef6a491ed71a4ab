// haar.cu -- Haar-wavelet sparsity of the object and its gradient; object error
// against ground truth after global-phase alignment (FP64).
//
// Replaces haar_wavelet_sparsity_loss (utils/loss.py:60-83), added to the
// loss at Recovery.py:309-313 when sparsity_weight != 0: with the 2x2 blocks
// a = img[0::2, 0::2], b = img[0::2, 1::2], c = img[1::2, 0::2],
// d = img[1::2, 1::2], the loss is the L1 norm of the three detail subbands
//   |a - b + c - d| + |a + b - c - d| + |a - b - c + d|,
// summed over the blocks and over the real and imaginary parts.
// Forward: k_haar_part sums a fixed range of blocks per thread (FP32 terms,
// FP64 accumulation), then a fixed shuffle tree per CTA -> partial[CTA];
// k_haar_final sums the partials in CTA order.  Deterministic.
// Backward (torch's convention, abs' = sign with sign(0) = 0): per block and
// part, with s_i = sign(t_i): da = s1+s2+s3, db = -s1+s2-s3, dc = s1-s2-s3,
// dd = -s1-s2+s3, times the upstream gradient read from device memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace pty {
namespace hr {

constexpr int NT = 256, PER = 1, MAXG = 1184;  // one 2x2 block per thread: enough warps to cover latency

PTY_DEVI float sgnf(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

__global__ void __launch_bounds__(NT) k_haar_part(const float2* __restrict__ img, int H, int W,
                                                  double* __restrict__ part) {
  __shared__ double red[NT / 32];
  const int bw = W / 2, nb = (H / 2) * bw;
  double s = 0.0;
  for (int q = blockIdx.x * NT + threadIdx.x; q < nb; q += gridDim.x * NT) {
    const int by = q / bw, bx = q - by * bw;
    const float2* r0 = img + size_t(2 * by) * W + 2 * bx;
    const float2 a = __ldg(r0), b = __ldg(r0 + 1), c = __ldg(r0 + W), d = __ldg(r0 + W + 1);
    const float t = fabsf(a.x - b.x + c.x - d.x) + fabsf(a.x + b.x - c.x - d.x) + fabsf(a.x - b.x - c.x + d.x);
    const float u = fabsf(a.y - b.y + c.y - d.y) + fabsf(a.y + b.y - c.y - d.y) + fabsf(a.y - b.y - c.y + d.y);
    s += double(t) + double(u);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) t += red[i];
    part[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(32) k_haar_final(const double* __restrict__ part, int G, double* __restrict__ out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < G; i += 32) s += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) out[0] = s;
}

__global__ void __launch_bounds__(NT) k_haar_bwd(const float2* __restrict__ img, int H, int W,
                                                 const double* __restrict__ gscale, float2* __restrict__ gimg) {
  const int bw = W / 2, nb = (H / 2) * bw;
  const float g = float(gscale[0]);
  for (int q = blockIdx.x * NT + threadIdx.x; q < nb; q += gridDim.x * NT) {
    const int by = q / bw, bx = q - by * bw;
    const size_t o = size_t(2 * by) * W + 2 * bx;
    const float2 a = __ldg(img + o), b = __ldg(img + o + 1), c = __ldg(img + o + W), d = __ldg(img + o + W + 1);
    const float p1 = sgnf(a.x - b.x + c.x - d.x), p2 = sgnf(a.x + b.x - c.x - d.x), p3 = sgnf(a.x - b.x - c.x + d.x);
    const float q1 = sgnf(a.y - b.y + c.y - d.y), q2 = sgnf(a.y + b.y - c.y - d.y), q3 = sgnf(a.y - b.y - c.y + d.y);
    gimg[o] = make_float2(g * (p1 + p2 + p3), g * (q1 + q2 + q3));
    gimg[o + 1] = make_float2(g * (-p1 + p2 - p3), g * (-q1 + q2 - q3));
    gimg[o + W] = make_float2(g * (p1 - p2 - p3), g * (q1 - q2 - q3));
    gimg[o + W + 1] = make_float2(g * (-p1 - p2 + p3), g * (-q1 - q2 + q3));
  }
}

inline int grid_for(int H, int W) {
  const int nb = (H / 2) * (W / 2);
  const int g = (nb + NT * PER - 1) / (NT * PER);
  return g < 1 ? 1 : (g < MAXG ? g : MAXG);
}

}  // namespace hr
}  // namespace pty

using namespace pty;

extern "C" {

size_t ptycho_haar_sparsity_workspace_size(int H, int W) {
  if (H <= 0 || W <= 0) return 0;
  return size_t(hr::grid_for(H, W)) * sizeof(double);
}

int ptycho_haar_sparsity(const float* img, int H, int W, double* loss_out, void* workspace,
                         size_t workspace_bytes, ptycho_stream_t stream) {
  if (!img || !loss_out || H <= 0 || W <= 0) return PTYCHO_ERR_INVALID_ARG;
  if ((H & 1) || (W & 1)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (!workspace || workspace_bytes < ptycho_haar_sparsity_workspace_size(H, W)) return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(img, 8) || !pty_aligned(loss_out, 8) || !pty_aligned(workspace, 8)) return PTYCHO_ERR_MISALIGNED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int G = hr::grid_for(H, W);
  double* part = static_cast<double*>(workspace);
  hr::k_haar_part<<<G, hr::NT, 0, s>>>(reinterpret_cast<const float2*>(img), H, W, part);
  hr::k_haar_final<<<1, 32, 0, s>>>(part, G, loss_out);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_haar_sparsity_backward(const float* img, int H, int W, const double* grad_loss, float* grad_img,
                                  ptycho_stream_t stream) {
  if (!img || !grad_loss || !grad_img || H <= 0 || W <= 0) return PTYCHO_ERR_INVALID_ARG;
  if ((H & 1) || (W & 1)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (!pty_aligned(img, 8) || !pty_aligned(grad_loss, 8) || !pty_aligned(grad_img, 8)) return PTYCHO_ERR_MISALIGNED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  hr::k_haar_bwd<<<hr::grid_for(H, W), hr::NT, 0, s>>>(reinterpret_cast<const float2*>(img), H, W, grad_loss,
                                                        reinterpret_cast<float2*>(grad_img));
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // extern "C"

// ---- object error after global-phase alignment (FP64) ----------------------
// Over the box [y0, y1) x [x0, x1) of recon R and ground truth T (both [H][W]
// complex64): c = sum conj(R) T, nR = sum |R|^2, nT = sum |T|^2 in FP64 (fixed
// per-thread ranges, per-CTA trees, CTA-order sum).  The phase exp(i a) with
// a = arg(c) minimises ||R e^{ia} - T|| (resolve_global_phase,
// scripts/compare_object_ssim.py:92-98), and then
//   NRMSE = sqrt((nR + nT - 2 |c|) / nT).
// With the least-squares complex factor g = c / nR (phase and the probe/object
// scale ambiguity both removed), ||g R - T||^2 / nT = 1 - |c|^2 / (nR nT).
// out[0] = NRMSE, out[1], out[2] = cos a, sin a, out[3] = |c|, out[4] = nR,
// out[5] = nT, out[6] = sqrt(1 - |c|^2 / (nR nT)).
namespace pty {
namespace oe {

constexpr int NT = 256, MAXG = 1184;

__global__ void __launch_bounds__(NT) k_obj_err_part(const float2* __restrict__ R, const float2* __restrict__ T,
                                                     int W, int y0, int y1, int x0, int x1,
                                                     double* __restrict__ part) {
  __shared__ double red[4][NT / 32];
  const int bw = x1 - x0;
  const long long n = (long long)(y1 - y0) * bw;
  double cr = 0.0, ci = 0.0, nr = 0.0, nt = 0.0;
  for (long long q = (long long)blockIdx.x * NT + threadIdx.x; q < n; q += (long long)gridDim.x * NT) {
    const int y = y0 + int(q / bw), x = x0 + int(q % bw);
    const float2 r = __ldg(R + size_t(y) * W + x), t = __ldg(T + size_t(y) * W + x);
    cr += double(r.x) * t.x + double(r.y) * t.y;  // Re(conj(r) t)
    ci += double(r.x) * t.y - double(r.y) * t.x;  // Im(conj(r) t)
    nr += double(r.x) * r.x + double(r.y) * r.y;
    nt += double(t.x) * t.x + double(t.y) * t.y;
  }
  double v[4] = {cr, ci, nr, nt};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0.0;
    for (int i = 0; i < NT / 32; ++i) s += red[threadIdx.x][i];
    part[blockIdx.x * 4 + threadIdx.x] = s;
  }
}

__global__ void __launch_bounds__(32) k_obj_err_final(const double* __restrict__ part, int G, double* __restrict__ out) {
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < G; i += 32)
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] += part[i * 4 + k];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if (threadIdx.x == 0) {
    const double mag = sqrt(v[0] * v[0] + v[1] * v[1]);
    const double nt = v[3];
    out[0] = nt > 0.0 ? sqrt(fmax(v[2] + nt - 2.0 * mag, 0.0) / nt) : 0.0;
    out[1] = mag > 0.0 ? v[0] / mag : 1.0;
    out[2] = mag > 0.0 ? v[1] / mag : 0.0;
    out[3] = mag;
    out[4] = v[2];
    out[5] = nt;
    out[6] = (v[2] > 0.0 && nt > 0.0) ? sqrt(fmax(1.0 - (mag / v[2]) * (mag / nt), 0.0)) : 1.0;
  }
}

inline int grid_for(long long n) {
  const long long g = (n + NT * 2 - 1) / (NT * 2);
  return g < 1 ? 1 : (g > MAXG ? MAXG : int(g));
}

}  // namespace oe
}  // namespace pty

extern "C" {

size_t ptycho_object_error_workspace_size(void) { return size_t(pty::oe::MAXG) * 4 * sizeof(double); }

int ptycho_object_error(const float* recon, const float* truth, int H, int W, int y0, int y1, int x0, int x1,
                        double* out, void* workspace, size_t workspace_bytes, ptycho_stream_t stream) {
  if (!recon || !truth || !out || H <= 0 || W <= 0) return PTYCHO_ERR_INVALID_ARG;
  if (y0 < 0 || x0 < 0 || y1 > H || x1 > W || y0 >= y1 || x0 >= x1) return PTYCHO_ERR_INVALID_ARG;
  if (!workspace || workspace_bytes < ptycho_object_error_workspace_size()) return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(recon, 8) || !pty_aligned(truth, 8) || !pty_aligned(out, 8) || !pty_aligned(workspace, 8))
    return PTYCHO_ERR_MISALIGNED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int G = pty::oe::grid_for((long long)(y1 - y0) * (x1 - x0));
  double* part = static_cast<double*>(workspace);
  pty::oe::k_obj_err_part<<<G, pty::oe::NT, 0, s>>>(reinterpret_cast<const float2*>(recon),
                                                    reinterpret_cast<const float2*>(truth), W, y0, y1, x0, x1, part);
  pty::oe::k_obj_err_final<<<1, 32, 0, s>>>(part, G, out);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // extern "C"
