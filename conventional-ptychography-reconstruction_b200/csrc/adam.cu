// adam.cu -- fused multi-tensor Adam step (torch.optim.Adam semantics).
//
// Replaces optimizer.step() of Recovery.py:321 (Adam built at :238-241) for
// float32 parameter tensors; complex parameters are passed as their real
// view, so real and imaginary parts get independent moments exactly as
// torch.optim.Adam treats complex tensors.  Per element, with t = step:
//   m = m + (1 - b1) (g - m);  v = b2 v + (1 - b2) g^2
//   p = p - (lr / (1 - b1^t)) * m / (sqrt(v) / sqrt(1 - b2^t) + eps)
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "common.cuh"

namespace pty {

constexpr int kAdamMaxTensors = 48;

struct AdamList {
  float* p[kAdamMaxTensors];
  const float* g[kAdamMaxTensors];
  float* m[kAdamMaxTensors];
  float* v[kAdamMaxTensors];
  long long end[kAdamMaxTensors];  // cumulative element counts
  int blk_end[kAdamMaxTensors];    // cumulative block counts (chunked launch)
  int vec[kAdamMaxTensors];        // p, g, m, v all 16-byte aligned
  int n;
};

constexpr int kAdamChunk = 256 * 4;  // elements per block of the chunked launch

// one element of the update (the expressions of both launch forms)
PTY_DEVI void adam_elem(float g, float& m, float& v, float& p, float lr_bc1, float b1, float b2,
                        float inv_sqrt_bc2, float eps) {
  m = fmaf(1.0f - b1, g - m, m);
  v = fmaf(1.0f - b2, g * g, b2 * v);
  const float denom = sqrtf(v) * inv_sqrt_bc2 + eps;
  p -= lr_bc1 * (m / denom);
}

__global__ void __launch_bounds__(256) k_adam(const AdamList L, long long total, float lr_bc1, float b1, float b2,
                                              float inv_sqrt_bc2, float eps) {
  for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < total; i += (long long)gridDim.x * 256) {
    int k = 0;
    while (L.end[k] <= i) ++k;
    const long long j = i - (k ? L.end[k - 1] : 0);
    const float g = L.g[k][j];
    float m = L.m[k][j], v = L.v[k][j];
    m = fmaf(1.0f - b1, g - m, m);
    v = fmaf(1.0f - b2, g * g, b2 * v);
    const float denom = sqrtf(v) * inv_sqrt_bc2 + eps;
    L.p[k][j] -= lr_bc1 * (m / denom);
    L.m[k][j] = m;
    L.v[k][j] = v;
  }
}

// capturable form: step counter and learning rate live in device memory, so a
// CUDA graph that replays the step stays correct; k_adam_tick advances the
// counter, every block derives the bias corrections from it
__global__ void k_adam_tick(int* step) { step[0] += 1; }

// capturable step, chunked: block b owns elements [1024 c, 1024 c + 1024) of one
// tensor (found once per block from the cumulative block counts), four per
// thread with 16-byte accesses where the tensor allows; the per-element
// arithmetic is adam_elem, so results equal the element-wise form bitwise.
__global__ void __launch_bounds__(256) k_adam_dev_chunked(const AdamList L, const int* __restrict__ step,
                                                          const float* __restrict__ lr, float b1, float b2,
                                                          float eps) {
  __shared__ float sc[2];
  if (threadIdx.x == 0) {
    const double t = (double)step[0];
    const double bc1 = 1.0 - pow((double)b1, t), bc2 = 1.0 - pow((double)b2, t);
    sc[0] = (float)((double)lr[0] / bc1);
    sc[1] = (float)(1.0 / sqrt(bc2));
  }
  __syncthreads();
  const float lr_bc1 = sc[0], inv_sqrt_bc2 = sc[1];
  const int b = blockIdx.x;
  int k = 0;
  while (k < L.n - 1 && L.blk_end[k] <= b) ++k;
  const long long base = k ? L.end[k - 1] : 0;
  const long long numel = L.end[k] - base;
  const long long j0 = (long long)(b - (k ? L.blk_end[k - 1] : 0)) * kAdamChunk + 4 * threadIdx.x;
  float* P = L.p[k];
  const float* G = L.g[k];
  float* Mv = L.m[k];
  float* V = L.v[k];
  if (L.vec[k] && j0 + 3 < numel) {
    const float4 g = *reinterpret_cast<const float4*>(G + j0);
    float4 m = *reinterpret_cast<const float4*>(Mv + j0), v = *reinterpret_cast<const float4*>(V + j0);
    float4 p = *reinterpret_cast<const float4*>(P + j0);
    adam_elem(g.x, m.x, v.x, p.x, lr_bc1, b1, b2, inv_sqrt_bc2, eps);
    adam_elem(g.y, m.y, v.y, p.y, lr_bc1, b1, b2, inv_sqrt_bc2, eps);
    adam_elem(g.z, m.z, v.z, p.z, lr_bc1, b1, b2, inv_sqrt_bc2, eps);
    adam_elem(g.w, m.w, v.w, p.w, lr_bc1, b1, b2, inv_sqrt_bc2, eps);
    *reinterpret_cast<float4*>(P + j0) = p;
    *reinterpret_cast<float4*>(Mv + j0) = m;
    *reinterpret_cast<float4*>(V + j0) = v;
  } else {
    for (int q = 0; q < 4; ++q) {
      const long long j = j0 + q;
      if (j < numel) {
        float m = Mv[j], v = V[j], p = P[j];
        adam_elem(G[j], m, v, p, lr_bc1, b1, b2, inv_sqrt_bc2, eps);
        P[j] = p;
        Mv[j] = m;
        V[j] = v;
      }
    }
  }
}

static int make_list(float* const* params, const float* const* grads, float* const* exp_avg,
                     float* const* exp_avg_sq, const long long* numels, int n_tensors, AdamList* L,
                     long long* total) {
  if (n_tensors < 0 || n_tensors > kAdamMaxTensors) return PTYCHO_ERR_INVALID_ARG;
  if (n_tensors > 0 && (!params || !grads || !exp_avg || !exp_avg_sq || !numels)) return PTYCHO_ERR_INVALID_ARG;
  *total = 0;
  for (int k = 0; k < n_tensors; ++k) {
    if (numels[k] < 0 || (numels[k] > 0 && (!params[k] || !grads[k] || !exp_avg[k] || !exp_avg_sq[k])))
      return PTYCHO_ERR_INVALID_ARG;
    L->p[k] = params[k];
    L->g[k] = grads[k];
    L->m[k] = exp_avg[k];
    L->v[k] = exp_avg_sq[k];
    *total += numels[k];
    L->end[k] = *total;
    const long long blocks = (numels[k] + kAdamChunk - 1) / kAdamChunk;
    const long long prev = k ? L->blk_end[k - 1] : 0;
    if (prev + blocks >= (1ll << 31)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
    L->blk_end[k] = int(prev + blocks);
    L->vec[k] = pty_aligned(params[k], 16) && pty_aligned(grads[k], 16) && pty_aligned(exp_avg[k], 16) &&
                pty_aligned(exp_avg_sq[k], 16);
  }
  L->n = n_tensors;
  return PTYCHO_OK;
}

}  // namespace pty

using namespace pty;

extern "C" int ptycho_adam_step_dev(float* const* params, const float* const* grads, float* const* exp_avg,
                                    float* const* exp_avg_sq, const long long* numels, int n_tensors,
                                    int32_t* step, const float* lr, float beta1, float beta2, float eps,
                                    ptycho_stream_t stream) {
  if (!step || !lr) return PTYCHO_ERR_INVALID_ARG;
  AdamList L{};
  long long total = 0;
  int st = make_list(params, grads, exp_avg, exp_avg_sq, numels, n_tensors, &L, &total);
  if (st) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  k_adam_tick<<<1, 1, 0, s>>>(step);
  if (total > 0 && L.blk_end[n_tensors - 1] > 0)
    k_adam_dev_chunked<<<L.blk_end[n_tensors - 1], 256, 0, s>>>(L, step, lr, beta1, beta2, eps);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

extern "C" int ptycho_adam_step(float* const* params, const float* const* grads, float* const* exp_avg,
                                float* const* exp_avg_sq, const long long* numels, int n_tensors, int step,
                                float lr, float beta1, float beta2, float eps, ptycho_stream_t stream) {
  if (n_tensors < 0 || n_tensors > kAdamMaxTensors || step < 1 || !(lr >= 0.f)) return PTYCHO_ERR_INVALID_ARG;
  if (n_tensors == 0) return PTYCHO_OK;
  if (!params || !grads || !exp_avg || !exp_avg_sq || !numels) return PTYCHO_ERR_INVALID_ARG;
  AdamList L{};
  long long total = 0;
  for (int k = 0; k < n_tensors; ++k) {
    if (numels[k] < 0 || (numels[k] > 0 && (!params[k] || !grads[k] || !exp_avg[k] || !exp_avg_sq[k])))
      return PTYCHO_ERR_INVALID_ARG;
    L.p[k] = params[k];
    L.g[k] = grads[k];
    L.m[k] = exp_avg[k];
    L.v[k] = exp_avg_sq[k];
    total += numels[k];
    L.end[k] = total;
  }
  L.n = n_tensors;
  if (total == 0) return PTYCHO_OK;
  const double bc1 = 1.0 - pow((double)beta1, (double)step);
  const double bc2 = 1.0 - pow((double)beta2, (double)step);
  const long long blocks = (total + 255) / 256;
  const int grid = (int)(blocks < 148 * 16 ? blocks : 148 * 16);
  k_adam<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(L, total, (float)(lr / bc1), beta1, beta2,
                                                                   (float)(1.0 / sqrt(bc2)), eps);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

// ---- chain rule through the fused loss: scaled copies of dO and dP --------
// The fused forward/adjoint produces dL/dO and dL/dP for a unit upstream
// gradient; autograd's backward multiplies both by the upstream scalar g
// (the FP64 loss's gradient, a device double).  One grid-stride launch covers both arrays (float4 where
// both pointers are 16-byte aligned), out of place so the saved gradients stay
// valid for a second backward.
namespace pty {
namespace gsc {

__global__ void __launch_bounds__(256) k_scale_pair(const float* __restrict__ a, float* __restrict__ ao, long long na,
                                                    const float* __restrict__ b, float* __restrict__ bo, long long nb,
                                                    const double* __restrict__ g, int vec_a, int vec_b) {
  const float s = float(__ldg(g));
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long qa = vec_a ? na / 4 : 0, qb = vec_b ? nb / 4 : 0;
  for (long long i = t0; i < qa; i += stride) {
    float4 v = __ldg(reinterpret_cast<const float4*>(a) + i);
    reinterpret_cast<float4*>(ao)[i] = make_float4(v.x * s, v.y * s, v.z * s, v.w * s);
  }
  for (long long i = 4 * qa + t0; i < na; i += stride) ao[i] = a[i] * s;
  for (long long i = t0; i < qb; i += stride) {
    float4 v = __ldg(reinterpret_cast<const float4*>(b) + i);
    reinterpret_cast<float4*>(bo)[i] = make_float4(v.x * s, v.y * s, v.z * s, v.w * s);
  }
  for (long long i = 4 * qb + t0; i < nb; i += stride) bo[i] = b[i] * s;
}

}  // namespace gsc
}  // namespace pty

extern "C" int ptycho_scale_pair(const float* a, float* a_out, long long na, const float* b, float* b_out,
                                 long long nb, const double* scale, ptycho_stream_t stream) {
  if (!scale || na < 0 || nb < 0 || (na > 0 && (!a || !a_out)) || (nb > 0 && (!b || !b_out)))
    return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(a, 4) || !pty_aligned(a_out, 4) || !pty_aligned(b, 4) || !pty_aligned(b_out, 4) ||
      !pty_aligned(scale, 8))
    return PTYCHO_ERR_MISALIGNED;
  if (na + nb == 0) return PTYCHO_OK;
  static PtyDevCache nsm_cache;
  int dev = 0;
  int nsm = nsm_cache.get(&dev);
  if (nsm == 0 && dev >= 0) {
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) nsm = 0;
    nsm_cache.put(dev, nsm > 0 ? nsm : 0);
  }
  if (nsm <= 0) nsm = 148;
  const long long work = (na + nb) / 4 + 1;
  const long long want = (work + 255) / 256;
  const int grid = int(want < 8LL * nsm ? want : 8LL * nsm);
  const int va = pty_aligned(a, 16) && pty_aligned(a_out, 16), vb = pty_aligned(b, 16) && pty_aligned(b_out, 16);
  pty::gsc::k_scale_pair<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a, a_out, na, b, b_out, nb,
                                                                                    scale, va, vb);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

// ---- residual composition k * m + init (models/complex_inr.py:132-135) ----
// k is a real float32 scalar in device memory, m and init complex64 [n].
// Forward: out = k m + init.  Backward (torch's complex convention, k real):
// gm = k g and gk = sum Re(conj(g) m), the sum in FP64 with fixed per-thread
// ranges, a fixed tree per CTA and the CTA partials added in order by the
// last-arriving CTA (integer counter, reset for the next call): one launch.
namespace pty {
namespace rsd {

constexpr int NT = 256, MAXG = 592;

__global__ void __launch_bounds__(NT) k_residual_fwd(const float* __restrict__ k, const float2* __restrict__ m,
                                                     const float2* __restrict__ init, long long n,
                                                     float2* __restrict__ out) {
  const float kk = __ldg(k);
  for (long long i = (long long)blockIdx.x * NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT) {
    const float2 a = __ldg(m + i), b = __ldg(init + i);
    out[i] = make_float2(fmaf(kk, a.x, b.x), fmaf(kk, a.y, b.y));
  }
}

__global__ void __launch_bounds__(NT) k_residual_bwd(const float* __restrict__ k, const float2* __restrict__ m,
                                                     const float2* __restrict__ g, long long n,
                                                     float2* __restrict__ gm, float* __restrict__ gk,
                                                     double* __restrict__ part, unsigned* __restrict__ counter) {
  __shared__ double red[NT / 32];
  __shared__ bool last;
  const float kk = __ldg(k);
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT) {
    const float2 a = __ldg(m + i), d = __ldg(g + i);
    if (gm) gm[i] = make_float2(kk * d.x, kk * d.y);
    s += double(d.x) * a.x + double(d.y) * a.y;  // Re(conj(g) m)
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < NT / 32; ++w) t += red[w];
    part[blockIdx.x] = t;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x < 32) {
    __threadfence();
    double t = 0.0;
    for (int b = threadIdx.x; b < int(gridDim.x); b += 32) t += __ldcg(part + b);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) {
      *gk = float(t);
      *counter = 0u;  // ready for the next call
    }
  }
}

inline int grid_for(long long n) {
  const long long g = (n + NT * 4 - 1) / (NT * 4);
  return g < 1 ? 1 : (g > MAXG ? MAXG : int(g));
}

}  // namespace rsd
}  // namespace pty

extern "C" {

size_t ptycho_residual_workspace_size(void) { return size_t(pty::rsd::MAXG) * sizeof(double) + 256; }

int ptycho_residual(const float* k, const float* m, const float* init, long long n, float* out,
                    ptycho_stream_t stream) {
  if (!k || !m || !init || !out || n < 0) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(k, 4) || !pty_aligned(m, 8) || !pty_aligned(init, 8) || !pty_aligned(out, 8))
    return PTYCHO_ERR_MISALIGNED;
  if (n == 0) return PTYCHO_OK;
  pty::rsd::k_residual_fwd<<<pty::rsd::grid_for(n), pty::rsd::NT, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      k, reinterpret_cast<const float2*>(m), reinterpret_cast<const float2*>(init), n,
      reinterpret_cast<float2*>(out));
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_residual_backward(const float* k, const float* m, const float* g, long long n, float* gm, float* gk,
                             void* workspace, size_t workspace_bytes, ptycho_stream_t stream) {
  if (!k || !m || !g || !gk || n < 0) return PTYCHO_ERR_INVALID_ARG;
  if (!workspace || workspace_bytes < ptycho_residual_workspace_size()) return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(k, 4) || !pty_aligned(m, 8) || !pty_aligned(g, 8) || !pty_aligned(gm, 8) ||
      !pty_aligned(gk, 4) || !pty_aligned(workspace, 256))
    return PTYCHO_ERR_MISALIGNED;
  double* part = static_cast<double*>(workspace);
  unsigned* counter = reinterpret_cast<unsigned*>(static_cast<char*>(workspace) +
                                                  size_t(pty::rsd::MAXG) * sizeof(double));
  pty::rsd::k_residual_bwd<<<pty::rsd::grid_for(n), pty::rsd::NT, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      k, reinterpret_cast<const float2*>(m), reinterpret_cast<const float2*>(g), n, reinterpret_cast<float2*>(gm),
      gk, part, counter);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // extern "C"
