// general.cu -- forward model, losses and adjoint for probes of any M x N.
//
// The fused kernels cover square 64, 128 and 256 probes.  Recovery.py takes
// the probe shape from the data (Recovery.py:290, utils/optics.py:102-112:
// any M x N window), so every other shape runs here, as a short pipeline of
// kernels over a workspace X [B][M][N] complex64:
//   gather     X_b = P * O[tlY_b : tlY_b + M, tlX_b : tlX_b + N]
//   rows       DFT of length N along every row        (line_fft.cuh plans)
//   columns    DFT of length M along every column     -> spectrum F_b
//   loss       per pattern: I = |F|^2 read against Imeas at the fftshifted
//              index ((p + M/2) mod M, (q + N/2) mod N), the loss terms of
//              Recovery.py:294-305 summed in a fixed order (FP64 across
//              threads), and X_b <- 2 dL/dI F_b
//   columns, rows   inverse (unnormalised) DFTs       -> E_b = dL/dpsi_b
// followed by the assembly of dO and dP (assemble.cu, without the (-1)^(x+y)
// factor the fused kernels fold in for even M).  The FD loss works on the
// shifted grid with circular neighbours, through three float planes per
// pattern in the workspace.  Every reduction has a fixed order: results are
// bitwise deterministic.
#include <cuda_runtime.h>
#include <stdint.h>

#include "assemble.cuh"
#include "fused.cuh"
#include "general.cuh"
#include "line_fft.cuh"

namespace pty {
namespace gen {

using lfft::LinePlan;
using lfft::kLineNT;
using lfft::pad16;

constexpr size_t kLineSmemCap = 200 * 1024;

// X_b = P * O[window_b]; resolves frame ids and windows (status on failure)
__global__ void __launch_bounds__(256) k_gather(const FusedArgs a, int M, int N, float2* __restrict__ X,
                                                int2* __restrict__ tlb) {
  const int b = blockIdx.y;
  const int f = a.batch ? __ldg(a.batch + b) : b;
  int2 c = make_int2(-1, -1);
  bool ok = f >= 0 && f < a.F;
  if (ok) {
    c = __ldg(a.tl + f);
    ok = c.x >= 0 && c.y >= 0 && c.x <= a.H - M && c.y <= a.W - N;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (tlb) tlb[b] = ok ? c : make_int2(-1, -1);
    if (!ok) pty_raise(a.status, PTYCHO_ERR_WINDOW);
  }
  const int MN = M * N;
  float2* Xb = X + size_t(b) * MN;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < MN; i += gridDim.x * 256) {
    float2 v = make_float2(0.f, 0.f);
    if (ok) {
      const int y = i / N, x = i - (i / N) * N;
      v = c_mul(__ldg(a.P + i), __ldg(a.O + size_t(c.x + y) * a.W + (c.y + x)));
    }
    Xb[i] = v;
  }
}

// in-place DFTs along rows (COL = false: B*M lines of length N) or columns
// (COL = true: B*N lines of length M, LINES adjacent columns per CTA)
template <bool COL, bool INV>
__global__ void __launch_bounds__(kLineNT) k_lines(float2* __restrict__ X, int M, int N, int nlines,
                                                   const LinePlan plan, int lines, int ls) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* bufA = reinterpret_cast<float2*>(smem);
  float2* bufB = bufA + size_t(lines) * ls;
  float2* tw = bufB + size_t(lines) * ls;
  const int L = plan.L, t = threadIdx.x;
  const int l0 = blockIdx.x * lines;
  const size_t MN = size_t(M) * N;
  for (int k = t; k < L; k += kLineNT) {
    double sn, cs;
    sincospi(-2.0 * double(k) / double(L), &sn, &cs);
    tw[k] = make_float2(float(cs), float(sn));
  }
  // element k of line l
  auto at = [&](int l, int k) -> float2* {
    if (COL) {
      const int b = l / N, col = l - (l / N) * N;
      return X + size_t(b) * MN + size_t(k) * N + col;
    }
    return X + size_t(l) * N + k;
  };
  for (int idx = t; idx < lines * L; idx += kLineNT) {
    int l, k;
    if (COL) {
      l = idx % lines;
      k = idx / lines;
    } else {
      l = idx / L;
      k = idx - l * L;
    }
    bufA[l * ls + pad16(k)] = l0 + l < nlines ? *at(l0 + l, k) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = lfft::transform<INV>(plan, bufA, bufB, tw, lines, ls, L, t);
  for (int idx = t; idx < lines * L; idx += kLineNT) {
    int l, k;
    if (COL) {
      l = idx % lines;
      k = idx / lines;
    } else {
      l = idx / L;
      k = idx - l * L;
    }
    if (l0 + l < nlines) *at(l0 + l, k) = res[l * ls + pad16(k)];
  }
}

// shifted (measurement) index of spectrum element (p, q)
PTY_DEVI int shifted(int p, int q, int M, int N) {
  int u = p + M / 2, v = q + N / 2;
  if (u >= M) u -= M;
  if (v >= N) v -= N;
  return u * N + v;
}

// FP64 block sum in a fixed order (result valid in thread 0)
PTY_DEVI double block_sum256(double x, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < 8; ++i) s += red[i];
  __syncthreads();
  return s;
}

// One CTA per pattern: per-pattern mean loss, and (GRAD) X_b <- 2 dL/dI F_b.
// MODE_INTENSITY-like output is done by k_intensity.  scr: 3 float planes of
// M*N per pattern on the shifted grid (FD only).
template <int LOSS, bool GRAD>
__global__ void __launch_bounds__(256) k_loss(float2* __restrict__ X, const FusedArgs a, int M, int N,
                                              const int2* __restrict__ tlb_in, float* __restrict__ scr,
                                              double* __restrict__ loss_pat) {
  __shared__ double red[8];
  const int b = blockIdx.x;
  const int MN = M * N;
  const float inv_mn = 1.0f / float(MN);
  float2* Xb = X + size_t(b) * MN;
  // frame and window (the gather resolved them; recompute here for MODE_LOSS)
  const int f = a.batch ? __ldg(a.batch + b) : b;
  bool ok = f >= 0 && f < a.F;
  if (ok) {
    const int2 c = tlb_in ? tlb_in[b] : __ldg(a.tl + f);
    ok = c.x >= 0 && c.y >= 0 && c.x <= a.H - M && c.y <= a.W - N;
  }
  if (!ok) {  // uniform; the gather zeroed X_b and raised the status
    if (threadIdx.x == 0 && loss_pat) loss_pat[b] = (double)__int_as_float(0x7fc00000);
    return;
  }
  const float* Im = a.Imeas + size_t(f) * MN;
  double acc = 0.0;
  if constexpr (LOSS != PTYCHO_LOSS_FD) {
    for (int i = threadIdx.x; i < MN; i += 256) {
      const int p = i / N, q = i - (i / N) * N;
      const float2 F = Xb[i];
      const float meas = __ldg(Im + shifted(p, q, M, N));
      const float I = fmaf(F.x, F.x, F.y * F.y);
      float term, g;
      if constexpr (LOSS == PTYCHO_LOSS_INTENSITY_GRAD) {
        term = I * meas * float(MN);
        g = meas;
      } else if constexpr (LOSS == PTYCHO_LOSS_SMOOTH_L1) {
        const float dd = I - meas;
        const float ad = fabsf(dd);
        term = ad < 1.0f ? 0.5f * dd * dd : ad - 0.5f;
        g = (ad < 1.0f ? dd : copysignf(1.0f, dd)) * inv_mn;
      } else {
        const float Ie = I + kEps;
        term = fmaf(-meas, __logf(Ie), I);
        g = (1.0f - __fdividef(meas, Ie)) * inv_mn;
      }
      acc += (double)term;
      if (GRAD) Xb[i] = c_scale(F, 2.0f * g);
    }
  } else {
    // shifted grid: dW, then ax = Rx / G, ay = Ry / G, then the stencil adjoint
    float* dW = scr + size_t(b) * 3 * MN;
    float* ax = dW + MN;
    float* ay = ax + MN;
    for (int i = threadIdx.x; i < MN; i += 256) {
      const int p = i / N, q = i - (i / N) * N;
      const float2 F = Xb[i];
      const int s = shifted(p, q, M, N);
      const float I = fmaf(F.x, F.x, F.y * F.y);
      dW[s] = sqrtf(__ldg(Im + s) + kEps) - sqrtf(I + kEps);
    }
    __syncthreads();
    for (int s = threadIdx.x; s < MN; s += 256) {
      const int u = s / N, v = s - (s / N) * N;
      const float d = dW[s];
      const float rx = dW[u * N + (v + 1 == N ? 0 : v + 1)] - d;
      const float ry = dW[(u + 1 == M ? 0 : u + 1) * N + v] - d;
      const float G = sqrtf(fmaf(rx, rx, fmaf(ry, ry, kEps)));
      acc += (double)G;
      ax[s] = rx / G;
      ay[s] = ry / G;
    }
    if (GRAD) {
      __syncthreads();
      for (int i = threadIdx.x; i < MN; i += 256) {
        const int p = i / N, q = i - (i / N) * N;
        const int s = shifted(p, q, M, N);
        const int u = s / N, v = s - (s / N) * N;
        const float dl = (ax[u * N + (v == 0 ? N - 1 : v - 1)] - ax[s] + ay[(u == 0 ? M - 1 : u - 1) * N + v] - ay[s]) *
                         inv_mn;
        const float2 F = Xb[i];
        const float I = fmaf(F.x, F.x, F.y * F.y);
        const float g = dl * (-0.5f / sqrtf(I + kEps));
        Xb[i] = c_scale(F, 2.0f * g);
      }
    }
  }
  const double tot = block_sum256(acc, red);
  if (threadIdx.x == 0 && loss_pat) loss_pat[b] = tot / double(MN);
}

// |F|^2 written at the fftshifted index
__global__ void __launch_bounds__(256) k_intensity(const float2* __restrict__ X, int M, int N, const FusedArgs a) {
  const int b = blockIdx.y;
  const int MN = M * N;
  const int f = a.batch ? __ldg(a.batch + b) : b;
  bool ok = f >= 0 && f < a.F;
  if (ok) {
    const int2 c = __ldg(a.tl + f);
    ok = c.x >= 0 && c.y >= 0 && c.x <= a.H - M && c.y <= a.W - N;
  }
  float* Ib = a.I_out + size_t(b) * MN;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < MN; i += gridDim.x * 256) {
    const int p = i / N, q = i - (i / N) * N;
    const float2 F = X[size_t(b) * MN + i];
    Ib[shifted(p, q, M, N)] = ok ? fmaf(F.x, F.x, F.y * F.y) : __int_as_float(0x7fc00000);
  }
}

static size_t line_smem(int lines, int ls, int L) { return (size_t(2) * lines * ls + size_t(L)) * sizeof(float2); }

template <bool COL, bool INV>
static int run_lines(float2* X, int B, int M, int N, cudaStream_t s) {
  const int L = COL ? M : N;
  LinePlan plan;
  if (!lfft::make_plan(L, &plan)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  const int nlines = COL ? B * N : B * M;
  const int ls = pad16(L - 1) + 1;
  int lines = L >= 4096 ? 1 : 4096 / L;
  if (COL && lines < 4) lines = 4;
  while (lines > 1 && line_smem(lines, ls, L) > kLineSmemCap) --lines;
  const size_t smem = line_smem(lines, ls, L);
  auto kern = k_lines<COL, INV>;
  static PtyDevCache attr_set;
  int dev = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    if (!attr_set.get(&dev)) {
      if (dev < 0) return PTYCHO_ERR_LAUNCH;
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kLineSmemCap)) != cudaSuccess)
        return PTYCHO_ERR_LAUNCH;
      attr_set.put(dev, 1);
    }
    kern<<<(nlines + lines - 1) / lines, kLineNT, smem, s>>>(X, M, N, nlines, plan, lines, ls);
    if (cudaGetLastError() == cudaSuccess) return PTYCHO_OK;
    attr_set.put(dev, 0);
  }
  return PTYCHO_ERR_LAUNCH;
}

static dim3 elem_grid(int B, int M, int N) {
  const int per = (M * N + 255) / 256;
  return dim3(per < 64 ? per : 64, B);
}

template <bool GRAD>
static int launch_loss(int loss, float2* X, const FusedArgs& a, int M, int N, const int2* tlb, float* scr,
                       double* lp, cudaStream_t s) {
  switch (loss) {
    case PTYCHO_LOSS_SMOOTH_L1: k_loss<PTYCHO_LOSS_SMOOTH_L1, GRAD><<<a.B, 256, 0, s>>>(X, a, M, N, tlb, scr, lp); break;
    case PTYCHO_LOSS_FD: k_loss<PTYCHO_LOSS_FD, GRAD><<<a.B, 256, 0, s>>>(X, a, M, N, tlb, scr, lp); break;
    case PTYCHO_LOSS_POISSON: k_loss<PTYCHO_LOSS_POISSON, GRAD><<<a.B, 256, 0, s>>>(X, a, M, N, tlb, scr, lp); break;
    default: k_loss<PTYCHO_LOSS_INTENSITY_GRAD, GRAD><<<a.B, 256, 0, s>>>(X, a, M, N, tlb, scr, lp); break;
  }
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // namespace gen

bool general_supported(int M, int N) { return M >= 1 && N >= 1 && M <= kGeneralMaxDim && N <= kGeneralMaxDim; }

int general_forward_intensity(const FusedArgs& a, int M, int N, float2* X, cudaStream_t s) {
  using namespace gen;
  k_gather<<<elem_grid(a.B, M, N), 256, 0, s>>>(a, M, N, X, nullptr);
  if (cudaGetLastError() != cudaSuccess) return PTYCHO_ERR_LAUNCH;
  int st = run_lines<false, false>(X, a.B, M, N, s);
  if (st) return st;
  st = run_lines<true, false>(X, a.B, M, N, s);
  if (st) return st;
  k_intensity<<<elem_grid(a.B, M, N), 256, 0, s>>>(X, M, N, a);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int general_fwd_adj(const FusedArgs& a, int M, int N, int loss, bool grad, float2* X, float* scr, int2* tlb,
                    cudaStream_t s) {
  using namespace gen;
  k_gather<<<elem_grid(a.B, M, N), 256, 0, s>>>(a, M, N, X, tlb);
  if (cudaGetLastError() != cudaSuccess) return PTYCHO_ERR_LAUNCH;
  int st = run_lines<false, false>(X, a.B, M, N, s);
  if (!st) st = run_lines<true, false>(X, a.B, M, N, s);
  if (st) return st;
  st = grad ? launch_loss<true>(loss, X, a, M, N, tlb, scr, a.loss_pat, s)
            : launch_loss<false>(loss, X, a, M, N, tlb, scr, a.loss_pat, s);
  if (st || !grad) return st;
  st = run_lines<true, true>(X, a.B, M, N, s);
  if (!st) st = run_lines<false, true>(X, a.B, M, N, s);
  return st;
}

}  // namespace pty
