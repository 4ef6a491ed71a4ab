// probe_prep.cu -- probe centring and energy normalisation as two device kernels.
//
// Replaces the per-minibatch probe preparation of Recovery.py:262-285 (the
// centre-of-mass roll of utils center_probe and the scaling to
// sum |P|^2 = M*N), which the reference runs as a few dozen small torch ops
// with host synchronisations, and the autograd backward through it.
//
// Forward (one CTA): a(y, x) = |P|^2 with FP64 row sums r_y and column sums
// c_x (fixed-order warp trees), tot = sum r_y.  The reference's
//   cp = trunc([M, N]/2 - [M, N] * mean(cumsum(marginal)) / tot + 1)
// uses mean(cumsum(r)) = sum_y r_y (M - y) / M, so
//   cy = trunc(M/2 - sum_y r_y (M - y) / tot + 1)   (cx likewise; 0 if tot == 0).
// P_r = roll(P, (-cy, -cx)), k = sqrt(M N / e) with e = sum |P_r|^2 = tot
// (k = 1 if e == 0), P_out = k P_r.  state = {cy, cx, k, e} (doubles).
//
// Backward (one CTA), torch's complex convention: with G the gradient of
// P_out, S = sum Re(conj(G) P_out) and k^2 e = M N,
//   dL/dP_r = k (G - S P_out / (M N))   (e > 0),   G (e == 0),
// rolled back by (cy, cx).  The e term is the gradient through the energy
// normalisation that autograd carries in the reference.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace pty {
namespace pp {

constexpr int NT = 1024, MAXD = 1024;

PTY_DEVI double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

PTY_DEVI double abs2(float2 p) { return double(p.x) * double(p.x) + double(p.y) * double(p.y); }

// Probes of up to kStageMax elements are first staged in shared memory (every
// thread's loads independent, one memory round trip); the sums and the roll
// then read shared memory, in the same order as the unstaged kernel, so both
// give identical results.
constexpr int kStageMax = 16384;

template <bool STAGED>
__global__ void __launch_bounds__(NT) k_probe_prep(const float2* __restrict__ P, int M, int N,
                                                   float2* __restrict__ out, double* __restrict__ state) {
  __shared__ double rs[MAXD], cs[MAXD];
  __shared__ double cpart[NT];  // column partials of the row groups
  __shared__ double sh[4];
  extern __shared__ float2 sP[];  // STAGED: the probe, [M][N]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if constexpr (STAGED) {
#pragma unroll
    for (int k = 0; k < kStageMax / NT; ++k) {
      const int idx = threadIdx.x + k * NT;
      if (idx < M * N) sP[idx] = __ldg(P + idx);
    }
    __syncthreads();
  }
  auto ld = [&](int idx) -> float2 {
    if constexpr (STAGED) return sP[idx];
    else return __ldg(P + idx);
  };
  for (int y = w; y < M; y += 32) {  // row sums: one warp per row, coalesced
    double s = 0.0;
    for (int x = lane; x < N; x += 32) s += abs2(ld(y * N + x));
    s = warp_sum(s);
    if (lane == 0) rs[y] = s;
  }
  {  // column sums: thread (g, x) sums rows g, g + G, ... of column x (coalesced),
     // then the G group partials of each column are added in group order
    const int G = NT / N > 0 ? NT / N : 1;
    const int t = threadIdx.x, x = t % N, g = t / N;
    double s = 0.0;
    if (g < G)
      for (int y = g; y < M; y += G) s += abs2(ld(y * N + x));
    if (g < G) cpart[g * N + x] = s;
    __syncthreads();
    for (int xx = t; xx < N; xx += NT) {
      double c = 0.0;
      for (int gg = 0; gg < G; ++gg) c += cpart[gg * N + xx];
      cs[xx] = c;
    }
  }
  __syncthreads();
  if (w == 0) {
    double tot = 0.0, wy = 0.0, wx = 0.0;
    for (int y = lane; y < M; y += 32) {
      tot += rs[y];
      wy += rs[y] * double(M - y);
    }
    for (int x = lane; x < N; x += 32) wx += cs[x] * double(N - x);
    tot = warp_sum(tot);
    wy = warp_sum(wy);
    wx = warp_sum(wx);
    if (lane == 0) {
      double cy = 0.0, cx = 0.0, k = 1.0;
      if (tot > 0.0) {
        cy = trunc(0.5 * double(M) - wy / tot + 1.0);
        cx = trunc(0.5 * double(N) - wx / tot + 1.0);
        k = sqrt(double(M) * double(N) / tot);
      }
      sh[0] = cy;
      sh[1] = cx;
      sh[2] = k;
      sh[3] = tot;
      if (state) {
        state[0] = cy;
        state[1] = cx;
        state[2] = k;
        state[3] = tot;
      }
    }
  }
  __syncthreads();
  // roll by (-cy, -cx): out[i][j] = P[(i + cy) mod M][(j + cx) mod N], times k
  const int cy = int(sh[0]), cx = int(sh[1]);
  const int oy = ((cy % M) + M) % M, ox = ((cx % N) + N) % N;
  const float k = float(sh[2]);
  for (int idx = threadIdx.x; idx < M * N; idx += NT) {
    const int i = idx / N, j = idx - (idx / N) * N;
    int si = i + oy, sj = j + ox;
    si -= si >= M ? M : 0;
    sj -= sj >= N ? N : 0;
    const float2 p = ld(si * N + sj);
    out[idx] = make_float2(p.x * k, p.y * k);
  }
}

__global__ void __launch_bounds__(NT) k_probe_prep_bwd(const float2* __restrict__ Pout,
                                                       const double* __restrict__ state,
                                                       const float2* __restrict__ g, int M, int N,
                                                       float2* __restrict__ gin) {
  __shared__ double red[32];
  __shared__ double Sh;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double s = 0.0;
#pragma unroll 8
  for (int idx = threadIdx.x; idx < M * N; idx += NT) {
    const float2 a = __ldg(g + idx), b = __ldg(Pout + idx);
    s += double(a.x) * double(b.x) + double(a.y) * double(b.y);  // Re(conj(G) P_out)
  }
  s = warp_sum(s);
  if (lane == 0) red[w] = s;
  __syncthreads();
  if (w == 0) {
    double t = red[lane];
    t = warp_sum(t);
    if (lane == 0) Sh = t;
  }
  __syncthreads();
  const double e = state[3];
  const int cy = int(state[0]), cx = int(state[1]);
  const int oy = ((cy % M) + M) % M, ox = ((cx % N) + N) % N;
  const bool norm = e > 0.0;
  const float k = float(state[2]);
  const float c = norm ? float(Sh / (double(M) * double(N))) : 0.f;
#pragma unroll 8
  for (int idx = threadIdx.x; idx < M * N; idx += NT) {
    const int i = idx / N, j = idx - (idx / N) * N;
    int si = i + oy, sj = j + ox;
    si -= si >= M ? M : 0;
    sj -= sj >= N ? N : 0;
    const float2 a = __ldg(g + idx);
    float2 r = a;
    if (norm) {
      const float2 b = __ldg(Pout + idx);
      r = make_float2(k * fmaf(-c, b.x, a.x), k * fmaf(-c, b.y, a.y));
    }
    gin[size_t(si) * N + sj] = r;
  }
}

}  // namespace pp
}  // namespace pty

using namespace pty;

extern "C" {

int ptycho_probe_center_normalize(const float* P, int M, int N, float* P_out, double* state,
                                  ptycho_stream_t stream) {
  if (!P || !P_out || !state || M <= 0 || N <= 0) return PTYCHO_ERR_INVALID_ARG;
  if (M > pp::MAXD || N > pp::MAXD) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (P == P_out) return PTYCHO_ERR_INVALID_ARG;  // the roll reads P while P_out is written
  if (!pty_aligned(P, 8) || !pty_aligned(P_out, 8) || !pty_aligned(state, 8)) return PTYCHO_ERR_MISALIGNED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (M * N <= pp::kStageMax) {
    const int smem = M * N * int(sizeof(float2));
    static PtyDevCache attr_set;  // per device: the dynamic shared-memory limit, once
    int dev = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      if (!attr_set.get(&dev)) {
        if (dev < 0) return PTYCHO_ERR_LAUNCH;
        if (cudaFuncSetAttribute(pp::k_probe_prep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 pp::kStageMax * int(sizeof(float2))) != cudaSuccess)
          return PTYCHO_ERR_LAUNCH;
        attr_set.put(dev, 1);
      }
      pp::k_probe_prep<true><<<1, pp::NT, smem, s>>>(reinterpret_cast<const float2*>(P), M, N,
                                                     reinterpret_cast<float2*>(P_out), state);
      if (cudaGetLastError() == cudaSuccess) return PTYCHO_OK;
      attr_set.put(dev, 0);  // the attribute was lost (device reset): set it again once
    }
    return PTYCHO_ERR_LAUNCH;
  } else {
    pp::k_probe_prep<false><<<1, pp::NT, 0, s>>>(reinterpret_cast<const float2*>(P), M, N,
                                                 reinterpret_cast<float2*>(P_out), state);
  }
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_probe_center_normalize_backward(const float* P_out, const double* state, const float* grad_out,
                                           int M, int N, float* grad_in, ptycho_stream_t stream) {
  if (!P_out || !state || !grad_out || !grad_in || M <= 0 || N <= 0) return PTYCHO_ERR_INVALID_ARG;
  if (M > pp::MAXD || N > pp::MAXD) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (grad_out == grad_in) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(P_out, 8) || !pty_aligned(state, 8) || !pty_aligned(grad_out, 8) || !pty_aligned(grad_in, 8))
    return PTYCHO_ERR_MISALIGNED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  pp::k_probe_prep_bwd<<<1, pp::NT, 0, s>>>(reinterpret_cast<const float2*>(P_out), state,
                                            reinterpret_cast<const float2*>(grad_out), M, N,
                                            reinterpret_cast<float2*>(grad_in));
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // extern "C"
