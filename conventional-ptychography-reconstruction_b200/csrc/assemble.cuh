// assemble.cuh -- launchers for the gradient assembly kernels (assemble.cu).
#pragma once
#include "common.cuh"

namespace pty {

constexpr int kTile = 32;   // canvas tile height for dO (its width: 32 or 64, by window width)
constexpr int kGroup = 16;  // patterns per dP partial sum
constexpr int kPixBlock = 256;  // probe pixels per dP block

// number of arrival counters the dP reduction needs for M x N windows (zeroed
// before the first call; every call leaves them zeroed)
inline int dp_counters(int M, int N) { return (M * N + kPixBlock - 1) / kPixBlock; }

// FP64 sum of the per-pattern losses in a fixed order (a strided pass per
// thread, a shuffle tree, the eight warp sums in order) by one block of 256
// threads; every thread of the block calls it
PTY_DEVI void loss_sum_block(const double* __restrict__ loss_pat, int B, double* loss_total) {
  __shared__ double red[8];
  double s = 0.0;
  for (int b = threadIdx.x; b < B; b += 256) s += loss_pat[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < 8; ++i) t += red[i];
    loss_total[0] = t;
  }
}

// dP (group partials, then the last-arriving block sums them in group order),
// dO (tile owner sums in ascending pattern order) and the FP64 loss total in
// one launch; any output may be null.  E' is only read; with fftshift_sign
// it carries the fused kernels' (-1)^(x+y) factor (M = N even).  `done` holds
// dp_counters(M, N) zeroed counters and is left zeroed.
int launch_assemble(const float2* Eb, const float2* O, const float2* P, const int2* tlb, int B, int H, int W,
                    int M, int N, bool fftshift_sign, float2* dO, float2* dP, float2* part, unsigned* done,
                    const double* loss_pat, double* loss_total, bool accumulate, cudaStream_t s);

}  // namespace pty
