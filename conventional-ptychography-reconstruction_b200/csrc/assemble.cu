// assemble.cu -- deterministic assembly of object and probe gradients.
//
// Replaces the accumulation that torch autograd performs for
// `probe * object[tlY:brY, tlX:brX]` (Recovery.py:290, backward at :316):
//   dP += dL/dpsi_b conj(O[window_b]),   dO[window_b] += dL/dpsi_b conj(P),
// with dL/dpsi_b(x, y) = (-1)^(x+y) E'_b(x, y) (E'_b written by the fused kernel).
//
// One launch, two kinds of blocks, both only reading E' (which the fused
// kernel has just written and which is still in L2):
//   * dP blocks (p, g) own kPixBlock x 2 probe pixels for the patterns
//     [g kGroup, (g+1) kGroup) and write one group partial per pixel; the last
//     block of pixel block p to arrive (integer arrival counter) sums the group
//     partials in group order;
//   * dO blocks own one canvas tile (32 rows x 32 or 64 columns), compact the overlapping
//     patterns in ascending order and sum E'_b conj(P) over them per pixel.
//     The sign (-1)^(lx+ly) of a local pixel splits into (-1)^(X+Y) of the
//     canvas pixel, applied once to the sum, and (-1)^(tlY+tlX) of the
//     pattern, uniform over the tile.
// Windows are M x N.  The fused kernels fold fftshift into E' as (-1)^(x+y)
// (SIGNED); the general path's E is dL/dpsi itself.  dP blocks take two
// adjacent pixels per thread (16-byte loads) when N is even, else one.
// No floating-point atomics: every output element is owned by one thread that
// sums its contributions in a fixed order, so results are bitwise deterministic.
#include "assemble.cuh"

namespace pty {

PTY_DEVI float2 c_xor_sign(float2 a, unsigned m) {
  return make_float2(__uint_as_float(__float_as_uint(a.x) ^ m), __uint_as_float(__float_as_uint(a.y) ^ m));
}

__global__ void __launch_bounds__(256) k_loss_total(const double* __restrict__ loss_pat, int B,
                                                    double* __restrict__ loss_total) {
  loss_sum_block(loss_pat, B, loss_total);
}

struct AsmArgs {
  const float2* Eb;
  const float2* O;
  const float2* P;
  const int2* tlb;
  int B, H, W, M, N;  // windows are M x N
  float2* dO;
  float2* dP;
  float2* part;
  unsigned* done;
  const double* loss_pat;
  double* loss_total;
  int accumulate;
  int np, ng;   // dP blocks: pixel blocks x pattern groups (0 when dP is not wanted)
  int ntx;      // dO tiles per canvas row
};

// dP role: block (p, g), PAIR = 2 adjacent probe pixels per thread (16-byte
// E' loads; N even) or 1, four patterns' loads in flight
template <bool SIGNED, int PAIR>
PTY_DEVI void dp_block(const AsmArgs& a, int p, int g) {
  __shared__ int last;
  const int N = a.N;
  const size_t MN = size_t(a.M) * N;
  const int idx = PAIR * (p * kPixBlock + threadIdx.x);  // PAIR 2: (x, x + 1) share a row
  const bool in = idx < int(MN);
  const int y = idx / N, x = idx - (idx / N) * N;
  if (in) {
    const int odd = SIGNED ? (x + y) & 1 : 0;
    float2 acc0 = make_float2(0.f, 0.f), acc1 = make_float2(0.f, 0.f);
    const int b1 = min(a.B, (g + 1) * kGroup);
    constexpr int U = 4;
    for (int b = g * kGroup; b < b1; b += U) {
      float2 e0[U], e1[U], o0[U], o1[U];
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const int2 c = b + k < b1 ? __ldg(a.tlb + b + k) : make_int2(-1, -1);
        e0[k] = e1[k] = o0[k] = o1[k] = make_float2(0.f, 0.f);
        if (c.x >= 0) {
          const float2* o = a.O + size_t(c.x + y) * a.W + c.y + x;
          if constexpr (PAIR == 2) {
            const float4 e = __ldg(reinterpret_cast<const float4*>(a.Eb + size_t(b + k) * MN + idx));
            e0[k] = make_float2(e.x, e.y);
            e1[k] = make_float2(e.z, e.w);
            o1[k] = __ldg(o + 1);
          } else {
            e0[k] = __ldg(a.Eb + size_t(b + k) * MN + idx);
          }
          o0[k] = __ldg(o);
        }
      }
#pragma unroll
      for (int k = 0; k < U; ++k) {  // ascending pattern order
        c_fma_conj(acc0, e0[k], o0[k]);
        if constexpr (PAIR == 2) c_fma_conj(acc1, e1[k], o1[k]);
      }
    }
    const float2 r0 = c_negif(acc0, odd), r1 = c_negif(acc1, odd ^ int(SIGNED));
    if constexpr (PAIR == 2)
      __stcg(reinterpret_cast<float4*>(a.part + size_t(g) * MN + idx), make_float4(r0.x, r0.y, r1.x, r1.y));
    else
      __stcg(a.part + size_t(g) * MN + idx, r0);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(a.done + p, 1u) == unsigned(a.ng - 1));
  __syncthreads();
  if (last) {
    __threadfence();
    if (in) {
      float2 r0 = make_float2(0.f, 0.f), r1 = make_float2(0.f, 0.f);
      for (int gg = 0; gg < a.ng; ++gg) {
        if constexpr (PAIR == 2) {
          const float4 v = __ldcg(reinterpret_cast<const float4*>(a.part + size_t(gg) * MN + idx));
          r0 = c_add(r0, make_float2(v.x, v.y));
          r1 = c_add(r1, make_float2(v.z, v.w));
        } else {
          r0 = c_add(r0, __ldcg(a.part + size_t(gg) * MN + idx));
        }
      }
      if (a.accumulate) {
        r0 = c_add(a.dP[idx], r0);
        if constexpr (PAIR == 2) r1 = c_add(a.dP[idx + 1], r1);
      }
      a.dP[idx] = r0;
      if constexpr (PAIR == 2) a.dP[idx + 1] = r1;
    }
    if (threadIdx.x == 0) a.done[p] = 0u;  // ready for the next call
  }
}

// dO role: one TW x kTile canvas tile; lane + 32 h = column, warp w = rows w + 8 j
template <bool SIGNED, int TW>
PTY_DEVI void do_block(const AsmArgs& a, int tile) {
  __shared__ int lb[256];
  __shared__ int2 lc[256];
  __shared__ int wcnt[8];
  static_assert(TW % 32 == 0, "dO tile width");
  constexpr int CH = TW / 32;  // columns per thread
  const int M = a.M, N = a.N;
  const size_t MN = size_t(M) * N;
  const int ty0 = (tile / a.ntx) * kTile, tx0 = (tile % a.ntx) * TW;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int X = tx0 + lane;
  const int Y0 = ty0 + w;
  constexpr int R = kTile / 8;
  float2 acc[R][CH];
#pragma unroll
  for (int j = 0; j < R; ++j)
#pragma unroll
    for (int h = 0; h < CH; ++h) acc[j][h] = make_float2(0.f, 0.f);
  for (int b0 = 0; b0 < a.B; b0 += 256) {
    const int b = b0 + threadIdx.x;
    bool hit = false;
    int2 c = make_int2(-1, -1);
    if (b < a.B) {
      c = __ldg(a.tlb + b);
      hit = c.x >= 0 && c.x < ty0 + kTile && c.x + M > ty0 && c.y < tx0 + TW && c.y + N > tx0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) wcnt[w] = __popc(m);
    __syncthreads();
    int off = 0, n = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      off += i < w ? wcnt[i] : 0;
      n += wcnt[i];
    }
    if (hit) {
      const int s = off + __popc(m & ((1u << lane) - 1u));
      lb[s] = b;
      lc[s] = c;
    }
    __syncthreads();
    for (int i = 0; i < n; ++i) {
      const int bb = lb[i];
      const int2 cc = lc[i];
      const unsigned sg = SIGNED ? unsigned((cc.x + cc.y) & 1) << 31 : 0u;  // (-1)^(tlY + tlX) of the pattern
      const int lx = X - cc.y;
      const int ly0 = Y0 - cc.x;
      const float2* Eg = a.Eb + size_t(bb) * MN;
      float2 e[R][CH], p[R][CH];
      const bool full = cc.x <= ty0 && cc.x + M >= ty0 + kTile && cc.y <= tx0 && cc.y + N >= tx0 + TW;
      if (full) {  // uniform: the window covers the whole tile
#pragma unroll
        for (int j = 0; j < R; ++j)
#pragma unroll
          for (int h = 0; h < CH; ++h) {
            const int o = (ly0 + 8 * j) * N + lx + 32 * h;
            e[j][h] = __ldg(Eg + o);
            p[j][h] = __ldg(a.P + o);
          }
      } else {
#pragma unroll
        for (int j = 0; j < R; ++j)
#pragma unroll
          for (int h = 0; h < CH; ++h) {
            const int ly = ly0 + 8 * j, lxh = lx + 32 * h;
            e[j][h] = p[j][h] = make_float2(0.f, 0.f);
            if (lxh >= 0 && lxh < N && ly >= 0 && ly < M) {
              e[j][h] = __ldg(Eg + ly * N + lxh);
              p[j][h] = __ldg(a.P + ly * N + lxh);
            }
          }
      }
#pragma unroll
      for (int j = 0; j < R; ++j)
#pragma unroll
        for (int h = 0; h < CH; ++h) c_fma_conj(acc[j][h], c_xor_sign(e[j][h], sg), p[j][h]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < R; ++j)
#pragma unroll
    for (int h = 0; h < CH; ++h) {
      const int Y = Y0 + 8 * j, Xh = X + 32 * h;
      if (Y < a.H && Xh < a.W) {
        const float2 v = SIGNED ? c_negif(acc[j][h], (Xh + Y) & 1) : acc[j][h];
        float2* o = a.dO + size_t(Y) * a.W + Xh;
        *o = a.accumulate ? c_add(*o, v) : v;
      }
    }
}

// blocks [0, np * ng): dP role; the rest: dO tiles
template <bool SIGNED, int PAIR, int TW>
__global__ void __launch_bounds__(256) k_assemble(const AsmArgs a) {
  const int bid = blockIdx.x;
  const int ndp = a.np * a.ng;
  if (bid < ndp) {
    const int p = bid % a.np, g = bid / a.np;
    dp_block<SIGNED, PAIR>(a, p, g);
    if (p == 0 && g == 0 && a.loss_total) {
      __syncthreads();
      loss_sum_block(a.loss_pat, a.B, a.loss_total);
    }
  } else {
    do_block<SIGNED, TW>(a, bid - ndp);
  }
}

int launch_assemble(const float2* Eb, const float2* O, const float2* P, const int2* tlb, int B, int H, int W,
                    int M, int N, bool fftshift_sign, float2* dO, float2* dP, float2* part, unsigned* done,
                    const double* loss_pat, double* loss_total, bool accumulate, cudaStream_t s) {
  if (!dO && !dP) {
    if (loss_total) k_loss_total<<<1, 256, 0, s>>>(loss_pat, B, loss_total);
    return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
  }
  const int pair = N % 2 == 0 ? 2 : 1;
  AsmArgs a{};
  a.Eb = Eb;
  a.O = O;
  a.P = P;
  a.tlb = tlb;
  a.B = B;
  a.H = H;
  a.W = W;
  a.M = M;
  a.N = N;
  a.dO = dO;
  a.dP = dP;
  a.part = part;
  a.done = done;
  a.loss_pat = loss_pat;
  a.loss_total = loss_total;
  a.accumulate = accumulate ? 1 : 0;
  a.np = dP ? (M * N / pair + kPixBlock - 1) / kPixBlock : 0;
  a.ng = dP ? (B + kGroup - 1) / kGroup : 0;
  // dO tiles 64 columns wide for windows of 256 columns or more (fewer
  // blocks scanning the batch, more pixels per hit: c3 +3 %, c4 +6 %), 32
  // below (c1: 64 measured 1 % slower)
  const int tw = N >= 256 ? 64 : 32;
  a.ntx = (W + tw - 1) / tw;
  const int ntiles = dO ? a.ntx * ((H + kTile - 1) / kTile) : 0;
  const int grid = a.np * a.ng + ntiles;
  if (!dP && loss_total) k_loss_total<<<1, 256, 0, s>>>(loss_pat, B, loss_total);
  if (tw == 64) {
    if (fftshift_sign)
      k_assemble<true, 2, 64><<<grid, 256, 0, s>>>(a);  // fused path: M = N even
    else if (pair == 2)
      k_assemble<false, 2, 64><<<grid, 256, 0, s>>>(a);
    else
      k_assemble<false, 1, 64><<<grid, 256, 0, s>>>(a);
  } else {
    if (fftshift_sign)
      k_assemble<true, 2, 32><<<grid, 256, 0, s>>>(a);
    else if (pair == 2)
      k_assemble<false, 2, 32><<<grid, 256, 0, s>>>(a);
    else
      k_assemble<false, 1, 32><<<grid, 256, 0, s>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // namespace pty
