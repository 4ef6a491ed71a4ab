// assemble.cu -- deterministic assembly of object and probe gradients.
//
// Replaces the accumulation that torch autograd performs for
// `probe * object[tlY:brY, tlX:brX]` (Recovery.py:290, backward at :316):
//   dP += dL/dpsi_b conj(O[window_b]),   dO[window_b] += dL/dpsi_b conj(P),
// with dL/dpsi_b = (-1)^(x+y) E'_b (E'_b written by the fused kernel).
// k_dP_terms runs first: it reduces dP and turns E'_b in place into the
// object-gradient terms G_b, which k_dO then only has to sum.
// No floating-point atomics: every output element is owned by one thread
// that sums its contributions in ascending pattern order; the dP group
// partials are summed in group order by whichever block arrives last (an
// integer arrival counter picks it, the order of the sum does not depend on it).
#include "assemble.cuh"

namespace pty {

PTY_DEVI float2 c_negif(float2 a, int odd) { return odd ? make_float2(-a.x, -a.y) : a; }

// dO over one kTile x kTile canvas tile, 256 threads x kTile/8 rows: the
// overlapping patterns are compacted in ascending order, then each thread sums
// their terms G_b = dL/dpsi_b conj(P) at its 4 pixels (k_dP_terms wrote G_b).
__global__ void __launch_bounds__(256) k_dO(const float2* __restrict__ Gb, const int2* __restrict__ tlb, int B,
                                            int H, int W, int M, int ntx, float2* __restrict__ dO,
                                            int accumulate) {
  __shared__ int list[256];
  __shared__ int wcnt[8];
  const int tile = blockIdx.x;
  const int ty0 = (tile / ntx) * kTile, tx0 = (tile % ntx) * kTile;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int X = tx0 + lane;
  const int Y0 = ty0 + w;
  constexpr int R = kTile / 8;
  float2 acc[R];
#pragma unroll
  for (int j = 0; j < R; ++j) acc[j] = make_float2(0.f, 0.f);
  for (int b0 = 0; b0 < B; b0 += 256) {
    const int b = b0 + threadIdx.x;
    bool hit = false;
    if (b < B) {
      const int2 c = __ldg(tlb + b);
      hit = c.x >= 0 && c.x < ty0 + kTile && c.x + M > ty0 && c.y < tx0 + kTile && c.y + M > tx0;
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
    if (hit) list[off + __popc(m & ((1u << lane) - 1u))] = b;
    __syncthreads();
    // two patterns per iteration: loads first, then the adds in list order
    for (int i = 0; i < n; i += 2) {
      float2 c0[R], c1[R];
      {
        const int bb = list[i];
        const int2 c = __ldg(tlb + bb);
        const int lx = X - c.y;
        const float2* Gp = Gb + size_t(bb) * M * M;
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const int ly = Y0 + 8 * j - c.x;
          c0[j] = make_float2(0.f, 0.f);
          if (lx >= 0 && lx < M && ly >= 0 && ly < M) c0[j] = __ldg(Gp + ly * M + lx);
        }
      }
      const bool two = i + 1 < n;
      if (two) {
        const int bb = list[i + 1];
        const int2 c = __ldg(tlb + bb);
        const int lx = X - c.y;
        const float2* Gp = Gb + size_t(bb) * M * M;
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const int ly = Y0 + 8 * j - c.x;
          c1[j] = make_float2(0.f, 0.f);
          if (lx >= 0 && lx < M && ly >= 0 && ly < M) c1[j] = __ldg(Gp + ly * M + lx);
        }
      }
#pragma unroll
      for (int j = 0; j < R; ++j) {
        acc[j] = c_add(acc[j], c0[j]);
        if (two) acc[j] = c_add(acc[j], c1[j]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int Y = Y0 + 8 * j;
    if (Y < H && X < W) {
      float2* o = dO + size_t(Y) * W + X;
      *o = accumulate ? c_add(*o, acc[j]) : acc[j];
    }
  }
}

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

__global__ void __launch_bounds__(256) k_loss_total(const double* __restrict__ loss_pat, int B,
                                                    double* __restrict__ loss_total) {
  loss_sum_block(loss_pat, B, loss_total);
}

// Per-pattern gradient terms and dP.  Block (p, g) owns kPixBlock probe
// pixels for the patterns [g*kGroup, (g+1)*kGroup); each (pattern, pixel)
// pair is visited by exactly one thread, which
//  * adds E'_b conj(O[window_b]) to its dP group partial (want_dP), and
//  * overwrites E'_b in place with G_b = (-1)^(x+y) E'_b conj(P) (want_G), the
//    object-gradient term k_dO then sums (the pixel's P is loaded once).
// E' is read with ld.global.cg (it is rewritten in this kernel).  The last of
// the G blocks of pixel block p sums the dP group partials in group order.
__global__ void __launch_bounds__(kPixBlock, 6) k_dP_terms(float2* __restrict__ Eb, const float2* __restrict__ O,
                                                        const float2* __restrict__ P, const int2* __restrict__ tlb,
                                                        int B, int W, int M, float2* __restrict__ part,
                                                        unsigned* __restrict__ done, float2* __restrict__ dP,
                                                        int want_G, int accumulate,
                                                        const double* __restrict__ loss_pat,
                                                        double* __restrict__ loss_total) {
  __shared__ int last;
  const int p = blockIdx.x, g = blockIdx.y, G = gridDim.y;
  const int idx = p * kPixBlock + threadIdx.x;
  const bool in = idx < M * M;
  const int y = idx / M, x = idx - (idx / M) * M;
  const bool want_dP = dP != nullptr;
  if (in) {
    const int odd = (x + y) & 1;
    const float2 pc = want_G ? __ldg(P + idx) : make_float2(0.f, 0.f);
    float2 acc = make_float2(0.f, 0.f);
    const int b1 = min(B, (g + 1) * kGroup);
    constexpr int U = 4;  // patterns whose loads are in flight together
    for (int b = g * kGroup; b < b1; b += U) {
      float2 e[U], t[U];
      bool ok[U];
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const int2 c = b + k < b1 ? __ldg(tlb + b + k) : make_int2(-1, -1);
        ok[k] = c.x >= 0;
        e[k] = make_float2(0.f, 0.f);
        t[k] = make_float2(0.f, 0.f);
        if (ok[k]) {
          e[k] = __ldcg(Eb + size_t(b + k) * M * M + idx);
          if (want_dP) t[k] = c_mulc(e[k], __ldg(O + size_t(c.x + y) * W + c.y + x));
        }
      }
#pragma unroll
      for (int k = 0; k < U; ++k) {
        acc = c_add(acc, t[k]);  // ascending pattern order
        if (want_G && ok[k]) __stcg(Eb + size_t(b + k) * M * M + idx, c_negif(c_mulc(e[k], pc), odd));
      }
    }
    if (want_dP) __stcg(reinterpret_cast<float2*>(part + size_t(g) * M * M + idx), c_negif(acc, odd));
  }
  if (want_dP) {  // uniform over the grid
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(done + p, 1u) == unsigned(G - 1));
    __syncthreads();
    if (last) {
      __threadfence();
      if (in) {
        float2 acc = make_float2(0.f, 0.f);
        for (int gg = 0; gg < G; ++gg) acc = c_add(acc, __ldcg(part + size_t(gg) * M * M + idx));
        dP[idx] = accumulate ? c_add(dP[idx], acc) : acc;
      }
      if (threadIdx.x == 0) done[p] = 0u;  // ready for the next call
    }
  }
  if (p == 0 && g == 0 && loss_total) loss_sum_block(loss_pat, B, loss_total);
}

// k_dP_terms with two adjacent probe pixels per thread: E', G and the partials
// move as 16-byte loads and stores and each pattern's window corner is read
// once per pair.  Same terms, same order, bitwise the same results (P must be
// 16-byte aligned; the launcher falls back to k_dP_terms otherwise).
__global__ void __launch_bounds__(kPixBlock, 4) k_dP_terms2(float2* __restrict__ Eb, const float2* __restrict__ O,
                                                         const float2* __restrict__ P, const int2* __restrict__ tlb,
                                                         int B, int W, int M, float2* __restrict__ part,
                                                         unsigned* __restrict__ done, float2* __restrict__ dP,
                                                         int want_G, int accumulate,
                                                         const double* __restrict__ loss_pat,
                                                         double* __restrict__ loss_total) {
  __shared__ int last;
  const int p = blockIdx.x, g = blockIdx.y, G = gridDim.y;
  const int idx = 2 * (p * kPixBlock + threadIdx.x);  // even: the pair (x, x + 1) shares a row
  const bool in = idx < M * M;
  const int y = idx / M, x = idx - (idx / M) * M;
  const bool want_dP = dP != nullptr;
  const size_t MM = size_t(M) * M;
  if (in) {
    const int odd = (x + y) & 1;
    float4 pc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (want_G) pc = __ldg(reinterpret_cast<const float4*>(P + idx));
    float2 acc0 = make_float2(0.f, 0.f), acc1 = make_float2(0.f, 0.f);
    const int b1 = min(B, (g + 1) * kGroup);
    constexpr int U = 4;  // patterns whose loads are in flight together
    for (int b = g * kGroup; b < b1; b += U) {
      float4 e[U];
      float2 t0[U], t1[U];
      bool ok[U];
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const int2 c = b + k < b1 ? __ldg(tlb + b + k) : make_int2(-1, -1);
        ok[k] = c.x >= 0;
        e[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        t0[k] = t1[k] = make_float2(0.f, 0.f);
        if (ok[k]) {
          e[k] = __ldcg(reinterpret_cast<const float4*>(Eb + size_t(b + k) * MM + idx));
          if (want_dP) {
            const float2* o = O + size_t(c.x + y) * W + c.y + x;
            t0[k] = c_mulc(make_float2(e[k].x, e[k].y), __ldg(o));
            t1[k] = c_mulc(make_float2(e[k].z, e[k].w), __ldg(o + 1));
          }
        }
      }
#pragma unroll
      for (int k = 0; k < U; ++k) {
        acc0 = c_add(acc0, t0[k]);  // ascending pattern order
        acc1 = c_add(acc1, t1[k]);
        if (want_G && ok[k]) {
          const float2 g0 = c_negif(c_mulc(make_float2(e[k].x, e[k].y), make_float2(pc.x, pc.y)), odd);
          const float2 g1 = c_negif(c_mulc(make_float2(e[k].z, e[k].w), make_float2(pc.z, pc.w)), odd ^ 1);
          __stcg(reinterpret_cast<float4*>(Eb + size_t(b + k) * MM + idx), make_float4(g0.x, g0.y, g1.x, g1.y));
        }
      }
    }
    if (want_dP) {
      const float2 a0 = c_negif(acc0, odd), a1 = c_negif(acc1, odd ^ 1);
      __stcg(reinterpret_cast<float4*>(part + size_t(g) * MM + idx), make_float4(a0.x, a0.y, a1.x, a1.y));
    }
  }
  if (want_dP) {  // uniform over the grid
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(done + p, 1u) == unsigned(G - 1));
    __syncthreads();
    if (last) {
      __threadfence();
      if (in) {
        float2 r0 = make_float2(0.f, 0.f), r1 = make_float2(0.f, 0.f);
        for (int gg = 0; gg < G; ++gg) {
          const float4 v = __ldcg(reinterpret_cast<const float4*>(part + size_t(gg) * MM + idx));
          r0 = c_add(r0, make_float2(v.x, v.y));
          r1 = c_add(r1, make_float2(v.z, v.w));
        }
        if (accumulate) {
          r0 = c_add(dP[idx], r0);
          r1 = c_add(dP[idx + 1], r1);
        }
        dP[idx] = r0;
        dP[idx + 1] = r1;
      }
      if (threadIdx.x == 0) done[p] = 0u;  // ready for the next call
    }
  }
  if (p == 0 && g == 0 && loss_total) loss_sum_block(loss_pat, B, loss_total);
}

int launch_assemble(float2* Eb, const float2* O, const float2* P, const int2* tlb, int B, int H, int W, int M,
                    float2* dO, float2* dP, float2* part, unsigned* done, const double* loss_pat,
                    double* loss_total, bool accumulate, cudaStream_t s) {
  if (dO || dP) {  // dP partials and, for dO, the in-place E' -> G conversion
    const int G = (B + kGroup - 1) / kGroup;
    if ((reinterpret_cast<uintptr_t>(P) & 15) == 0) {  // pairs of pixels, 16-byte accesses
      dim3 grid((M * M / 2 + kPixBlock - 1) / kPixBlock, G);
      k_dP_terms2<<<grid, kPixBlock, 0, s>>>(Eb, O, P, tlb, B, W, M, part, done, dP, dO ? 1 : 0,
                                             accumulate ? 1 : 0, loss_pat, loss_total);
    } else {
      dim3 grid(dp_counters(M), G);
      k_dP_terms<<<grid, kPixBlock, 0, s>>>(Eb, O, P, tlb, B, W, M, part, done, dP, dO ? 1 : 0,
                                            accumulate ? 1 : 0, loss_pat, loss_total);
    }
  } else if (loss_total) {
    k_loss_total<<<1, 256, 0, s>>>(loss_pat, B, loss_total);
  }
  if (dO) {
    const int ntx = (W + kTile - 1) / kTile, nty = (H + kTile - 1) / kTile;
    k_dO<<<ntx * nty, 256, 0, s>>>(Eb, tlb, B, H, W, M, ntx, dO, accumulate ? 1 : 0);
  }
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // namespace pty
