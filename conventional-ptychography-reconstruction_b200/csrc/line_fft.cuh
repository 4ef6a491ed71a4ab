// line_fft.cuh -- batched DFTs of any length along lines held in shared memory.
//
// A LinePlan factors the length L into Stockham passes: powers of two as
// radix 16, 8, 4, 2, then 3, 5, 7 (register butterflies, dft_regs.cuh), and
// every other prime factor p as a direct p-term sum per output with table
// twiddles.  Passes ping-pong between two shared-memory buffers of float2 with
// one float2 of padding every 16 (pad16: breaks the stride-2^k bank conflicts
// of the first passes); natural order in and out.  Twiddles come from a table
// exp(-2 pi i j / LMAX) that a length-L pass reads with stride LMAX / L (L
// divides LMAX).  `transform` runs all passes over `lines` lines of padded
// stride `ls` with kLineNT threads and returns the buffer holding the result.
#pragma once
#include "common.cuh"
#include "dft_regs.cuh"

namespace pty {
namespace lfft {

constexpr int kLineNT = 512;
constexpr int kMaxFactors = 16;
constexpr int kMaxLen = 8192;

struct LinePlan {
  int L;
  int nf;
  int radix[kMaxFactors];
};

// factor L into passes: powers of two as 16, 8, 4, 2; then 3, 5, 7; any
// other prime factor gets its own direct-sum pass
inline bool make_plan(int L, LinePlan* p) {
  if (L < 1 || L > kMaxLen) return false;
  p->L = L;
  p->nf = 0;
  int r = L;
  auto push = [&](int f) {
    if (p->nf >= kMaxFactors) return false;
    p->radix[p->nf++] = f;
    r /= f;
    return true;
  };
  for (int f : {16, 8, 4, 2})
    while (r % f == 0)
      if (!push(f)) return false;
  for (int f : {3, 5, 7})
    while (r % f == 0)
      if (!push(f)) return false;
  for (int f = 11; r > 1; f += 2)
    while (r % f == 0)
      if (!push(f)) return false;
  return true;
}

__host__ __device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }

template <int R, bool INV>
PTY_DEVI void pass_r(const float2* __restrict__ src, float2* __restrict__ dst, const float2* __restrict__ tw,
                     int L, int NS, int lines, int ls, int lmax, int t) {
  const int bpl = L / R;
  const int tws = lmax / (NS * R);
  for (int b = t; b < lines * bpl; b += kLineNT) {
    const int line = b / bpl, j = b - line * bpl;
    const int k = j % NS;
    const float2* sl = src + line * ls;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = sl[pad16(j + r * bpl)];
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[k * r * tws];
        if (INV) w.y = -w.y;
        v[r] = c_mul(v[r], w);
      }
    }
    dft<R, INV, 1>(v);
    float2* dl = dst + line * ls;
    const int o = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dl[pad16(o + r * NS)] = v[r];
  }
}

// direct sum for a prime factor p: output o = (j / NS) NS p + k + r NS gets
// sum_m x[j + m L/p] exp(-+2 pi i m (k + r NS) / (NS p))
template <bool INV>
PTY_DEVI void pass_generic(const float2* __restrict__ src, float2* __restrict__ dst, const float2* __restrict__ tw,
                           int L, int p, int NS, int lines, int ls, int lmax, int t) {
  const int bpl = L / p;
  const int blk = NS * p;
  const int tws = lmax / blk;
  for (int e = t; e < lines * L; e += kLineNT) {
    const int line = e / L, o = e - line * L;
    const int ob = o / blk, rem = o - ob * blk;
    const int r = rem / NS, k = rem - r * NS;
    const int j = ob * NS + k;
    const int q = (k + r * NS) * tws;  // < lmax
    const float2* sl = src + line * ls;
    float2 acc = make_float2(0.f, 0.f);
    int idx = 0;
    for (int m = 0; m < p; ++m) {
      float2 w = tw[idx];
      if (INV) w.y = -w.y;
      const float2 x = sl[pad16(j + m * bpl)];
      acc.x = fmaf(x.x, w.x, fmaf(-x.y, w.y, acc.x));
      acc.y = fmaf(x.x, w.y, fmaf(x.y, w.x, acc.y));
      idx += q;
      if (idx >= lmax) idx -= lmax;
    }
    dst[line * ls + pad16(o)] = acc;
  }
}

template <bool INV>
PTY_DEVI void run_pass(int R, const float2* src, float2* dst, const float2* tw, int L, int NS, int lines, int ls,
                       int lmax, int t) {
  switch (R) {
    case 2: pass_r<2, INV>(src, dst, tw, L, NS, lines, ls, lmax, t); break;
    case 3: pass_r<3, INV>(src, dst, tw, L, NS, lines, ls, lmax, t); break;
    case 4: pass_r<4, INV>(src, dst, tw, L, NS, lines, ls, lmax, t); break;
    case 5: pass_r<5, INV>(src, dst, tw, L, NS, lines, ls, lmax, t); break;
    case 7: pass_r<7, INV>(src, dst, tw, L, NS, lines, ls, lmax, t); break;
    case 8: pass_r<8, INV>(src, dst, tw, L, NS, lines, ls, lmax, t); break;
    case 16: pass_r<16, INV>(src, dst, tw, L, NS, lines, ls, lmax, t); break;
    default: pass_generic<INV>(src, dst, tw, L, R, NS, lines, ls, lmax, t); break;
  }
}

// all passes of one plan; returns the buffer that holds the result
template <bool INV>
PTY_DEVI float2* transform(const LinePlan& pl, float2* a, float2* b, const float2* tw, int lines, int ls, int lmax,
                           int t) {
  int NS = 1;
  for (int i = 0; i < pl.nf; ++i) {
    const int R = pl.radix[i];
    run_pass<INV>(R, a, b, tw, pl.L, NS, lines, ls, lmax, t);
    __syncthreads();
    NS *= R;
    float2* c = a;
    a = b;
    b = c;
  }
  return a;
}

}  // namespace lfft
}  // namespace pty
