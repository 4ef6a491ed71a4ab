// fwd_adj.cu -- fused far-field ptychography forward model, loss and adjoint.
//
// Replaces, for a batch of scan positions, the per-frame loop of
// Recovery.py:288-307 (crop * probe -> fft2 -> fftshift -> |.|^2 -> loss) and
// the autograd backward of Recovery.py:316, plus utils/optics.py:102-112
// (forward_imaging_model).  See include/ptycho_b200.h for the ABI.
//
// Kernel K1 (k_fused): one CTA per pattern.  The M x M exit wave lives in
// registers (E complex values per thread); the 2-D DFT is a decimation-in-
// frequency Cooley-Tukey over the 2*log2(M) position bits, done in three
// register passes with two shared-memory exchanges (re/im planes, padded
// pitch, conflict-free for each pass's lane mapping).  fftshift is folded in
// as a (-1)^(x+y) sign on the input.  The spectrum stays in digit-reversed
// order: the loss reads Imeas at the bit-permuted frequency index, and the
// adjoint runs the three passes backwards (conjugate twiddles, inverse
// radix kernels), which returns natural order -- no reorder pass.
// The exit-wave gradient E_b = dL/dpsi_b is written once to the workspace.
//
// K2 (deterministic gradient assembly, no floating-point atomics):
//   k_bin      -- per 32x32 canvas tile, the ordered list of patterns whose
//                 window overlaps it (ballot compaction, ascending b);
//   k_dO       -- per tile, dO = sum over its list of E_b * conj(P), in list order;
//   k_dP_part  -- per group of GS patterns, sum of E_b * conj(O_window_b);
//   k_dP_final -- fixed-order sum over groups (and the FP64 loss total).
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <type_traits>

#include "common.cuh"
#include "dft_regs.cuh"

namespace pty {

// ---------------------------------------------------------------------------
// pass plans
// ---------------------------------------------------------------------------
// Position bits: [0, LOGM) are x (column) bits, [LOGM, 2 LOGM) are y (row) bits.
struct PassDesc {
  int ne;        // element bits per thread (E = 1 << ne)
  int ebit[6];   // element bit j -> position bit; x-stage digit bits first,
                 // then y-stage digit bits, then repeat bits
  int nt;        // thread-index bits: 5 lane bits then warp bits
  int tbit[10];  // thread bit j -> position bit
  int nbx, lox;  // x DIF stage of this pass: digit width (0 = none), lowest bit
  int nby, loy;  // y DIF stage
};

struct FreqMap {
  int fx[8];  // x position bit -> x frequency bit
  int fy[8];  // y position bit -> y frequency bit
};

template <int M>
struct Plan;

// M = 64: x = 16 * 4, y = 4 * 16; 256 threads x 16 values.
template <>
struct Plan<64> {
  static constexpr int LOGM = 6, NT = 256, E = 16, PITCH = 65;
  static constexpr PassDesc P1 = {4, {2, 3, 4, 5}, 8, {0, 1, 8, 9, 10, 6, 7, 11}, 4, 2, 0, 0};
  static constexpr PassDesc P2 = {4, {0, 1, 10, 11}, 8, {6, 7, 2, 3, 4, 5, 8, 9}, 2, 0, 2, 4};
  static constexpr PassDesc P3 = {4, {6, 7, 8, 9}, 8, {0, 1, 2, 3, 4, 5, 10, 11}, 0, 0, 4, 0};
  // position bit -> frequency bit after all DIF stages (digit reversal)
  static constexpr FreqMap F = {{4, 5, 0, 1, 2, 3}, {2, 3, 4, 5, 0, 1}};
};

// M = 128: x = 16 * 8, y = 2 * 4 * 16; 512 threads x 32 values.
template <>
struct Plan<128> {
  static constexpr int LOGM = 7, NT = 512, E = 32, PITCH = 129;
  static constexpr PassDesc P1 = {5, {3, 4, 5, 6, 13}, 9, {0, 1, 2, 10, 11, 7, 8, 9, 12}, 4, 3, 1, 6};
  static constexpr PassDesc P2 = {5, {0, 1, 2, 11, 12}, 9, {7, 8, 9, 3, 4, 5, 6, 10, 13}, 3, 0, 2, 4};
  static constexpr PassDesc P3 = {5, {7, 8, 9, 10, 5}, 9, {0, 1, 2, 3, 4, 6, 11, 12, 13}, 0, 0, 4, 0};
  static constexpr FreqMap F = {{4, 5, 6, 0, 1, 2, 3}, {3, 4, 5, 6, 1, 2, 0}};
};

template <int M, int PASS>
__host__ __device__ constexpr PassDesc desc() {
  if constexpr (PASS == 1) return Plan<M>::P1;
  else if constexpr (PASS == 2) return Plan<M>::P2;
  else return Plan<M>::P3;
}

// compile-time x / y offset of element e within a pass
template <int M, int PASS>
__host__ __device__ constexpr int eoff_x(int e) {
  constexpr PassDesc d = desc<M, PASS>();
  int r = 0;
  for (int j = 0; j < d.ne; ++j)
    if (((e >> j) & 1) && d.ebit[j] < Plan<M>::LOGM) r += 1 << d.ebit[j];
  return r;
}
template <int M, int PASS>
__host__ __device__ constexpr int eoff_y(int e) {
  constexpr PassDesc d = desc<M, PASS>();
  int r = 0;
  for (int j = 0; j < d.ne; ++j)
    if (((e >> j) & 1) && d.ebit[j] >= Plan<M>::LOGM) r += 1 << (d.ebit[j] - Plan<M>::LOGM);
  return r;
}
// frequency index of a position (bit permutation from the DIF digit order)
template <int M>
__host__ __device__ constexpr int freq_x(int px) {
  constexpr FreqMap f = Plan<M>::F;
  int r = 0;
  for (int i = 0; i < Plan<M>::LOGM; ++i)
    if ((px >> i) & 1) r |= 1 << f.fx[i];
  return r;
}
template <int M>
__host__ __device__ constexpr int freq_y(int py) {
  constexpr FreqMap f = Plan<M>::F;
  int r = 0;
  for (int i = 0; i < Plan<M>::LOGM; ++i)
    if ((py >> i) & 1) r |= 1 << f.fy[i];
  return r;
}
// value of thread bit J in a pass: its x / y position weight (compile time)
template <int M, int PASS, int J>
__host__ __device__ constexpr int tw_x() {
  constexpr int pb = desc<M, PASS>().tbit[J];
  return pb < Plan<M>::LOGM ? (1 << pb) : 0;
}
template <int M, int PASS, int J>
__host__ __device__ constexpr int tw_y() {
  constexpr int pb = desc<M, PASS>().tbit[J];
  return pb >= Plan<M>::LOGM ? (1 << (pb - Plan<M>::LOGM)) : 0;
}
template <int M, int PASS, int... J>
PTY_DEVI void tbase_seq(int t, int& bx, int& by, std::integer_sequence<int, J...>) {
  bx = (0 | ... | (((t >> J) & 1) * tw_x<M, PASS, J>()));
  by = (0 | ... | (((t >> J) & 1) * tw_y<M, PASS, J>()));
}
// run-time thread base position (bx, by) of a pass
template <int M, int PASS>
PTY_DEVI void tbase(int t, int& bx, int& by) {
  tbase_seq<M, PASS>(t, bx, by, std::make_integer_sequence<int, desc<M, PASS>().nt>{});
}

// unrolled loop whose index is a compile-time constant
template <typename F, int... I>
PTY_DEVI void static_for_seq(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
PTY_DEVI void static_for(F&& f) {
  static_for_seq(f, std::make_integer_sequence<int, N>{});
}

// ---------------------------------------------------------------------------
// one DIF pass (forward) or its adjoint, on the register array v
// ---------------------------------------------------------------------------
template <int M, int E, bool ADJ, int RX, int RY, int LOX, int NBX, int LOY, int NBY>
PTY_DEVI void run_pass(float2 (&v)[E], int bx, int by, const float2* __restrict__ tw) {
  constexpr int LOGM = Plan<M>::LOGM;
  constexpr int REP = E / (RX * RY);
  static_assert(RX * RY * REP == E, "pass shape");
  // x stage -----------------------------------------------------------------
  if constexpr (RX > 1) {
    const int n2 = bx & ((1 << LOX) - 1);
    constexpr int SH = LOGM - LOX - NBX;
    if constexpr (!ADJ) {
#pragma unroll
      for (int j = 0; j < RY * REP; ++j) dft<RX, false, 1>(v + RX * j);
    }
    if constexpr (LOX > 0) {
#pragma unroll
      for (int k = 1; k < RX; ++k) {
        float2 w = tw[((n2 * k) << SH) & (M - 1)];
        if constexpr (ADJ) w.y = -w.y;
#pragma unroll
        for (int j = 0; j < RY * REP; ++j) v[k + RX * j] = c_mul(v[k + RX * j], w);
      }
    }
    if constexpr (ADJ) {
#pragma unroll
      for (int j = 0; j < RY * REP; ++j) dft<RX, true, 1>(v + RX * j);
    }
  }
  // y stage -----------------------------------------------------------------
  if constexpr (RY > 1) {
    const int n2 = by & ((1 << LOY) - 1);
    constexpr int SH = LOGM - LOY - NBY;
    if constexpr (!ADJ) {
#pragma unroll
      for (int r = 0; r < REP; ++r)
#pragma unroll
        for (int ix = 0; ix < RX; ++ix) dft<RY, false, RX>(v + ix + RX * RY * r);
    }
    if constexpr (LOY > 0) {
#pragma unroll
      for (int k = 1; k < RY; ++k) {
        float2 w = tw[((n2 * k) << SH) & (M - 1)];
        if constexpr (ADJ) w.y = -w.y;
#pragma unroll
        for (int r = 0; r < REP; ++r)
#pragma unroll
          for (int ix = 0; ix < RX; ++ix) {
            const int e = ix + RX * k + RX * RY * r;
            v[e] = c_mul(v[e], w);
          }
      }
    }
    if constexpr (ADJ) {
#pragma unroll
      for (int r = 0; r < REP; ++r)
#pragma unroll
        for (int ix = 0; ix < RX; ++ix) dft<RY, true, RX>(v + ix + RX * RY * r);
    }
  }
}

template <int M, bool ADJ, int PASS>
PTY_DEVI void pass(float2 (&v)[Plan<M>::E], int t, const float2* __restrict__ tw) {
  constexpr PassDesc d = desc<M, PASS>();
  int bx, by;
  tbase<M, PASS>(t, bx, by);
  run_pass<M, Plan<M>::E, ADJ, (1 << d.nbx), (1 << d.nby), d.lox, d.nbx, d.loy, d.nby>(v, bx, by, tw);
}

// write v (layout PA) to the re/im planes, barrier, read back in layout PB
template <int M, int PA, int PB>
PTY_DEVI void exchange(float2 (&v)[Plan<M>::E], int t, float* re, float* im) {
  constexpr int PITCH = Plan<M>::PITCH, E = Plan<M>::E;
  int ax, ay, bx, by;
  tbase<M, PA>(t, ax, ay);
  tbase<M, PB>(t, bx, by);
  float* rea = re + ay * PITCH + ax;
  float* ima = im + ay * PITCH + ax;
  const float* reb = re + by * PITCH + bx;
  const float* imb = im + by * PITCH + bx;
  __syncthreads();  // previous readers of the planes are done
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    constexpr int off = eoff_y<M, PA>(e) * PITCH + eoff_x<M, PA>(e);
    rea[off] = v[e].x;
    ima[off] = v[e].y;
  });
  __syncthreads();
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    constexpr int off = eoff_y<M, PB>(e) * PITCH + eoff_x<M, PB>(e);
    v[e] = make_float2(reb[off], imb[off]);
  });
}

// frequency-index base of a thread in the pass-3 layout: fold over thread bits
template <int M, int... J>
PTY_DEVI void fbase_seq(int t, int& fx, int& fy, std::integer_sequence<int, J...>) {
  fx = (0 | ... | (((t >> J) & 1) * freq_x<M>(tw_x<M, 3, J>())));
  fy = (0 | ... | (((t >> J) & 1) * freq_y<M>(tw_y<M, 3, J>())));
}
template <int M>
PTY_DEVI void fbase(int t, int& fx, int& fy) {
  fbase_seq<M>(t, fx, fy, std::make_integer_sequence<int, desc<M, 3>().nt>{});
}
// frequency-index offset of element e in the pass-3 layout (compile time)
template <int M>
__host__ __device__ constexpr int efreq(int e, int pitch) {
  return freq_y<M>(eoff_y<M, 3>(e)) * pitch + freq_x<M>(eoff_x<M, 3>(e));
}

// ---------------------------------------------------------------------------
// loss: value (accumulated in FP64) and v <- 2 * dL/dI * v
// ---------------------------------------------------------------------------
constexpr float kEps = 1e-8f;

template <int M>
PTY_DEVI double loss_pointwise(float2 (&v)[Plan<M>::E], int t, const float* __restrict__ Im_b,
                               int loss_type, float* re, float* im) {
  constexpr int E = Plan<M>::E, PITCH = Plan<M>::PITCH;
  constexpr float inv_mn = 1.0f / float(M * M);
  int fx0, fy0;
  fbase<M>(t, fx0, fy0);
  const float* Ib = Im_b + fy0 * M + fx0;  // pitch M in global memory
  double acc = 0.0;
  if (loss_type == PTYCHO_LOSS_INTENSITY_GRAD) {
    // upstream dL/dI given directly: G_F = 2 * dL/dI * F
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const float g = __ldg(Ib + efreq<M>(e, M));
      const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      acc += (double)(I * g);
      v[e] = c_scale(v[e], 2.0f * g);
    });
    return acc * double(M * M);  // caller divides by M*M
  }
  if (loss_type == PTYCHO_LOSS_SMOOTH_L1 || loss_type == PTYCHO_LOSS_POISSON) {
    const bool l1 = loss_type == PTYCHO_LOSS_SMOOTH_L1;
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const float meas = __ldg(Ib + efreq<M>(e, M));
      const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      float l, g;
      if (l1) {
        const float dd = I - meas;
        const float ad = fabsf(dd);
        l = ad < 1.0f ? 0.5f * dd * dd : ad - 0.5f;
        g = ad < 1.0f ? dd : copysignf(1.0f, dd);
      } else {
        const float Ie = I + kEps;
        l = I - meas * logf(Ie);
        g = 1.0f - meas / Ie;
      }
      acc += (double)l;
      v[e] = c_scale(v[e], 2.0f * g * inv_mn);
    });
  } else {  // FD (gradient-difference) loss: 5-point circular stencil via smem
    // natural (fy, fx) layout in the planes, pitch PITCH
    float q[E];
    const int sb = fy0 * PITCH + fx0;
    __syncthreads();
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const float meas = __ldg(Ib + efreq<M>(e, M));
      const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      im[sb + efreq<M>(e, PITCH)] = sqrtf(meas + kEps) - sqrtf(I + kEps);  // dW
    });
    __syncthreads();
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      constexpr int fxe = freq_x<M>(eoff_x<M, 3>(e)), fye = freq_y<M>(eoff_y<M, 3>(e));
      const int fx = fx0 | fxe, fy = fy0 | fye;
      const float dw = im[fy * PITCH + fx];
      const float rx = im[fy * PITCH + ((fx + 1) & (M - 1))] - dw;
      const float ry = im[((fy + 1) & (M - 1)) * PITCH + fx] - dw;
      const float G = sqrtf(fmaf(rx, rx, fmaf(ry, ry, kEps)));
      acc += (double)G;
      re[fy * PITCH + fx] = rx / G;
      q[e] = ry / G;
    });
    __syncthreads();
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      constexpr int fxe = freq_x<M>(eoff_x<M, 3>(e)), fye = freq_y<M>(eoff_y<M, 3>(e));
      const int fx = fx0 | fxe, fy = fy0 | fye;
      im[fy * PITCH + fx] = q[e];
      q[e] = re[fy * PITCH + ((fx - 1) & (M - 1))] - re[fy * PITCH + fx];
    });
    __syncthreads();
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      constexpr int fxe = freq_x<M>(eoff_x<M, 3>(e)), fye = freq_y<M>(eoff_y<M, 3>(e));
      const int fx = fx0 | fxe, fy = fy0 | fye;
      const float dl = (q[e] + im[((fy - 1) & (M - 1)) * PITCH + fx] - im[fy * PITCH + fx]) * inv_mn;
      const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      const float g = dl * (-0.5f / sqrtf(I + kEps));
      v[e] = c_scale(v[e], 2.0f * g);
    });
  }
  return acc;
}

// deterministic block sum of one double per thread (fixed shuffle tree, then
// warp partials in warp order); result valid in thread 0
template <int NT>
PTY_DEVI double block_sum(double x, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) s += red[i];
  }
  return s;
}

enum { MODE_INTENSITY = 0, MODE_LOSS = 1, MODE_ADJ = 2 };

template <int M>
constexpr size_t fused_smem_bytes() {
  return size_t(2) * M * Plan<M>::PITCH * sizeof(float) + size_t(M) * sizeof(float2) +
         size_t(Plan<M>::NT / 32) * sizeof(double);
}

template <int M, int MODE>
__global__ void __launch_bounds__(Plan<M>::NT, 1)
    k_fused(const float2* __restrict__ O, int H, int W, const float2* __restrict__ P,
            const int2* __restrict__ tl, const float* __restrict__ Imeas, int F,
            const int* __restrict__ batch, int loss_type, float* __restrict__ I_out,
            double* __restrict__ loss_pat, float2* __restrict__ Eout, int2* __restrict__ tlb,
            int32_t* status) {
  using PL = Plan<M>;
  constexpr int E = PL::E, NT = PL::NT, PITCH = PL::PITCH;
  extern __shared__ __align__(16) float smem[];
  float* re = smem;
  float* im = smem + M * PITCH;
  float2* tw = reinterpret_cast<float2*>(smem + 2 * M * PITCH);
  double* red = reinterpret_cast<double*>(tw + M);

  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const int f = batch ? batch[b] : b;  // frame id
  const int2 c = (f >= 0 && f < F) ? tl[f] : make_int2(-1, -1);  // (tlY, tlX)
  const bool ok = f >= 0 && f < F && c.x >= 0 && c.y >= 0 && c.x <= H - M && c.y <= W - M;
  if constexpr (MODE == MODE_ADJ) {
    if (t == 0) tlb[b] = ok ? c : make_int2(-1, -1);  // resolved windows for the assembly
  }
  if (!ok) {  // uniform across the block
    if (t == 0) pty_raise(status, PTYCHO_ERR_WINDOW);
    const float nan = __int_as_float(0x7fc00000);
    if constexpr (MODE == MODE_INTENSITY) {
      for (int i = t; i < M * M; i += NT) I_out[size_t(b) * M * M + i] = nan;
    } else {
      if (t == 0 && loss_pat) loss_pat[b] = (double)nan;
      if constexpr (MODE == MODE_ADJ)
        for (int i = t; i < M * M; i += NT) Eout[size_t(b) * M * M + i] = make_float2(0.f, 0.f);
    }
    return;
  }

  // twiddle table W_M^j = exp(-2 pi i j / M), rounded from double precision
  for (int j = t; j < M; j += NT) {
    double s, co;
    sincospi(-2.0 * double(j) / double(M), &s, &co);
    tw[j] = make_float2((float)co, (float)s);
  }

  float2 v[E];
  // ---- pass 1: gather window, multiply by probe, fftshift sign -----------
  {
    int bx, by;
    tbase<M, 1>(t, bx, by);
    const float2* Ob = O + size_t(c.x + by) * W + (c.y + bx);
    const float2* Pb = P + by * M + bx;
    const int par = (bx + by) & 1;
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      constexpr int ox = eoff_x<M, 1>(e), oy = eoff_y<M, 1>(e);
      const float2 o = __ldg(Ob + size_t(oy) * W + ox);
      const float2 p = __ldg(Pb + oy * M + ox);
      const float2 psi = c_mul(p, o);
      const int sgn = par ^ ((ox + oy) & 1);
      v[e] = sgn ? make_float2(-psi.x, -psi.y) : psi;
    });
  }
  __syncthreads();  // twiddle table ready
  pass<M, false, 1>(v, t, tw);
  exchange<M, 1, 2>(v, t, re, im);
  pass<M, false, 2>(v, t, tw);
  exchange<M, 2, 3>(v, t, re, im);
  pass<M, false, 3>(v, t, tw);

  if constexpr (MODE == MODE_INTENSITY) {
    int fx0, fy0;
    fbase<M>(t, fx0, fy0);
    float* Ib = I_out + size_t(b) * M * M + fy0 * M + fx0;
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      Ib[efreq<M>(e, M)] = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
    });
    return;
  } else {
    const double acc = loss_pointwise<M>(v, t, Imeas + size_t(f) * M * M, loss_type, re, im);
    const double tot = block_sum<NT>(acc, red);
    if (t == 0 && loss_pat) loss_pat[b] = tot / double(M * M);
    if constexpr (MODE == MODE_ADJ) {
      pass<M, true, 3>(v, t, tw);
      exchange<M, 3, 2>(v, t, re, im);
      pass<M, true, 2>(v, t, tw);
      exchange<M, 2, 1>(v, t, re, im);
      pass<M, true, 1>(v, t, tw);
      int bx, by;
      tbase<M, 1>(t, bx, by);
      float2* Eb = Eout + size_t(b) * M * M + by * M + bx;
      const int par = (bx + by) & 1;
      static_for<E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        constexpr int ox = eoff_x<M, 1>(e), oy = eoff_y<M, 1>(e);
        const int sgn = par ^ ((ox + oy) & 1);
        Eb[oy * M + ox] = sgn ? make_float2(-v[e].x, -v[e].y) : v[e];
      });
    }
  }
}

// ---------------------------------------------------------------------------
// K2: deterministic gradient assembly
// ---------------------------------------------------------------------------
constexpr int kTile = 32;     // canvas tile edge for dO
constexpr int kGroup = 16;    // patterns per dP partial sum

// resolved windows (from k_fused): (-1, -1) marks a skipped pattern
PTY_DEVI bool window_ok(int2 c) { return c.x >= 0; }

// per tile: ascending list of overlapping valid patterns
__global__ void __launch_bounds__(256) k_bin(const int2* __restrict__ tl, int B, int H, int W, int M,
                                             int ntx, int* __restrict__ list, int* __restrict__ cnt) {
  __shared__ int wsum[8];
  const int tile = blockIdx.x;
  const int ty0 = (tile / ntx) * kTile, tx0 = (tile % ntx) * kTile;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int base = 0;
  int* out = list + size_t(tile) * B;
  for (int b0 = 0; b0 < B; b0 += 256) {
    const int b = b0 + threadIdx.x;
    bool hit = false;
    if (b < B) {
      const int2 c = tl[b];
      hit = window_ok(c) && c.x < ty0 + kTile && c.x + M > ty0 && c.y < tx0 + kTile &&
            c.y + M > tx0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) wsum[w] = __popc(m);
    __syncthreads();
    int off = base;
    for (int i = 0; i < w; ++i) off += wsum[i];
    int tot = 0;
    for (int i = 0; i < 8; ++i) tot += wsum[i];
    if (hit) out[off + __popc(m & ((1u << lane) - 1u))] = b;
    base += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) cnt[tile] = base;
}

// dO over one 32x32 tile: 256 threads, 4 rows each
__global__ void __launch_bounds__(256) k_dO(const float2* __restrict__ Eb, const float2* __restrict__ P,
                                            const int2* __restrict__ tl, int B, int H, int W, int M,
                                            int ntx, const int* __restrict__ list,
                                            const int* __restrict__ cnt, float2* __restrict__ dO,
                                            int accumulate) {
  const int tile = blockIdx.x;
  const int ty0 = (tile / ntx) * kTile, tx0 = (tile % ntx) * kTile;
  const int X = tx0 + (threadIdx.x & 31);
  const int Y0 = ty0 + (threadIdx.x >> 5);
  float2 acc[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) acc[j] = make_float2(0.f, 0.f);
  const int n = cnt[tile];
  const int* lst = list + size_t(tile) * B;
  for (int i = 0; i < n; ++i) {
    const int b = lst[i];
    const int2 c = __ldg(tl + b);
    const int lx = X - c.y;
    const float2* Ep = Eb + size_t(b) * M * M;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int ly = Y0 + 8 * j - c.x;
      if (lx >= 0 && lx < M && ly >= 0 && ly < M) {
        const float2 e = __ldg(Ep + ly * M + lx);
        const float2 p = __ldg(P + ly * M + lx);
        acc[j] = c_add(acc[j], c_mulc(e, p));
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int Y = Y0 + 8 * j;
    if (Y < H && X < W) {
      float2* o = dO + size_t(Y) * W + X;
      *o = accumulate ? c_add(*o, acc[j]) : acc[j];
    }
  }
}

// dP partial sums over groups of kGroup patterns
__global__ void __launch_bounds__(256) k_dP_part(const float2* __restrict__ Eb, const float2* __restrict__ O,
                                                 const int2* __restrict__ tl, int B, int H, int W, int M,
                                                 float2* __restrict__ part) {
  const int idx = blockIdx.x * 256 + threadIdx.x;
  const int g = blockIdx.y;
  if (idx >= M * M) return;
  const int y = idx / M, x = idx - (idx / M) * M;
  float2 acc = make_float2(0.f, 0.f);
  const int b1 = min(B, (g + 1) * kGroup);
  for (int b = g * kGroup; b < b1; ++b) {
    const int2 c = __ldg(tl + b);
    if (!window_ok(c)) continue;
    const float2 e = __ldg(Eb + size_t(b) * M * M + idx);
    const float2 o = __ldg(O + size_t(c.x + y) * W + c.y + x);
    acc = c_add(acc, c_mulc(e, o));
  }
  part[size_t(g) * M * M + idx] = acc;
}

// dP = sum of group partials in group order; block 0 also sums the loss
__global__ void __launch_bounds__(256) k_dP_final(const float2* __restrict__ part, int G, int M,
                                                  float2* __restrict__ dP, int accumulate,
                                                  const double* __restrict__ loss_pat, int B,
                                                  double* __restrict__ loss_total) {
  const int idx = blockIdx.x * 256 + threadIdx.x;
  if (dP && idx < M * M) {
    float2 acc = make_float2(0.f, 0.f);
    for (int g = 0; g < G; ++g) acc = c_add(acc, part[size_t(g) * M * M + idx]);
    dP[idx] = accumulate ? c_add(dP[idx], acc) : acc;
  }
  if (blockIdx.x == 0 && loss_total) {
    __shared__ double red[8];
    double s = 0.0;
    for (int b = threadIdx.x; b < B; b += 256) s += loss_pat[b];
    s = block_sum<256>(s, red);
    if (threadIdx.x == 0) loss_total[0] = s;
  }
}

__global__ void k_zero2(float2* p, size_t n) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) p[i] = make_float2(0.f, 0.f);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct WsLayout {
  size_t E, list, cnt, part, loss, tlb, total;
};

static WsLayout ws_layout(int H, int W, int M, int B) {
  const size_t ntiles = size_t((H + kTile - 1) / kTile) * ((W + kTile - 1) / kTile);
  const size_t G = (size_t(B) + kGroup - 1) / kGroup;
  WsLayout L;
  size_t off = 0;
  L.E = off;
  off += pty_align_up(size_t(B) * M * M * sizeof(float2), 256);
  L.list = off;
  off += pty_align_up(ntiles * size_t(B) * sizeof(int), 256);
  L.cnt = off;
  off += pty_align_up(ntiles * sizeof(int), 256);
  L.part = off;
  off += pty_align_up(G * M * M * sizeof(float2), 256);
  L.loss = off;
  off += pty_align_up(size_t(B) * sizeof(double), 256);
  L.tlb = off;
  off += pty_align_up(size_t(B) * sizeof(int2), 256);
  L.total = off;
  return L;
}

static int check_common(const float* O, int H, int W, const float* P, int M, int N, const int32_t* tl,
                        int F, const int32_t* batch, int B) {
  if (!O || !P || (B > 0 && !tl) || H <= 0 || W <= 0 || B < 0 || F < 0) return PTYCHO_ERR_INVALID_ARG;
  if (!batch && B > F) return PTYCHO_ERR_INVALID_ARG;
  if (M != N || (M != 64 && M != 128)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (H < M || W < M) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(O, 8) || !pty_aligned(P, 8) || !pty_aligned(tl, 8) || !pty_aligned(batch, 4))
    return PTYCHO_ERR_MISALIGNED;
  return PTYCHO_OK;
}

template <int M, int MODE>
static int launch_fused(const float* O, int H, int W, const float* P, const int32_t* tl,
                        const float* Imeas, int F, const int32_t* batch, int B, int loss_type,
                        float* I_out, double* loss_pat, float2* Eout, int2* tlb, int32_t* status,
                        cudaStream_t s) {
  constexpr size_t smem = fused_smem_bytes<M>();
  auto kern = k_fused<M, MODE>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return PTYCHO_ERR_LAUNCH;
  kern<<<B, Plan<M>::NT, smem, s>>>(reinterpret_cast<const float2*>(O), H, W,
                                    reinterpret_cast<const float2*>(P),
                                    reinterpret_cast<const int2*>(tl), Imeas, F, batch, loss_type,
                                    I_out, loss_pat, Eout, tlb, status);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
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

int ptycho_version(void) { return 100; }

int ptycho_forward_intensity(const float* O, int H, int W, const float* P, int M, int N,
                             const int32_t* tl, int F, const int32_t* batch, int B, float* I_out,
                             int32_t* status_out, ptycho_stream_t stream) {
  int st = check_common(O, H, W, P, M, N, tl, F, batch, B);
  if (st) return st;
  if (B == 0) return PTYCHO_OK;
  if (!I_out) return PTYCHO_ERR_INVALID_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (M == 64)
    return launch_fused<64, MODE_INTENSITY>(O, H, W, P, tl, nullptr, F, batch, B, 0, I_out, nullptr,
                                            nullptr, nullptr, status_out, s);
  return launch_fused<128, MODE_INTENSITY>(O, H, W, P, tl, nullptr, F, batch, B, 0, I_out, nullptr,
                                           nullptr, nullptr, status_out, s);
}

size_t ptycho_fwd_adj_workspace_size(int H, int W, int M, int N, int B) {
  if (H <= 0 || W <= 0 || M <= 0 || N <= 0 || B < 0) return 0;
  return ws_layout(H, W, M, B).total;
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
  if ((dO && !pty_aligned(dO, 8)) || (dP && !pty_aligned(dP, 8))) return PTYCHO_ERR_MISALIGNED;
  const WsLayout L = ws_layout(H, W, M, B);
  if (!workspace || workspace_bytes < L.total) return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(workspace, 256)) return PTYCHO_ERR_MISALIGNED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const bool acc = (flags & PTYCHO_FLAG_ACCUMULATE) != 0;
  char* ws = static_cast<char*>(workspace);
  float2* Ews = reinterpret_cast<float2*>(ws + L.E);
  int* list = reinterpret_cast<int*>(ws + L.list);
  int* cnt = reinterpret_cast<int*>(ws + L.cnt);
  float2* part = reinterpret_cast<float2*>(ws + L.part);
  double* lp = loss_per_pattern ? loss_per_pattern : reinterpret_cast<double*>(ws + L.loss);
  int2* tlb = reinterpret_cast<int2*>(ws + L.tlb);

  if (B == 0) {  // empty batch: zero gradients and loss
    if (!acc) {
      if (dO) cudaMemsetAsync(dO, 0, size_t(H) * W * sizeof(float2), s);
      if (dP) cudaMemsetAsync(dP, 0, size_t(M) * M * sizeof(float2), s);
    }
    if (loss_total) cudaMemsetAsync(loss_total, 0, sizeof(double), s);
    return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
  }
  const bool adj = dO || dP;
  if (adj) {
    st = M == 64 ? launch_fused<64, MODE_ADJ>(O, H, W, P, tl, Imeas, F, batch, B, loss_type, nullptr,
                                               lp, Ews, tlb, status_out, s)
                 : launch_fused<128, MODE_ADJ>(O, H, W, P, tl, Imeas, F, batch, B, loss_type, nullptr,
                                                lp, Ews, tlb, status_out, s);
  } else {
    st = M == 64 ? launch_fused<64, MODE_LOSS>(O, H, W, P, tl, Imeas, F, batch, B, loss_type, nullptr,
                                                lp, nullptr, nullptr, status_out, s)
                 : launch_fused<128, MODE_LOSS>(O, H, W, P, tl, Imeas, F, batch, B, loss_type, nullptr,
                                                 lp, nullptr, nullptr, status_out, s);
  }
  if (st) return st;
  const int2* tl2 = tlb;
  if (dO) {
    const int ntx = (W + kTile - 1) / kTile, nty = (H + kTile - 1) / kTile;
    k_bin<<<ntx * nty, 256, 0, s>>>(tl2, B, H, W, M, ntx, list, cnt);
    k_dO<<<ntx * nty, 256, 0, s>>>(Ews, reinterpret_cast<const float2*>(P), tl2, B, H, W, M, ntx, list,
                                   cnt, reinterpret_cast<float2*>(dO), acc ? 1 : 0);
  }
  const int G = (B + kGroup - 1) / kGroup;
  if (dP) {
    dim3 grid((M * M + 255) / 256, G);
    k_dP_part<<<grid, 256, 0, s>>>(Ews, reinterpret_cast<const float2*>(O), tl2, B, H, W, M, part);
  }
  if (dP || loss_total) {
    k_dP_final<<<dP ? (M * M + 255) / 256 : 1, 256, 0, s>>>(part, G, M, reinterpret_cast<float2*>(dP),
                                                            acc ? 1 : 0, lp, B, loss_total);
  }
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // extern "C"
