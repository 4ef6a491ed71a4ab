// fused.cuh -- persistent fused forward / loss / adjoint kernel for one probe size.
//
// Replaces, per pattern, Recovery.py:290-305 (crop * probe -> fft2 -> fftshift
// -> |.|^2 -> loss) and the autograd backward of Recovery.py:316 down to the
// exit wave; utils/optics.py:102-112 in MODE_INTENSITY.
//
// One CTA per SM loops over patterns b = blockIdx.x, blockIdx.x + gridDim.x, ...
// While pattern b is computed, the measurement of the CTA's next pattern is
// copied global -> shared by a TMA bulk copy (mbarrier-tracked, bounded wait)
// and its object window is prefetched into L2, so the next gather and loss
// read warm data.  Per pattern:
//   pass 1: v = (-1)^(x+y) P * O[window]  (fftshift folded in as a sign)
//   3 DIF passes + 2 shared-memory exchanges -> spectrum F (digit-reversed)
//   loss on I = |F|^2 against Imeas (read from shared memory at the permuted
//   frequency index), FP64 accumulation; v <- 2 * dL/dI * F
//   3 adjoint passes + 2 exchanges -> E'_b = (-1)^(x+y) dL/dpsi_b, written once
#pragma once
#include "async_copy.cuh"
#include "fft_plan.cuh"

namespace pty {

enum { MODE_INTENSITY = 0, MODE_LOSS = 1, MODE_ADJ = 2 };

struct FusedArgs {
  const float2* O;
  int H, W;
  const float2* P;   // probe [M][M]
  const int2* tl;    // [F] windows (tlY, tlX)
  const float* Imeas;  // [F][M][M]
  int F;
  const int* batch;  // [B] frame ids or nullptr
  int B;
  float* I_out;       // [B][M][M]        (MODE_INTENSITY)
  double* loss_pat;   // [B]              (MODE_LOSS / MODE_ADJ)
  float2* Eout;       // [B][M][M]        (MODE_ADJ)
  int2* tlb;          // [B] resolved windows, (-1,-1) = skipped (MODE_ADJ)
  unsigned* done;     // dP arrival counters to zero (MODE_ADJ), or nullptr
  int ndone;
  int32_t* status;
};

constexpr float kEps = 1e-8f;

template <int M>
struct FusedSmem {
  static constexpr int PITCH = Plan<M>::PITCH, NT = Plan<M>::NT;
  static constexpr size_t re = 0;
  static constexpr size_t im = re + size_t(M) * PITCH * 4;
  static constexpr size_t meas = pty_align_up_c(im + size_t(M) * PITCH * 4, 16);
  static constexpr size_t tw = meas + size_t(M) * M * 4;
  static constexpr size_t red = tw + size_t(M) * 8;
  static constexpr size_t bar = red + size_t(NT / 32) * 8;
  static constexpr size_t total = bar + 16;
};

template <int M>
PTY_DEVI bool resolve(const FusedArgs& a, int b, int& f, int2& c) {
  f = a.batch ? __ldg(a.batch + b) : b;
  if (f < 0 || f >= a.F) {
    c = make_int2(-1, -1);
    return false;
  }
  c = __ldg(a.tl + f);
  return c.x >= 0 && c.y >= 0 && c.x <= a.H - M && c.y <= a.W - M;
}

// threads < M prefetch one object row of pattern nb's window into L2
template <int M>
PTY_DEVI void prefetch_window(const FusedArgs& a, int nb, int t) {
  int f;
  int2 c;
  if (t < M && resolve<M>(a, nb, f, c)) {
    const char* row = reinterpret_cast<const char*>(a.O + size_t(c.x + t) * a.W + c.y);
    prefetch_l2_range(row, row + M * sizeof(float2), reinterpret_cast<const char*>(a.O),
                      reinterpret_cast<const char*>(a.O + size_t(a.H) * a.W));
  }
}

// thread 0 starts the bulk copy of pattern nb's measurement into shared memory
template <int M>
PTY_DEVI void fetch_meas(const FusedArgs& a, int nb, float* sm, uint64_t* bar) {
  int f;
  int2 c;
  if (resolve<M>(a, nb, f, c)) {
    mbar_arrive_expect_tx(bar, M * M * 4);
    bulk_g2s(sm, a.Imeas + size_t(f) * M * M, M * M * 4, bar);
  }
}

// per-element loss and v <- 2 dL/dI v; returns the thread's FP64 partial sum
template <int M, int LOSS>
PTY_DEVI double loss_pointwise(float2 (&v)[Plan<M>::E], int t, const float* sm, float* re, float* im) {
  constexpr int E = Plan<M>::E, PITCH = Plan<M>::PITCH;
  constexpr float inv_mn = 1.0f / float(M * M);
  int fx0, fy0;
  fbase<M>(t, fx0, fy0);
  const float* Ib = sm + fy0 * M + fx0;
  float part[E];  // per-element loss terms, summed pairwise (fixed order) then in FP64
  if constexpr (LOSS == PTYCHO_LOSS_INTENSITY_GRAD) {
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const float g = Ib[efreq<M>(e, M)];
      const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      part[e] = I * g * float(M * M);
      v[e] = c_scale(v[e], 2.0f * g);
    });
  } else if constexpr (LOSS == PTYCHO_LOSS_SMOOTH_L1 || LOSS == PTYCHO_LOSS_POISSON) {
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const float meas = Ib[efreq<M>(e, M)];
      const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      float g;
      if constexpr (LOSS == PTYCHO_LOSS_SMOOTH_L1) {
        const float dd = I - meas;
        const float ad = fabsf(dd);
        part[e] = ad < 1.0f ? 0.5f * dd * dd : ad - 0.5f;
        g = ad < 1.0f ? dd : copysignf(1.0f, dd);
      } else {
        const float Ie = I + kEps;
        part[e] = fmaf(-meas, __logf(Ie), I);
        g = 1.0f - __fdividef(meas, Ie);
      }
      v[e] = c_scale(v[e], 2.0f * g * inv_mn);
    });
  } else {  // FD: 5-point circular stencil over the natural frequency grid (planes, pitch PITCH)
    float q[E];
    const int sb = fy0 * PITCH + fx0;
    __syncthreads();
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const float meas = Ib[efreq<M>(e, M)];
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
      part[e] = G;
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
  // pairwise tree over the E terms (fixed order), then one FP64 conversion
#pragma unroll
  for (int w = 1; w < E; w <<= 1)
#pragma unroll
    for (int i = 0; i < E; i += 2 * w) part[i] += part[i + w];
  return (double)part[0];
}

// deterministic block sum (fixed shuffle tree, then warp partials in order);
// the result is valid in thread 0; contains two barriers
template <int NT>
PTY_DEVI double block_sum(double x, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) s += red[i];
  }
  return s;
}

template <int M, int MODE, int LOSS>
__global__ void __launch_bounds__(Plan<M>::NT, Plan<M>::MIN_BLOCKS) k_fused(const FusedArgs a) {
  using PL = Plan<M>;
  using SM = FusedSmem<M>;
  constexpr int E = PL::E, NT = PL::NT;
  extern __shared__ __align__(16) unsigned char smem[];
  float* re = reinterpret_cast<float*>(smem + SM::re);
  float* im = reinterpret_cast<float*>(smem + SM::im);
  float* sm = reinterpret_cast<float*>(smem + SM::meas);
  float2* tw = reinterpret_cast<float2*>(smem + SM::tw);
  double* red = reinterpret_cast<double*>(smem + SM::red);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + SM::bar);
  constexpr bool kMeas = MODE != MODE_INTENSITY;

  const int t = threadIdx.x;
  const int G = gridDim.x;
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  if (a.done && blockIdx.x == 0)
    for (int i = t; i < a.ndone; i += NT) a.done[i] = 0u;
  // twiddle table W_M^j = exp(-2 pi i j / M), rounded from double precision
  for (int j = t; j < M; j += NT) {
    double s, co;
    sincospi(-2.0 * double(j) / double(M), &s, &co);
    tw[j] = make_float2((float)co, (float)s);
  }
  __syncthreads();
  if (blockIdx.x < a.B) {
    prefetch_window<M>(a, blockIdx.x, t);
    if (kMeas && t == 0) fetch_meas<M>(a, blockIdx.x, sm, bar);
  }
  uint32_t phase = 0;

  for (int b = blockIdx.x; b < a.B; b += G) {
    int f;
    int2 c;
    const bool ok = resolve<M>(a, b, f, c);
    if constexpr (MODE == MODE_ADJ) {
      if (t == 0) a.tlb[b] = ok ? c : make_int2(-1, -1);
    }
    const int nb = b + G;
    if (!ok) {  // uniform: skipped pattern (no copy was issued for it)
      if (t == 0) pty_raise(a.status, PTYCHO_ERR_WINDOW);
      const float nan = __int_as_float(0x7fc00000);
      if constexpr (MODE == MODE_INTENSITY) {
        for (int i = t; i < M * M; i += NT) a.I_out[size_t(b) * M * M + i] = nan;
      } else {
        if (t == 0 && a.loss_pat) a.loss_pat[b] = (double)nan;
      }
      if (nb < a.B) {
        prefetch_window<M>(a, nb, t);
        if (kMeas && t == 0) fetch_meas<M>(a, nb, sm, bar);
      }
      continue;
    }

    float2 v[E];
    // ---- pass 1: gather the window times the probe, fftshift sign --------
    {
      int bx, by;
      tbase<M, 1>(t, bx, by);
      const float2* Ob = a.O + size_t(c.x + by) * a.W + (c.y + bx);
      const float2* Pb = a.P + by * M + bx;
      const unsigned par = unsigned((bx + by) & 1) << 31;
      static_for<E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        constexpr int ox = eoff_x<M, 1>(e), oy = eoff_y<M, 1>(e);
        constexpr unsigned ce = unsigned((ox + oy) & 1) << 31;
        float2 p = __ldg(Pb + oy * M + ox);
        p.x = __uint_as_float(__float_as_uint(p.x) ^ (par ^ ce));
        p.y = __uint_as_float(__float_as_uint(p.y) ^ (par ^ ce));
        v[e] = c_mul(p, __ldg(Ob + size_t(oy) * a.W + ox));
      });
    }
    if (nb < a.B) prefetch_window<M>(a, nb, t);
    pass<M, false, 1>(v, t, tw);
    exchange<M, 1, 2>(v, t, re, im);
    pass<M, false, 2>(v, t, tw);
    exchange<M, 2, 3>(v, t, re, im);
    pass<M, false, 3>(v, t, tw);

    if constexpr (MODE == MODE_INTENSITY) {
      int fx0, fy0;
      fbase<M>(t, fx0, fy0);
      float* Ib = a.I_out + size_t(b) * M * M + fy0 * M + fx0;
      static_for<E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        Ib[efreq<M>(e, M)] = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      });
    } else {
      const bool got = mbar_wait_bounded(bar, phase);
      phase ^= 1u;
      if (__syncthreads_or(!got)) {  // uniform give-up after a bounded wait
        if (t == 0) pty_raise(a.status, PTYCHO_ERR_TIMEOUT);
        return;
      }
      const double acc = loss_pointwise<M, LOSS>(v, t, sm, re, im);
      const double tot = block_sum<NT>(acc, red);  // all reads of sm are done after this
      if (t == 0) {
        if (a.loss_pat) a.loss_pat[b] = tot / double(M * M);
        if (nb < a.B) fetch_meas<M>(a, nb, sm, bar);
      }
      if constexpr (MODE == MODE_ADJ) {
        pass<M, true, 3>(v, t, tw);
        exchange<M, 3, 2>(v, t, re, im);
        pass<M, true, 2>(v, t, tw);
        exchange<M, 2, 1>(v, t, re, im);
        pass<M, true, 1>(v, t, tw);
        int bx, by;
        tbase<M, 1>(t, bx, by);
        float2* Eb = a.Eout + size_t(b) * M * M + by * M + bx;
        static_for<E>([&](auto ec) {
          constexpr int e = decltype(ec)::value;
          constexpr int ox = eoff_x<M, 1>(e), oy = eoff_y<M, 1>(e);
          Eb[oy * M + ox] = v[e];
        });
      }
    }
  }
}

// launch helper: persistent grid of min(B, #SMs) CTAs
template <int M, int MODE, int LOSS>
int launch_fused_t(const FusedArgs& a, cudaStream_t s) {
  constexpr size_t smem = FusedSmem<M>::total;
  auto kern = k_fused<M, MODE, LOSS>;
  // the shared-memory attribute and the resident-CTA count are set up once per
  // device (a per-call host cost otherwise)
  static PtyDevCache slots_cache;
  int dev = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    int slots = slots_cache.get(&dev);
    if (dev < 0) return PTYCHO_ERR_LAUNCH;
    if (slots == 0) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return PTYCHO_ERR_LAUNCH;
      int nsm = 148, per_sm = 1;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Plan<M>::NT, smem) != cudaSuccess ||
          per_sm < 1)
        per_sm = 1;
      slots = nsm * per_sm;
      slots_cache.put(dev, slots);
    }
    const int grid = a.B < slots ? a.B : slots;
    kern<<<grid, Plan<M>::NT, smem, s>>>(a);
    if (cudaGetLastError() == cudaSuccess) return PTYCHO_OK;
    slots_cache.put(dev, 0);  // e.g. the attribute was lost with a device reset: set up again once
  }
  return PTYCHO_ERR_LAUNCH;
}

template <int M>
int launch_fused_m(int mode, int loss, const FusedArgs& a, cudaStream_t s) {
  if (mode == MODE_INTENSITY) return launch_fused_t<M, MODE_INTENSITY, 0>(a, s);
  if (mode == MODE_LOSS) {
    switch (loss) {
      case 0: return launch_fused_t<M, MODE_LOSS, 0>(a, s);
      case 1: return launch_fused_t<M, MODE_LOSS, 1>(a, s);
      case 2: return launch_fused_t<M, MODE_LOSS, 2>(a, s);
      default: return launch_fused_t<M, MODE_LOSS, 3>(a, s);
    }
  }
  switch (loss) {
    case 0: return launch_fused_t<M, MODE_ADJ, 0>(a, s);
    case 1: return launch_fused_t<M, MODE_ADJ, 1>(a, s);
    case 2: return launch_fused_t<M, MODE_ADJ, 2>(a, s);
    default: return launch_fused_t<M, MODE_ADJ, 3>(a, s);
  }
}

// defined in fused_m64.cu / fused_m128.cu / fused256.cu (4-CTA cluster per pattern)
int launch_fused_64(int mode, int loss, const FusedArgs& a, cudaStream_t s);
int launch_fused_128(int mode, int loss, const FusedArgs& a, cudaStream_t s);
int launch_fused_256(int mode, int loss, const FusedArgs& a, cudaStream_t s);

// split256.cu: M = 256 as three line-DFT kernels (smooth-L1, Poisson and the
// intensity-gradient losses in MODE_LOSS / MODE_ADJ); a.Eout is the scratch,
// lpart holds B * kSplit256Blocks doubles.  With dp_part (MODE_ADJ, batches of
// at least kDpFuseMinB patterns) the inverse-row kernel also leaves the probe
// gradient as ceil(B / kDpGroup) partials of 256 x 256 in dp_part, which
// split256_dp_sum adds into dP (and writes the loss total); the assembly then
// runs without its dP role.
constexpr int kSplit256Blocks = 16;
constexpr int kDpGroup = 8;
#ifndef PTY_S256_DP_FUSE_MIN_B
#define PTY_S256_DP_FUSE_MIN_B 192
#endif
constexpr int kDpFuseMinB = PTY_S256_DP_FUSE_MIN_B;
bool split256_supported(int mode, int loss);
int launch_split256(int mode, int loss, const FusedArgs& a, double* lpart, float2* dp_part, cudaStream_t s);
int split256_dp_sum(const float2* dp_part, int B, float2* dP, bool accumulate, const double* loss_pat,
                    double* loss_total, cudaStream_t s);

}  // namespace pty
