// cmlp.cu -- complex-exponential MLP on the 5th-generation tensor cores (tcgen05).
//
// Replaces ComplexMLP.net of models/complex_inr.py:6-82 (as called through
// _get_complex_output, :308-314) for the configuration every reference config
// uses: 32 input features (16 hash levels x 2), hidden_features 64 (32
// complex units), hidden_layers 2, one complex output:
//   z1 = W1 x + b1 (real 32x32),          h1 = exp(i w1 z1)
//   z2 = W2 h1 + b2 (complex 32x32),      h2 = exp(i w2 z2)
//   z3 = W3 h2 + b3,                      h3 = exp(i w3 z3)
//   y  = Wo h3 + bo (complex 1x32).
// A complex layer acts on [Re h; Im h] as the real 64x64 block [[A,-B],[B,A]]
// (W = A + iB).  Operands are BF16 in shared memory, accumulators FP32 in
// tensor memory; the hidden activations entering layer 2, layer 3 and the
// output layer are split into bf16(h) + bf16(h - bf16(h)), two MMAs into one
// accumulator (with h rounded once to BF16, training on 1e3-photon Poisson data
// stalled at about 3x the residual an FP32 MLP reached); one CTA handles tiles of 128 coordinates and loops over
// tiles (persistent).  256 threads: warp w reads TMEM lane quarter w & 3 (tile
// rows 32 (w & 3) .. +31) and does the elementwise work of half w >> 2 of each
// layer's complex units, so the sin / cos / exp chains between two MMAs are
// split over 8 warps.
//
// Backward (training): the kernel recomputes the forward of its tile (keeping
// the FP32 h2, h3 in shared memory for the gradient steps), then
//   G_h3 = Wo_r^T G_y,  G_z = conj(i w h) G_h (complex layers),
//   G_z1 = Re(conj(G_h1) i w1 h1),  G_h(prev) = W_r^T G_z,  G_x = W1^T G_z1
// on the tensor core, and accumulates the weight gradients
//   sum_c [G_z3 | G_z2]_c^T [h2 | h1 | 1]_c,   sum_c G_z1_c^T [x | 1]_c,
//   sum_c G_y_c^T [h3 | 1]_c
// in TMEM across all its tiles (the appended ones column yields the bias
// gradients).  Each CTA writes its raw accumulators once; k_cmlp_reduce sums
// the CTA partials in a fixed order and folds the real-form blocks back into
// complex gradients (G_W = (P+S) + i(R-Q) for [[P,Q],[R,S]]) -- deterministic,
// no atomics.  Gradients follow torch's complex convention.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "async_copy.cuh"
#include "common.cuh"
#include "tc_umma.cuh"

namespace pty {
namespace cm {

constexpr int kThreads = 256;
constexpr int GRP = 2048;  // one group of 8 bf16 features x 128 rows

// ---- shared-memory map (bytes) --------------------------------------------
constexpr int S_W1 = 0;             // W1  [32 out][32 in]   K-major, LBO 512
constexpr int S_W2 = S_W1 + 2048;   // Wr2 [64][64]          LBO 1024
constexpr int S_W3 = S_W2 + 8192;   // Wr3 [64][64]
constexpr int S_WO = S_W3 + 8192;   // Wor [16][64] (rows 0,1 used), LBO 256
constexpr int kWBytes = S_WO + 2048;  // 20480
constexpr int S_PAR = kWBytes;      // fp32 biases and omegas
constexpr int S_BAR = S_PAR + 1024;
constexpr int S_TMEM = S_BAR + 16;
constexpr int S_RED = S_TMEM + 16;  // 24 floats: omega-gradient partials of 8 warps
constexpr int S_X = S_RED + 128;    // 6 groups: x (4), ones, zeros
constexpr int S_H = S_X + 6 * GRP;  // 18 groups: h2 (8), h1 (8), ones, zeros
constexpr int S_H3 = S_H + 18 * GRP;  // 10 groups: h3 (8), ones, zeros
constexpr int S_GY = S_H3 + 10 * GRP;  // 2 groups: (G_yr, G_yi, 0, ...), zeros
constexpr int S_GZ1 = S_GY + 2 * GRP;  // 4 groups: G_z1
constexpr int S_GZ = S_GZ1 + 4 * GRP;  // 16 groups: G_z3 (8), G_z2 (8)
constexpr int S_ACT_END = S_GZ + 16 * GRP;
// FP32 h2, h3 of the tile (backward only): [layer][re, im][32 units][128 rows],
// kept from the forward recompute for the layer-3 and layer-2 gradients
constexpr int S_HF = S_ACT_END;
// BF16 residuals h - bf16(h) of the input of layer 2, 3 or the output layer (8
// groups, rewritten layer by layer): each of those MMAs runs once on bf16(h) and
// once on the residual into the same accumulator, so the hidden activations
// reach the tensor core with about 16 significant bits instead of 8
constexpr int S_LO_BWD = int(pty_align_up_c(S_HF + 2 * 2 * 32 * 128 * 4, 1024));
constexpr int kSmemBwd = S_LO_BWD + 8 * GRP;  // 219136 bytes: one CTA per SM
constexpr int S_LO_FWD = S_GY;                // the forward needs x, h, h3 and the residual plane only
constexpr int kSmemFwd = S_LO_FWD + 8 * GRP;  // 107648 bytes: two CTAs per SM
static_assert(kSmemBwd <= 232448 && 2 * (kSmemFwd + 1024) <= 233472, "shared-memory budget");

// every MMA footprint used below stays inside [0, S_ACT_END)
static_assert(S_GY + 16 * GRP <= S_ACT_END, "output-grad A footprint");
static_assert(S_GZ1 + 16 * GRP <= S_ACT_END, "layer-1 grad A footprint");

// ---- fp32 parameter block (floats) ------------------------------------------
constexpr int P_B1 = 0, P_B2R = 32, P_B2I = 64, P_B3R = 96, P_B3I = 128, P_BOR = 160, P_BOI = 161,
              P_W1 = 162, P_W2 = 163, P_W3 = 164, kParFloats = 168;
constexpr int kPackedBytes = kWBytes + kParFloats * 4;  // 21152

// ---- TMEM columns -------------------------------------------------------------
constexpr uint32_t T_D1 = 0, T_D2 = 32, T_D3 = 96, T_DO = 160, T_ACC = 224, T_ACC1 = 368, T_ACCO = 416;
constexpr uint32_t kColsBwd = 512, kColsFwd = 256;

// ---- raw per-CTA gradient partials (floats) ----------------------------------
constexpr int R_W3 = 0, R_B3 = 4096, R_W2 = 4160, R_B2 = 8256, R_W1 = 8320, R_B1 = 9344, R_WO = 9376,
              R_BO = 9504, R_OM = 9506, kPartFloats = 9512;
// ---- final gradient blob (floats; complex entries interleaved re, im) --------
constexpr int G_W1 = 0, G_B1 = 1024, G_OM1 = 1056, G_W2 = 1058, G_B2 = 3106, G_OM2 = 3170, G_W3 = 3172,
              G_B3 = 5220, G_OM3 = 5284, G_WO = 5286, G_BO = 5350, kGradFloats = 5352;

// byte offset of (row c, feature f) in an activation buffer
PTY_DEVI int cm_off(int c, int f) { return (f >> 3) * GRP + (c >> 3) * 128 + (c & 7) * 16 + (f & 7) * 2; }
// byte offset of (n, k) in a weight matrix with nout rows (K-major view)
__host__ __device__ constexpr int wm_off(int n, int k, int nout) {
  return (k >> 3) * (nout * 16) + (n >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
}

PTY_DEVI uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}
// store 8 consecutive features [f0, f0+8) of row c (f0 % 8 == 0)
PTY_DEVI void st8(unsigned char* base, int c, int f0, const float* v) {
  uint4 q;
  q.x = pack_bf16x2(v[0], v[1]);
  q.y = pack_bf16x2(v[2], v[3]);
  q.z = pack_bf16x2(v[4], v[5]);
  q.w = pack_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4*>(base + cm_off(c, f0)) = q;
}
// the same 8 values as bf16(v) at feature f0 of `hi` and as bf16(v - bf16(v))
// at feature f_lo of `lo`
PTY_DEVI void st8_split(unsigned char* hi, int f0, unsigned char* lo, int f_lo, int c, const float* v) {
  float h[8], r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    h[k] = __bfloat162float(__float2bfloat16_rn(v[k]));
    r[k] = v[k] - h[k];
  }
  st8(hi, c, f0, h);
  st8(lo, c, f_lo, r);
}

// sin and cos of a after Cody-Waite reduction by 2 pi (two-constant split of
// 2 pi: the float nearest 2 pi plus its residual), then the SFU on [-pi, pi]
PTY_DEVI void sincos_rr(float a, float* s, float* c) {
  const float k = rintf(a * 0.159154943091895336f);
  float r = fmaf(-k, 6.28318548202514648f, a);
  r = fmaf(-k, -1.74845553e-7f, r);
  __sincosf(r, s, c);
}

// ---- GEMM issue helpers (single thread) --------------------------------------
// D[128 x N] (+)= A[128 x K] * B[N x K]^T, A activations (K-major), B weights (K-major)
PTY_DEVI void gemm_act_w(uint32_t d, uint32_t sa, uint32_t sb, uint32_t nout, int N, int K, bool acc) {
  const uint32_t id = tc::idesc_bf16(128, N, false, false);
  const uint32_t lbo_b = nout * 16;
  for (int s = 0; s < K / 16; ++s)
    tc::mma(d, tc::desc(sa + s * 2 * GRP, GRP, 128), tc::desc(sb + s * 2 * lbo_b, lbo_b, 128), id,
            (acc || s > 0) ? 1u : 0u);
}
// D[128 x N] = A[128 x K] * W where W[K out][N in] is stored K-major (n contiguous): MN-major B
PTY_DEVI void gemm_act_wT(uint32_t d, uint32_t sa, uint32_t sb, uint32_t nout, int N, int K) {
  const uint32_t id = tc::idesc_bf16(128, N, false, true);
  for (int s = 0; s < K / 16; ++s)
    tc::mma(d, tc::desc(sa + s * 2 * GRP, GRP, 128), tc::desc(sb + s * 2 * 128, 128, nout * 16), id,
            s > 0 ? 1u : 0u);
}
// D[128 x N] (+)= sum over the tile's 128 rows of a_c b_c^T: both operands are
// activation buffers read MN-major (feature = M or N, row = K)
PTY_DEVI void gemm_outer(uint32_t d, uint32_t sa, uint32_t sb, int N, bool acc) {
  const uint32_t id = tc::idesc_bf16(128, N, true, true);
  for (int s = 0; s < 8; ++s)
    tc::mma(d, tc::desc(sa + s * 256, 128, GRP), tc::desc(sb + s * 256, 128, GRP), id, (acc || s > 0) ? 1u : 0u);
}

struct Args {
  const unsigned char* packed;
  const float* x;    // [N][32]
  const float2* gy;  // [N]
  int N;
  float2* y;         // [N] or null
  float* gx;         // [N][32] (or [32][N] when gx_planar) or null
  float* part;       // [gridDim.x][kPartFloats]
  int32_t* status;
  int gx_planar;     // gx feature-major: feature f of row c at gx[f * N + c]
  int x_planar;      // x feature-major: feature f of row c at x[f * N + c]
};

template <bool BWD>
__global__ void __launch_bounds__(kThreads, BWD ? 1 : 2) k_cmlp(const Args a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, w = t >> 5;
  const int quarter = w & 3;                // TMEM lane quarter of this warp
  const int hh = w >> 2;                    // half of each layer's units handled here
  const int row = 32 * quarter + (t & 31);  // tile row (TMEM lane) of this thread
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + S_TMEM);
  float* par = reinterpret_cast<float*>(sm + S_PAR);
  float* red = reinterpret_cast<float*>(sm + S_RED);
  float* hf = reinterpret_cast<float*>(sm + S_HF);  // valid in the backward only
  constexpr int S_LO = BWD ? S_LO_BWD : S_LO_FWD;
  auto hfi = [&](int layer, int part, int unit) { return ((layer * 2 + part) * 32 + unit) * 128 + row; };
  constexpr uint32_t NCOLS = BWD ? kColsBwd : kColsFwd;
  const uint32_t sbase = tc::smem_addr(sm);

  // -- set-up: zero activations, copy weights and parameters, ones columns ----
  constexpr int kActEnd = BWD ? S_ACT_END : S_GY;
  for (int i = t; i < (kActEnd - S_X) / 16; i += kThreads)
    reinterpret_cast<uint4*>(sm + S_X)[i] = make_uint4(0u, 0u, 0u, 0u);
  for (int i = t; i < kWBytes / 16; i += kThreads)
    reinterpret_cast<uint4*>(sm)[i] = __ldg(reinterpret_cast<const uint4*>(a.packed) + i);
  for (int i = t; i < kParFloats; i += kThreads)
    par[i] = __ldg(reinterpret_cast<const float*>(a.packed + kWBytes) + i);
  __syncthreads();
  if (hh == 0) {
    const __nv_bfloat16 one = __float2bfloat16(1.0f);
    *reinterpret_cast<__nv_bfloat16*>(sm + S_X + cm_off(row, 32)) = one;
    *reinterpret_cast<__nv_bfloat16*>(sm + S_H + cm_off(row, 128)) = one;
    *reinterpret_cast<__nv_bfloat16*>(sm + S_H3 + cm_off(row, 64)) = one;
  }
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  if (w == 0) {
    tc::tmem_alloc(tslot, NCOLS);
    tc::tmem_relinquish();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tm = *tslot;
  const uint32_t lo = uint32_t(quarter * 32) << 16;  // this warp's TMEM lane quarter
  const float w1 = par[P_W1], w2 = par[P_W2], w3 = par[P_W3];
  uint32_t phase = 0;
  bool abort = false;

  // barrier + fences, then thread 0 issues `issue`, commits, everybody waits
  auto step = [&](auto issue) {
    tc::fence_smem_async();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (t == 0) {
      issue();
      tc::commit(bar);
    }
    const bool ok = mbar_wait_bounded(bar, phase);
    if (__syncthreads_or(!ok)) abort = true;  // phase stays at the unfinished one
    else phase ^= 1u;
    tc::fence_after();
  };

  float om1 = 0.f, om2 = 0.f, om3 = 0.f;
  bool first = true;
  const int ntiles = (a.N + 127) / 128;
  // this half's 16 of row c's 32 input features (and, backward, G_y of row c)
  auto load_inputs = [&](int cc, float (&xv)[16], float2& g) {
    const bool ok = cc < a.N;
    if (a.x_planar) {  // per feature, a warp reads 32 consecutive rows
#pragma unroll
      for (int i = 0; i < 16; ++i) xv[i] = ok ? __ldg(a.x + size_t(16 * hh + i) * a.N + cc) : 0.f;
    } else {
      const float4* xp = reinterpret_cast<const float4*>(a.x + size_t(ok ? cc : 0) * 32 + 16 * hh);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float4 v = ok ? __ldg(xp + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        xv[4 * q] = v.x;
        xv[4 * q + 1] = v.y;
        xv[4 * q + 2] = v.z;
        xv[4 * q + 3] = v.w;
      }
    }
    if constexpr (BWD) g = (ok && hh == 0) ? __ldg(a.gy + cc) : make_float2(0.f, 0.f);
  };
  // The tile loop is a chain of dependent MMA / elementwise steps, so a tile's
  // input loads would stall it: the backward (registers to spare) loads the
  // next tile's inputs while this tile computes; the forward (at its register
  // cap) has them prefetched into L2.
  auto prefetch_l2 = [&](int nt) {
    if (nt < ntiles) {
      if (a.x_planar) {  // 32 features x 512 bytes: one 64-byte piece per thread
        const int f = t >> 3, piece = t & 7;
        const int r0 = nt * 128 + piece * 16;
        if (r0 < a.N) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.x + size_t(f) * a.N + r0));
      } else {  // 128 rows x 128 bytes: 16 KB, one 64-byte piece per thread
        const size_t off = size_t(nt) * 128 * 32 + size_t(t) * 16;
        if (off < size_t(a.N) * 32) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.x + off));
      }
    }
  };
  float xnext[16];
  float2 gnext = make_float2(0.f, 0.f);
  if constexpr (BWD) load_inputs(blockIdx.x * 128 + row, xnext, gnext);
  for (int tile = blockIdx.x; tile < ntiles && !abort; tile += gridDim.x) {
    const int c = tile * 128 + row;
    const bool valid = c < a.N;
    // -- inputs ------------------------------------------------------------------
    {
      float xv[16];
      float2 g;
      if constexpr (BWD) {
#pragma unroll
        for (int i = 0; i < 16; ++i) xv[i] = xnext[i];
        g = gnext;
        load_inputs((tile + gridDim.x) * 128 + row, xnext, gnext);  // lands during this tile
      } else {
        load_inputs(c, xv, g);
        prefetch_l2(tile + gridDim.x);
      }
      st8(sm + S_X, row, 16 * hh, xv);
      st8(sm + S_X, row, 16 * hh + 8, xv + 8);
      if constexpr (BWD) {
        if (hh == 0) {
          const float v8[8] = {g.x, g.y, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
          st8(sm + S_GY, row, 0, v8);
        }
      }
    }
    // -- layer 1 ---------------------------------------------------------------
    step([&] { gemm_act_w(tm + T_D1, sbase + S_X, sbase + S_W1, 32, 32, 32, false); });
    if (abort) break;
    {
      const int h = hh;
      float d[16], hr[16], hi[16];
      tc::ld16(tm + lo + T_D1 + 16 * h, d);
#pragma unroll
      for (int k = 0; k < 16; ++k) sincos_rr(w1 * (d[k] + par[P_B1 + 16 * h + k]), &hi[k], &hr[k]);
      st8_split(sm + S_H, 64 + 16 * h, sm + S_LO, 16 * h, row, hr);
      st8_split(sm + S_H, 72 + 16 * h, sm + S_LO, 8 + 16 * h, row, hr + 8);
      st8_split(sm + S_H, 96 + 16 * h, sm + S_LO, 32 + 16 * h, row, hi);
      st8_split(sm + S_H, 104 + 16 * h, sm + S_LO, 40 + 16 * h, row, hi + 8);
    }
    // -- complex layers 2 and 3 ------------------------------------------------
    step([&] {
      gemm_act_w(tm + T_D2, sbase + S_H + 8 * GRP, sbase + S_W2, 64, 64, 64, false);
      gemm_act_w(tm + T_D2, sbase + S_LO, sbase + S_W2, 64, 64, 64, true);
    });
    if (abort) break;
    {
      const int h = hh;
      float zr[16], zi[16], hr[16], hi[16];
      tc::ld16(tm + lo + T_D2 + 16 * h, zr);
      tc::ld16(tm + lo + T_D2 + 32 + 16 * h, zi);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const float r = zr[k] + par[P_B2R + 16 * h + k], i = zi[k] + par[P_B2I + 16 * h + k];
        const float amp = __expf(-w2 * i);
        float s, co;
        sincos_rr(w2 * r, &s, &co);
        hr[k] = amp * co;
        hi[k] = amp * s;
        if constexpr (BWD) {
          hf[hfi(0, 0, 16 * h + k)] = hr[k];
          hf[hfi(0, 1, 16 * h + k)] = hi[k];
        }
      }
      st8_split(sm + S_H, 16 * h, sm + S_LO, 16 * h, row, hr);
      st8_split(sm + S_H, 8 + 16 * h, sm + S_LO, 8 + 16 * h, row, hr + 8);
      st8_split(sm + S_H, 32 + 16 * h, sm + S_LO, 32 + 16 * h, row, hi);
      st8_split(sm + S_H, 40 + 16 * h, sm + S_LO, 40 + 16 * h, row, hi + 8);
    }
    step([&] {
      gemm_act_w(tm + T_D3, sbase + S_H, sbase + S_W3, 64, 64, 64, false);
      gemm_act_w(tm + T_D3, sbase + S_LO, sbase + S_W3, 64, 64, 64, true);
    });
    if (abort) break;
    {
      const int h = hh;
      float zr[16], zi[16], hr[16], hi[16];
      tc::ld16(tm + lo + T_D3 + 16 * h, zr);
      tc::ld16(tm + lo + T_D3 + 32 + 16 * h, zi);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const float r = zr[k] + par[P_B3R + 16 * h + k], i = zi[k] + par[P_B3I + 16 * h + k];
        const float amp = __expf(-w3 * i);
        float s, co;
        sincos_rr(w3 * r, &s, &co);
        hr[k] = amp * co;
        hi[k] = amp * s;
        if constexpr (BWD) {
          hf[hfi(1, 0, 16 * h + k)] = hr[k];
          hf[hfi(1, 1, 16 * h + k)] = hi[k];
        }
      }
      st8_split(sm + S_H3, 16 * h, sm + S_LO, 16 * h, row, hr);
      st8_split(sm + S_H3, 8 + 16 * h, sm + S_LO, 8 + 16 * h, row, hr + 8);
      st8_split(sm + S_H3, 32 + 16 * h, sm + S_LO, 32 + 16 * h, row, hi);
      st8_split(sm + S_H3, 40 + 16 * h, sm + S_LO, 40 + 16 * h, row, hi + 8);
    }
    // -- output layer ----------------------------------------------------------
    step([&] {
      gemm_act_w(tm + T_DO, sbase + S_H3, sbase + S_WO, 16, 16, 64, false);
      gemm_act_w(tm + T_DO, sbase + S_LO, sbase + S_WO, 16, 16, 64, true);
    });
    if (abort) break;
    if (hh == 0) {  // warp-uniform
      float d[16];
      tc::ld16(tm + lo + T_DO, d);
      if (a.y && valid) a.y[c] = make_float2(d[0] + par[P_BOR], d[1] + par[P_BOI]);
    }
    if constexpr (BWD) {
      // G_h3 = Wo_r^T G_y ; output-layer gradient accumulation
      step([&] {
        gemm_act_wT(tm + T_DO, sbase + S_GY, sbase + S_WO, 16, 64, 16);
        gemm_outer(tm + T_ACCO, sbase + S_GY, sbase + S_H3, 80, !first);
      });
      if (abort) break;
      // G_z3 = conj(i w3 h3) G_h3 (h3 recomputed from z3 in TMEM)
      {
        const int h = hh;
        float gr[16], gi[16], zr[16], zi[16];
        tc::ld16(tm + lo + T_DO + 16 * h, gr);
        tc::ld16(tm + lo + T_DO + 32 + 16 * h, gi);
        tc::ld16(tm + lo + T_D3 + 16 * h, zr);
        tc::ld16(tm + lo + T_D3 + 32 + 16 * h, zi);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const float r = zr[k] + par[P_B3R + 16 * h + k], i = zi[k] + par[P_B3I + 16 * h + k];
          const float hr = hf[hfi(1, 0, 16 * h + k)], hi = hf[hfi(1, 1, 16 * h + k)];  // h3 of this tile
          om3 += gi[k] * (r * hr - i * hi) - gr[k] * (r * hi + i * hr);
          zr[k] = w3 * (hr * gi[k] - hi * gr[k]);
          zi[k] = -w3 * (hr * gr[k] + hi * gi[k]);
        }
        st8(sm + S_GZ, row, 16 * h, zr);
        st8(sm + S_GZ, row, 8 + 16 * h, zr + 8);
        st8(sm + S_GZ, row, 32 + 16 * h, zi);
        st8(sm + S_GZ, row, 40 + 16 * h, zi + 8);
      }
      step([&] { gemm_act_wT(tm + T_D3, sbase + S_GZ, sbase + S_W3, 64, 64, 64); });
      if (abort) break;
      // G_z2
      {
        const int h = hh;
        float gr[16], gi[16], zr[16], zi[16];
        tc::ld16(tm + lo + T_D3 + 16 * h, gr);
        tc::ld16(tm + lo + T_D3 + 32 + 16 * h, gi);
        tc::ld16(tm + lo + T_D2 + 16 * h, zr);
        tc::ld16(tm + lo + T_D2 + 32 + 16 * h, zi);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const float r = zr[k] + par[P_B2R + 16 * h + k], i = zi[k] + par[P_B2I + 16 * h + k];
          const float hr = hf[hfi(0, 0, 16 * h + k)], hi = hf[hfi(0, 1, 16 * h + k)];  // h2 of this tile
          om2 += gi[k] * (r * hr - i * hi) - gr[k] * (r * hi + i * hr);
          zr[k] = w2 * (hr * gi[k] - hi * gr[k]);
          zi[k] = -w2 * (hr * gr[k] + hi * gi[k]);
        }
        st8(sm + S_GZ, row, 64 + 16 * h, zr);
        st8(sm + S_GZ, row, 72 + 16 * h, zr + 8);
        st8(sm + S_GZ, row, 96 + 16 * h, zi);
        st8(sm + S_GZ, row, 104 + 16 * h, zi + 8);
      }
      step([&] { gemm_act_wT(tm + T_D2, sbase + S_GZ + 8 * GRP, sbase + S_W2, 64, 64, 64); });
      if (abort) break;
      // G_z1 = Re(conj(G_h1) i w1 h1)
      {
        const int h = hh;
        float gr[16], gi[16], z[16];
        tc::ld16(tm + lo + T_D2 + 16 * h, gr);
        tc::ld16(tm + lo + T_D2 + 32 + 16 * h, gi);
        tc::ld16(tm + lo + T_D1 + 16 * h, z);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const float zz = z[k] + par[P_B1 + 16 * h + k];
          float s, co;
          sincos_rr(w1 * zz, &s, &co);
          const float q = co * gi[k] - s * gr[k];
          om1 += zz * q;
          z[k] = w1 * q;
        }
        st8(sm + S_GZ1, row, 16 * h, z);
        st8(sm + S_GZ1, row, 8 + 16 * h, z + 8);
      }
      // G_x = W1^T G_z1 ; hidden / layer-1 weight-gradient accumulation
      step([&] {
        gemm_act_wT(tm + T_D1, sbase + S_GZ1, sbase + S_W1, 32, 32, 32);
        gemm_outer(tm + T_ACC, sbase + S_GZ, sbase + S_H, 144, !first);
        gemm_outer(tm + T_ACC1, sbase + S_GZ1, sbase + S_X, 48, !first);
      });
      if (abort) break;
      if (a.gx) {
        {
          const int h = hh;
          float d[16];
          tc::ld16(tm + lo + T_D1 + 16 * h, d);
          if (valid) {
            if (a.gx_planar) {  // per feature, a warp stores 32 consecutive rows
#pragma unroll
              for (int i = 0; i < 16; ++i) a.gx[size_t(16 * h + i) * a.N + c] = d[i];
            } else {
              float4* gp = reinterpret_cast<float4*>(a.gx + size_t(c) * 32 + 16 * h);
#pragma unroll
              for (int q = 0; q < 4; ++q) gp[q] = make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
            }
          }
        }
      }
      first = false;
    }
  }

  if (abort) {  // bounded wait gave up: report, let the tensor core drain, free TMEM
    if (t == 0) pty_raise(a.status, PTYCHO_ERR_TIMEOUT);
    mbar_wait_bounded(bar, phase);
  }
  if constexpr (BWD) {
    if (!abort) {
      // -- raw accumulators -> this CTA's partial --------------------------------
      float* P = a.part + size_t(blockIdx.x) * kPartFloats;
      auto rd = [&](uint32_t col, float (&d)[16]) {
        if (first) {
#pragma unroll
          for (int i = 0; i < 16; ++i) d[i] = 0.f;
        } else {
          tc::ld16(tm + lo + col, d);
        }
      };
      float d[16];
      if (hh == 1) {
        // the raw accumulators are read by warps 0..3 (one per lane quarter)
      } else if (quarter < 2) {  // rows 0..63: W3 real form and b3
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          rd(T_ACC + 16 * q, d);
#pragma unroll
          for (int i = 0; i < 16; ++i) P[R_W3 + row * 64 + 16 * q + i] = d[i];
        }
        rd(T_ACC + 128, d);
        P[R_B3 + row] = d[0];
      } else {  // rows 64..127: W2 real form and b2
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          rd(T_ACC + 64 + 16 * q, d);
#pragma unroll
          for (int i = 0; i < 16; ++i) P[R_W2 + (row - 64) * 64 + 16 * q + i] = d[i];
        }
        rd(T_ACC + 128, d);
        P[R_B2 + row - 64] = d[0];
      }
      if (w == 0) {  // rows 0..31: W1, b1 ; rows 0,1: Wo real form, bo
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          rd(T_ACC1 + 16 * q, d);
#pragma unroll
          for (int i = 0; i < 16; ++i) P[R_W1 + row * 32 + 16 * q + i] = d[i];
        }
        rd(T_ACC1 + 32, d);
        P[R_B1 + row] = d[0];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          rd(T_ACCO + 16 * q, d);
          if (row < 2) {
#pragma unroll
            for (int i = 0; i < 16; ++i) P[R_WO + row * 64 + 16 * q + i] = d[i];
          }
        }
        rd(T_ACCO + 64, d);
        if (row < 2) P[R_BO + row] = d[0];
      }
      // omega gradients: fixed shuffle tree, then warps in order
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        om1 += __shfl_xor_sync(0xffffffffu, om1, o);
        om2 += __shfl_xor_sync(0xffffffffu, om2, o);
        om3 += __shfl_xor_sync(0xffffffffu, om3, o);
      }
      if ((t & 31) == 0) {
        red[w] = om1;
        red[8 + w] = om2;
        red[16 + w] = om3;
      }
      __syncthreads();
      if (t == 0) {
#pragma unroll
        for (int l = 0; l < 3; ++l) {
          float s = 0.f;
#pragma unroll
          for (int i = 0; i < 8; ++i) s += red[8 * l + i];  // warps in order
          P[R_OM + l] = s;
        }
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_free(tm, NCOLS);
}

// sum the CTA partials in a fixed order and fold the real-form blocks
// Block b owns outputs 32 b .. 32 b + 31, one per lane, so each warp's loads of
// one partial touch neighbouring raw entries; warp k sums partials k, k + 8, ...
// in order and the eight warp sums are added in warp order.
__global__ void __launch_bounds__(256) k_cmlp_reduce(const float* __restrict__ part, int nparts,
                                                     float* __restrict__ grad) {
  __shared__ float wsum[8][32];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int e = blockIdx.x * 32 + lane;
  // each output is a (sign-weighted) sum of at most two raw entries
  int i0 = -1, i1 = -1;
  float s1 = 0.f;
  if (e < G_B1) {
    i0 = R_W1 + (e - G_W1);
  } else if (e < G_OM1) {
    i0 = R_B1 + (e - G_B1);
  } else if (e == G_OM1) {
    i0 = R_OM + 0;
  } else if (e == G_OM1 + 1) {
  } else if (e < G_B2 || (e >= G_W3 && e < G_B3)) {  // complex W2 / W3 [o][i][re,im]
    const bool l2 = e < G_B2;
    const int base = l2 ? R_W2 : R_W3;
    const int j = e - (l2 ? G_W2 : G_W3);
    const int o = j / 64, i = (j % 64) / 2, im = j & 1;
    if (!im) {  // P + S
      i0 = base + o * 64 + i;
      i1 = base + (32 + o) * 64 + 32 + i;
      s1 = 1.f;
    } else {  // R - Q
      i0 = base + (32 + o) * 64 + i;
      i1 = base + o * 64 + 32 + i;
      s1 = -1.f;
    }
  } else if (e < G_OM2 || (e >= G_B3 && e < G_OM3)) {  // complex b2 / b3
    const bool l2 = e < G_OM2;
    const int j = e - (l2 ? G_B2 : G_B3);
    i0 = (l2 ? R_B2 : R_B3) + (j & 1) * 32 + j / 2;
  } else if (e == G_OM2) {
    i0 = R_OM + 1;
  } else if (e == G_OM3) {
    i0 = R_OM + 2;
  } else if (e >= G_WO && e < G_BO) {
    const int j = e - G_WO;
    const int i = j / 2, im = j & 1;
    if (!im) {
      i0 = R_WO + i;
      i1 = R_WO + 64 + 32 + i;
      s1 = 1.f;
    } else {
      i0 = R_WO + 64 + i;
      i1 = R_WO + 32 + i;
      s1 = -1.f;
    }
  } else if (e >= G_BO) {
    i0 = R_BO + (e - G_BO);
  }
  float acc = 0.f;
  if (e < kGradFloats && i0 >= 0) {
    int p = wp;
    for (; p + 24 < nparts; p += 32) {  // four partials' loads in flight, added in order
      float v[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float* P = part + size_t(p + 8 * k) * kPartFloats;
        v[k] = P[i0];
        if (i1 >= 0) v[k] = fmaf(s1, P[i1], v[k]);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) acc += v[k];
    }
    for (; p < nparts; p += 8) {
      const float* P = part + size_t(p) * kPartFloats;
      float v = P[i0];
      if (i1 >= 0) v = fmaf(s1, P[i1], v);
      acc += v;
    }
  }
  wsum[wp][lane] = acc;
  __syncthreads();
  if (wp == 0 && e < kGradFloats) {
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += wsum[k][lane];  // warps in order
    grad[e] = t;
  }
}

// pack torch-layout parameters into the kernel's bf16 operand blob + fp32 block
struct PackArgs {
  const float *W1, *b1, *w1, *W2, *b2, *w2, *W3, *b3, *w3, *Wo, *bo;
  unsigned char* out;
};

__global__ void __launch_bounds__(256) k_cmlp_pack(const PackArgs p) {
  const int e = blockIdx.x * 256 + threadIdx.x;
  __nv_bfloat16* wb = reinterpret_cast<__nv_bfloat16*>(p.out);
  float* fb = reinterpret_cast<float*>(p.out + kWBytes);
  if (e < 1024) {  // W1 [32 out][32 in]
    const int n = e / 32, k = e % 32;
    wb[(S_W1 + wm_off(n, k, 32)) / 2] = __float2bfloat16(p.W1[e]);
  } else if (e < 1024 + 2 * 4096) {  // Wr2, Wr3: [[A,-B],[B,A]]
    const int j = e - 1024;
    const int layer = j / 4096, r = (j % 4096) / 64, k = j % 64;
    const float* W = layer ? p.W3 : p.W2;  // complex [32][32] interleaved
    const int ro = r % 32, ko = k % 32;
    const float A = W[2 * (ro * 32 + ko)], B = W[2 * (ro * 32 + ko) + 1];
    const float v = (r < 32) ? (k < 32 ? A : -B) : (k < 32 ? B : A);
    wb[((layer ? S_W3 : S_W2) + wm_off(r, k, 64)) / 2] = __float2bfloat16(v);
  } else if (e < 1024 + 8192 + 1024) {  // Wor [16][64]: row 0 = [Re Wo, -Im Wo], row 1 = [Im Wo, Re Wo]
    const int j = e - 1024 - 8192;
    const int r = j / 64, k = j % 64;
    float v = 0.f;
    if (r < 2) {
      const int ko = k % 32;
      const float A = p.Wo[2 * ko], B = p.Wo[2 * ko + 1];
      v = (r == 0) ? (k < 32 ? A : -B) : (k < 32 ? B : A);
    }
    wb[(S_WO + wm_off(r, k, 16)) / 2] = __float2bfloat16(v);
  } else if (e < 1024 + 8192 + 1024 + kParFloats) {
    const int j = e - 1024 - 8192 - 1024;
    float v = 0.f;
    if (j < 32) v = p.b1[j];
    else if (j < 64) v = p.b2[2 * (j - 32)];
    else if (j < 96) v = p.b2[2 * (j - 64) + 1];
    else if (j < 128) v = p.b3[2 * (j - 96)];
    else if (j < 160) v = p.b3[2 * (j - 128) + 1];
    else if (j == P_BOR) v = p.bo[0];
    else if (j == P_BOI) v = p.bo[1];
    else if (j == P_W1) v = p.w1[0];
    else if (j == P_W2) v = p.w2[0];
    else if (j == P_W3) v = p.w3[0];
    fb[j] = v;
  }
}

template <bool BWD>
static int launch(const Args& a, cudaStream_t s, int* grid_out) {
  auto kern = k_cmlp<BWD>;
  constexpr int smem = BWD ? kSmemBwd : kSmemFwd;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return PTYCHO_ERR_LAUNCH;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (a.N + 127) / 128;
  const int per_sm = BWD ? 1 : 2;  // TMEM: 512 columns (backward) or 2 x 256 (forward) per SM
  const int grid = ntiles < nsm * per_sm ? ntiles : nsm * per_sm;
  if (grid_out) *grid_out = grid;
  if (grid == 0) return PTYCHO_OK;
  kern<<<grid, kThreads, smem, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // namespace cm
}  // namespace pty

using namespace pty;

extern "C" {

size_t ptycho_cmlp_packed_bytes(void) { return cm::kPackedBytes; }

int ptycho_cmlp_grad_floats(void) { return cm::kGradFloats; }

int ptycho_cmlp_pack(const float* W1, const float* b1, const float* omega1, const float* W2, const float* b2,
                     const float* omega2, const float* W3, const float* b3, const float* omega3, const float* Wo,
                     const float* bo, void* packed, ptycho_stream_t stream) {
  if (!W1 || !b1 || !omega1 || !W2 || !b2 || !omega2 || !W3 || !b3 || !omega3 || !Wo || !bo || !packed)
    return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(packed, 16)) return PTYCHO_ERR_MISALIGNED;
  cm::PackArgs p{W1, b1, omega1, W2, b2, omega2, W3, b3, omega3, Wo, bo, static_cast<unsigned char*>(packed)};
  const int total = 1024 + 8192 + 1024 + cm::kParFloats;
  cm::k_cmlp_pack<<<(total + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

static int cmlp_forward(int planar, const void* packed, const float* x, int N, float* y, int32_t* status_out,
                        ptycho_stream_t stream) {
  if (!packed || N < 0 || (N > 0 && (!x || !y))) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(packed, 16) || !pty_aligned(x, planar ? 4 : 16) || !pty_aligned(y, 8))
    return PTYCHO_ERR_MISALIGNED;
  cm::Args a{static_cast<const unsigned char*>(packed), x, nullptr, N, reinterpret_cast<float2*>(y), nullptr,
             nullptr, status_out, 0, planar};
  return cm::launch<false>(a, reinterpret_cast<cudaStream_t>(stream), nullptr);
}

int ptycho_cmlp_forward(const void* packed, const float* x, int N, float* y, int32_t* status_out,
                        ptycho_stream_t stream) {
  return cmlp_forward(0, packed, x, N, y, status_out, stream);
}

int ptycho_cmlp_forward_planar(const void* packed, const float* x_planar, int N, float* y, int32_t* status_out,
                               ptycho_stream_t stream) {
  return cmlp_forward(1, packed, x_planar, N, y, status_out, stream);
}

size_t ptycho_cmlp_backward_workspace_size(int N) {
  if (N < 0) return 0;
  const int ntiles = (N + 127) / 128;
  const int parts = ntiles < 1024 ? ntiles : 1024;  // at most one partial per SM is used
  return pty_align_up(size_t(parts > 0 ? parts : 1) * cm::kPartFloats * sizeof(float), 256);
}

static int cmlp_backward(int planar, const void* packed, const float* x, const float* gy, int N, float* gx, float* grad,
                         float* y, void* workspace, size_t workspace_bytes, int32_t* status_out,
                         ptycho_stream_t stream) {
  if (!packed || !grad || N < 0 || (N > 0 && (!x || !gy))) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(packed, 16) || !pty_aligned(x, 16) || !pty_aligned(gy, 8) || !pty_aligned(gx, 16) ||
      !pty_aligned(y, 8))
    return PTYCHO_ERR_MISALIGNED;
  if (!workspace || workspace_bytes < ptycho_cmlp_backward_workspace_size(N)) return PTYCHO_ERR_WORKSPACE;
  {  // the persistent grid writes one partial per CTA: min(tiles, SMs) <= the sized count
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = (N + 127) / 128;
    const int grid = ntiles < nsm ? ntiles : nsm;
    if (size_t(grid) * cm::kPartFloats * sizeof(float) > workspace_bytes) return PTYCHO_ERR_WORKSPACE;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (N == 0) {
    cudaMemsetAsync(grad, 0, sizeof(float) * cm::kGradFloats, s);
    return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
  }
  cm::Args a{static_cast<const unsigned char*>(packed), x, reinterpret_cast<const float2*>(gy), N,
             reinterpret_cast<float2*>(y), gx, static_cast<float*>(workspace), status_out, planar, planar};
  int grid = 0;
  int st = cm::launch<true>(a, s, &grid);
  if (st) return st;
  cm::k_cmlp_reduce<<<(cm::kGradFloats + 31) / 32, 256, 0, s>>>(static_cast<const float*>(workspace), grid,
                                                                  grad);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_cmlp_backward(const void* packed, const float* x, const float* gy, int N, float* gx, float* grad,
                         float* y, void* workspace, size_t workspace_bytes, int32_t* status_out,
                         ptycho_stream_t stream) {
  return cmlp_backward(0, packed, x, gy, N, gx, grad, y, workspace, workspace_bytes, status_out, stream);
}

int ptycho_cmlp_backward_planar(const void* packed, const float* x, const float* gy, int N, float* gx,
                                float* grad, float* y, void* workspace, size_t workspace_bytes,
                                int32_t* status_out, ptycho_stream_t stream) {
  return cmlp_backward(1, packed, x, gy, N, gx, grad, y, workspace, workspace_bytes, status_out, stream);
}

}  // extern "C"
