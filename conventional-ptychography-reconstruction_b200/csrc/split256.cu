// split256.cu -- forward / loss / adjoint for 256 x 256 probes as three
// line-DFT kernels over the E' workspace (smooth-L1, Poisson and the
// intensity-gradient losses; the FD loss and MODE_INTENSITY keep the
// cluster kernel of fused256.cu).
//
// Same contract as the fused kernels (fused.cuh): per pattern b of the batch,
//   A  rows:     X_b[y][.] = DFT_x( (-1)^(x+y) P[y][x] O[tlY+y][tlX+x] )
//   B  columns:  F_b[.][fx] = DFT_y(X_b[.][fx])   (= fftshift(fft2(P * O_w)))
//                loss terms against Imeas[f_b] at the same index (the sign
//                folds fftshift in), FP64 partial per column block;
//                G = 2 dL/dI F;  X_b[.][fx] = IDFT_y(G[.][fx])  (unnormalised)
//   C  rows:     E'_b[y][.] = IDFT_x(X_b[y][.]); per-pattern loss from the
//                column-block partials in a fixed order
// so E'_b = (-1)^(x+y) dL/dpsi_b, the layout the assembly (assemble.cu)
// reads.  X_b is E'_b's own workspace slot: no other scratch.  Batches
// above kChunk patterns run in chunks of kChunk.
//
// Line DFT of length 256 = 16 x 16.  Rows: a half-warp per row, lane j
// holding x[j + 16 k] in registers; a 16-point DFT over k, the twiddle
// W256^(j p), a 16 x 16 transpose through shared memory (padded rows of 17:
// the two half-warps of a warp hit disjoint banks), a second 16-point DFT;
// lane p then holds X[p + 16 q], the input layout, so lines chain without
// reordering.  Columns: the same factorisation with the 16 values of a
// column spread over 16 half-warps (a half-warp = 16 adjacent columns, so
// every global access is a 64- or 128-byte row piece) and the transpose
// across warps.  Everything is a fixed sequence: results are bitwise
// deterministic.
#include <cuda_runtime.h>
#include <stdint.h>

#include "assemble.cuh"
#include "dft_regs.cuh"
#include "fused.cuh"

// Build-time tuning (measured on B200, c3 = 64 and c4 = 512 patterns): one
// launch per kernel for up to 512 patterns beat chunks of 64 that keep the
// scratch in L2 (c4 515 vs 551 us: fuller waves, fewer launches); three
// column CTAs per SM at 85 registers beat four at 64 with a 20-byte spill.
#ifndef PTY_S256_CHUNK
#define PTY_S256_CHUNK 512
#endif
#ifndef PTY_S256_COLS_MINB
#define PTY_S256_COLS_MINB 3
#endif
#ifndef PTY_S256_ROWS_MINB
#define PTY_S256_ROWS_MINB 4
#endif

namespace pty {
namespace s256 {

constexpr int M = 256;
constexpr int NT = 256;            // 16 lines x 16 lanes per CTA
constexpr int LINES = 16;
constexpr int TP = 17;             // padded row of a 16 x 16 transpose / tile
constexpr int BUF = LINES * 16 * TP;  // floats per plane (re or im): 4352
constexpr int NCB = M / LINES;     // column (or row) blocks per pattern: 16
static_assert(NCB == kSplit256Blocks, "loss partials per pattern");
constexpr int kChunk = PTY_S256_CHUNK;
static_assert(kChunk % kDpGroup == 0, "probe-gradient groups do not straddle chunks");

// shared memory: twiddles, two transpose planes (re, im), reduction
constexpr size_t SM_TW = 0;
constexpr size_t SM_RE = SM_TW + M * 8;
constexpr size_t SM_IM = SM_RE + BUF * 4;
constexpr size_t SM_RED = SM_IM + BUF * 4;
constexpr size_t SMEM_ROWS = SM_RED;              // kernels A and C
constexpr size_t SMEM_COLS = SM_RED + 8 * 8;      // kernel B

struct Args {
  FusedArgs f;
  double* lpart;  // [B][NCB] FP64 loss partial of each column block
  int b0;         // first pattern of this chunk
};

// The line twiddles W256^(j p), j, p = 0..15 (forward sign), stored at
// p * 16 + j: the row lanes j of a half-warp read 16 adjacent entries (no bank
// conflict), the column half-warps read one entry (a broadcast).  One entry
// per thread.
PTY_DEVI void fill_twiddles(float2* tw) {
  const int p = threadIdx.x >> 4, j = threadIdx.x & 15;
  float s, c;
  sincospif(-float(j * p) / 128.0f, &s, &c);
  tw[threadIdx.x] = make_float2(c, s);
}

// 256-point DFT (INV: unnormalised inverse) of one line held by a half-warp.
// In: lane j holds x[j + 16 k] in v[k].  Out: lane j holds X[j + 16 q] in v[q].
// bre / bim: this line's private 16 x 17 transpose planes.
template <bool INV>
PTY_DEVI void line256(float2 (&v)[16], int j, float* bre, float* bim, const float2* tw) {
  dft16<INV, 1>(v);  // v[p] = sum_k x[j + 16 k] W16^(k p)
#pragma unroll
  for (int p = 1; p < 16; ++p) {
    const float2 w = tw[p * 16 + j];
    v[p] = c_mul(v[p], INV ? c_conj(w) : w);
  }
  __syncwarp();
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    bre[p * TP + j] = v[p].x;
    bim[p * TP + j] = v[p].y;
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = make_float2(bre[j * TP + i], bim[j * TP + i]);
  dft16<INV, 1>(v);  // v[q] = X[j + 16 q]
}

PTY_DEVI bool window_ok(const FusedArgs& a, int b, int& f, int2& w) {
  f = a.batch ? __ldg(a.batch + b) : b;
  if (f < 0 || f >= a.F) {
    w = make_int2(-1, -1);
    return false;
  }
  w = __ldg(a.tl + f);
  return w.x >= 0 && w.y >= 0 && w.x <= a.H - M && w.y <= a.W - M;
}

// A: gather + row DFTs.  grid (NCB, chunk): CTA (rb, b - b0) owns rows
// 16 rb .. 16 rb + 15 of pattern b.  Also resolves the window (tlb, status)
// and, once per call, zeroes the assembly's dP arrival counters.
__global__ void __launch_bounds__(NT, PTY_S256_ROWS_MINB) k_rows_fwd(const Args g) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* tw = reinterpret_cast<float2*>(smem + SM_TW);
  float* pre = reinterpret_cast<float*>(smem + SM_RE);
  float* pim = reinterpret_cast<float*>(smem + SM_IM);
  const FusedArgs& a = g.f;
  const int t = threadIdx.x, r = t >> 4, j = t & 15;
  const int b = g.b0 + blockIdx.y;
  const int y = blockIdx.x * LINES + r;
  if (g.b0 == 0 && blockIdx.x == 0 && blockIdx.y == 0 && a.done)
    for (int i = t; i < a.ndone; i += NT) a.done[i] = 0u;
  int f;
  int2 w;
  const bool ok = window_ok(a, b, f, w);
  if (blockIdx.x == 0 && t == 0) {
    a.tlb[b] = ok ? w : make_int2(-1, -1);
    if (!ok) pty_raise(a.status, PTYCHO_ERR_WINDOW);
  }
  if (!ok) return;  // uniform over the CTA
  fill_twiddles(tw);
  float2 v[16];
  {
    const float2* Or = a.O + size_t(w.x + y) * a.W + w.y + j;
    const float2* Pr = a.P + y * M + j;
    const unsigned sg = unsigned((j + y) & 1) << 31;  // (-1)^(x+y), x = j + 16 k
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      float2 pv = __ldg(Pr + 16 * k);
      pv.x = __uint_as_float(__float_as_uint(pv.x) ^ sg);
      pv.y = __uint_as_float(__float_as_uint(pv.y) ^ sg);
      v[k] = c_mul(pv, __ldg(Or + 16 * k));
    }
  }
  __syncthreads();  // twiddles ready
  line256<false>(v, j, pre + r * 16 * TP, pim + r * 16 * TP, tw);
  float2* Xr = a.Eout + size_t(b) * M * M + size_t(y) * M + j;
#pragma unroll
  for (int q = 0; q < 16; ++q) Xr[16 * q] = v[q];
}

// C: inverse row DFTs in place -> E'.  grid (NCB, chunk).  CTA (0, b)
// also writes the pattern's loss: its NCB column-block partials summed in
// order, / M^2 (NaN for a skipped window).
__global__ void __launch_bounds__(NT, PTY_S256_ROWS_MINB) k_rows_inv(const Args g) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* tw = reinterpret_cast<float2*>(smem + SM_TW);
  float* pre = reinterpret_cast<float*>(smem + SM_RE);
  float* pim = reinterpret_cast<float*>(smem + SM_IM);
  const FusedArgs& a = g.f;
  const int t = threadIdx.x, r = t >> 4, j = t & 15;
  const int b = g.b0 + blockIdx.y;
  const int y = blockIdx.x * LINES + r;
  const bool ok = __ldg(&a.tlb[b].x) >= 0;
  if (blockIdx.x == 0 && t == 0 && a.loss_pat) {
    double s = 0.0;
    for (int cb = 0; cb < NCB; ++cb) s += g.lpart[size_t(b) * NCB + cb];
    a.loss_pat[b] = ok ? s / double(M * M) : (double)__int_as_float(0x7fc00000);
  }
  if (!ok) return;
  fill_twiddles(tw);
  float2* Xr = a.Eout + size_t(b) * M * M + size_t(y) * M + j;
  float2 v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = Xr[16 * k];
  __syncthreads();
  line256<true>(v, j, pre + r * 16 * TP, pim + r * 16 * TP, tw);
#pragma unroll
  for (int q = 0; q < 16; ++q) Xr[16 * q] = v[q];
}

// C with the probe gradient (large batches): grid (NCB, groups of kDpGroup
// patterns).  The CTA runs C for rows 16 rb .. 16 rb + 15 of its group's
// patterns in ascending order and, while E' is in registers, accumulates
// sum_b E'_b conj(O_b) over those rows; the group's partial, with the
// (-1)^(x+y) factor applied once, goes to part[group].  The assembly then
// never reads E' for dP (it reads it once, for dO), and k_dp_sum adds the
// partials in group order.
__global__ void __launch_bounds__(NT, 2) k_rows_inv_dp(const Args g, float2* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* tw = reinterpret_cast<float2*>(smem + SM_TW);
  float* pre = reinterpret_cast<float*>(smem + SM_RE);
  float* pim = reinterpret_cast<float*>(smem + SM_IM);
  const FusedArgs& a = g.f;
  const int t = threadIdx.x, r = t >> 4, j = t & 15;
  const int y = blockIdx.x * LINES + r;
  const int grp = g.b0 / kDpGroup + blockIdx.y;
  const int b1 = min(a.B, (grp + 1) * kDpGroup);
  fill_twiddles(tw);
  __syncthreads();
  float2 acc[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) acc[q] = make_float2(0.f, 0.f);
  for (int b = grp * kDpGroup; b < b1; ++b) {
    const int2 w = __ldg(a.tlb + b);
    const bool ok = w.x >= 0;
    if (blockIdx.x == 0 && t == 0 && a.loss_pat) {
      double s = 0.0;
      for (int cb = 0; cb < NCB; ++cb) s += g.lpart[size_t(b) * NCB + cb];
      a.loss_pat[b] = ok ? s / double(M * M) : (double)__int_as_float(0x7fc00000);
    }
    if (!ok) continue;  // uniform over the CTA
    float2* Xr = a.Eout + size_t(b) * M * M + size_t(y) * M + j;
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = Xr[16 * k];
    line256<true>(v, j, pre + r * 16 * TP, pim + r * 16 * TP, tw);
    const float2* Or = a.O + size_t(w.x + y) * a.W + w.y + j;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      Xr[16 * q] = v[q];
      c_fma_conj(acc[q], v[q], __ldg(Or + 16 * q));
    }
  }
  float2* pr = part + size_t(grp) * M * M + size_t(y) * M + j;
  const int odd = (j + y) & 1;  // x = j + 16 q has the parity of j
#pragma unroll
  for (int q = 0; q < 16; ++q) __stcg(pr + 16 * q, c_negif(acc[q], odd));
}

// dP = (accumulate ? dP : 0) + sum over groups of part[group], in group
// order: four threads per pixel pair each add a quarter of the groups (eight
// loads in flight), then the quarters are added in order.  Block 0 also
// writes the FP64 loss total.
__global__ void __launch_bounds__(256) k_dp_sum(const float2* __restrict__ part, int ngroups,
                                                 float2* __restrict__ dP, int accumulate,
                                                 const double* __restrict__ loss_pat, int B, double* loss_total) {
  __shared__ float4 quarter[4][64];
  const int qd = threadIdx.x >> 6, pl = threadIdx.x & 63;
  const int i = blockIdx.x * 64 + pl;  // pixel pair
  const float4* p4 = reinterpret_cast<const float4*>(part) + i;
  constexpr size_t kStride = M * M / 2;
  const int gq = (ngroups + 3) / 4;
  const int g1 = min(ngroups, (qd + 1) * gq);
  float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
  int gi = qd * gq;
  for (; gi + 8 <= g1; gi += 8) {
    float4 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = __ldcg(p4 + size_t(gi + u) * kStride);
#pragma unroll
    for (int u = 0; u < 8; ++u) s = make_float4(s.x + v[u].x, s.y + v[u].y, s.z + v[u].z, s.w + v[u].w);
  }
  for (; gi < g1; ++gi) {
    const float4 v = __ldcg(p4 + size_t(gi) * kStride);
    s = make_float4(s.x + v.x, s.y + v.y, s.z + v.z, s.w + v.w);
  }
  quarter[qd][pl] = s;
  __syncthreads();
  if (qd == 0) {
    s = quarter[0][pl];
#pragma unroll
    for (int k = 1; k < 4; ++k) {
      const float4 v = quarter[k][pl];
      s = make_float4(s.x + v.x, s.y + v.y, s.z + v.z, s.w + v.w);
    }
    float2* d = dP + 2 * i;  // dP is only required to be 8-byte aligned
    if (accumulate) {
      const float2 o0 = d[0], o1 = d[1];
      s = make_float4(o0.x + s.x, o0.y + s.y, o1.x + s.z, o1.y + s.w);
    }
    d[0] = make_float2(s.x, s.y);
    d[1] = make_float2(s.z, s.w);
  }
  if (blockIdx.x == 0 && loss_total) loss_sum_block(loss_pat, B, loss_total);
}

// 256-point DFT of one column per thread slot, spread over the CTA: thread
// (j, c) = (t >> 4, t & 15) holds x[j + 16 k] of column c in v[k]; a 16-point
// DFT over k, the twiddle W256^(j p), a transpose across warps through the
// planes (row p of the transpose at p * CT, so the two half-warps of a warp
// hit disjoint banks when writing and when reading), a second 16-point DFT.
// Thread (p, c) then holds X[p + 16 q] in v[q] -- the input layout again.
// Contains two barriers: every thread of the CTA calls it, with the twiddle
// table already published by a barrier.
constexpr int CT = 16 * 16 + 16;  // floats per transpose row p (16 j x 16 c + pad)
template <bool INV>
PTY_DEVI void col256(float2 (&v)[16], int j, int c, float* bre, float* bim, const float2* tw) {
  dft16<INV, 1>(v);
#pragma unroll
  for (int p = 1; p < 16; ++p) {
    const float2 w = tw[p * 16 + j];
    v[p] = c_mul(v[p], INV ? c_conj(w) : w);
  }
  __syncthreads();  // earlier readers of the planes are done
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    bre[p * CT + j * 16 + c] = v[p].x;
    bim[p * CT + j * 16 + c] = v[p].y;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = make_float2(bre[j * CT + i * 16 + c], bim[j * CT + i * 16 + c]);
  dft16<INV, 1>(v);
}
static_assert(16 * CT <= BUF, "column transpose planes fit the plane size");

// B: column DFTs, loss, and (GRAD) the gradient's inverse column DFTs.
// grid (NCB, chunk): CTA (cb, b - b0) owns columns 16 cb .. 16 cb + 15 of
// pattern b.  Thread (j, c) reads rows j + 16 k of column c: a half-warp
// reads 16 adjacent columns of one row (128 bytes), and so for the
// measurement (64 bytes) and the write-back.
template <int LOSS, bool GRAD>
__global__ void __launch_bounds__(NT, PTY_S256_COLS_MINB) k_cols(const Args g) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* tw = reinterpret_cast<float2*>(smem + SM_TW);
  float* bre = reinterpret_cast<float*>(smem + SM_RE);
  float* bim = reinterpret_cast<float*>(smem + SM_IM);
  double* red = reinterpret_cast<double*>(smem + SM_RED);
  const FusedArgs& a = g.f;
  const int t = threadIdx.x, j = t >> 4, c = t & 15;
  const int b = g.b0 + blockIdx.y;
  const int fx0 = blockIdx.x * LINES;
  if (__ldg(&a.tlb[b].x) < 0) return;  // skipped window (uniform)
  const int f = a.batch ? __ldg(a.batch + b) : b;
  float2* Xc = a.Eout + size_t(b) * M * M + fx0 + c;
  const float* Ic = a.Imeas + size_t(f) * M * M + fx0 + c;
  // the measurement block (256 rows x 64 bytes) towards L2 while the DFT runs
  asm volatile("prefetch.global.L2 [%0];" ::"l"(Ic - c + size_t(t) * M));
  fill_twiddles(tw);
  float2 v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = Xc[size_t(j + 16 * k) * M];
  __syncthreads();  // twiddles ready
  col256<false>(v, j, c, bre, bim, tw);  // v[q] = F[j + 16 q][fx0 + c]

  constexpr float inv_mn = 1.0f / float(M * M);
  float part[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const float meas = __ldg(Ic + size_t(j + 16 * q) * M);
    const float I = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
    if constexpr (LOSS == PTYCHO_LOSS_INTENSITY_GRAD) {
      part[q] = I * meas * float(M * M);
      v[q] = c_scale(v[q], 2.0f * meas);
    } else {
      float gq;
      if constexpr (LOSS == PTYCHO_LOSS_SMOOTH_L1) {
        const float dd = I - meas;
        const float ad = fabsf(dd);
        part[q] = ad < 1.0f ? 0.5f * dd * dd : ad - 0.5f;
        gq = ad < 1.0f ? dd : copysignf(1.0f, dd);
      } else {
        const float Ie = I + kEps;
        part[q] = fmaf(-meas, __logf(Ie), I);
        gq = 1.0f - __fdividef(meas, Ie);
      }
      v[q] = c_scale(v[q], 2.0f * gq * inv_mn);
    }
  }
#pragma unroll
  for (int w = 1; w < 16; w <<= 1)
#pragma unroll
    for (int i = 0; i < 16; i += 2 * w) part[i] += part[i + w];
  const double tot = block_sum<NT>((double)part[0], red);
  if (t == 0) g.lpart[size_t(b) * NCB + blockIdx.x] = tot;
  if constexpr (GRAD) {
    col256<true>(v, j, c, bre, bim, tw);  // v[q] = X2[j + 16 q][fx0 + c]
#pragma unroll
    for (int q = 0; q < 16; ++q) Xc[size_t(j + 16 * q) * M] = v[q];
  }
}

// MODE_LOSS: per-pattern losses from the column-block partials (fixed order)
__global__ void k_loss_pat(const Args g) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= g.f.B || !g.f.loss_pat) return;
  const bool ok = g.f.tlb[b].x >= 0;
  double s = 0.0;
  for (int cb = 0; cb < NCB; ++cb) s += g.lpart[size_t(b) * NCB + cb];
  g.f.loss_pat[b] = ok ? s / double(M * M) : (double)__int_as_float(0x7fc00000);
}

template <typename K>
static bool set_smem(K kern, size_t bytes, PtyDevCache& cache) {
  int dev;
  if (cache.get(&dev)) return true;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)) != cudaSuccess)
    return false;
  cache.put(dev, 1);
  return true;
}

template <int LOSS>
static int launch_t(bool adj, const FusedArgs& fa, double* lpart, float2* dp_part, cudaStream_t s) {
  // "shared-memory attribute set" per device and kernel; cleared when a
  // launch is refused (a device reset drops the attribute), so the next
  // call sets it again
  static PtyDevCache c_rows_fwd, c_rows_inv, c_rows_inv_dp, c_cols_adj, c_cols_loss;
  PtyDevCache& c_cols = adj ? c_cols_adj : c_cols_loss;
  auto kcols = adj ? k_cols<LOSS, true> : k_cols<LOSS, false>;
  if (!set_smem(k_rows_fwd, SMEM_ROWS, c_rows_fwd) || !set_smem(k_rows_inv, SMEM_ROWS, c_rows_inv) ||
      !set_smem(k_rows_inv_dp, SMEM_ROWS, c_rows_inv_dp) || !set_smem(kcols, SMEM_COLS, c_cols))
    return PTYCHO_ERR_LAUNCH;
  Args g{fa, lpart, 0};
  for (int b0 = 0; b0 < fa.B; b0 += kChunk) {
    const int n = fa.B - b0 < kChunk ? fa.B - b0 : kChunk;
    g.b0 = b0;
    const dim3 grid(NCB, n);
    k_rows_fwd<<<grid, NT, SMEM_ROWS, s>>>(g);
    kcols<<<grid, NT, SMEM_COLS, s>>>(g);
    if (adj && dp_part)
      k_rows_inv_dp<<<dim3(NCB, (n + kDpGroup - 1) / kDpGroup), NT, SMEM_ROWS, s>>>(g, dp_part);
    else if (adj)
      k_rows_inv<<<grid, NT, SMEM_ROWS, s>>>(g);
  }
  if (!adj) k_loss_pat<<<(fa.B + 255) / 256, 256, 0, s>>>(g);
  if (cudaGetLastError() == cudaSuccess) return PTYCHO_OK;
  int dev;
  for (PtyDevCache* c : {&c_rows_fwd, &c_rows_inv, &c_rows_inv_dp, &c_cols})
    if (c->get(&dev)) c->put(dev, 0);
  return PTYCHO_ERR_LAUNCH;
}

}  // namespace s256
}  // namespace pty

namespace pty {

bool split256_supported(int mode, int loss) {
  return (mode == MODE_LOSS || mode == MODE_ADJ) &&
         (loss == PTYCHO_LOSS_SMOOTH_L1 || loss == PTYCHO_LOSS_POISSON || loss == PTYCHO_LOSS_INTENSITY_GRAD);
}

// a.Eout (B M^2 complex64) is the scratch and, in MODE_ADJ, the output E';
// a.tlb receives the resolved windows in both modes; lpart holds B * 16 doubles
int launch_split256(int mode, int loss, const FusedArgs& a, double* lpart, float2* dp_part, cudaStream_t s) {
  using namespace s256;
  if (!split256_supported(mode, loss) || !a.Eout || !a.tlb || !lpart) return PTYCHO_ERR_INVALID_ARG;
  const bool adj = mode == MODE_ADJ;
  switch (loss) {
    case PTYCHO_LOSS_SMOOTH_L1: return launch_t<PTYCHO_LOSS_SMOOTH_L1>(adj, a, lpart, dp_part, s);
    case PTYCHO_LOSS_POISSON: return launch_t<PTYCHO_LOSS_POISSON>(adj, a, lpart, dp_part, s);
    default: return launch_t<PTYCHO_LOSS_INTENSITY_GRAD>(adj, a, lpart, dp_part, s);
  }
}

int split256_dp_sum(const float2* dp_part, int B, float2* dP, bool accumulate, const double* loss_pat,
                    double* loss_total, cudaStream_t s) {
  using namespace s256;
  const int ngroups = (B + kDpGroup - 1) / kDpGroup;
  k_dp_sum<<<M * M / 2 / 64, 256, 0, s>>>(dp_part, ngroups, dP, accumulate ? 1 : 0, loss_pat, B, loss_total);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // namespace pty
