// gsplat.cu -- 2-D complex Gaussian splatting (real and imaginary channels) on
// 16 x 16 pixel tiles: preprocess, render and a deterministic backward.
//
// Replaces the reference's gscp rasteriser (gscp/csrc/gscp_rasterizer:
// preprocessCUDA / preprocessCUDA_cholesky forward.cu:18-170, renderCUDA
// forward.cu:175-250, renderCUDA_backward backward.cu:21-133 and the
// preprocess backward passes backward.cu:138-275), bound to Python by
// gscp/cuda/_wrapper.py:18-163.  Same per-Gaussian arithmetic and the same
// per-pixel terms and skip rules (the exponent regrouped so pixels of one column
// share work, equal up to rounding; exp is __expf, which the reference's
// fast-math build also evaluates); the pipeline around it is different:
//
// * Binning without a sort or a host round trip.  The reference counts
//   tile overlaps, scans them, reads the total back to the host, duplicates
//   (tile, index) keys and radix-sorts them so each tile sees its Gaussians in
//   ascending index order.  Here each Gaussian sets its bit in a per-tile
//   bitmask (integer atomicOr, so the result does not depend on timing) and a
//   second-level mask marks the non-empty 32-bit words.  A tile reads its
//   masks in index order, so its list comes out ascending with no sort, the
//   whole forward is stream-ordered (graph-capturable) and needs no host sync.
// * Render: one CTA of 128 threads per tile, two pixels per thread (rows y and
//   y + 8 of one column, sharing the Gaussian's column terms); the tile's list
//   is compacted from the masks 4096 Gaussians at a time (block scan of the
//   word popcounts) and the Gaussians are staged through shared memory 128 at
//   a time.  Each pixel sums in ascending Gaussian index, as the reference.
//   (Four pixels per thread in 64-thread CTAs measured slower: 1024 tiles
//   then leave too few warps per SM.)
// * Backward: one warp per Gaussian walks the tiles of its rectangle and sums
//   its seven per-pixel terms in a fixed order (lane-strided pixels, then an
//   XOR tree), then applies the preprocess chain rule.  No float atomics: the
//   gradients are bitwise reproducible (the reference's warp sums + atomicAdd
//   are not).
//
// The preprocess is written with explicit round-to-nearest intrinsics, so
// radii and tile rectangles follow the float32 operation sequence exactly
// (no FMA contraction) and a float32 restatement reproduces them bit for bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace pty {
namespace gs {

constexpr int TILE = 16, NPIX = TILE * TILE, NTR = 128, CHUNK_WORDS = NTR, WARPS_BWD = 8;

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Layout {
  size_t mean, conic, rect, radius, mask1, mask2, total;
  int tx, ty, NW, NV;
};

inline Layout layout(int N, int H, int W) {
  Layout L;
  L.tx = (W + TILE - 1) / TILE;
  L.ty = (H + TILE - 1) / TILE;
  L.NW = (N + 31) / 32;
  L.NV = (L.NW + 31) / 32;
  const size_t T = size_t(L.tx) * L.ty;
  size_t o = 0;
  L.mean = o;   o = align256(o + size_t(N) * sizeof(float2));
  L.conic = o;  o = align256(o + size_t(N) * sizeof(float4));
  L.rect = o;   o = align256(o + size_t(N) * sizeof(int4));
  L.radius = o; o = align256(o + size_t(N) * sizeof(int));
  L.mask1 = o;  o = align256(o + T * L.NW * sizeof(uint32_t));
  L.mask2 = o;  o = align256(o + T * L.NV * sizeof(uint32_t));
  L.total = o;
  return L;
}

struct Geom {
  float2* mean;
  float4* conic;  // (x, y, z, unused) = inverse covariance (c, -b, a) / det
  int4* rect;     // tile rectangle x0, y0, x1, y1 (exclusive ends)
  int* radius;
  uint32_t* mask1;  // [tiles][NW]: bit i of word w = Gaussian 32 w + i covers the tile
  uint32_t* mask2;  // [tiles][NV]: bit j of word v = mask1 word 32 v + j is non-zero
};

inline Geom geom(void* ws, const Layout& L) {
  char* b = static_cast<char*>(ws);
  return {reinterpret_cast<float2*>(b + L.mean), reinterpret_cast<float4*>(b + L.conic),
          reinterpret_cast<int4*>(b + L.rect), reinterpret_cast<int*>(b + L.radius),
          reinterpret_cast<uint32_t*>(b + L.mask1), reinterpret_cast<uint32_t*>(b + L.mask2)};
}

PTY_DEVI float clampf(float v, float lo, float hi) { return fminf(hi, fmaxf(lo, v)); }

// Covariance [[a, b], [b, c]] and determinant of Gaussian i (float32, rn).
template <int KIND>
PTY_DEVI void covariance(const float* __restrict__ p1, const float* __restrict__ p2, int i, float mxs, float mns,
                         float& a, float& b, float& c, float& det) {
  if constexpr (KIND == PTYCHO_GS_RS) {
    const float sx = clampf(expf(p1[2 * i + 0]), mns, mxs), sy = clampf(expf(p1[2 * i + 1]), mns, mxs);
    const float sx2 = __fmul_rn(sx, sx), sy2 = __fmul_rn(sy, sy);
    const float th = p2[i];
    const float ct = cosf(th), st = sinf(th);
    const float cc = __fmul_rn(ct, ct), ss = __fmul_rn(st, st), cs = __fmul_rn(ct, st);
    a = __fadd_rn(__fmul_rn(cc, sx2), __fmul_rn(ss, sy2));
    b = __fmul_rn(cs, __fsub_rn(sx2, sy2));
    c = __fadd_rn(__fmul_rn(ss, sx2), __fmul_rn(cc, sy2));
    det = __fsub_rn(__fmul_rn(a, c), __fmul_rn(b, b));
  } else {
    const float l11 = clampf(expf(p1[2 * i + 0]), mns, mxs), l22 = clampf(expf(p1[2 * i + 1]), mns, mxs);
    const float l21 = p2[i];
    a = __fmul_rn(l11, l11);
    b = __fmul_rn(l11, l21);
    c = __fadd_rn(__fmul_rn(l21, l21), __fmul_rn(l22, l22));
    det = __fmul_rn(__fmul_rn(a, l22), l22);
  }
}

// One thread per Gaussian: mean, conic, radius, tile rectangle, mask bits.
template <int KIND>
__global__ void __launch_bounds__(256) k_gs_pre(const float* __restrict__ xy, const float* __restrict__ p1,
                                                const float* __restrict__ p2, int N, int H, int W, int tx, int ty,
                                                int NW, int NV, float mxs, float mns, Geom g,
                                                int* __restrict__ radii_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float mx = clampf(xy[2 * i + 0], 0.f, float(W - 1)), my = clampf(xy[2 * i + 1], 0.f, float(H - 1));
  float a, b, c, det;
  covariance<KIND>(p1, p2, i, mxs, mns, a, b, c, det);
  int radius = 0;
  float4 con = make_float4(0.f, 0.f, 0.f, 0.f);
  if (det > 0.f) {
    const float dinv = __fdiv_rn(1.f, det);
    con = make_float4(__fmul_rn(c, dinv), __fmul_rn(-b, dinv), __fmul_rn(a, dinv), 0.f);
    const float mid = __fmul_rn(0.5f, __fadd_rn(a, c));
    const float lam = __fadd_rn(mid, __fsqrt_rn(fmaxf(0.1f, __fsub_rn(__fmul_rn(mid, mid), det))));
    radius = int(ceilf(__fmul_rn(3.f, __fsqrt_rn(lam))));
  }
  int4 rc = make_int4(0, 0, 0, 0);
  if (radius > 0) {
    const float r = float(radius);
    rc.x = min(tx, max(0, int(__fdiv_rn(__fsub_rn(mx, r), float(TILE)))));
    rc.y = min(ty, max(0, int(__fdiv_rn(__fsub_rn(my, r), float(TILE)))));
    rc.z = min(tx, max(0, int(__fdiv_rn(__fadd_rn(__fadd_rn(mx, r), float(TILE - 1)), float(TILE)))));
    rc.w = min(ty, max(0, int(__fdiv_rn(__fadd_rn(__fadd_rn(my, r), float(TILE - 1)), float(TILE)))));
  } else {
    radius = 0;
  }
  g.mean[i] = make_float2(mx, my);
  g.conic[i] = con;
  g.rect[i] = rc;
  g.radius[i] = radius;
  if (radii_out) radii_out[i] = radius;
  const uint32_t b1 = 1u << (i & 31), b2 = 1u << ((i >> 5) & 31);
  for (int y = rc.y; y < rc.w; ++y)
    for (int x = rc.x; x < rc.z; ++x) {
      const size_t t = size_t(y) * tx + x;
      atomicOr(g.mask1 + t * NW + (i >> 5), b1);
      atomicOr(g.mask2 + t * NV + (i >> 10), b2);
    }
}

// Per-pixel exponent of one Gaussian, rearranged so a thread's two pixels
// (one column, rows dy apart) share the column terms:
//   power = -0.5 (cx dx^2 + cz dy^2) - cy dx dy = p0 - dy (0.5 cz dy + cy dx),
// p0 = -0.5 cx dx^2.  The term is kept where power <= 0 and exp(power) >= 1e-7
// (a select, so the warp does not diverge); exp is __expf, the exponential the
// reference's fast-math build evaluates.
PTY_DEVI float gauss_term(float p0, float h, float czh, float dy) {
  const float power = fmaf(-dy, fmaf(czh, dy, h), p0);
  const float G = __expf(power);
  return (power <= 0.f && G >= 1e-7f) ? G : 0.f;
}

// One CTA of NTR threads per tile; thread (x, y) owns the pixels
// (x, y + RSTEP r), r < ROWS, which share the Gaussian's column terms.
__global__ void __launch_bounds__(NTR) k_gs_render(const float2* __restrict__ weight, int H, int W, int tx, int NW,
                                                   int NV, Geom g, float* __restrict__ out) {
  constexpr int ROWS = NPIX / NTR, RSTEP = TILE / ROWS;
  __shared__ int s_ids[CHUNK_WORDS * 32];
  __shared__ float2 s_mean[NTR];
  __shared__ float4 s_con[NTR];  // (0.5 cx, cy, 0.5 cz, unused)
  __shared__ float2 s_w[NTR];
  __shared__ int s_warp[NTR / 32];
  const int t = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int px = (t % tx) * TILE + (threadIdx.x & (TILE - 1));
  const int py = (t / tx) * TILE + (threadIdx.x / TILE);
  const float pxf = float(px);
  float pyf[ROWS], acc_re[ROWS], acc_im[ROWS];
#pragma unroll
  for (int r = 0; r < ROWS; ++r) {
    pyf[r] = float(py + RSTEP * r);
    acc_re[r] = 0.f;
    acc_im[r] = 0.f;
  }
  const uint32_t* m1 = g.mask1 + size_t(t) * NW;
  const uint32_t* m2 = g.mask2 + size_t(t) * NV;
  for (int w0 = 0; w0 < NW; w0 += CHUNK_WORDS) {
    const int w = w0 + threadIdx.x;
    uint32_t bits = 0;
    if (w < NW && ((__ldg(m2 + (w >> 5)) >> (w & 31)) & 1u)) bits = __ldg(m1 + w);
    // block exclusive scan of the word popcounts -> list positions (index order)
    const int cnt = __popc(bits);
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += v;
    }
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    int base = 0, total = 0;
#pragma unroll
    for (int k = 0; k < NTR / 32; ++k) {
      const int v = s_warp[k];
      base += k < wid ? v : 0;
      total += v;
    }
    int pos = base + inc - cnt;
    while (bits) {
      s_ids[pos++] = (w << 5) + (__ffs(bits) - 1);
      bits &= bits - 1;
    }
    __syncthreads();
    for (int c0 = 0; c0 < total; c0 += NTR) {
      const int j = c0 + threadIdx.x;
      if (j < total) {
        const int id = s_ids[j];
        const float4 con = g.conic[id];
        s_mean[threadIdx.x] = g.mean[id];
        s_con[threadIdx.x] = make_float4(0.5f * con.x, con.y, 0.5f * con.z, 0.f);
        s_w[threadIdx.x] = __ldg(weight + id);
      }
      __syncthreads();
      const int nb = min(NTR, total - c0);
      for (int k = 0; k < nb; ++k) {
        const float2 m = s_mean[k];
        const float4 con = s_con[k];
        const float2 wk = s_w[k];
        const float dx = m.x - pxf;
        const float p0 = -con.x * dx * dx, h = con.y * dx;
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
          const float G = gauss_term(p0, h, con.z, m.y - pyf[r]);
          acc_re[r] = fmaf(wk.x, G, acc_re[r]);
          acc_im[r] = fmaf(wk.y, G, acc_im[r]);
        }
      }
      __syncthreads();
    }
  }
  const size_t plane = size_t(H) * W;
#pragma unroll
  for (int r = 0; r < ROWS; ++r) {
    const int y = py + RSTEP * r;
    if (px < W && y < H) {
      out[size_t(y) * W + px] = acc_re[r];
      out[plane + size_t(y) * W + px] = acc_im[r];
    }
  }
}

PTY_DEVI float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One warp per Gaussian: the per-pixel terms of every tile in its rectangle
// (the pixels the reference's tile loop visits for it), fixed-order sums, then
// the preprocess chain rule.
template <int KIND>
__global__ void __launch_bounds__(32 * WARPS_BWD) k_gs_bwd(const float* __restrict__ xy, const float* __restrict__ p1,
                                                           const float* __restrict__ p2,
                                                           const float2* __restrict__ weight, int N, int H, int W,
                                                           float mxs, float mns, Geom g,
                                                           const float* __restrict__ gout, float* __restrict__ dxy,
                                                           float* __restrict__ dp1, float* __restrict__ dp2,
                                                           float* __restrict__ dweight) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * WARPS_BWD + (threadIdx.x >> 5);
  if (i >= N) return;  // warp-uniform
  const int radius = g.radius[i];
  float gw0 = 0.f, gw1 = 0.f, gmx = 0.f, gmy = 0.f, gc0 = 0.f, gc1 = 0.f, gc2 = 0.f;
  if (radius > 0) {
    const int4 rc = g.rect[i];
    const float2 m = g.mean[i];
    const float4 con = g.conic[i];
    const float2 w = __ldg(weight + i);
    const float* g0 = gout;
    const float* g1 = gout + size_t(H) * W;
    const float czh = 0.5f * con.z;
    const int lx = lane & (TILE - 1), ly = lane / TILE;  // lane -> pixel (lx, ly + 2k) of each tile
    for (int ty = rc.y; ty < rc.w; ++ty)
      for (int tx = rc.x; tx < rc.z; ++tx) {
        const int px = tx * TILE + lx;
        const float dx = m.x - float(px);
        const float p0 = -0.5f * con.x * dx * dx, h = con.y * dx;
        const float mxc = -con.x * dx, myc = -con.y * dx, c0c = -0.5f * dx * dx;
#pragma unroll
        for (int k = 0; k < NPIX / 32; ++k) {
          const int py = ty * TILE + ly + 2 * k;
          const float dy = m.y - float(py);
          float G = gauss_term(p0, h, czh, dy);
          const bool ok = G != 0.f && px < W && py < H;  // terms that are zero add nothing
          G = ok ? G : 0.f;
          const size_t q = size_t(py) * W + px;
          const float d0 = ok ? __ldg(g0 + q) : 0.f, d1 = ok ? __ldg(g1 + q) : 0.f;
          const float u = G * fmaf(w.y, d1, w.x * d0);  // G dL/dG
          gw0 = fmaf(G, d0, gw0);
          gw1 = fmaf(G, d1, gw1);
          gmx = fmaf(u, fmaf(-con.y, dy, mxc), gmx);  // dG/ddx = G (-cx dx - cy dy)
          gmy = fmaf(u, fmaf(-con.z, dy, myc), gmy);  // dG/ddy = G (-cz dy - cy dx)
          const float v = u * dy;
          gc0 = fmaf(u, c0c, gc0);         // -0.5 G dx^2 dL/dG
          gc1 = fmaf(-dx, v, gc1);         // -G dx dy dL/dG
          gc2 = fmaf(-0.5f * dy, v, gc2);  // -0.5 G dy^2 dL/dG
        }
      }
  }
  gw0 = warp_sum_f(gw0);
  gw1 = warp_sum_f(gw1);
  gmx = warp_sum_f(gmx);
  gmy = warp_sum_f(gmy);
  gc0 = warp_sum_f(gc0);
  gc1 = warp_sum_f(gc1);
  gc2 = warp_sum_f(gc2);
  if (lane != 0) return;
  if (radius <= 0) {
    dxy[2 * i] = dxy[2 * i + 1] = 0.f;
    dp1[2 * i] = dp1[2 * i + 1] = 0.f;
    dp2[i] = 0.f;
    dweight[2 * i] = dweight[2 * i + 1] = 0.f;
    return;
  }
  dweight[2 * i] = gw0;
  dweight[2 * i + 1] = gw1;
  dxy[2 * i] = gmx;  // positions are in pixels: the mean gradient passes through
  dxy[2 * i + 1] = gmy;
  float a, b, c, det;
  covariance<KIND>(p1, p2, i, mxs, mns, a, b, c, det);
  const float d2 = 1.f / (det * det + 1e-7f);
  const float da = d2 * (-c * c * gc0 + b * c * gc1 + (det - a * c) * gc2);
  const float db = d2 * (2.f * b * c * gc0 - (det + 2.f * b * b) * gc1 + 2.f * a * b * gc2);
  const float dc = d2 * ((det - a * c) * gc0 + a * b * gc1 - a * a * gc2);
  if constexpr (KIND == PTYCHO_GS_RS) {
    const float th = p2[i];
    const float ct = cosf(th), st = sinf(th);
    const float sxr = expf(p1[2 * i]), syr = expf(p1[2 * i + 1]);
    const float sx = clampf(sxr, mns, mxs), sy = clampf(syr, mns, mxs);
    const float sx2 = sx * sx, sy2 = sy * sy;
    const float dsx2 = ct * ct * da + ct * st * db + st * st * dc;
    const float dsy2 = st * st * da - ct * st * db + ct * ct * dc;
    const float dth = 2.f * ct * st * (sy2 - sx2) * da + (ct * ct - st * st) * (sx2 - sy2) * db +
                      2.f * st * ct * (sx2 - sy2) * dc;
    const float inx = (sxr >= mns && sxr <= mxs) ? 1.f : 0.f, iny = (syr >= mns && syr <= mxs) ? 1.f : 0.f;
    dp1[2 * i] = dsx2 * 2.f * sx2 * inx;
    dp1[2 * i + 1] = dsy2 * 2.f * sy2 * iny;
    dp2[i] = dth;
  } else {
    const float l11r = expf(p1[2 * i]), l22r = expf(p1[2 * i + 1]);
    const float l11 = clampf(l11r, mns, mxs), l22 = clampf(l22r, mns, mxs);
    const float l21 = p2[i];
    const float dl11 = 2.f * l11 * da + l21 * db;
    const float dl21 = l11 * db + 2.f * l21 * dc;
    const float dl22 = 2.f * l22 * dc;
    const float in11 = (l11r >= mns && l11r <= mxs) ? 1.f : 0.f, in22 = (l22r >= mns && l22r <= mxs) ? 1.f : 0.f;
    dp1[2 * i] = dl11 * l11 * in11;
    dp1[2 * i + 1] = dl22 * l22 * in22;
    dp2[i] = dl21;
  }
}

inline int check_common(int kind, const float* xy, const float* p1, const float* p2, const float* weight, int N,
                        int H, int W, int max_patch_radius, float min_scale) {
  if (kind != PTYCHO_GS_RS && kind != PTYCHO_GS_CHOLESKY) return PTYCHO_ERR_INVALID_ARG;
  if (N < 0 || H <= 0 || W <= 0 || max_patch_radius <= 0 || !(min_scale >= 0.f)) return PTYCHO_ERR_INVALID_ARG;
  if (N > (1 << 28) || H > 65536 || W > 65536) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (N > 0 && (!xy || !p1 || !p2 || !weight)) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(xy, 8) || !pty_aligned(weight, 8) || !pty_aligned(p1, 8) || !pty_aligned(p2, 4))
    return PTYCHO_ERR_MISALIGNED;
  return PTYCHO_OK;
}

}  // namespace gs
}  // namespace pty

using namespace pty;

extern "C" {

size_t ptycho_gs_workspace_size(int N, int H, int W) {
  if (N < 0 || H <= 0 || W <= 0) return 0;
  return gs::layout(N, H, W).total;
}

int ptycho_gs_forward(int kind, const float* xy, const float* p1, const float* p2, const float* weight, int N, int H,
                      int W, int max_patch_radius, float min_scale, float* out, int* radii_out, void* workspace,
                      size_t workspace_bytes, ptycho_stream_t stream) {
  int st = gs::check_common(kind, xy, p1, p2, weight, N, H, W, max_patch_radius, min_scale);
  if (st != PTYCHO_OK) return st;
  if (!out || (!workspace && N > 0)) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(out, 4) || !pty_aligned(workspace, 256)) return PTYCHO_ERR_MISALIGNED;
  const gs::Layout L = gs::layout(N, H, W);
  if (workspace_bytes < L.total) return PTYCHO_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const gs::Geom g = gs::geom(workspace, L);
  if (N == 0) {
    cudaMemsetAsync(out, 0, size_t(2) * H * W * sizeof(float), s);
    return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
  }
  const size_t T = size_t(L.tx) * L.ty;
  cudaMemsetAsync(g.mask1, 0, T * L.NW * sizeof(uint32_t), s);
  cudaMemsetAsync(g.mask2, 0, T * L.NV * sizeof(uint32_t), s);
  const int nb = (N + 255) / 256;
  const float mxs = float(max_patch_radius);
  if (kind == PTYCHO_GS_RS)
    gs::k_gs_pre<PTYCHO_GS_RS><<<nb, 256, 0, s>>>(xy, p1, p2, N, H, W, L.tx, L.ty, L.NW, L.NV, mxs, min_scale, g,
                                                  radii_out);
  else
    gs::k_gs_pre<PTYCHO_GS_CHOLESKY><<<nb, 256, 0, s>>>(xy, p1, p2, N, H, W, L.tx, L.ty, L.NW, L.NV, mxs, min_scale,
                                                        g, radii_out);
  gs::k_gs_render<<<unsigned(T), gs::NTR, 0, s>>>(reinterpret_cast<const float2*>(weight), H, W, L.tx, L.NW, L.NV,
                                                   g, out);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_gs_backward(int kind, const float* xy, const float* p1, const float* p2, const float* weight, int N, int H,
                       int W, int max_patch_radius, float min_scale, const float* grad_out, const void* workspace,
                       size_t workspace_bytes, float* dxy, float* dp1, float* dp2, float* dweight,
                       ptycho_stream_t stream) {
  int st = gs::check_common(kind, xy, p1, p2, weight, N, H, W, max_patch_radius, min_scale);
  if (st != PTYCHO_OK) return st;
  if (N == 0) return PTYCHO_OK;
  if (!grad_out || !workspace || !dxy || !dp1 || !dp2 || !dweight) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(grad_out, 4) || !pty_aligned(workspace, 256) || !pty_aligned(dxy, 4) || !pty_aligned(dp1, 4) ||
      !pty_aligned(dp2, 4) || !pty_aligned(dweight, 4))
    return PTYCHO_ERR_MISALIGNED;
  const gs::Layout L = gs::layout(N, H, W);
  if (workspace_bytes < L.total) return PTYCHO_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const gs::Geom g = gs::geom(const_cast<void*>(workspace), L);
  const int nb = (N + gs::WARPS_BWD - 1) / gs::WARPS_BWD;
  const float mxs = float(max_patch_radius);
  const float2* w2 = reinterpret_cast<const float2*>(weight);
  if (kind == PTYCHO_GS_RS)
    gs::k_gs_bwd<PTYCHO_GS_RS><<<nb, 32 * gs::WARPS_BWD, 0, s>>>(xy, p1, p2, w2, N, H, W, mxs, min_scale, g, grad_out,
                                                                 dxy, dp1, dp2, dweight);
  else
    gs::k_gs_bwd<PTYCHO_GS_CHOLESKY><<<nb, 32 * gs::WARPS_BWD, 0, s>>>(xy, p1, p2, w2, N, H, W, mxs, min_scale, g,
                                                                       grad_out, dxy, dp1, dp2, dweight);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // extern "C"
