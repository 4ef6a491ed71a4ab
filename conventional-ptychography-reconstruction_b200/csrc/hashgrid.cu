// hashgrid.cu -- multi-resolution hash encoding (forward, deterministic backward).
//
// Replaces the tiny-cuda-nn HashGrid encoding the reference consumes at
// models/complex_inr.py:130-145 (called at :279 and :294): 2-D coordinates
// in [0,1] -> n_levels x F features.  Level l has scale
// s_l = base * per_level_scale^l - 1 and r_l = ceil(s_l) + 1 vertices per
// axis; a coordinate maps to x * s_l + 0.5, whose floor is the cell corner and
// whose fraction gives the bilinear weights.  A level whose r_l^2 (rounded up
// to a multiple of 8) fits in T = 2^log2_hashmap_size entries is indexed
// densely (ix + iy * r_l), otherwise by (ix * 1) ^ (iy * 2654435761) mod T.
// Level l's entries start at the sum of the previous levels' entry counts;
// each entry holds F = 2 floats (the table is [entries][2] float32).
//
// Backward: the coordinates of an INR are fixed, so the (entry, coordinate,
// weight) contributions are static.  ptycho_hashgrid_contrib emits them; the
// caller sorts them by entry once (stable) and passes the CSR to
// ptycho_hashgrid_backward, which gathers each entry's contributions in that
// fixed order -- a deterministic table-gradient "scatter" without atomics.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "common.cuh"

namespace pty {

constexpr int kMaxLevels = 32;
constexpr uint32_t kPrimeY = 2654435761u;

struct LevelTable {
  float scale[kMaxLevels];
  int res[kMaxLevels];
  int n[kMaxLevels];       // entries in the level
  int offset[kMaxLevels];  // first entry of the level
  int dense[kMaxLevels];
  int levels;
  int total;  // total entries
};

static int make_levels(int n_levels, int log2_T, int base_res, float per_level_scale, LevelTable* L) {
  if (n_levels < 1 || n_levels > kMaxLevels || log2_T < 4 || log2_T > 26 || base_res < 1 ||
      !(per_level_scale >= 1.0f))
    return PTYCHO_ERR_INVALID_ARG;
  const long long T = 1ll << log2_T;
  long long off = 0;
  for (int l = 0; l < n_levels; ++l) {
    const double scale = double(base_res) * pow(double(per_level_scale), double(l)) - 1.0;
    const long long res = (long long)ceil(scale) + 1;
    long long dn = res * res;
    dn = (dn + 7) / 8 * 8;
    const long long n = dn < T ? dn : T;
    L->scale[l] = (float)scale;
    L->res[l] = (int)res;
    L->n[l] = (int)n;
    L->offset[l] = (int)off;
    L->dense[l] = dn <= T;
    off += n;
  }
  L->levels = n_levels;
  L->total = (int)off;
  return off < (1ll << 31) ? PTYCHO_OK : PTYCHO_ERR_INVALID_ARG;
}

// entry of corner (cx, cy) of level l: index mod n_l.  A hashed level has
// n_l = 2^log2_hashmap_size (a mask); a dense level's index cx + cy*r is below
// n_l except for corners on the far edge, which take the modulo.
PTY_DEVI int corner_entry(const LevelTable& L, int l, int cx, int cy) {
  const uint32_t n = uint32_t(L.n[l]);
  uint32_t e;
  if (L.dense[l]) {
    e = uint32_t(cx) + uint32_t(cy) * uint32_t(L.res[l]);
    if (e >= n) e %= n;
  } else {
    e = uint32_t(cx) ^ (uint32_t(cy) * kPrimeY);
    e = (n & (n - 1)) == 0 ? (e & (n - 1)) : (e % n);
  }
  return L.offset[l] + int(e);
}

// one thread per coordinate, all levels: adjacent threads hold adjacent
// coordinates, so each level's corner gathers of a warp fall on neighbouring
// cells, and a thread writes its n_levels x 2 features contiguously
__global__ void __launch_bounds__(256) k_hash_fwd(const float2* __restrict__ coords, int N,
                                                  const float2* __restrict__ table, const LevelTable L,
                                                  float2* __restrict__ feat) {
  const int n = blockIdx.x * 256 + threadIdx.x;
  if (n >= N) return;
  const float2 x = __ldg(coords + n);
  float2* out = feat + (long long)n * L.levels;
#pragma unroll 4
  for (int l = 0; l < L.levels; ++l) {
    const float s = L.scale[l];
    const float px = fmaf(x.x, s, 0.5f), py = fmaf(x.y, s, 0.5f);
    const float gx = floorf(px), gy = floorf(py);
    const float fx = px - gx, fy = py - gy;
    const int ix = int(gx), iy = int(gy);
    const float2 t00 = __ldg(table + corner_entry(L, l, ix, iy));
    const float2 t10 = __ldg(table + corner_entry(L, l, ix + 1, iy));
    const float2 t01 = __ldg(table + corner_entry(L, l, ix, iy + 1));
    const float2 t11 = __ldg(table + corner_entry(L, l, ix + 1, iy + 1));
    const float w00 = (1.f - fx) * (1.f - fy), w10 = fx * (1.f - fy), w01 = (1.f - fx) * fy, w11 = fx * fy;
    float2 o;
    o.x = fmaf(w11, t11.x, fmaf(w01, t01.x, fmaf(w10, t10.x, w00 * t00.x)));
    o.y = fmaf(w11, t11.y, fmaf(w01, t01.y, fmaf(w10, t10.y, w00 * t00.y)));
    out[l] = o;
  }
}

// feature-major forward: blockIdx.y = level, one thread per coordinate; writes
// features [2L][N] (feature 2l + c of coordinate n at (2l + c) * N + n), so
// every store is coalesced and the grid has L times the threads
__global__ void __launch_bounds__(256) k_hash_fwd_planar(const float2* __restrict__ coords, int N,
                                                         const float2* __restrict__ table, const LevelTable L,
                                                         float* __restrict__ feat) {
  const int n = blockIdx.x * 256 + threadIdx.x;
  const int l = blockIdx.y;
  if (n >= N) return;
  const float2 x = __ldg(coords + n);
  const float s = L.scale[l];
  const float px = fmaf(x.x, s, 0.5f), py = fmaf(x.y, s, 0.5f);
  const float gx = floorf(px), gy = floorf(py);
  const float fx = px - gx, fy = py - gy;
  const int ix = int(gx), iy = int(gy);
  const float2 t00 = __ldg(table + corner_entry(L, l, ix, iy));
  const float2 t10 = __ldg(table + corner_entry(L, l, ix + 1, iy));
  const float2 t01 = __ldg(table + corner_entry(L, l, ix, iy + 1));
  const float2 t11 = __ldg(table + corner_entry(L, l, ix + 1, iy + 1));
  const float w00 = (1.f - fx) * (1.f - fy), w10 = fx * (1.f - fy), w01 = (1.f - fx) * fy, w11 = fx * fy;
  feat[size_t(2 * l) * N + n] = fmaf(w11, t11.x, fmaf(w01, t01.x, fmaf(w10, t10.x, w00 * t00.x)));
  feat[size_t(2 * l + 1) * N + n] = fmaf(w11, t11.y, fmaf(w01, t01.y, fmaf(w10, t10.y, w00 * t00.y)));
}

// feature-major forward, one thread per coordinate over all levels: the
// coordinate is read once (not once per level) and each level's two stores
// are still coalesced across the warp
__global__ void __launch_bounds__(256) k_hash_fwd_planar_all(const float2* __restrict__ coords, int N,
                                                             const float2* __restrict__ table, const LevelTable L,
                                                             float* __restrict__ feat) {
  const int n = blockIdx.x * 256 + threadIdx.x;
  if (n >= N) return;
  const float2 x = __ldg(coords + n);
#pragma unroll 4
  for (int l = 0; l < L.levels; ++l) {
    const float s = L.scale[l];
    const float px = fmaf(x.x, s, 0.5f), py = fmaf(x.y, s, 0.5f);
    const float gx = floorf(px), gy = floorf(py);
    const float fx = px - gx, fy = py - gy;
    const int ix = int(gx), iy = int(gy);
    const float2 t00 = __ldg(table + corner_entry(L, l, ix, iy));
    const float2 t10 = __ldg(table + corner_entry(L, l, ix + 1, iy));
    const float2 t01 = __ldg(table + corner_entry(L, l, ix, iy + 1));
    const float2 t11 = __ldg(table + corner_entry(L, l, ix + 1, iy + 1));
    const float w00 = (1.f - fx) * (1.f - fy), w10 = fx * (1.f - fy), w01 = (1.f - fx) * fy, w11 = fx * fy;
    feat[size_t(2 * l) * N + n] = fmaf(w11, t11.x, fmaf(w01, t01.x, fmaf(w10, t10.x, w00 * t00.x)));
    feat[size_t(2 * l + 1) * N + n] = fmaf(w11, t11.y, fmaf(w01, t01.y, fmaf(w10, t10.y, w00 * t00.y)));
  }
}

// contributions: for coordinate n, level l, corner k -> key = entry,
// item = n * levels + l (feature pair index), weight
__global__ void __launch_bounds__(256) k_hash_contrib(const float2* __restrict__ coords, int N, const LevelTable L,
                                                      int* __restrict__ key, int* __restrict__ item,
                                                      float* __restrict__ weight) {
  const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
  if (i >= (long long)N * L.levels) return;
  const int n = int(i / L.levels), l = int(i - (long long)n * L.levels);
  const float2 x = __ldg(coords + n);
  const float s = L.scale[l];
  const float px = fmaf(x.x, s, 0.5f), py = fmaf(x.y, s, 0.5f);
  const float gx = floorf(px), gy = floorf(py);
  const float fx = px - gx, fy = py - gy;
  const int ix = int(gx), iy = int(gy);
  const long long base = i * 4;
  const int it = n * L.levels + l;
  key[base + 0] = corner_entry(L, l, ix, iy);
  key[base + 1] = corner_entry(L, l, ix + 1, iy);
  key[base + 2] = corner_entry(L, l, ix, iy + 1);
  key[base + 3] = corner_entry(L, l, ix + 1, iy + 1);
  weight[base + 0] = (1.f - fx) * (1.f - fy);
  weight[base + 1] = fx * (1.f - fy);
  weight[base + 2] = (1.f - fx) * fy;
  weight[base + 3] = fx * fy;
#pragma unroll
  for (int k = 0; k < 4; ++k) item[base + k] = it;
}

// segment starts from sorted keys: start[e] = first position with key >= e
__global__ void __launch_bounds__(256) k_seg_starts(const int* __restrict__ skey, long long K, int E,
                                                    int* __restrict__ start) {
  const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
  if (i > K) return;
  const int prev = i == 0 ? -1 : skey[i - 1];
  const int cur = i == K ? E : skey[i];
  for (int e = prev + 1; e <= cur; ++e) start[e] = int(i);
}

// feature gradient of a contribution: PLANAR = false -> item = n*L + l into
// [N][L] float2; PLANAR = true -> item = 2*l*N + n into feature-major [2L][N]
// floats (real part at item, imaginary part N further), which makes the
// gathers of one entry's spatially adjacent coordinates coalesced
template <bool PLANAR>
PTY_DEVI float2 dfeat_at(const float* __restrict__ dfeat, int item, int N) {
  if constexpr (PLANAR) return make_float2(__ldg(dfeat + item), __ldg(dfeat + item + N));
  else return __ldg(reinterpret_cast<const float2*>(dfeat) + item);
}

// long segments (coarse levels): a group of G lanes per entry (G = 32: one warp;
// G = 8: four entries per warp, for hashed levels' segments of 16 to 31), lanes stride the
// segment in order, fixed xor tree within the group.  Entries [e0, e1).
template <bool PLANAR, int G>
__global__ void __launch_bounds__(256) k_hash_bwd_warp(const int* __restrict__ start, const int* __restrict__ item,
                                                       const float* __restrict__ weight,
                                                       const float* __restrict__ dfeat, int N, int e0, int e1,
                                                       float2* __restrict__ dtable, int accumulate) {
  static_assert(G == 8 || G == 16 || G == 32, "lane group");
  const int lane = threadIdx.x & 31, gl = lane % G;
  const int e = e0 + (blockIdx.x * 8 + (threadIdx.x >> 5)) * (32 / G) + lane / G;
  const bool in = e < e1;  // every lane stays for the shuffles
  const int s0 = in ? start[e] : 0, s1 = in ? start[e + 1] : 0;
  float ax = 0.f, ay = 0.f;
  int j = s0 + gl;
  // four strides' loads in flight, then the adds in the same order as one at a time
  for (; j + 3 * G < s1; j += 4 * G) {
    float w[4];
    float2 g[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      w[k] = __ldg(weight + j + G * k);
      g[k] = dfeat_at<PLANAR>(dfeat, __ldg(item + j + G * k), N);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      ax = fmaf(w[k], g[k].x, ax);
      ay = fmaf(w[k], g[k].y, ay);
    }
  }
  for (; j < s1; j += G) {
    const float w = __ldg(weight + j);
    const float2 g = dfeat_at<PLANAR>(dfeat, __ldg(item + j), N);
    ax = fmaf(w, g.x, ax);
    ay = fmaf(w, g.y, ay);
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
  }
  if (in && gl == 0) {
    float2 r = make_float2(ax, ay);
    if (accumulate) {
      const float2 old = dtable[e];
      r = make_float2(old.x + r.x, old.y + r.y);
    }
    dtable[e] = r;
  }
}

// short segments (fine levels): one thread per entry, sequential in order
template <bool PLANAR>
__global__ void __launch_bounds__(256) k_hash_bwd_thread(const int* __restrict__ start, const int* __restrict__ item,
                                                         const float* __restrict__ weight,
                                                         const float* __restrict__ dfeat, int N, int e0, int E,
                                                         float2* __restrict__ dtable, int accumulate) {
  const int e = e0 + blockIdx.x * 256 + threadIdx.x;
  if (e >= E) return;
  const int s0 = start[e], s1 = start[e + 1];
  float ax = 0.f, ay = 0.f;
  int j = s0;
  for (; j + 3 < s1; j += 4) {  // four items' loads in flight, adds in order
    float w[4];
    float2 g[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      w[k] = __ldg(weight + j + k);
      g[k] = dfeat_at<PLANAR>(dfeat, __ldg(item + j + k), N);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      ax = fmaf(w[k], g[k].x, ax);
      ay = fmaf(w[k], g[k].y, ay);
    }
  }
  for (; j < s1; ++j) {
    const float w = __ldg(weight + j);
    const float2 g = dfeat_at<PLANAR>(dfeat, __ldg(item + j), N);
    ax = fmaf(w, g.x, ax);
    ay = fmaf(w, g.y, ay);
  }
  float2 r = make_float2(ax, ay);
  if (accumulate) {
    const float2 old = dtable[e];
    r = make_float2(old.x + r.x, old.y + r.y);
  }
  dtable[e] = r;
}

// ---------------------------------------------------------------------------
// Grid backward.  When the coordinates are a tensor-product grid (coordinate
// n = i * Bj + j at (ax0[j], ax1[i]), both axes non-decreasing -- an INR's
// pixel centres), the contributors of one level's vertex (cx, cy) are the
// rectangle of coordinates with ix0[j] in {cx - 1, cx} and iy1[i] in
// {cy - 1, cy}: j in [lo0[cx - 1], lo0[cx + 1]), i in [lo1[cy - 1],
// lo1[cy + 1]).  Phase 1 sums each vertex's rectangle with the forward's
// bilinear weights (wx * wy, wx = 1 - fx on the cell's own corner, fx on the
// next) into G[vertex]; phase 2 sums, per table entry, the G of the vertices
// mapping to it (a hashed level's collisions, a dense level's far-edge
// aliases) in the order of the vertex list sorted by entry.  Both phases have
// fixed orders: deterministic, no atomics, and the only per-step state is
// the per-axis tables and one list entry per vertex (the host builds them,
// hashgrid.py GridPlan).
// ---------------------------------------------------------------------------
struct GridArgs {
  const int* ix0;
  const int* iy1;
  const int* lo0;
  const int* lo1;
  const int* vstart;
  const int* vorder;
  const float* fx0;
  const float* fy1;
  const float* dfeat;
  int planar;
  int N, A, Bj, L;
  int E0[kMaxLevels], E1[kMaxLevels];
  int cw0[kMaxLevels], cw1[kMaxLevels];  // most axis values in one cell
  int lo0off[kMaxLevels], lo1off[kMaxLevels];
  long long voff[kMaxLevels + 1];
  float2* G;
  // the separable levels (k = 0 .. nsep-1): level, lanes of the row and column
  // passes, offset of the level's rows in H, first block of each pass
  int nsep;
  int sep_l[kMaxLevels], sep_gr[kMaxLevels], sep_gc[kMaxLevels];
  long long sep_h[kMaxLevels], sep_rb[kMaxLevels + 1], sep_cb[kMaxLevels + 1];
  // the tiled fine levels: level, tiles per row, first block
  int ntile;
  int tile_l[kMaxLevels], tile_gx[kMaxLevels];
  long long tile_b[kMaxLevels + 1];
  float4* H;  // (S0, S1) row sums of the separable levels
};

PTY_DEVI float2 grid_dfeat(const GridArgs& g, int l, int n) {
  if (g.planar) {
    const float* p = g.dfeat + size_t(2 * l) * g.N + n;
    return make_float2(__ldg(p), __ldg(p + g.N));
  }
  return __ldg(reinterpret_cast<const float2*>(g.dfeat) + size_t(n) * g.L + l);
}

// level, cx, cy and the contributor ranges of global vertex v
struct VertexRange {
  int l, cx, cy, i0, i1, j0, j1;
};
PTY_DEVI VertexRange vertex_range(const GridArgs& g, long long v) {
  VertexRange r;
  int l = 0;
  while (l + 1 < g.L && v >= g.voff[l + 1]) ++l;
  const int local = int(v - g.voff[l]);
  const int E0 = g.E0[l];
  r.l = l;
  r.cy = local / E0;
  r.cx = local - r.cy * E0;
  const int* lo0 = g.lo0 + g.lo0off[l];
  const int* lo1 = g.lo1 + g.lo1off[l];
  r.j0 = lo0[max(r.cx - 1, 0)];
  r.j1 = lo0[r.cx + 1];
  r.i0 = lo1[max(r.cy - 1, 0)];
  r.i1 = lo1[r.cy + 1];
  return r;
}

PTY_DEVI float axis_weight(const int* ix, const float* fx, int k, int c) {
  const float f = __ldg(fx + k);
  return __ldg(ix + k) == c ? 1.f - f : f;
}

// Sum over the flattened rectangle of vertex r: terms k = tid, tid + step, ...
// (i = i0 + k / nj, j = j0 + k % nj), four terms' loads in flight, added in k
// order per thread.  The row / column of the next term follow by a constant
// increment (one division per thread).
PTY_DEVI void rect_sum(const GridArgs& g, const VertexRange& r, int tid, int step, float& ax, float& ay) {
  const int nj = r.j1 - r.j0, ni = r.i1 - r.i0;
  const int total = ni * nj;
  if (tid >= total) return;
  const int* ix0 = g.ix0 + size_t(r.l) * g.Bj;
  const float* fx0 = g.fx0 + size_t(r.l) * g.Bj;
  const int* iy1 = g.iy1 + size_t(r.l) * g.A;
  const float* fy1 = g.fy1 + size_t(r.l) * g.A;
  const int dq = step / nj, dr = step - dq * nj;
  int i = tid / nj, j = tid - (tid / nj) * nj;
  int k = tid;
  auto advance = [&]() {
    k += step;
    j += dr;
    i += dq;
    if (j >= nj) {
      j -= nj;
      ++i;
    }
  };
  for (; k + 3 * step < total;) {
    float w[4];
    float2 d[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int ii = r.i0 + i, jj = r.j0 + j;
      w[u] = axis_weight(ix0, fx0, jj, r.cx) * axis_weight(iy1, fy1, ii, r.cy);
      d[u] = grid_dfeat(g, r.l, ii * g.Bj + jj);
      advance();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      ax = fmaf(w[u], d[u].x, ax);
      ay = fmaf(w[u], d[u].y, ay);
    }
  }
  for (; k < total; advance()) {
    const int ii = r.i0 + i, jj = r.j0 + j;
    const float wt = axis_weight(ix0, fx0, jj, r.cx) * axis_weight(iy1, fy1, ii, r.cy);
    const float2 d = grid_dfeat(g, r.l, ii * g.Bj + jj);
    ax = fmaf(wt, d.x, ax);
    ay = fmaf(wt, d.y, ay);
  }
}

// G lanes per vertex (G = 1 .. 32, a power of two; 32 / G vertices per warp):
// the group strides the flattened rectangle, then a fixed xor tree within it
template <int G>
__global__ void __launch_bounds__(256) k_gvert_group(const GridArgs g, long long v0, long long v1) {
  const int t = threadIdx.x, gl = t % G;
  const long long v = v0 + ((long long)blockIdx.x * 256 + t) / G;
  const bool in = v < v1;
  float ax = 0.f, ay = 0.f;
  if (in) {
    const VertexRange r = vertex_range(g, v);
    rect_sum(g, r, gl, G, ax, ay);
  }
  if constexpr (G > 1) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      ax += __shfl_xor_sync(0xffffffffu, ax, o);
      ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
  }
  if (in && gl == 0) g.G[v] = make_float2(ax, ay);
}

// Coarse levels (cw0 * cw1 >= 16) separably, since a term's weight is
// wx(j, cx) * wy(i, cy).  Row pass: per row i and cell c (the j with
// ix0[j] = c), S0 = sum (1 - fx) g and S1 = sum fx g, so every gradient value
// is read once.  Column pass: G[cy][cx] = sum over i in [lo1[cy - 1],
// lo1[cy + 1]) of wy (S1[i][cx - 1] + S0[i][cx]).  One launch per pass covers
// every separable level (blocks by level); G lanes (uniform in a block) share
// one output, striding its range, then a fixed xor tree.

PTY_DEVI void lane_reduce(float& ax, float& ay, int G) {
  for (int o = G >> 1; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
  }
}

// the separable level of block b of a pass whose levels start at `first`
PTY_DEVI int sep_slot(const GridArgs& g, const long long* first, long long b) {
  int k = 0;
  while (k + 1 < g.nsep && b >= first[k + 1]) ++k;
  return k;
}

__global__ void __launch_bounds__(256) k_gsep_rows(const GridArgs g) {
  const long long b = blockIdx.x;
  const int k = sep_slot(g, g.sep_rb, b);
  const int l = g.sep_l[k], G = g.sep_gr[k];
  const int t = threadIdx.x, gl = t & (G - 1);
  // 32-bit index math (A * E0 < 2^31; G is a power of two)
  const unsigned item = unsigned(int(b - g.sep_rb[k]) * 256 + t) >> (__ffs(G) - 1);
  const unsigned E0 = unsigned(g.E0[l]);
  const bool in = item < unsigned(g.A) * E0;
  float s0x = 0.f, s0y = 0.f, s1x = 0.f, s1y = 0.f;
  if (in) {
    const int i = int(item / E0);
    const int c = int(item - unsigned(i) * E0);
    const int* lo0 = g.lo0 + g.lo0off[l];
    const int j0 = lo0[c], j1 = lo0[c + 1];
    const float* fx0 = g.fx0 + size_t(l) * g.Bj;
    const int rowbase = i * g.Bj;
    int j = j0 + gl;
    for (; j + 3 * G < j1; j += 4 * G) {
      float f[4];
      float2 d[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        f[u] = __ldg(fx0 + j + u * G);
        d[u] = grid_dfeat(g, l, rowbase + j + u * G);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float w0 = 1.f - f[u];
        s0x = fmaf(w0, d[u].x, s0x);
        s0y = fmaf(w0, d[u].y, s0y);
        s1x = fmaf(f[u], d[u].x, s1x);
        s1y = fmaf(f[u], d[u].y, s1y);
      }
    }
    for (; j < j1; j += G) {
      const float f = __ldg(fx0 + j);
      const float2 d = grid_dfeat(g, l, rowbase + j);
      s0x = fmaf(1.f - f, d.x, s0x);
      s0y = fmaf(1.f - f, d.y, s0y);
      s1x = fmaf(f, d.x, s1x);
      s1y = fmaf(f, d.y, s1y);
    }
  }
  lane_reduce(s0x, s0y, G);
  lane_reduce(s1x, s1y, G);
  if (in && gl == 0) g.H[g.sep_h[k] + item] = make_float4(s0x, s0y, s1x, s1y);
}

__global__ void __launch_bounds__(256) k_gsep_cols(const GridArgs g) {
  const long long b = blockIdx.x;
  const int k = sep_slot(g, g.sep_cb, b);
  const int l = g.sep_l[k], G = g.sep_gc[k];
  const int t = threadIdx.x, gl = t & (G - 1);
  const unsigned item = unsigned(int(b - g.sep_cb[k]) * 256 + t) >> (__ffs(G) - 1);
  const int E0 = g.E0[l], E1 = g.E1[l];
  const bool in = item < unsigned(E0) * unsigned(E1);
  const float4* H = g.H + g.sep_h[k];
  float ax = 0.f, ay = 0.f;
  if (in) {
    const int cy = int(item / unsigned(E0)), cx = int(item - unsigned(cy) * unsigned(E0));
    auto Hat = [&](int i) {  // H[i][cx] = S1[i][cx - 1] + S0[i][cx]
      const float4 a0 = H[size_t(i) * E0 + cx];
      float2 h = make_float2(a0.x, a0.y);
      if (cx > 0) {
        const float4 a1 = H[size_t(i) * E0 + cx - 1];
        h = make_float2(a1.z + h.x, a1.w + h.y);
      }
      return h;
    };
    const int* lo1 = g.lo1 + g.lo1off[l];
    const int i0 = lo1[max(cy - 1, 0)], i1 = lo1[cy + 1];
    const int* iy1 = g.iy1 + size_t(l) * g.A;
    const float* fy1 = g.fy1 + size_t(l) * g.A;
    int i = i0 + gl;
    for (; i + 3 * G < i1; i += 4 * G) {
      float w[4];
      float2 h[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        w[u] = axis_weight(iy1, fy1, i + u * G, cy);
        h[u] = Hat(i + u * G);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        ax = fmaf(w[u], h[u].x, ax);
        ay = fmaf(w[u], h[u].y, ay);
      }
    }
    for (; i < i1; i += G) {
      const float w = axis_weight(iy1, fy1, i, cy);
      const float2 h = Hat(i);
      ax = fmaf(w, h.x, ax);
      ay = fmaf(w, h.y, ay);
    }
  }
  lane_reduce(ax, ay, G);
  if (in && gl == 0) g.G[g.voff[l] + item] = make_float2(ax, ay);
}

// lanes for a sum of about n terms: the power of two nearest n / 4 in 1 .. 32
static int lanes_for_terms(double n) {
  int G = 1;
  while (G < 32 && 8.0 * G <= n) G *= 2;
  return G;
}

// a level takes the separable passes when its cells hold at least 16 terms
static bool separable_level(const int32_t* extents, int l) { return extents[4 * l + 2] * extents[4 * l + 3] >= 16; }

// Fine levels (a few contributors per vertex): one CTA per kTX x kTY vertices of
// a level, all tiled levels in one launch (blocks by level).  The gradient sub-rectangle those vertices touch (rows i in
// [lo1[cy0 - 1], lo1[cy0 + kTY + 1]), columns likewise) and its axis tables are
// staged in shared memory with coalesced loads; each thread then sums its
// vertex's rectangle from shared memory in row-major order.
constexpr int kTX = 32, kTY = 8;
constexpr size_t kTileSmemCap = 96 * 1024;

__global__ void __launch_bounds__(256) k_gvert_tile(const GridArgs g) {
  extern __shared__ __align__(16) unsigned char tsm[];
  const long long b = blockIdx.x;
  int k = 0;
  while (k + 1 < g.ntile && b >= g.tile_b[k + 1]) ++k;
  const int l = g.tile_l[k];
  const int bl = int(b - g.tile_b[k]);
  const int E0 = g.E0[l], E1 = g.E1[l];
  const int cx0 = (bl % g.tile_gx[k]) * kTX, cy0 = (bl / g.tile_gx[k]) * kTY;
  const int* lo0 = g.lo0 + g.lo0off[l];
  const int* lo1 = g.lo1 + g.lo1off[l];
  const int j_lo = lo0[max(cx0 - 1, 0)], j_hi = lo0[min(cx0 + kTX + 1, E0)];
  const int i_lo = lo1[max(cy0 - 1, 0)], i_hi = lo1[min(cy0 + kTY + 1, E1)];
  const int nc = j_hi - j_lo, nr = i_hi - i_lo;
  float* sre = reinterpret_cast<float*>(tsm);
  float* sim = sre + nr * nc;
  int* six = reinterpret_cast<int*>(sim + nr * nc);
  float* sfx = reinterpret_cast<float*>(six + nc);
  int* siy = reinterpret_cast<int*>(sfx + nc);
  float* sfy = reinterpret_cast<float*>(siy + nr);
  const int t = threadIdx.x;
  for (int q = t; q < nc; q += 256) {
    six[q] = __ldg(g.ix0 + size_t(l) * g.Bj + j_lo + q);
    sfx[q] = __ldg(g.fx0 + size_t(l) * g.Bj + j_lo + q);
  }
  for (int q = t; q < nr; q += 256) {
    siy[q] = __ldg(g.iy1 + size_t(l) * g.A + i_lo + q);
    sfy[q] = __ldg(g.fy1 + size_t(l) * g.A + i_lo + q);
  }
  for (int r = t >> 5; r < nr; r += 8) {  // a warp per row, lanes along it
    for (int c = t & 31; c < nc; c += 32) {
      const float2 d = grid_dfeat(g, l, (i_lo + r) * g.Bj + j_lo + c);
      sre[r * nc + c] = d.x;
      sim[r * nc + c] = d.y;
    }
  }
  __syncthreads();
  const int cx = cx0 + (t % kTX), cy = cy0 + (t / kTX);
  if (cx >= E0 || cy >= E1) return;
  // (splitting each row's sum at lo0[cx] into two loops without the cell test
  // measured slower on c4: 219 against 181 us)
  const int j0 = lo0[max(cx - 1, 0)] - j_lo, j1 = lo0[cx + 1] - j_lo;
  const int i0 = lo1[max(cy - 1, 0)] - i_lo, i1 = lo1[cy + 1] - i_lo;
  float ax = 0.f, ay = 0.f;
  for (int i = i0; i < i1; ++i) {
    const float fy = sfy[i];
    const float wy = siy[i] == cy ? 1.f - fy : fy;
    for (int j = j0; j < j1; ++j) {
      const float fx = sfx[j];
      const float w = (six[j] == cx ? 1.f - fx : fx) * wy;
      ax = fmaf(w, sre[i * nc + j], ax);
      ay = fmaf(w, sim[i * nc + j], ay);
    }
  }
  g.G[g.voff[l] + (long long)cy * E0 + cx] = make_float2(ax, ay);
}

// shared memory of a tile of level l (rows and columns bounded by the cell widths)
static size_t tile_smem(const GridArgs& g, int l) {
  const size_t nc = size_t(kTX + 2) * g.cw0[l], nr = size_t(kTY + 2) * g.cw1[l];
  return (2 * nr * nc + 2 * nc + 2 * nr) * 4;
}

// WPB warps (1 or 8) per vertex: the WPB * 32 threads stride the flattened
// rectangle; fixed xor tree per warp, then the warps' partials in warp order
template <int WPB>
__global__ void __launch_bounds__(256) k_gvert_warp(const GridArgs g, long long v0, long long v1) {
  __shared__ float2 part[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int slot = w / WPB, ww = w % WPB;  // 8 / WPB vertices per block
  const long long v = v0 + (long long)blockIdx.x * (8 / WPB) + slot;
  const bool in = v < v1;
  float ax = 0.f, ay = 0.f;
  if (in) {
    const VertexRange r = vertex_range(g, v);
    rect_sum(g, r, ww * 32 + lane, WPB * 32, ax, ay);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
  }
  if (WPB == 1) {
    if (in && lane == 0) g.G[v] = make_float2(ax, ay);
    return;
  }
  if (lane == 0) part[w] = make_float2(ax, ay);
  __syncthreads();
  if (in && ww == 0 && lane == 0) {
    float2 t = part[w];
    for (int k = 1; k < WPB; ++k) t = c_add(t, part[w + k]);
    g.G[v] = t;
  }
}

// per table entry: the G of its vertices, in vertex-list order
__global__ void __launch_bounds__(256) k_gentry(const int* __restrict__ vstart, const int* __restrict__ vorder,
                                                const float2* __restrict__ G, int E, float2* __restrict__ dtable,
                                                int accumulate) {
  const int e = blockIdx.x * 256 + threadIdx.x;
  if (e >= E) return;
  const int s0 = __ldg(vstart + e), s1 = __ldg(vstart + e + 1);
  float2 r = make_float2(0.f, 0.f);
  for (int k = s0; k < s1; ++k) r = c_add(r, G[__ldg(vorder + k)]);
  if (accumulate) r = c_add(dtable[e], r);
  dtable[e] = r;
}

}  // namespace pty

using namespace pty;

extern "C" {

int ptycho_hashgrid_entries(int n_levels, int log2_hashmap_size, int base_resolution, float per_level_scale) {
  LevelTable L;
  if (make_levels(n_levels, log2_hashmap_size, base_resolution, per_level_scale, &L)) return -1;
  return L.total;
}

int ptycho_hashgrid_forward(const float* coords, int N, const float* table, int n_levels,
                            int log2_hashmap_size, int base_resolution, float per_level_scale,
                            float* features, ptycho_stream_t stream) {
  LevelTable L;
  int st = make_levels(n_levels, log2_hashmap_size, base_resolution, per_level_scale, &L);
  if (st) return st;
  if (N < 0 || (N > 0 && (!coords || !table || !features))) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(coords, 8) || !pty_aligned(table, 8) || !pty_aligned(features, 8))
    return PTYCHO_ERR_MISALIGNED;
  if (N == 0) return PTYCHO_OK;
  k_hash_fwd<<<(unsigned)((N + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float2*>(coords), N, reinterpret_cast<const float2*>(table), L,
      reinterpret_cast<float2*>(features));
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_hashgrid_forward_planar(const float* coords, int N, const float* table, int n_levels,
                                   int log2_hashmap_size, int base_resolution, float per_level_scale,
                                   float* features_planar, ptycho_stream_t stream) {
  LevelTable L;
  int st = make_levels(n_levels, log2_hashmap_size, base_resolution, per_level_scale, &L);
  if (st) return st;
  if (N < 0 || (N > 0 && (!coords || !table || !features_planar))) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(coords, 8) || !pty_aligned(table, 8) || !pty_aligned(features_planar, 4))
    return PTYCHO_ERR_MISALIGNED;
  if (N == 0) return PTYCHO_OK;
#ifndef PTY_HASH_FWD_PER_LEVEL
  k_hash_fwd_planar_all<<<(unsigned)((N + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float2*>(coords), N, reinterpret_cast<const float2*>(table), L, features_planar);
#else
  const dim3 grid((unsigned)((N + 255) / 256), (unsigned)L.levels);
  k_hash_fwd_planar<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float2*>(coords), N, reinterpret_cast<const float2*>(table), L, features_planar);
#endif
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_hashgrid_contrib(const float* coords, int N, int n_levels, int log2_hashmap_size,
                            int base_resolution, float per_level_scale, int32_t* key, int32_t* item,
                            float* weight, ptycho_stream_t stream) {
  LevelTable L;
  int st = make_levels(n_levels, log2_hashmap_size, base_resolution, per_level_scale, &L);
  if (st) return st;
  if (N < 0 || (N > 0 && (!coords || !key || !item || !weight))) return PTYCHO_ERR_INVALID_ARG;
  if ((long long)N * n_levels * 4 >= (1ll << 31)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (N == 0) return PTYCHO_OK;
  const long long work = (long long)N * n_levels;
  k_hash_contrib<<<(unsigned)((work + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float2*>(coords), N, L, key, item, weight);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_hashgrid_segments(const int32_t* sorted_key, long long K, int n_entries, int32_t* start,
                             ptycho_stream_t stream) {
  if (K < 0 || n_entries < 1 || !start || (K > 0 && !sorted_key)) return PTYCHO_ERR_INVALID_ARG;
  k_seg_starts<<<(unsigned)((K + 1 + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      sorted_key, K, n_entries, start);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

static int hash_backward(bool planar, const int32_t* start, const int32_t* item, const float* weight,
                         const float* dfeatures, int N, int n_levels, int log2_hashmap_size, int base_resolution,
                         float per_level_scale, float* dtable, int accumulate, ptycho_stream_t stream) {
  LevelTable L;
  int st = make_levels(n_levels, log2_hashmap_size, base_resolution, per_level_scale, &L);
  if (st) return st;
  if (N < 0 || !start || !item || !weight || !dfeatures || !dtable) return PTYCHO_ERR_INVALID_ARG;
  if (!pty_aligned(dfeatures, planar ? 4 : 8) || !pty_aligned(dtable, 8)) return PTYCHO_ERR_MISALIGNED;
  // by average segment length 4N / n_l (levels run coarse to fine, so each rule
  // holds for a prefix): >= 32, or >= 16 on a dense level, a warp per entry;
  // >= 16 on a hashed level eight lanes per entry; shorter a thread per entry
  // (measured: eight lanes gained on 2^20-entry hashed levels with segments of
  // 16 and lost on dense levels with segments of 16 to 31)
  int split32 = 0, split = 0;
  for (int l = 0; l < L.levels; ++l) {
    const long long seg4 = (long long)N * 4;
    if (seg4 >= 32ll * L.n[l] || (L.dense[l] && seg4 >= 16ll * L.n[l])) split32 = L.offset[l] + L.n[l];
    if ((long long)N * 4 >= 16ll * L.n[l]) split = L.offset[l] + L.n[l];
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  float2* dt = reinterpret_cast<float2*>(dtable);
  if (split32 > 0) {
    const unsigned g = unsigned((split32 + 7) / 8);
    if (planar)
      k_hash_bwd_warp<true, 32><<<g, 256, 0, s>>>(start, item, weight, dfeatures, N, 0, split32, dt, accumulate);
    else
      k_hash_bwd_warp<false, 32><<<g, 256, 0, s>>>(start, item, weight, dfeatures, N, 0, split32, dt, accumulate);
  }
  if (split > split32) {
    const unsigned g = unsigned((split - split32 + 31) / 32);  // 8 warps x 4 entries per block
    if (planar)
      k_hash_bwd_warp<true, 8><<<g, 256, 0, s>>>(start, item, weight, dfeatures, N, split32, split, dt, accumulate);
    else
      k_hash_bwd_warp<false, 8><<<g, 256, 0, s>>>(start, item, weight, dfeatures, N, split32, split, dt, accumulate);
  }
  if (L.total > split) {
    const unsigned g = (L.total - split + 255) / 256;
    if (planar)
      k_hash_bwd_thread<true><<<g, 256, 0, s>>>(start, item, weight, dfeatures, N, split, L.total, dt, accumulate);
    else
      k_hash_bwd_thread<false><<<g, 256, 0, s>>>(start, item, weight, dfeatures, N, split, L.total, dt, accumulate);
  }
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

int ptycho_hashgrid_backward(const int32_t* start, const int32_t* item, const float* weight,
                             const float* dfeatures, int N, int n_levels, int log2_hashmap_size,
                             int base_resolution, float per_level_scale, float* dtable, int accumulate,
                             ptycho_stream_t stream) {
  return hash_backward(false, start, item, weight, dfeatures, N, n_levels, log2_hashmap_size, base_resolution,
                       per_level_scale, dtable, accumulate, stream);
}

int ptycho_hashgrid_backward_planar(const int32_t* start, const int32_t* item_planar, const float* weight,
                                    const float* dfeatures_planar, int N, int n_levels, int log2_hashmap_size,
                                    int base_resolution, float per_level_scale, float* dtable, int accumulate,
                                    ptycho_stream_t stream) {
  if ((long long)2 * n_levels * N > 0x7fffffffll) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  return hash_backward(true, start, item_planar, weight, dfeatures_planar, N, n_levels, log2_hashmap_size,
                       base_resolution, per_level_scale, dtable, accumulate, stream);
}

size_t ptycho_hashgrid_grid_scratch_size(const int32_t* extents, int n_levels, int A, int Bj) {
  if (!extents || n_levels < 1 || n_levels > kMaxLevels || A < 1 || Bj < 1) return 0;
  size_t n = 0, h = 0;
  for (int l = 0; l < n_levels; ++l) {
    if (extents[4 * l] < 1 || extents[4 * l + 1] < 1 || extents[4 * l + 2] < 1 || extents[4 * l + 3] < 1) return 0;
    n += size_t(extents[4 * l]) * size_t(extents[4 * l + 1]);
    if (separable_level(extents, l)) h += size_t(A) * size_t(extents[4 * l]);
  }
  // vertex sums (float2), then every separable level's (S0, S1) rows (float4)
  return n * sizeof(float2) + 16 + h * sizeof(float4);
}

int ptycho_hashgrid_backward_grid(const int32_t* grid_int, const float* grid_frac, const int32_t* extents, int A,
                                  int Bj, const float* dfeatures, int planar, int n_levels, int log2_hashmap_size,
                                  int base_resolution, float per_level_scale, float* dtable, int accumulate,
                                  void* scratch, size_t scratch_bytes, ptycho_stream_t stream) {
  LevelTable L;
  int st = make_levels(n_levels, log2_hashmap_size, base_resolution, per_level_scale, &L);
  if (st) return st;
  if (!grid_int || !grid_frac || !extents || !dfeatures || !dtable || A < 1 || Bj < 1) return PTYCHO_ERR_INVALID_ARG;
  const long long N = (long long)A * Bj;
  if (N * 4 >= (1ll << 31) || (planar && 2ll * n_levels * N >= (1ll << 31))) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  const size_t need = ptycho_hashgrid_grid_scratch_size(extents, n_levels, A, Bj);
  if (need == 0) return PTYCHO_ERR_INVALID_ARG;
  if (!scratch || scratch_bytes < need) return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(dfeatures, planar ? 4 : 8) || !pty_aligned(dtable, 8) || !pty_aligned(scratch, 8) ||
      !pty_aligned(grid_int, 4) || !pty_aligned(grid_frac, 4))
    return PTYCHO_ERR_MISALIGNED;
  GridArgs g{};
  g.dfeat = dfeatures;
  g.planar = planar ? 1 : 0;
  g.N = int(N);
  g.A = A;
  g.Bj = Bj;
  g.L = n_levels;
  // layout of grid_int: ix0 [L][Bj], iy1 [L][A], lo0 [sum (E0 + 1)], lo1 [sum (E1 + 1)],
  // vstart [entries + 1], vorder [vertices]; grid_frac: fx0 [L][Bj], fy1 [L][A]
  size_t off = 0;
  g.ix0 = grid_int + off;
  off += size_t(n_levels) * Bj;
  g.iy1 = grid_int + off;
  off += size_t(n_levels) * A;
  g.lo0 = grid_int + off;
  int o0 = 0, o1 = 0;
  long long nv = 0;
  for (int l = 0; l < n_levels; ++l) {
    g.E0[l] = extents[4 * l];
    g.E1[l] = extents[4 * l + 1];
    g.cw0[l] = extents[4 * l + 2];
    g.cw1[l] = extents[4 * l + 3];
    g.lo0off[l] = o0;
    g.lo1off[l] = o1;
    o0 += g.E0[l] + 1;
    o1 += g.E1[l] + 1;
    g.voff[l] = nv;
    nv += (long long)g.E0[l] * g.E1[l];
  }
  g.voff[n_levels] = nv;
  off += size_t(o0);
  g.lo1 = grid_int + off;
  off += size_t(o1);
  g.vstart = grid_int + off;
  off += size_t(L.total) + 1;
  g.vorder = grid_int + off;
  g.fx0 = grid_frac;
  g.fy1 = grid_frac + size_t(n_levels) * Bj;
  g.G = static_cast<float2*>(scratch);
  // lanes per vertex by the level's average contributors per vertex: 256 (a
  // block) from 2048 terms, else the power of two nearest terms / 4 in 1 .. 32
  // (about four terms per lane); levels run coarse to fine, so equal choices
  // form runs of levels, one launch each
  auto lanes_for = [&](int l) {
    const double terms = (2.0 * Bj / g.E0[l]) * (2.0 * A / g.E1[l]);
    if (terms >= 2048.0) return 256;
    int G = 1;
    while (G < 32 && 4.0 * G * 2 <= terms) G *= 2;
    return G;
  };
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  g.H = reinterpret_cast<float4*>(pty_align_up(reinterpret_cast<uintptr_t>(g.G + g.voff[n_levels]), 16));
  // plan the levels: separable ones (two launches for all of them), tiled fine
  // levels (one launch), the rest per vertex with G lanes (runs of equal G)
  long long hoff = 0, rb = 0, cb = 0, tb = 0;
  size_t tsmem = 0;
  int rest[kMaxLevels], nrest = 0;
  for (int l = 0; l < n_levels; ++l) {
    if (separable_level(extents, l)) {
      const int k = g.nsep++;
      g.sep_l[k] = l;
      g.sep_gr[k] = lanes_for_terms(double(g.cw0[l]));  // one cell per row item
      g.sep_gc[k] = lanes_for_terms(2.0 * A / g.E1[l]);
      g.sep_h[k] = hoff;
      hoff += (long long)A * g.E0[l];
      g.sep_rb[k] = rb;
      rb += ((long long)A * g.E0[l] * g.sep_gr[k] + 255) / 256;
      g.sep_cb[k] = cb;
      cb += ((long long)g.E0[l] * g.E1[l] * g.sep_gc[k] + 255) / 256;
    } else if (lanes_for(l) <= 8 && tile_smem(g, l) <= kTileSmemCap) {
      const int k = g.ntile++;
      g.tile_l[k] = l;
      g.tile_gx[k] = (g.E0[l] + kTX - 1) / kTX;
      g.tile_b[k] = tb;
      tb += (long long)g.tile_gx[k] * ((g.E1[l] + kTY - 1) / kTY);
      tsmem = tile_smem(g, l) > tsmem ? tile_smem(g, l) : tsmem;
    } else {
      rest[nrest++] = l;
    }
  }
  g.sep_rb[g.nsep] = rb;
  g.sep_cb[g.nsep] = cb;
  g.tile_b[g.ntile] = tb;
  if (g.nsep) {
    k_gsep_rows<<<unsigned(rb), 256, 0, s>>>(g);
    k_gsep_cols<<<unsigned(cb), 256, 0, s>>>(g);
  }
  if (g.ntile) {
    if (tsmem > 48 * 1024 &&
        cudaFuncSetAttribute(k_gvert_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTileSmemCap)) !=
            cudaSuccess)
      return PTYCHO_ERR_LAUNCH;
    k_gvert_tile<<<unsigned(tb), 256, tsmem, s>>>(g);
  }
  for (int r = 0; r < nrest;) {
    const int l0 = rest[r], G = lanes_for(l0);
    int r1 = r + 1;
    while (r1 < nrest && rest[r1] == rest[r1 - 1] + 1 && lanes_for(rest[r1]) == G) ++r1;
    const long long va = g.voff[l0], vb = g.voff[rest[r1 - 1] + 1], nvv = vb - va;
    switch (G) {
      case 256: k_gvert_warp<8><<<unsigned(nvv), 256, 0, s>>>(g, va, vb); break;
      case 32: k_gvert_group<32><<<unsigned((nvv * 32 + 255) / 256), 256, 0, s>>>(g, va, vb); break;
      case 16: k_gvert_group<16><<<unsigned((nvv * 16 + 255) / 256), 256, 0, s>>>(g, va, vb); break;
      case 8: k_gvert_group<8><<<unsigned((nvv * 8 + 255) / 256), 256, 0, s>>>(g, va, vb); break;
      case 4: k_gvert_group<4><<<unsigned((nvv * 4 + 255) / 256), 256, 0, s>>>(g, va, vb); break;
      case 2: k_gvert_group<2><<<unsigned((nvv * 2 + 255) / 256), 256, 0, s>>>(g, va, vb); break;
      default: k_gvert_group<1><<<unsigned((nvv + 255) / 256), 256, 0, s>>>(g, va, vb); break;
    }
    r = r1;
  }
  k_gentry<<<unsigned((L.total + 255) / 256), 256, 0, s>>>(g.vstart, g.vorder, g.G, L.total,
                                                           reinterpret_cast<float2*>(dtable), accumulate);
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // extern "C"
