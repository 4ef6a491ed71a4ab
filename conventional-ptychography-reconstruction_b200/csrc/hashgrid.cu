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
  const dim3 grid((unsigned)((N + 255) / 256), (unsigned)L.levels);
  k_hash_fwd_planar<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float2*>(coords), N, reinterpret_cast<const float2*>(table), L, features_planar);
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

}  // extern "C"
