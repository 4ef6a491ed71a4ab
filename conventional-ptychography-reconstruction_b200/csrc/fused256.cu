// fused256.cu -- fused forward / loss / adjoint for 256 x 256 probes on a
// cluster of 4 CTAs per pattern (the pattern, 512 KB of complex64, does not
// fit one SM).
//
// Same contract as k_fused (fused.cuh); per pattern:
//   pass 1 (each CTA: the 64 rows whose y bits 4,5 equal its rank): gather
//          (-1)^(x+y) P * O[window], radix-16 x stage + radix-2 y stage
//   local exchange, pass 2: radix-16 x + radix-2 y
//   cluster exchange through distributed shared memory (DSMEM): each value
//          is stored into the shared memory of the CTA owning its row band
//          y bits 6,7 (mapa + st.shared::cluster), between cluster barriers
//   pass 3: radix-16 y, local exchange, pass 4: radix-4 y -> spectrum
//   loss against the measurement rows of this CTA's frequency residue class
//   (64 bulk copies of 1 KB, mbarrier-tracked, prefetched one pattern ahead);
//   FP64 per-pattern loss summed over the cluster in rank order via DSMEM
//   (the FD loss reads its neighbouring frequency rows from the other CTAs)
//   adjoint: the four passes backwards, the DSMEM exchange reversed, then
//          E'_b = (-1)^(x+y) dL/dpsi_b written once (same layout as M <= 128).
// Shared-memory planes are 64 x 256 floats per CTA with no padding: the
// column swizzle x ^ ((x >> 4) << 1) and a local-row swizzle make every
// pass's lane map and the measurement reads bank-conflict free.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "async_copy.cuh"
#include "fft_plan.cuh"
#include "fused.cuh"

namespace cg = cooperative_groups;

namespace pty {
namespace f256 {

constexpr int M = 256, E = 32, NT = 512, CL = 4;
constexpr size_t S_RE = 0, S_IM = 65536, S_MEAS = 131072, S_TW = 196608, S_RED = S_TW + 256 * 8,
                 S_LOSS = S_RED + 16 * 8, S_BAR = S_LOSS + 4 * 8, S_ABORT = S_BAR + 8, SMEM = S_ABORT + 8;

// local row of a position in the two cluster layouts
__host__ __device__ constexpr int ly12(int y) { return (y & 15) | (((y >> 6) & 3) << 4); }  // passes 1-2
__host__ __device__ constexpr int ly34(int y) { return y & 63; }                             // passes 3-4
__host__ __device__ constexpr int gly(int ly) { return ((ly & 1) << 4) | ((ly >> 1) & 1); }

// local plane offset (floats) = base + element part; the XOR parts are linear
struct Addr {
  int row;  // ly_base * 256
  int xr;   // swz(bx) ^ gly(ly_base)
};
template <int PASS, int LAYOUT>
PTY_DEVI Addr addr_base(int bx, int by) {
  const int ly = LAYOUT == 12 ? ly12(by) : ly34(by);
  return Addr{ly * 256, swz<M>(bx) ^ gly(ly)};
}
template <int PASS, int LAYOUT, int e>
__host__ __device__ constexpr int addr_row(int /*unused*/ = 0) {
  return (LAYOUT == 12 ? ly12(eoff_y<M, PASS>(e)) : ly34(eoff_y<M, PASS>(e))) * 256;
}
template <int PASS, int LAYOUT, int e>
__host__ __device__ constexpr int addr_x() {
  return swz<M>(eoff_x<M, PASS>(e)) ^ gly(LAYOUT == 12 ? ly12(eoff_y<M, PASS>(e)) : ly34(eoff_y<M, PASS>(e)));
}

template <int PASS>
PTY_DEVI void pos_base(int t, int r, int& bx, int& by) {
  tbase<M, PASS>(t, bx, by);
  rbase<M, PASS>(r, bx, by);
}

template <bool ADJ, int PASS>
PTY_DEVI void pass(float2 (&v)[E], int t, int r, const float2* __restrict__ tw) {
  constexpr PassDesc d = desc<M, PASS>();
  int bx, by;
  pos_base<PASS>(t, r, bx, by);
  run_pass<M, E, ADJ, (1 << d.nbx), (1 << d.nby), d.lox, d.nbx, d.loy, d.nby>(v, bx, by, tw);
}

// exchange inside the CTA (both passes use the same local layout)
template <int PA, int PB, int LAYOUT>
PTY_DEVI void exch_local(float2 (&v)[E], int t, int r, float* re, float* im) {
  int ax, ay, bx, by;
  pos_base<PA>(t, r, ax, ay);
  pos_base<PB>(t, r, bx, by);
  const Addr A = addr_base<PA, LAYOUT>(ax, ay), B = addr_base<PB, LAYOUT>(bx, by);
  __syncthreads();
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const int off = A.row + addr_row<PA, LAYOUT, e>() + (A.xr ^ addr_x<PA, LAYOUT, e>());
    re[off] = v[e].x;
    im[off] = v[e].y;
  });
  __syncthreads();
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const int off = B.row + addr_row<PB, LAYOUT, e>() + (B.xr ^ addr_x<PB, LAYOUT, e>());
    v[e] = make_float2(re[off], im[off]);
  });
}

PTY_DEVI uint32_t mapa(uint32_t saddr, uint32_t rank) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(saddr), "r"(rank));
  return out;
}
PTY_DEVI void st_cluster(uint32_t addr, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}
PTY_DEVI void st_cluster_v2(uint32_t addr, float a, float b) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(a), "f"(b) : "memory");
}
PTY_DEVI void st_cluster_v4(uint32_t addr, float a, float b, float c, float d) {
  asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}
PTY_DEVI void st_cluster_u32(uint32_t addr, unsigned v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
PTY_DEVI void st_cluster_f64(uint32_t addr, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}

// pass 2 -> pass 3 (forward, DIR = 0) or pass 3 -> pass 2 (adjoint, DIR = 1)
// through distributed shared memory, between cluster barriers
template <int DIR>
PTY_DEVI void exch_cluster(float2 (&v)[E], int t, int r, float* re, float* im, cg::cluster_group& cl) {
  constexpr int PS = DIR == 0 ? 2 : 3, PD = DIR == 0 ? 3 : 2;
  constexpr int LD = DIR == 0 ? 34 : 12;  // destination layout
  int sx, sy;
  pos_base<PS>(t, r, sx, sy);
  // destination address computed in the destination layout from the source positions
  const Addr A = addr_base<PS, LD>(sx, sy);
  // destination rank = y bits 6,7 (forward) or 4,5 (adjoint) of the position,
  // = (thread part) ^ (element part); the bases are indexed by the element part
  constexpr int SH = DIR == 0 ? 6 : 4;
  const int qs = (sy >> SH) & 3;
  // a CTA's shared memory maps linearly into the cluster window, so the
  // imaginary plane of rank q sits (S_IM - S_RE) bytes above its real plane
  uint32_t rre[4];
#pragma unroll
  for (int qe = 0; qe < 4; ++qe) rre[qe] = mapa(smem_u32(re), uint32_t(qs ^ qe));
  constexpr uint32_t IMOFF = uint32_t(S_IM - S_RE);
  cl.sync();  // every CTA is done reading its planes
  if constexpr (DIR == 0) {
    // Pass 2 holds x bits 0-3 (element bits 0-3) and y6 (bit 4): the 16 values
    // of one y6 half land in one aligned 16-float group of the destination
    // row, at column (A.xr ^ j).  Reorder them by the lane's XOR mask with four
    // conditional-swap stages, then write the group with 16-byte stores.
    static_for<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      static_assert(addr_row<PS, LD, e>() == 0 && addr_x<PS, LD, e>() == (e & 15), "pass-2 element map");
      static_assert(((eoff_y<M, PS>(e) >> SH) & 3) == (e >> 4), "pass-2 rank map");
    });
    const int pm = A.xr & 15;
    static_for<4>([&](auto bc) {
      constexpr int bit = 1 << decltype(bc)::value;
      const bool sw = (pm & bit) != 0;
      static_for<E>([&](auto ec) {
        constexpr int j = decltype(ec)::value;
        if constexpr ((j & bit) == 0) {
          const float2 a = v[j], b = v[j | bit];
          v[j] = sw ? b : a;
          v[j | bit] = sw ? a : b;
        }
      });
    });
    const uint32_t grp = 4u * uint32_t(A.row + (A.xr & ~15));
    static_for<8>([&](auto gc) {
      constexpr int g = decltype(gc)::value;  // y6 half g / 4, floats 4 (g % 4) .. +3
      constexpr int e0 = 4 * g;
      const uint32_t a = rre[g >> 2] + grp + 16u * uint32_t(g & 3);
      st_cluster_v4(a, v[e0].x, v[e0 + 1].x, v[e0 + 2].x, v[e0 + 3].x);
      st_cluster_v4(a + IMOFF, v[e0].y, v[e0 + 1].y, v[e0 + 2].y, v[e0 + 3].y);
    });
  } else {
    // Pass 3 holds y bits 2-5 (element bits 0-3) and x0 (bit 4): the values
    // e and e + 16 are adjacent columns (A.xr ^ x0) of one destination row;
    // order each pair by the lane's column bit 0 and write it with 8-byte stores.
    static_for<16>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      static_assert(addr_x<PS, LD, e>() == 0 && addr_x<PS, LD, e + 16>() == 1, "pass-3 column map");
      static_assert(addr_row<PS, LD, e + 16>() == addr_row<PS, LD, e>(), "pass-3 row map");
      static_assert(((eoff_y<M, PS>(e + 16) >> SH) & 3) == ((eoff_y<M, PS>(e) >> SH) & 3), "pass-3 rank map");
      constexpr int qe = (eoff_y<M, PS>(e) >> SH) & 3;
      const bool sw = (A.xr & 1) != 0;
      const float2 lo = sw ? v[e + 16] : v[e], hi = sw ? v[e] : v[e + 16];
      const uint32_t a = rre[qe] + 4u * uint32_t(A.row + addr_row<PS, LD, e>() + (A.xr & ~1));
      st_cluster_v2(a, lo.x, hi.x);
      st_cluster_v2(a + IMOFF, lo.y, hi.y);
    });
  }
  cl.sync();  // all values have landed
  int dx, dy;
  pos_base<PD>(t, r, dx, dy);
  const Addr B = addr_base<PD, LD>(dx, dy);
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const int off = B.row + addr_row<PD, LD, e>() + (B.xr ^ addr_x<PD, LD, e>());
    v[e] = make_float2(re[off], im[off]);
  });
}

// frequency index of a pass-4 position: staging row (fy >> 2) and column fx
template <int... J>
PTY_DEVI void fbase4_seq(int t, int& fx, int& fy, std::integer_sequence<int, J...>) {
  fx = (0 | ... | (((t >> J) & 1) * freq_x<M>(tw_x<M, 4, J>())));
  fy = (0 | ... | (((t >> J) & 1) * freq_y<M>(tw_y<M, 4, J>())));
}

PTY_DEVI float ld_cluster(uint32_t addr) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
  return v;
}

// FD loss (5-point circular stencil of dW = sqrt(Imeas + eps) - sqrt(I + eps)
// over the natural frequency grid).  CTA c holds the frequency rows
// fy = c + 4 j as rows j of its planes, so the rows fy +- 1 are read from the
// CTAs c +- 1 through distributed shared memory, between cluster barriers.
// part[e] <- the pixel's loss term; v[e] <- 2 dL/dI v[e].
PTY_DEVI void fd_terms(float2 (&v)[E], float (&part)[E], int c, int fx0, int fy0, const float* sm, float* re,
                       float* im, cg::cluster_group& cl) {
  constexpr float inv_mn = 1.0f / float(M * M);
  const int j0 = fy0 >> 2;
  const int c_up = (c + 1) & 3, c_dn = (c + 3) & 3;  // holders of rows fy + 1 and fy - 1
  const uint32_t im_up = mapa(smem_u32(im), uint32_t(((c_up >> 1) & 1) | ((c_up & 1) << 1)));
  const uint32_t im_dn = mapa(smem_u32(im), uint32_t(((c_dn >> 1) & 1) | ((c_dn & 1) << 1)));
  const int dj_up = c == 3 ? 1 : 0, dj_dn = c == 0 ? -1 : 0;
  float q[E];
  __syncthreads();  // earlier readers of the planes are done
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    constexpr int fxe = freq_x<M>(eoff_x<M, 4>(e)), fye = freq_y<M>(eoff_y<M, 4>(e));
    const int o = (j0 + (fye >> 2)) * M + (fx0 | fxe);
    const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
    im[o] = sqrtf(sm[o] + kEps) - sqrtf(I + kEps);  // dW
  });
  cl.sync();  // dW of every row is visible cluster-wide
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    constexpr int fxe = freq_x<M>(eoff_x<M, 4>(e)), fye = freq_y<M>(eoff_y<M, 4>(e));
    const int j = j0 + (fye >> 2), fx = fx0 | fxe;
    const float dw = im[j * M + fx];
    const float rx = im[j * M + ((fx + 1) & (M - 1))] - dw;
    const float ry = ld_cluster(im_up + 4u * uint32_t(((j + dj_up) & 63) * M + fx)) - dw;
    const float G = sqrtf(fmaf(rx, rx, fmaf(ry, ry, kEps)));
    part[e] = G;
    re[j * M + fx] = rx / G;
    q[e] = ry / G;
  });
  cl.sync();  // all reads of dW are done; rx / G is visible
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    constexpr int fxe = freq_x<M>(eoff_x<M, 4>(e)), fye = freq_y<M>(eoff_y<M, 4>(e));
    const int j = j0 + (fye >> 2), fx = fx0 | fxe;
    im[j * M + fx] = q[e];  // ry / G
    q[e] = re[j * M + ((fx - 1) & (M - 1))] - re[j * M + fx];
  });
  cl.sync();  // ry / G is visible cluster-wide
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    constexpr int fxe = freq_x<M>(eoff_x<M, 4>(e)), fye = freq_y<M>(eoff_y<M, 4>(e));
    const int j = j0 + (fye >> 2), fx = fx0 | fxe;
    const float up = ld_cluster(im_dn + 4u * uint32_t(((j + dj_dn) & 63) * M + fx));
    const float dl = (q[e] + up - im[j * M + fx]) * inv_mn;
    const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
    const float g = dl * (-0.5f / sqrtf(I + kEps));
    v[e] = c_scale(v[e], 2.0f * g);
  });
  cl.sync();  // remote reads of this CTA's planes are done before they are reused
}

template <int MODE, int LOSS>
__global__ void __launch_bounds__(NT, 1) k_fused256(const FusedArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* re = reinterpret_cast<float*>(smem + S_RE);
  float* im = reinterpret_cast<float*>(smem + S_IM);
  float* sm = reinterpret_cast<float*>(smem + S_MEAS);
  float2* tw = reinterpret_cast<float2*>(smem + S_TW);
  double* red = reinterpret_cast<double*>(smem + S_RED);
  double* lossbuf = reinterpret_cast<double*>(smem + S_LOSS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S_BAR);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + S_ABORT);
  constexpr bool kMeas = MODE != MODE_INTENSITY;

  cg::cluster_group cl = cg::this_cluster();
  const int t = threadIdx.x;
  const int r = int(cl.block_rank());
  const int cid = blockIdx.x / CL, ncl = gridDim.x / CL;
  // this CTA's measurement rows are the frequencies fy = c + 4 j
  const int c = ((r >> 1) & 1) | ((r & 1) << 1);
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    *abort_flag = 0;
  }
  for (int j = t; j < M; j += NT) {
    double s, co;
    sincospi(-2.0 * double(j) / double(M), &s, &co);
    tw[j] = make_float2((float)co, (float)s);
  }
  if (a.done && blockIdx.x == 0)
    for (int i = t; i < a.ndone; i += NT) a.done[i] = 0u;
  cl.sync();  // all CTAs of the cluster are running; barriers and tables ready

  auto resolve = [&](int b, int& f, int2& w) -> bool {
    f = a.batch ? __ldg(a.batch + b) : b;
    if (f < 0 || f >= a.F) {
      w = make_int2(-1, -1);
      return false;
    }
    w = __ldg(a.tl + f);
    return w.x >= 0 && w.y >= 0 && w.x <= a.H - M && w.y <= a.W - M;
  };
  auto prefetch = [&](int nb) {  // this CTA's 64 object rows of pattern nb -> L2
    int f;
    int2 w;
    if (t < 64 && resolve(nb, f, w)) {
      const int y = (t & 15) | (r << 4) | ((t >> 4) << 6);
      const char* row = reinterpret_cast<const char*>(a.O + size_t(w.x + y) * a.W + w.y);
      prefetch_l2_range(row, row + M * sizeof(float2), reinterpret_cast<const char*>(a.O),
                        reinterpret_cast<const char*>(a.O + size_t(a.H) * a.W));
    }
  };
  auto fetch = [&](int nb) {  // this CTA's 64 measurement rows of pattern nb -> shared memory
    int f;
    int2 w;
    if (t == 0 && resolve(nb, f, w)) {
      mbar_arrive_expect_tx(bar, 64 * M * 4);
      const float* src = a.Imeas + size_t(f) * M * M;
      for (int j = 0; j < 64; ++j) bulk_g2s(sm + j * M, src + size_t(c + 4 * j) * M, M * 4, bar);
    }
  };

  if (cid < a.B) {
    prefetch(cid);
    if (kMeas) fetch(cid);
  }
  uint32_t phase = 0;
  for (int b = cid; b < a.B; b += ncl) {
    int f;
    int2 w;
    const bool ok = resolve(b, f, w);  // uniform over the cluster
    if constexpr (MODE == MODE_ADJ) {
      if (t == 0 && r == 0) a.tlb[b] = ok ? w : make_int2(-1, -1);
    }
    const int nb = b + ncl;
    if (!ok) {
      if (t == 0 && r == 0) pty_raise(a.status, PTYCHO_ERR_WINDOW);
      const float nan = __int_as_float(0x7fc00000);
      if constexpr (MODE == MODE_INTENSITY) {
        for (int i = t; i < M * M / CL; i += NT) a.I_out[size_t(b) * M * M + size_t(r) * (M * M / CL) + i] = nan;
      } else {
        if (t == 0 && r == 0 && a.loss_pat) a.loss_pat[b] = (double)nan;
      }
      if (nb < a.B) {
        prefetch(nb);
        if (kMeas) fetch(nb);
      }
      continue;
    }
    float2 v[E];
    {  // pass-1 gather
      int bx, by;
      pos_base<1>(t, r, bx, by);
      const float2* Ob = a.O + size_t(w.x + by) * a.W + (w.y + bx);
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
    if (nb < a.B) prefetch(nb);
    pass<false, 1>(v, t, r, tw);
    exch_local<1, 2, 12>(v, t, r, re, im);
    pass<false, 2>(v, t, r, tw);
    exch_cluster<0>(v, t, r, re, im, cl);
    pass<false, 3>(v, t, r, tw);
    exch_local<3, 4, 34>(v, t, r, re, im);
    pass<false, 4>(v, t, r, tw);

    int fx0, fy0;
    fbase4_seq(t, fx0, fy0, std::make_integer_sequence<int, desc<M, 4>().nt>{});
    if constexpr (MODE == MODE_INTENSITY) {
      float* Ib = a.I_out + size_t(b) * M * M;
      const int fyr = (fy0 | c);  // rank bits give fy mod 4
      static_for<E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        constexpr int fxe = freq_x<M>(eoff_x<M, 4>(e)), fye = freq_y<M>(eoff_y<M, 4>(e));
        Ib[(fyr | fye) * M + (fx0 | fxe)] = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      });
    } else {
      // A copy that never lands must stop the whole cluster at the same
      // barrier: the CTA that gave up flags every CTA, the pattern finishes
      // on whatever is in the buffer (no cluster barrier is skipped), and all
      // four leave after the next cluster barrier.
      const bool bad = __syncthreads_or(!mbar_wait_bounded(bar, phase)) != 0;
      phase ^= 1u;
      if (bad && t == 0) {
        pty_raise(a.status, PTYCHO_ERR_TIMEOUT);
        for (int q = 0; q < CL; ++q) st_cluster_u32(mapa(smem_u32((const void*)abort_flag), q), 1u);
      }
      // loss (FP32 terms, pairwise, then FP64); staging row = fy >> 2
      constexpr float inv_mn = 1.0f / float(M * M);
      float part[E];
      const float* Sb = sm + (fy0 >> 2) * M + fx0;
      if constexpr (LOSS == PTYCHO_LOSS_FD) {
        fd_terms(v, part, c, fx0, fy0, sm, re, im, cl);
      } else static_for<E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        constexpr int fxe = freq_x<M>(eoff_x<M, 4>(e)), fye = freq_y<M>(eoff_y<M, 4>(e));
        const float meas = Sb[(fye >> 2) * M + fxe];
        const float I = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
        float g;
        if constexpr (LOSS == PTYCHO_LOSS_INTENSITY_GRAD) {
          part[e] = I * meas * float(M * M);
          g = meas;
          v[e] = c_scale(v[e], 2.0f * g);
        } else {
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
        }
      });
#pragma unroll
      for (int s2 = 1; s2 < E; s2 <<= 1)
#pragma unroll
        for (int i = 0; i < E; i += 2 * s2) part[i] += part[i + s2];
      const double tot = block_sum<NT>((double)part[0], red);  // barriers: all reads of sm are done
      if (t == 0) {
        st_cluster_f64(mapa(smem_u32(lossbuf + r), 0), tot);
        if (nb < a.B && !bad) fetch(nb);
      }
      if constexpr (MODE == MODE_ADJ) {
        pass<true, 4>(v, t, r, tw);
        exch_local<4, 3, 34>(v, t, r, re, im);
        pass<true, 3>(v, t, r, tw);
        exch_cluster<1>(v, t, r, re, im, cl);  // its first barrier also publishes lossbuf
        if (t == 0 && r == 0 && a.loss_pat)
          a.loss_pat[b] = (((lossbuf[0] + lossbuf[1]) + lossbuf[2]) + lossbuf[3]) / double(M * M);
        pass<true, 2>(v, t, r, tw);
        exch_local<2, 1, 12>(v, t, r, re, im);
        pass<true, 1>(v, t, r, tw);
        int bx, by;
        pos_base<1>(t, r, bx, by);
        float2* Eb = a.Eout + size_t(b) * M * M + by * M + bx;
        static_for<E>([&](auto ec) {
          constexpr int e = decltype(ec)::value;
          constexpr int ox = eoff_x<M, 1>(e), oy = eoff_y<M, 1>(e);
          Eb[oy * M + ox] = v[e];
        });
      } else {
        // publishes lossbuf; the next writes to it come after the next
        // pattern's first cluster barrier, which rank 0 reaches after reading
        cl.sync();
        if (t == 0 && r == 0 && a.loss_pat)
          a.loss_pat[b] = (((lossbuf[0] + lossbuf[1]) + lossbuf[2]) + lossbuf[3]) / double(M * M);
      }
      if (*abort_flag) break;  // uniform: set before a cluster barrier every CTA has passed
    }
  }
  cl.sync();  // no CTA leaves while others may still address its shared memory
}

template <int MODE, int LOSS>
static int launch_t(const FusedArgs& a, cudaStream_t s) {
  auto kern = k_fused256<MODE, LOSS>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM)) != cudaSuccess)
    return PTYCHO_ERR_LAUNCH;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = SMEM;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(CL);
  int nclusters = 0;
  if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1) nclusters = 1;
  const int ncl = a.B < nclusters ? a.B : nclusters;
  cfg.gridDim = dim3(CL * ncl);
  if (cudaLaunchKernelEx(&cfg, kern, a) != cudaSuccess) return PTYCHO_ERR_LAUNCH;
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

}  // namespace f256

int launch_fused_256(int mode, int loss, const FusedArgs& a, cudaStream_t s) {
  using namespace f256;
  if (mode == MODE_INTENSITY) return launch_t<MODE_INTENSITY, 0>(a, s);
  if (mode == MODE_LOSS) {
    switch (loss) {
      case 0: return launch_t<MODE_LOSS, 0>(a, s);
      case 1: return launch_t<MODE_LOSS, 1>(a, s);
      case 2: return launch_t<MODE_LOSS, 2>(a, s);
      default: return launch_t<MODE_LOSS, 3>(a, s);
    }
  }
  switch (loss) {
    case 0: return launch_t<MODE_ADJ, 0>(a, s);
    case 1: return launch_t<MODE_ADJ, 1>(a, s);
    case 2: return launch_t<MODE_ADJ, 2>(a, s);
    default: return launch_t<MODE_ADJ, 3>(a, s);
  }
}

}  // namespace pty
