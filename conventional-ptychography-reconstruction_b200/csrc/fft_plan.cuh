// fft_plan.cuh -- register/shared-memory 2-D DFT plans for one M x M pattern.
//
// A pattern of M*M complex values is spread over NT threads, E values each.
// The 2-D DFT is decimation-in-frequency Cooley-Tukey over the 2*log2(M)
// position bits (x = column bits [0, LOGM), y = row bits [LOGM, 2 LOGM)).
// Three register passes each apply one x-stage and/or one y-stage to the
// digits a thread holds; between passes the values move through two float
// planes (re, im) in shared memory.  A PassDesc gives, per pass, which
// position bit each element bit and each thread-index bit stands for, so
// every shared-memory address is a per-thread base plus a compile-time
// offset.  Columns are XOR-swizzled (bits 5,6 folded onto bits 1,2) so all
// three lane maps are bank-conflict free with a pitch of M+1 floats.
// The spectrum is left in digit-reversed order; FreqMap gives the bit
// permutation position -> frequency.  The adjoint runs the passes backwards.
#pragma once
#include <utility>
#include <type_traits>

#include "common.cuh"
#include "dft_regs.cuh"

namespace pty {

struct PassDesc {
  int ne;        // element bits per thread (E = 1 << ne)
  int ebit[6];   // element bit j -> position bit; x-stage digit bits first,
                 // then y-stage digit bits, then repeat bits
  int nt;        // thread-index bits: 5 lane bits then warp bits
  int tbit[10];  // thread bit j -> position bit
  int nbx, lox;  // x DIF stage of this pass: digit width (0 = none), lowest bit
  int nby, loy;  // y DIF stage
  int nr = 0;          // cluster-rank bits (patterns split over a CTA cluster)
  int rbit[2] = {0, 0};  // rank bit j -> position bit
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
  static constexpr int LOGM = 6, NT = 256, E = 16, PITCH = 65, SWZ = 2, MIN_BLOCKS = 2;
  static constexpr PassDesc P1 = {4, {2, 3, 4, 5}, 8, {0, 1, 8, 9, 10, 6, 7, 11}, 4, 2, 0, 0};
  static constexpr PassDesc P2 = {4, {0, 1, 10, 11}, 8, {6, 7, 2, 3, 4, 5, 8, 9}, 2, 0, 2, 4};
  static constexpr PassDesc P3 = {4, {6, 7, 8, 9}, 8, {2, 3, 4, 5, 0, 1, 10, 11}, 0, 0, 4, 0};
  static constexpr FreqMap F = {{4, 5, 0, 1, 2, 3}, {2, 3, 4, 5, 0, 1}};
};

// M = 128: x = 16 * 8, y = 2 * 4 * 16; 512 threads x 32 values.
template <>
struct Plan<128> {
  static constexpr int LOGM = 7, NT = 512, E = 32, PITCH = 129, SWZ = 6, MIN_BLOCKS = 1;
  static constexpr PassDesc P1 = {5, {3, 4, 5, 6, 13}, 9, {0, 1, 2, 10, 11, 7, 8, 9, 12}, 4, 3, 1, 6};
  static constexpr PassDesc P2 = {5, {0, 1, 2, 11, 12}, 9, {7, 8, 9, 3, 4, 5, 6, 10, 13}, 3, 0, 2, 4};
  static constexpr PassDesc P3 = {5, {7, 8, 9, 10, 1}, 9, {3, 4, 5, 6, 0, 2, 11, 12, 13}, 0, 0, 4, 0};
  static constexpr FreqMap F = {{4, 5, 6, 0, 1, 2, 3}, {3, 4, 5, 6, 1, 2, 0}};
};

// M = 256: a cluster of 4 CTAs per pattern (512 threads x 32 values each);
// x = 16 * 16, y = 2 * 2 * 16 * 4 in four passes.  Passes 1-2 split rows by
// y bits 4,5 across the cluster, passes 3-4 by y bits 6,7; the exchange
// between passes 2 and 3 goes through distributed shared memory.
template <>
struct Plan<256> {
  static constexpr int LOGM = 8, NT = 512, E = 32, CLUSTER = 4, MIN_BLOCKS = 1;
  static constexpr PassDesc P1 = {5, {4, 5, 6, 7, 15}, 9, {0, 1, 2, 3, 8, 9, 10, 11, 14}, 4, 4, 1, 7, 2, {12, 13}};
  static constexpr PassDesc P2 = {5, {0, 1, 2, 3, 14}, 9, {4, 5, 6, 7, 9, 8, 10, 11, 15}, 4, 0, 1, 6, 2, {12, 13}};
  static constexpr PassDesc P3 = {5, {10, 11, 12, 13, 0}, 9, {1, 2, 3, 7, 9, 4, 5, 6, 8}, 0, 0, 4, 2, 2, {14, 15}};
  static constexpr PassDesc P4 = {5, {8, 9, 1, 2, 3}, 9, {0, 4, 5, 6, 7, 10, 11, 12, 13}, 0, 0, 2, 0, 2, {14, 15}};
  static constexpr FreqMap F = {{4, 5, 6, 7, 0, 1, 2, 3}, {6, 7, 2, 3, 4, 5, 1, 0}};
};

// column swizzle: bits 5 (and 6) of the column are XOR-ed onto bits 1 (and 2)
template <int M>
__host__ __device__ constexpr int swz(int px) {
  if constexpr (M == 256) return px ^ (((px >> 4) & 0xF) << 1);
  else return px ^ ((px >> 4) & Plan<M>::SWZ);
}

template <int M, int PASS>
__host__ __device__ constexpr PassDesc desc() {
  if constexpr (PASS == 1) return Plan<M>::P1;
  else if constexpr (PASS == 2) return Plan<M>::P2;
  else if constexpr (PASS == 3) return Plan<M>::P3;
  else return Plan<M>::P4;
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
// weight of thread bit J of a pass in x / y (compile time)
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
// position contributed by the cluster rank in a pass (compile-time bit map)
template <int M, int PASS>
PTY_DEVI void rbase(int r, int& bx, int& by) {
  constexpr PassDesc d = desc<M, PASS>();
  if constexpr (d.nr > 0) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int pb = j == 0 ? d.rbit[0] : d.rbit[1];
      const int bit = (r >> j) & 1;
      if (pb < Plan<M>::LOGM) bx |= bit << pb;
      else by |= bit << (pb - Plan<M>::LOGM);
    }
  }
}

// unrolled loop whose index is a compile-time constant
template <typename Fn, int... I>
PTY_DEVI void static_for_seq(Fn&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename Fn>
PTY_DEVI void static_for(Fn&& f) {
  static_for_seq(f, std::make_integer_sequence<int, N>{});
}

// ---------------------------------------------------------------------------
// one DIF pass (forward) or its adjoint, on the register array v
// ---------------------------------------------------------------------------
// twiddle table entry i, read with a volatile shared-memory load: the loads
// are issued where they are used instead of all being hoisted ahead of the
// butterflies, which keeps the 32-value passes inside the register budget
PTY_DEVI float2 tw_load(const float2* __restrict__ tw, int i) {
  float2 w;
  asm volatile("ld.volatile.shared.v2.f32 {%0, %1}, [%2];"
               : "=f"(w.x), "=f"(w.y)
               : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(tw + i))));
  return w;
}

template <int M, int E, bool ADJ, int RX, int RY, int LOX, int NBX, int LOY, int NBY>
PTY_DEVI void run_pass(float2 (&v)[E], int bx, int by, const float2* __restrict__ tw) {
  constexpr int LOGM = Plan<M>::LOGM;
  constexpr int REP = E / (RX * RY);
  static_assert(RX * RY * REP == E, "pass shape");
  if constexpr (RX > 1) {
    const int n2 = bx & ((1 << LOX) - 1);
    constexpr int SH = LOGM - LOX - NBX;
    if constexpr (!ADJ) {
#pragma unroll
      for (int j = 0; j < RY * REP; ++j) dft<RX, false, 1>(v + RX * j);
      if constexpr (LOX > 0) {
#pragma unroll
        for (int k = 1; k < RX; ++k) {
          const float2 w = tw[((n2 * k) << SH) & (M - 1)];
#pragma unroll
          for (int j = 0; j < RY * REP; ++j) v[k + RX * j] = c_mul(v[k + RX * j], w);
        }
      }
    } else {
      // one line at a time: conjugate twiddles (volatile loads, issued where
      // they are used), then the inverse DFT
#pragma unroll
      for (int j = 0; j < RY * REP; ++j) {
        if constexpr (LOX > 0) {
#pragma unroll
          for (int k = 1; k < RX; ++k) {
            float2 w = tw_load(tw, ((n2 * k) << SH) & (M - 1));
            w.y = -w.y;
            v[k + RX * j] = c_mul(v[k + RX * j], w);
          }
        }
        dft<RX, true, 1>(v + RX * j);
      }
    }
  }
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

// write v (layout PA) to the swizzled re/im planes, barrier, read back in layout PB
template <int M, int PA, int PB>
PTY_DEVI void exchange(float2 (&v)[Plan<M>::E], int t, float* re, float* im) {
  constexpr int PITCH = Plan<M>::PITCH, E = Plan<M>::E;
  int ax, ay, bx, by;
  tbase<M, PA>(t, ax, ay);
  tbase<M, PB>(t, bx, by);
  const int sax = swz<M>(ax), sbx = swz<M>(bx);
  float* rea = re + ay * PITCH;
  float* ima = im + ay * PITCH;
  const float* reb = re + by * PITCH;
  const float* imb = im + by * PITCH;
  __syncthreads();  // previous readers of the planes are done
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    constexpr int row = eoff_y<M, PA>(e) * PITCH;
    constexpr int col = swz<M>(eoff_x<M, PA>(e));
    const int off = row + (sax ^ col);
    rea[off] = v[e].x;
    ima[off] = v[e].y;
  });
  __syncthreads();
  static_for<E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    constexpr int row = eoff_y<M, PB>(e) * PITCH;
    constexpr int col = swz<M>(eoff_x<M, PB>(e));
    const int off = row + (sbx ^ col);
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

}  // namespace pty
