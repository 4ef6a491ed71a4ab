// resample.cu -- Fourier (band-limited) upsampling of the object and its adjoint.
//
// Replaces models/complex_inr.py:252-271 (called at :287):
//   y = ifft2( ifftshift( zero_pad( fftshift( fft2(x) ) ) ) ) * s^2,
// x [h][w] -> y [h*s][w*s] complex64, and the gradient of that map (torch's
// complex convention, the conjugate-transpose operator).  The map is
// separable: per axis, y = (s / N) F_N^-1 P F_n x, where F is the
// unnormalised DFT and P places frequency f in [-n/2, n/2) of the length-n
// spectrum at f mod N of the length-N one (for even n and N this is what the
// shift / centred pad / inverse shift of the reference does).  Its adjoint is
// (s / N) F_n^-1 P^T F_N.  Both are "forward FFT of length L1, spectrum remap,
// inverse FFT of length L2, scale 1 / min(L1, L2)", so one kernel does all
// four line transforms:
//   row pass    -- lines are rows (contiguous), written as rows;
//   column pass -- lines are LINES adjacent columns (32-byte or wider
//                  segments per row), written the same way.
// Upsampling: row pass x -> t [h][w s], column pass t -> y.  Adjoint: row pass
// g -> t [h s][w], column pass t -> x-gradient.
//
// Each CTA loads LINES lines into two shared-memory planes (re, im; one float
// of padding every 32), runs radix-8 or radix-16 Stockham passes (8- or
// 16-value register slots; lines up to 1024 points use 8 for more threads) --
// natural order in and out, each thread holding one or two slots in
// registers, in place between barriers -- remaps the spectrum, runs the
// inverse passes and writes the lines back.  Twiddles come from the
// correctly rounded build-time table kTw4096 (twiddle4096.cuh, read through
// the L1 cache with stride 4096 / L), so no CTA spends time building one.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "dft_regs.cuh"
#include "line_fft.cuh"
#include "twiddle4096.cuh"

namespace pty {
namespace rs {

constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int cmin(int a, int b) { return a < b ? a : b; }

template <int L1, int L2, bool COL>
struct Cfg {
  static constexpr int LMAX = cmax(L1, L2);
  // row pass: 2048 values per CTA (>= 1 line); column pass: >= 4 lines
  // (32-byte segments) and 4096 values per CTA when lines are short (2 lines
  // of 4096, which would fit three CTAs per SM, ran slower: 16-byte pieces)
  static constexpr int LINES = COL ? cmax(4, 4096 / LMAX) : cmax(1, 2048 / LMAX);
  static constexpr int N = LINES * LMAX;            // values held by the CTA
  // values per register slot: 8 (radix-8 passes) for lines up to 1024 points,
  // which doubles the threads of these small, latency-bound transforms
  static constexpr int VPT = LMAX <= 1024 ? 8 : 16;
  static constexpr int NT = cmin(512, N / VPT);     // threads: one slot each, or two
  static constexpr int SPT = N / VPT / NT;          // slots per thread (1 or 2)
  static constexpr int PLANE = N + N / 32;          // padded plane length (floats)
  static constexpr size_t SMEM = size_t(2) * PLANE * 4;
  static_assert(SPT == 1 || SPT == 2, "slot count");
  static_assert(L1 >= 64 && L2 >= 64 && LMAX <= 4096, "supported line lengths");
};

PTY_DEVI int pad(int i) { return i + (i >> 5); }

// One Stockham pass of radix R over every line of length L: butterfly j of a
// line reads j + r L/R, applies exp(-+2 pi i (j mod NS) r / (NS R)) and the
// radix-R DFT, and writes (j / NS) NS R + (j mod NS) + r NS.  Twiddles are
// read from the 4096-entry table kTw4096 (global memory, L1-cached).
template <int L, int R, int NS, bool INV, int LINES, int NT, int SPT, int LMAX, int VPT>
PTY_DEVI void stockham(float* re, float* im, int t) {
  constexpr int BPL = L / R;              // butterflies per line
  constexpr int NB = LINES * BPL;         // butterflies in the CTA
  constexpr int PER = VPT / R;            // butterflies per VPT-value slot
  constexpr int NSLOT = NB / PER;         // slots in use (<= SPT * NT)
  constexpr int TWS = 4096 / (NS * R);    // twiddle table stride
  float2 v[SPT][VPT];
  int jj[SPT][PER], base[SPT][PER];
#pragma unroll
  for (int q = 0; q < SPT; ++q) {
    const int s = t + q * NT;
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int b = s + p * NSLOT;  // consecutive lanes -> consecutive j
      const int line = b / BPL, j = b - line * BPL;
      jj[q][p] = j;
      base[q][p] = line * LMAX;
      if (s < NSLOT) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = pad(base[q][p] + j + r * BPL);
          v[q][p * R + r] = make_float2(re[i], im[i]);
        }
      }
    }
  }
  __syncthreads();  // every value is read before any is overwritten
#pragma unroll
  for (int q = 0; q < SPT; ++q) {
    const int s = t + q * NT;
    if (s < NSLOT) {
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int j = jj[q][p];
        const int k = j % NS;
        if constexpr (NS > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            float2 w = __ldg(&kTw4096[k * r * TWS]);
            if constexpr (INV) w.y = -w.y;
            v[q][p * R + r] = c_mul(v[q][p * R + r], w);
          }
        }
        dft<R, INV, 1>(&v[q][p * R]);
        const int o = base[q][p] + (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = pad(o + r * NS);
          re[i] = v[q][p * R + r].x;
          im[i] = v[q][p * R + r].y;
        }
      }
    }
  }
  __syncthreads();
}

// all passes of a length-L transform: radix VPT while it divides the rest, then smaller
template <int L, bool INV, int LINES, int NT, int SPT, int LMAX, int VPT, int NS = 1>
PTY_DEVI void fft_lines(float* re, float* im, int t) {
  if constexpr (NS < L) {
    constexpr int REST = L / NS;
    constexpr int R = REST >= VPT ? VPT : REST;
    stockham<L, R, NS, INV, LINES, NT, SPT, LMAX, VPT>(re, im, t);
    fft_lines<L, INV, LINES, NT, SPT, LMAX, VPT, NS * R>(re, im, t);
  }
}

template <int L1, int L2, bool COL>
__global__ void __launch_bounds__(Cfg<L1, L2, COL>::NT) k_resample(const float2* __restrict__ in,
                                                                   float2* __restrict__ out, int nlines,
                                                                   long long ld_in, long long ld_out,
                                                                   float scale) {
  using C = Cfg<L1, L2, COL>;
  constexpr int LINES = C::LINES, NT = C::NT, LMAX = C::LMAX;
  extern __shared__ __align__(16) unsigned char smem[];
  float* re = reinterpret_cast<float*>(smem);
  float* im = re + C::PLANE;
  const int t = threadIdx.x;
  const int l0 = blockIdx.x * LINES;
  // load LINES lines of length L1 (lines past the end read as zero)
  for (int idx = t; idx < LINES * L1; idx += NT) {
    int l, k;
    if constexpr (COL) {
      l = idx % LINES;
      k = idx / LINES;
    } else {
      l = idx / L1;
      k = idx - l * L1;
    }
    float2 x = make_float2(0.f, 0.f);
    if (l0 + l < nlines)
      x = COL ? __ldg(in + k * ld_in + (l0 + l)) : __ldg(in + (l0 + l) * ld_in + k);
    const int i = pad(l * LMAX + k);
    re[i] = x.x;
    im[i] = x.y;
  }
  __syncthreads();
  fft_lines<L1, false, LINES, NT, C::SPT, LMAX, C::VPT>(re, im, t);
  // spectrum remap: frequency f in [-n/2, n/2), n = min(L1, L2), from f mod L1 to f mod L2
  if constexpr (L2 > L1) {
    for (int idx = t; idx < LINES * (L1 / 2); idx += NT) {  // negative frequencies move up
      const int l = idx / (L1 / 2), k = L1 / 2 + (idx - l * (L1 / 2));
      const int a = pad(l * LMAX + k), b = pad(l * LMAX + k + (L2 - L1));
      re[b] = re[a];
      im[b] = im[a];
    }
    __syncthreads();
    for (int idx = t; idx < LINES * (L2 - L1); idx += NT) {  // the new band is empty
      const int l = idx / (L2 - L1), k = L1 / 2 + (idx - l * (L2 - L1));
      const int a = pad(l * LMAX + k);
      re[a] = 0.f;
      im[a] = 0.f;
    }
    __syncthreads();
  } else if constexpr (L2 < L1) {
    for (int idx = t; idx < LINES * (L2 / 2); idx += NT) {  // negative frequencies move down
      const int l = idx / (L2 / 2), k = L2 / 2 + (idx - l * (L2 / 2));
      const int a = pad(l * LMAX + k + (L1 - L2)), b = pad(l * LMAX + k);
      re[b] = re[a];
      im[b] = im[a];
    }
    __syncthreads();
  }
  fft_lines<L2, true, LINES, NT, C::SPT, LMAX, C::VPT>(re, im, t);
  for (int idx = t; idx < LINES * L2; idx += NT) {
    int l, k;
    if constexpr (COL) {
      l = idx % LINES;
      k = idx / LINES;
    } else {
      l = idx / L2;
      k = idx - l * L2;
    }
    if (l0 + l < nlines) {
      const int i = pad(l * LMAX + k);
      const float2 y = make_float2(re[i] * scale, im[i] * scale);
      if constexpr (COL)
        out[k * ld_out + (l0 + l)] = y;
      else
        out[(l0 + l) * ld_out + k] = y;
    }
  }
}

template <int L1, int L2, bool COL>
int launch(const float2* in, float2* out, int nlines, long long ld_in, long long ld_out, cudaStream_t s) {
  using C = Cfg<L1, L2, COL>;
  auto kern = k_resample<L1, L2, COL>;
  if (C::SMEM > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(C::SMEM)) != cudaSuccess)
    return PTYCHO_ERR_LAUNCH;
  const int grid = (nlines + C::LINES - 1) / C::LINES;
  kern<<<grid, C::NT, C::SMEM, s>>>(in, out, nlines, ld_in, ld_out, 1.0f / float(L1 < L2 ? L1 : L2));
  return cudaGetLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_LAUNCH;
}

// dispatch over line lengths 2^6 .. 2^12 with L2 / L1 in {1/4, 1/2, 1, 2, 4}
template <bool COL>
int dispatch(int l1, int l2, const float2* in, float2* out, int nlines, long long ld_in, long long ld_out,
             cudaStream_t s) {
#define PTY_RS(A, B) \
  if (l1 == A && l2 == B) return launch<A, B, COL>(in, out, nlines, ld_in, ld_out, s);
#define PTY_RS_ROW(A) PTY_RS(A, A) PTY_RS(A, 2 * A) PTY_RS(2 * A, A) PTY_RS(A, 4 * A) PTY_RS(4 * A, A)
  PTY_RS_ROW(64)
  PTY_RS_ROW(128)
  PTY_RS_ROW(256)
  PTY_RS_ROW(512)
  PTY_RS_ROW(1024)
  PTY_RS(2048, 2048) PTY_RS(2048, 4096) PTY_RS(4096, 2048)
  PTY_RS(4096, 4096)
#undef PTY_RS_ROW
#undef PTY_RS
  return PTYCHO_ERR_UNSUPPORTED_SIZE;
}

bool supported(int n, int N) {
  auto pow2 = [](int v) { return v >= 64 && v <= 4096 && (v & (v - 1)) == 0; };
  if (!pow2(n) || !pow2(N)) return false;
  const int r = n > N ? n / N : N / n;
  return r == 1 || r == 2 || r == 4;
}

}  // namespace rs

// ---------------------------------------------------------------------------
// Any line length (the canvases Recovery.py builds are multiples of 6, so
// object grids are multiples of 3 and can hold large prime factors: 498 =
// 2 * 3 * 83).  Per line: forward DFT of length L1, band remap, inverse DFT
// of length L2, scale -- the same per-axis operator as above, with the remap
// written for odd lengths too.  With n = min(L1, L2), N = max(L1, L2) and the
// band k in [lo, lo + n), lo = -floor(n/2), the reference's fftshift /
// centred pad / ifftshift puts bin k of the length-n spectrum at bin
// (k + d) mod N of the length-N one, d = floor(n/2) + floor((N-n)/2) -
// floor(N/2): d = 0 for even n, or odd n and odd N; d = -1 for odd n and even
// N (the reference's half-bin asymmetry, kept).  The adjoint gathers back.
//
// Transforms are Stockham passes with a run-time plan: radix 16, 8, 4, 2, 3,
// 5, 7 as register butterflies (dft_regs.cuh), any other prime factor p as a
// direct p-term sum per output with table twiddles.  Passes ping-pong between
// two shared-memory buffers of float2 (one float2 of padding every 16 breaks
// the stride-2^k bank conflicts of the first passes).  Twiddles:
// exp(-2 pi i j / LMAX), LMAX = max(L1, L2) = s * min(L1, L2), rounded from
// double-precision sincospi; a length-L pass reads it with stride LMAX / L.
// ---------------------------------------------------------------------------
namespace rsg {

using lfft::LinePlan;
using lfft::make_plan;
using lfft::kMaxLen;
using lfft::pad16;
using lfft::transform;
constexpr int kNT = lfft::kLineNT;
constexpr size_t kSmemCap = 200 * 1024;

struct Args {
  const float2* in;
  float2* out;
  int nlines;
  long long ld_in, ld_out;
  LinePlan f1, f2;  // forward transform (length L1), inverse transform (length L2)
  int lmax;         // max(L1, L2): twiddle table length
  int lines;        // lines per CTA
  int ls;           // padded line stride in float2
  int d, lo;        // band remap offset and lowest band frequency
  float scale;
};

template <bool COL>
__global__ void __launch_bounds__(kNT) k_resample_any(const Args g) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lines = g.lines, ls = g.ls, lmax = g.lmax;
  float2* bufA = reinterpret_cast<float2*>(smem);
  float2* bufB = bufA + size_t(lines) * ls;
  float2* tw = bufB + size_t(lines) * ls;
  const int t = threadIdx.x;
  const int l0 = blockIdx.x * lines;
  const int L1 = g.f1.L, L2 = g.f2.L;
  for (int k = t; k < lmax; k += kNT) {
    double sn, cs;
    sincospi(-2.0 * double(k) / double(lmax), &sn, &cs);
    tw[k] = make_float2(float(cs), float(sn));
  }
  for (int idx = t; idx < lines * L1; idx += kNT) {
    int l, k;
    if (COL) {
      l = idx % lines;
      k = idx / lines;
    } else {
      l = idx / L1;
      k = idx - l * L1;
    }
    float2 x = make_float2(0.f, 0.f);
    if (l0 + l < g.nlines) x = COL ? __ldg(g.in + k * g.ld_in + (l0 + l)) : __ldg(g.in + (l0 + l) * g.ld_in + k);
    bufA[l * ls + pad16(k)] = x;
  }
  __syncthreads();
  float2* spec = transform<false>(g.f1, bufA, bufB, tw, lines, ls, lmax, t);
  float2* rem = spec == bufA ? bufB : bufA;
  // band remap into the other buffer
  const int n = L1 < L2 ? L1 : L2;
  for (int idx = t; idx < lines * L2; idx += kNT) {
    const int l = idx / L2, j = idx - l * L2;
    float2 v = make_float2(0.f, 0.f);
    if (L2 >= L1) {  // pad: bin j of the long spectrum holds band frequency k, or nothing
      int k = (j - g.d - g.lo) % L2;
      if (k < 0) k += L2;
      k += g.lo;
      if (k < g.lo + n) {
        int src = k % L1;
        if (src < 0) src += L1;
        v = spec[l * ls + pad16(src)];
      }
    } else {  // crop: bin j of the short spectrum is band frequency k of the long one
      int k = (j - g.lo) % n;
      if (k < 0) k += n;
      k += g.lo;
      int src = (k + g.d) % L1;
      if (src < 0) src += L1;
      v = spec[l * ls + pad16(src)];
    }
    rem[l * ls + pad16(j)] = v;
  }
  __syncthreads();
  float2* other = rem == bufA ? bufB : bufA;
  float2* res = transform<true>(g.f2, rem, other, tw, lines, ls, lmax, t);
  for (int idx = t; idx < lines * L2; idx += kNT) {
    int l, k;
    if (COL) {
      l = idx % lines;
      k = idx / lines;
    } else {
      l = idx / L2;
      k = idx - l * L2;
    }
    if (l0 + l < g.nlines) {
      const float2 y = res[l * ls + pad16(k)];
      const float2 o = make_float2(y.x * g.scale, y.y * g.scale);
      if (COL)
        g.out[k * g.ld_out + (l0 + l)] = o;
      else
        g.out[(l0 + l) * g.ld_out + k] = o;
    }
  }
}

static size_t smem_bytes(int lines, int ls, int lmax) {
  return (size_t(2) * lines * ls + size_t(lmax)) * sizeof(float2);
}

// true when the pair of line lengths is handled (one a whole multiple of the other)
static bool supported_pair(int l1, int l2) {
  if (l1 < 1 || l2 < 1 || l1 > kMaxLen || l2 > kMaxLen) return false;
  const int lo = l1 < l2 ? l1 : l2, hi = l1 < l2 ? l2 : l1;
  return hi % lo == 0;
}

// lines of length l1 -> lines of length l2: forward DFT, band remap, inverse DFT, scale 1 / min(l1, l2)
template <bool COL>
static int launch(int l1, int l2, const float2* in, float2* out, int nlines, long long ld_in, long long ld_out,
                  cudaStream_t s) {
  if (!supported_pair(l1, l2)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  Args g{};
  if (!make_plan(l1, &g.f1) || !make_plan(l2, &g.f2)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  g.in = in;
  g.out = out;
  g.nlines = nlines;
  g.ld_in = ld_in;
  g.ld_out = ld_out;
  const int n = l1 < l2 ? l1 : l2, N = l1 < l2 ? l2 : l1;
  g.lmax = N;
  g.lo = -(n / 2);
  g.d = n / 2 + (N - n) / 2 - N / 2;
  g.scale = 1.0f / float(n);
  g.ls = pad16(N - 1) + 1;
  // lines per CTA: ~8192 values, at least 4 adjacent columns (32-byte
  // segments) in the column pass, within the shared-memory cap
  int lines = N >= 8192 ? 1 : 8192 / N;
  if (COL && lines < 4) lines = 4;
  while (lines > 1 && smem_bytes(lines, g.ls, N) > kSmemCap) --lines;
  g.lines = lines;
  const size_t smem = smem_bytes(lines, g.ls, N);
  auto kern = k_resample_any<COL>;
  static PtyDevCache attr_set;
  int dev = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    if (!attr_set.get(&dev)) {
      if (dev < 0) return PTYCHO_ERR_LAUNCH;
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemCap)) != cudaSuccess)
        return PTYCHO_ERR_LAUNCH;
      attr_set.put(dev, 1);
    }
    kern<<<(nlines + lines - 1) / lines, kNT, smem, s>>>(g);
    if (cudaGetLastError() == cudaSuccess) return PTYCHO_OK;
    attr_set.put(dev, 0);
  }
  return PTYCHO_ERR_LAUNCH;
}

}  // namespace rsg
}  // namespace pty

using namespace pty;

namespace {

// power-of-two pairs keep the compile-time kernels; every other pair runs the
// run-time-planned one
template <bool COL>
int line_pass(int l1, int l2, const float2* in, float2* out, int nlines, long long ld_in, long long ld_out,
              cudaStream_t s) {
  if (rs::supported(l1, l2)) return rs::dispatch<COL>(l1, l2, in, out, nlines, ld_in, ld_out, s);
  return rsg::launch<COL>(l1, l2, in, out, nlines, ld_in, ld_out, s);
}

bool supported_upsample(int h, int w, int s) {
  if (h <= 0 || w <= 0 || s <= 0) return false;
  if (h > rsg::kMaxLen / s || w > rsg::kMaxLen / s) return false;
  return true;
}

}  // namespace

extern "C" {

size_t ptycho_fourier_upsample_workspace_size(int h, int w, int s) {
  if (h <= 0 || w <= 0 || s <= 0) return 0;
  return size_t(h) * size_t(w) * size_t(s) * sizeof(float2);
}

int ptycho_fourier_upsample(const float* x, int h, int w, int s, float* y, void* workspace,
                            size_t workspace_bytes, ptycho_stream_t stream) {
  if (!x || !y || h <= 0 || w <= 0 || s <= 0) return PTYCHO_ERR_INVALID_ARG;
  if (!supported_upsample(h, w, s)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (!workspace || workspace_bytes < ptycho_fourier_upsample_workspace_size(h, w, s))
    return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(x, 8) || !pty_aligned(y, 8) || !pty_aligned(workspace, 8)) return PTYCHO_ERR_MISALIGNED;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int W = w * s, H = h * s;
  float2* tmp = static_cast<float2*>(workspace);
  int rc = line_pass<false>(w, W, reinterpret_cast<const float2*>(x), tmp, h, w, W, st);  // rows
  if (rc) return rc;
  return line_pass<true>(h, H, tmp, reinterpret_cast<float2*>(y), W, W, W, st);           // columns
}

int ptycho_fourier_upsample_adjoint(const float* gy, int h, int w, int s, float* gx, void* workspace,
                                    size_t workspace_bytes, ptycho_stream_t stream) {
  if (!gy || !gx || h <= 0 || w <= 0 || s <= 0) return PTYCHO_ERR_INVALID_ARG;
  if (!supported_upsample(h, w, s)) return PTYCHO_ERR_UNSUPPORTED_SIZE;
  if (!workspace || workspace_bytes < ptycho_fourier_upsample_workspace_size(h, w, s))
    return PTYCHO_ERR_WORKSPACE;
  if (!pty_aligned(gy, 8) || !pty_aligned(gx, 8) || !pty_aligned(workspace, 8)) return PTYCHO_ERR_MISALIGNED;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int W = w * s, H = h * s;
  float2* tmp = static_cast<float2*>(workspace);  // [H][w]
  int rc = line_pass<false>(W, w, reinterpret_cast<const float2*>(gy), tmp, H, W, w, st);  // rows
  if (rc) return rc;
  return line_pass<true>(H, h, tmp, reinterpret_cast<float2*>(gx), w, w, w, st);           // columns
}

}  // extern "C"
