// dft_regs.cuh -- small DFTs held entirely in registers.
//
// dft<R, INV, S>(a) transforms the R complex values a[0], a[S], ..., a[(R-1)S]
// in place into natural order: afterwards a[k*S] = X[k] with
//   X[k] = sum_n a[n*S] * exp(-+ 2 pi i n k / R)   (minus: forward, plus: INV).
// All indices are compile-time constants, so after inlining the arrays live in
// registers.  Radix 16 is 4x4 Cooley-Tukey, radix 8 is 2x4; the internal
// twiddles are the exact constants cos/sin(pi/8), cos/sin(pi/4).  Radix 3, 5
// and 7 use the symmetric pair form with exact cos/sin(2 pi q / P).
#pragma once
#include "common.cuh"

namespace pty {

constexpr float kC8 = 0.70710678118654752440f;   // cos(pi/4)
constexpr float kC16 = 0.92387953251128675613f;  // cos(pi/8)
constexpr float kS16 = 0.38268343236508977173f;  // sin(pi/8)

// multiply by -i (forward) or +i (inverse)
template <bool INV>
PTY_DEVI float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// exp(-+ 2 pi i j / 16) for the j that occur in the 4x4 split (compile time)
template <int J, bool INV>
PTY_DEVI float2 w16_mul(float2 a) {
  constexpr int j = J & 15;
  if constexpr (j == 0) {
    return a;
  } else if constexpr (j == 4) {
    return mul_mi<INV>(a);
  } else if constexpr (j == 8) {
    return make_float2(-a.x, -a.y);
  } else if constexpr (j == 12) {
    return mul_mi<!INV>(a);
  } else {
    // generic: w = cos(2 pi j/16) -+ i sin(2 pi j/16)
    constexpr float cs[16] = {1.f, kC16, kC8, kS16, 0.f, -kS16, -kC8, -kC16,
                              -1.f, -kC16, -kC8, -kS16, 0.f, kS16, kC8, kC16};
    constexpr float sn[16] = {0.f, kS16, kC8, kC16, 1.f, kC16, kC8, kS16,
                              0.f, -kS16, -kC8, -kC16, -1.f, -kC16, -kC8, -kS16};
    const float c = cs[j];
    const float s = INV ? sn[j] : -sn[j];
    return make_float2(fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c));
  }
}

template <bool INV, int S>
PTY_DEVI void dft2(float2* a) {
  float2 t = a[0];
  a[0] = c_add(t, a[S]);
  a[S] = c_sub(t, a[S]);
}

template <bool INV, int S>
PTY_DEVI void dft4(float2* a) {
  float2 t0 = c_add(a[0], a[2 * S]);
  float2 t1 = c_sub(a[0], a[2 * S]);
  float2 t2 = c_add(a[S], a[3 * S]);
  float2 t3 = mul_mi<INV>(c_sub(a[S], a[3 * S]));
  a[0] = c_add(t0, t2);
  a[2 * S] = c_sub(t0, t2);
  a[S] = c_add(t1, t3);
  a[3 * S] = c_sub(t1, t3);
}

template <bool INV, int S>
PTY_DEVI void dft8(float2* a) {
  float2 u[4], w[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    u[n] = c_add(a[n * S], a[(n + 4) * S]);
    w[n] = c_sub(a[n * S], a[(n + 4) * S]);
  }
  w[1] = w16_mul<2, INV>(w[1]);
  w[2] = w16_mul<4, INV>(w[2]);
  w[3] = w16_mul<6, INV>(w[3]);
  dft4<INV, 1>(u);
  dft4<INV, 1>(w);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    a[(2 * k) * S] = u[k];
    a[(2 * k + 1) * S] = w[k];
  }
}

template <bool INV, int S>
PTY_DEVI void dft16(float2* a) {
  // n = 4*n1 + n2 ; k = k1 + 4*k2
  float2 t[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) t[i] = a[i * S];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) dft4<INV, 4>(t + n2);  // over n1 -> k1 at t[4*k1+n2]
  // twiddle W16^(n2*k1)
  t[5] = w16_mul<1, INV>(t[5]);
  t[6] = w16_mul<2, INV>(t[6]);
  t[7] = w16_mul<3, INV>(t[7]);
  t[9] = w16_mul<2, INV>(t[9]);
  t[10] = w16_mul<4, INV>(t[10]);
  t[11] = w16_mul<6, INV>(t[11]);
  t[13] = w16_mul<3, INV>(t[13]);
  t[14] = w16_mul<6, INV>(t[14]);
  t[15] = w16_mul<9, INV>(t[15]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4<INV, 1>(t + 4 * k1);  // over n2 -> k2 at t[4*k1+k2]
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) a[(k1 + 4 * k2) * S] = t[4 * k1 + k2];
}

// exact cos / sin(2 pi q / P) for the odd primes 3, 5, 7 (q = 0 .. P-1)
template <int P>
__host__ __device__ constexpr float odd_cos(int q) {
  q %= P;
  if (q > P / 2) q = P - q;
  if (q == 0) return 1.f;
  if constexpr (P == 3) return -0.5f;
  if constexpr (P == 5) return q == 1 ? 0.30901699437494742410f : -0.80901699437494742410f;
  return q == 1 ? 0.62348980185873353053f : (q == 2 ? -0.22252093395631440429f : -0.90096886790241912624f);
}
template <int P>
__host__ __device__ constexpr float odd_sin(int q) {
  q %= P;
  const float sg = q > P / 2 ? -1.f : 1.f;
  if (q > P / 2) q = P - q;
  if (q == 0) return 0.f;
  if constexpr (P == 3) return sg * 0.86602540378443864676f;
  if constexpr (P == 5) return sg * (q == 1 ? 0.95105651629515357212f : 0.58778525229247312917f);
  return sg * (q == 1 ? 0.78183148246802980871f : (q == 2 ? 0.97492791218182360702f : 0.43388373911755812048f));
}

// odd prime P: pairs a_m +- a_{P-m} give, for r = 1 .. (P-1)/2,
//   A_r = a_0 + sum_m (a_m + a_{P-m}) cos(2 pi m r / P)
//   B_r =       sum_m (a_m - a_{P-m}) sin(2 pi m r / P)
//   X_r = A_r -+ i B_r,  X_{P-r} = A_r +- i B_r   (upper sign: forward)
template <int P, bool INV, int S>
PTY_DEVI void dft_odd(float2* a) {
  constexpr int h = (P - 1) / 2;
  float2 sp[h], sm[h];
  float2 x0 = a[0], sum = a[0];
#pragma unroll
  for (int m = 1; m <= h; ++m) {
    sp[m - 1] = c_add(a[m * S], a[(P - m) * S]);
    sm[m - 1] = c_sub(a[m * S], a[(P - m) * S]);
    sum = c_add(sum, sp[m - 1]);
  }
#pragma unroll
  for (int r = 1; r <= h; ++r) {
    float2 A = x0, Bv = make_float2(0.f, 0.f);
#pragma unroll
    for (int m = 1; m <= h; ++m) {
      const float c = odd_cos<P>(m * r), s = odd_sin<P>(m * r);
      A = make_float2(fmaf(sp[m - 1].x, c, A.x), fmaf(sp[m - 1].y, c, A.y));
      Bv = make_float2(fmaf(sm[m - 1].x, s, Bv.x), fmaf(sm[m - 1].y, s, Bv.y));
    }
    // -i B = (B.y, -B.x); +i B = (-B.y, B.x)
    const float2 mib = INV ? make_float2(-Bv.y, Bv.x) : make_float2(Bv.y, -Bv.x);
    a[r * S] = c_add(A, mib);
    a[(P - r) * S] = c_sub(A, mib);
  }
  a[0] = sum;
}

template <int R, bool INV, int S>
PTY_DEVI void dft(float2* a) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2<INV, S>(a);
  } else if constexpr (R == 4) {
    dft4<INV, S>(a);
  } else if constexpr (R == 8) {
    dft8<INV, S>(a);
  } else if constexpr (R == 16) {
    dft16<INV, S>(a);
  } else if constexpr (R == 3 || R == 5 || R == 7) {
    dft_odd<R, INV, S>(a);
  } else {
    static_assert(R == 16, "unsupported radix");
  }
}

}  // namespace pty
