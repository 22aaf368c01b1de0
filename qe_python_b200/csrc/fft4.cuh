// Register-resident four-step line FFTs with compile-time factors.
//
// A line of length n = N1 * N2 is owned by G = max(N1, N2) consecutive lanes
// of one warp ("a line group"); a warp holds floor(32 / G) groups.  Two data
// distributions are used:
//   D1: lane j (j < N2) holds x[j + N2 * i], i < N1
//   D2: lane k (k < N1) holds x[k + N1 * i], i < N2
// The inverse (sign +1) transform takes D1 to D2, the forward (sign -1)
// transform takes D2 to D1:
//   inverse: a[i] = x[j + N2 i]; A = DFT_N1(a); A[k] *= w^(j k)   (lane j)
//            exchange through the group's shared scratch
//            b[i] = A_i[k];       X[k + N1 i] = DFT_N2(b)           (lane k)
//   forward: the mirror image (DFT_N2 first, twiddle w^(k q2), DFT_N1).
// with w = exp(s 2 pi i / n) read from the per-line table tw[m] (forward
// sign; conjugated for the inverse).  Small DFTs of length 2..16 run fully
// unrolled in registers: coprime composite lengths by the prime-factor
// mapping, the others (8, 9, 16) by the Cooley-Tukey split with their
// twiddles from __constant__ tables (filled on the host from long-double
// evaluations, see init_small_dft_twiddles).  A lane's index within its
// group is below G, so the role tests of the group whose size is G itself
// are resolved at compile time.
#pragma once

#include <type_traits>

#include "qeb_common.cuh"

namespace qeb {

// Offsets of the composite small-DFT tables: exp(-2 pi i m / N), m < N.
template <int N> struct SmallTw;
template <> struct SmallTw<6> { static constexpr int off = 0; };
template <> struct SmallTw<8> { static constexpr int off = 6; };
template <> struct SmallTw<9> { static constexpr int off = 14; };
template <> struct SmallTw<10> { static constexpr int off = 23; };
template <> struct SmallTw<12> { static constexpr int off = 33; };
template <> struct SmallTw<15> { static constexpr int off = 45; };
template <> struct SmallTw<16> { static constexpr int off = 60; };
constexpr int kSmallTwTotal = 76;

// Defined here (one translation unit includes this header; the library is
// built without relocatable device code, so each module owns its tables).
__constant__ double2 c_small_tw64[kSmallTwTotal];
__constant__ float2 c_small_tw32[kSmallTwTotal];

template <int N> struct Split { static constexpr int A = 1, B = N; };
template <> struct Split<6> { static constexpr int A = 2, B = 3; };
template <> struct Split<8> { static constexpr int A = 2, B = 4; };
template <> struct Split<9> { static constexpr int A = 3, B = 3; };
template <> struct Split<10> { static constexpr int A = 2, B = 5; };
template <> struct Split<12> { static constexpr int A = 3, B = 4; };
template <> struct Split<15> { static constexpr int A = 3, B = 5; };
template <> struct Split<16> { static constexpr int A = 4, B = 4; };

template <typename T, int N, bool BWD>
__device__ __forceinline__ C2<T> small_tw(int m) {
  if constexpr (sizeof(T) == 8) {
    const double2 w = c_small_tw64[SmallTw<N>::off + m];
    return mk<T>(w.x, BWD ? -w.y : w.y);
  } else {
    const float2 w = c_small_tw32[SmallTw<N>::off + m];
    return mk<T>(w.x, BWD ? -w.y : w.y);
  }
}

// u * exp(sgn 2 pi i m / 8) for the compile-time m = 1, 2, 3 of the length-8
// split: multiplications by (1 +- i)/sqrt(2) and +-i without table loads.
template <typename T, bool BWD>
__device__ __forceinline__ C2<T> mul_w8(C2<T> u, int m) {
  constexpr T r = T(0.70710678118654752440084436210484903928L);  // 1/sqrt(2)
  // forward (BWD false) rotates by -45 degrees per step, backward by +45
  if (m == 2) return BWD ? mk<T>(-u.im, u.re) : mk<T>(u.im, -u.re);
  if (m == 1)
    return BWD ? mk<T>(r * (u.re - u.im), r * (u.re + u.im))
               : mk<T>(r * (u.re + u.im), r * (u.im - u.re));
  return BWD ? mk<T>(-r * (u.re + u.im), r * (u.re - u.im))
             : mk<T>(r * (u.im - u.re), -r * (u.re + u.im));
}

constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }

// The inverse of a modulo m (a and m coprime, both small).
constexpr int inverse_mod_c(int a, int m) {
  for (int x = 1; x < m; ++x)
    if ((a * x) % m == 1) return x;
  return m == 1 ? 0 : -1;
}

// Calls fn(std::integral_constant<int, I>{}) for I = BEGIN .. END - 1: a loop
// whose index is a constant expression (a template argument inside fn).
template <int BEGIN, int END, class Fn>
__device__ __forceinline__ void static_for(Fn&& fn) {
  if constexpr (BEGIN < END) {
    fn(std::integral_constant<int, BEGIN>{});
    static_for<BEGIN + 1, END>(fn);
  }
}

// Known-zero mask of the inputs of the first-stage DFT u[n1] = v[m(n1)],
// n1 < A, from the mask Z of v: bit n1 of the result is bit m(n1) of Z.
template <int A, int N, unsigned Z, int STRIDE, int OFFSET>
constexpr unsigned sub_zero_mask() {
  unsigned m = 0;
  for (int n1 = 0; n1 < A; ++n1)
    if ((Z >> ((STRIDE * n1 + OFFSET) % N)) & 1u) m |= 1u << n1;
  return m;
}

// In-register DFT of compile-time length N (sign +1 if BWD else -1).
// Bit i of Z marks input i as zero: it is neither read nor added (the
// result is the same as the DFT of an input whose entry i is zero; an entry
// of v marked in Z need not be initialised).  Length 2 skips the addition
// of a zero; the first stage of a split passes the marks on; other lengths
// fill the marked entries with zeros.
// Coprime splits N = A B (6, 10, 12, 15) use the prime-factor (Good-Thomas)
// mapping: input n = (B n1 + A n2) mod N, output k with k = k1 (mod A) and
// k = k2 (mod B), so w_N^(n k) = w_A^(n1 k1) w_B^(n2 k2) and no twiddle
// multiplications sit between the two stages.  Other composite lengths use
// the Cooley-Tukey split with twiddles.
template <typename T, int N, bool BWD, unsigned Z = 0u>
__device__ __forceinline__ void dft(C2<T>* v) {
  constexpr T sgn = BWD ? T(1) : T(-1);
  constexpr unsigned kAll = (N >= 32) ? 0xffffffffu : ((1u << N) - 1u);
  if constexpr (N == 1) {
    if constexpr (Z & 1u) v[0] = mk<T>(0, 0);
    return;
  } else if constexpr ((Z & kAll) == kAll) {
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = mk<T>(0, 0);
  } else if constexpr (N == 2 && Z != 0u) {
    if constexpr (Z & 1u) {  // (0, b) -> (b, -b)
      v[0] = v[1];
      v[1] = mk<T>(-v[1].re, -v[1].im);
    } else {  // (a, 0) -> (a, a)
      v[1] = v[0];
    }
  } else if constexpr (N == 2 || N == 3 || N == 4 || N == 5) {
#pragma unroll
    for (int i = 0; i < N; ++i)
      if ((Z >> i) & 1u) v[i] = mk<T>(0, 0);
    dft_small(v, N, sgn);
  } else if constexpr (gcd_c(Split<N>::A, Split<N>::B) == 1) {
    constexpr int A = Split<N>::A, B = Split<N>::B;
    constexpr int eA = B * inverse_mod_c(B % A, A), eB = A * inverse_mod_c(A % B, B);
    static_assert(eA % A == 1 && eA % B == 0 && eB % B == 1 && eB % A == 0,
                  "CRT idempotents of the prime-factor split");
    C2<T> y[A][B];
    static_for<0, B>([&](auto c) {
      constexpr int n2 = decltype(c)::value;
      C2<T> u[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1)
        if (!((Z >> ((B * n1 + A * n2) % N)) & 1u)) u[n1] = v[(B * n1 + A * n2) % N];
      dft<T, A, BWD, sub_zero_mask<A, N, Z, B, A * n2>()>(u);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) y[k1][n2] = u[k1];
    });
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      dft<T, B, BWD>(y[k1]);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[(k1 * eA + k2 * eB) % N] = y[k1][k2];
    }
  } else {
    constexpr int A = Split<N>::A, B = Split<N>::B;
    C2<T> y[B][A];
    static_for<0, B>([&](auto c) {
      constexpr int n2 = decltype(c)::value;
      C2<T> u[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1)
        if (!((Z >> (B * n1 + n2)) & 1u)) u[n1] = v[B * n1 + n2];
      dft<T, A, BWD, sub_zero_mask<A, N, Z, B, n2>()>(u);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) {
        if (n2 * k1 == 0)
          y[n2][k1] = u[k1];
        else if constexpr (N == 8)
          y[n2][k1] = mul_w8<T, BWD>(u[k1], n2 * k1);
        else
          y[n2][k1] = cmul(u[k1], small_tw<T, N, BWD>(n2 * k1));
      }
    });
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      C2<T> w[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) w[n2] = y[n2][k1];
      dft<T, B, BWD>(w);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = w[k2];
    }
  }
}

// Line-group geometry of a four-step transform n = N1 * N2.
template <int N1_, int N2_>
struct Four {
  static constexpr int N1 = N1_, N2 = N2_, n = N1_ * N2_;
  static constexpr int G = (N1_ > N2_) ? N1_ : N2_;
  static constexpr int per_warp = 32 / G;
  static constexpr int R = G;  // registers (complex) per lane
  // exchange buffer of one group: N1 rows of N2 values at an odd stride, so
  // the N1 lanes reading one column of it (8-byte or 16-byte values) fall on
  // distinct banks: N2 + 1 for even N2, N2 itself for odd N2 (an even stride
  // such as 16 for N2 = 15 put all of them on one bank)
  static constexpr int xstride = N2_ | 1;
  static constexpr int scratch = N1_ * xstride;
};

// Inverse transform, D1 -> D2.  `v` holds N1 values (D1) on lanes j < N2 and
// returns N2 values (D2) on lanes k < N1.  `x` is the group's exchange
// scratch (F::scratch values), `tw` the forward table of length n.
template <typename T, class F>
__device__ __forceinline__ void four_inverse(C2<T>* v, int lane, C2<T>* x, const C2<T>* tw,
                                             unsigned mask) {
  if (F::N2 == F::G || lane < F::N2) {
    dft<T, F::N1, true>(v);
#pragma unroll
    for (int k = 1; k < F::N1; ++k) {
      C2<T> w = tw[(lane * k) % F::n];
      w.im = -w.im;
      v[k] = cmul(v[k], w);
    }
#pragma unroll
    for (int k = 0; k < F::N1; ++k) x[k * F::xstride + lane] = v[k];
  }
  __syncwarp(mask);
  if (F::N1 == F::G || lane < F::N1) {
#pragma unroll
    for (int i = 0; i < F::N2; ++i) v[i] = x[lane * F::xstride + i];
    dft<T, F::N2, true>(v);
  }
  __syncwarp(mask);
}

// Forward transform, D2 -> D1.  `v` holds N2 values (D2) on lanes k < N1 and
// returns N1 values (D1) on lanes j < N2.
template <typename T, class F>
__device__ __forceinline__ void four_forward(C2<T>* v, int lane, C2<T>* x, const C2<T>* tw,
                                             unsigned mask) {
  if (F::N1 == F::G || lane < F::N1) {
    dft<T, F::N2, false>(v);
#pragma unroll
    for (int q = 1; q < F::N2; ++q) v[q] = cmul(v[q], tw[(lane * q) % F::n]);
#pragma unroll
    for (int q = 0; q < F::N2; ++q) x[lane * F::xstride + q] = v[q];
  }
  __syncwarp(mask);
  if (F::N2 == F::G || lane < F::N2) {
#pragma unroll
    for (int k = 0; k < F::N1; ++k) v[k] = x[k * F::xstride + lane];
    dft<T, F::N1, false>(v);
  }
  __syncwarp(mask);
}

// Per-lane four-step twiddles held in registers: a line group processes
// many lines with the same lane roles, so lane j's inverse factors
// conj(w)^(j k), k < N1, and lane k's forward factors w^(k q), q < N2, are
// loaded once instead of once per line.
template <typename T, class F>
struct LaneTwiddles {
  C2<T> inv[F::N1];
  C2<T> fwd[F::N2];
  __device__ __forceinline__ void load(int lane, const C2<T>* tw) {
#pragma unroll
    for (int k = 0; k < F::N1; ++k) {
      C2<T> w = tw[(lane * k) % F::n];
      w.im = -w.im;
      inv[k] = w;
    }
#pragma unroll
    for (int q = 0; q < F::N2; ++q) fwd[q] = tw[(lane * q) % F::n];
  }
};

// Z: known-zero mask of the D1 inputs (bit i: x[j + N2 i] is zero on every
// lane j), passed to the first DFT, which then neither reads nor adds them.
template <typename T, class F, unsigned Z = 0u>
__device__ __forceinline__ void four_inverse(C2<T>* v, int lane, C2<T>* x,
                                             const LaneTwiddles<T, F>& w, unsigned mask) {
  if (F::N2 == F::G || lane < F::N2) {
    dft<T, F::N1, true, Z>(v);
#pragma unroll
    for (int k = 1; k < F::N1; ++k) v[k] = cmul(v[k], w.inv[k]);
#pragma unroll
    for (int k = 0; k < F::N1; ++k) x[k * F::xstride + lane] = v[k];
  }
  __syncwarp(mask);
  if (F::N1 == F::G || lane < F::N1) {
#pragma unroll
    for (int i = 0; i < F::N2; ++i) v[i] = x[lane * F::xstride + i];
    dft<T, F::N2, true>(v);
  }
  __syncwarp(mask);
}

template <typename T, class F>
__device__ __forceinline__ void four_forward(C2<T>* v, int lane, C2<T>* x,
                                             const LaneTwiddles<T, F>& w, unsigned mask) {
  if (F::N1 == F::G || lane < F::N1) {
    dft<T, F::N2, false>(v);
#pragma unroll
    for (int q = 1; q < F::N2; ++q) v[q] = cmul(v[q], w.fwd[q]);
#pragma unroll
    for (int q = 0; q < F::N2; ++q) x[lane * F::xstride + q] = v[q];
  }
  __syncwarp(mask);
  if (F::N2 == F::G || lane < F::N2) {
#pragma unroll
    for (int k = 0; k < F::N1; ++k) v[k] = x[k * F::xstride + lane];
    dft<T, F::N1, false>(v);
  }
  __syncwarp(mask);
}

// Host: upload the composite small-DFT twiddles to the current device.
int init_small_dft_twiddles();

}  // namespace qeb
