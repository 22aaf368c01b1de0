// Shared device/host helpers for the qe_b200 kernels (sm_100a).
//
// * C2<T>        : interleaved complex value (re, im), 8 or 16 bytes.
// * FftDesc      : a mixed-radix (2/3/4/5) Stockham factorisation of one
//                  transform length, passed by value to kernels.
// * fft_lines    : cooperative in-place FFT of many short lines held in
//                  shared memory, executed by the whole thread block.
// * error state  : thread-local message retrieved through qeb_last_error().
//
// Sign conventions follow the reference (qepy_pw/_native_fft.pyx:2020-2037):
// "backward" is the unnormalised sign +1 transform (G -> r), "forward" the
// unnormalised sign -1 transform (r -> G).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#define QEB_OK 0
#define QEB_EINVAL -1
#define QEB_EUNSUPPORTED -2
#define QEB_ECUDA -3
#define QEB_ESCRATCH -4
#define QEB_ENOPLAN -5

namespace qeb {

void set_error(const char* fmt, ...);
int cuda_status(cudaError_t err, const char* where);
// Process-wide count of kernels launched by this library (qeb_launch_count).
void count_launches(int n);

// Raise (never lower) a kernel's dynamic shared-memory limit on the current
// device: the attribute is per kernel, while plans of different sizes share
// the kernel.
template <typename Kernel>
cudaError_t raise_smem_limit(Kernel* kernel, size_t bytes) {
  cudaFuncAttributes attr;
  cudaError_t err = cudaFuncGetAttributes(&attr, reinterpret_cast<const void*>(kernel));
  if (err != cudaSuccess) return err;
  if ((size_t)attr.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(reinterpret_cast<const void*>(kernel),
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename T>
struct alignas(2 * sizeof(T)) C2 {
  T re, im;
};

template <typename T>
__host__ __device__ __forceinline__ C2<T> mk(T re, T im) {
  C2<T> c;
  c.re = re;
  c.im = im;
  return c;
}
template <typename T>
__device__ __forceinline__ C2<T> operator+(C2<T> a, C2<T> b) { return mk<T>(a.re + b.re, a.im + b.im); }
template <typename T>
__device__ __forceinline__ C2<T> operator-(C2<T> a, C2<T> b) { return mk<T>(a.re - b.re, a.im - b.im); }
template <typename T>
__device__ __forceinline__ C2<T> cmul(C2<T> a, C2<T> b) {
  return mk<T>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename T>
__device__ __forceinline__ C2<T> scale(C2<T> a, T s) { return mk<T>(a.re * s, a.im * s); }
// multiply by i*s
template <typename T>
__device__ __forceinline__ C2<T> imul(C2<T> a, T s) { return mk<T>(-a.im * s, a.re * s); }

constexpr int kMaxStages = 12;
constexpr int kMaxRadix = 5;

struct FftDesc {
  int n;
  int nstages;
  int radix[kMaxStages];
};

// Closed-form constants of the radix-3 and radix-5 DFT matrices.
// cos(2pi/3) = -1/2, sin(2pi/3) = sqrt(3)/2,
// cos(2pi/5) = (sqrt5-1)/4, cos(4pi/5) = -(sqrt5+1)/4,
// sin(2pi/5) = sqrt((5+sqrt5)/8), sin(4pi/5) = sqrt((5-sqrt5)/8).
constexpr double kSin60 = 0.86602540378443864676372317075294;
constexpr double kCos72 = 0.30901699437494742410229341718282;
constexpr double kCos144 = -0.80901699437494742410229341718282;
constexpr double kSin72 = 0.95105651629515357211643933337938;
constexpr double kSin144 = 0.58778525229247312916870595463907;

// In-register DFT of radix R on v[0..R-1]; sgn = -1 forward, +1 backward.
template <typename T>
__device__ __forceinline__ void dft_small(C2<T>* v, int R, T sgn) {
  if (R == 4) {
    C2<T> t0 = v[0] + v[2], t1 = v[0] - v[2];
    C2<T> t2 = v[1] + v[3], t3 = imul(v[1] - v[3], sgn);
    v[0] = t0 + t2;
    v[2] = t0 - t2;
    v[1] = t1 + t3;
    v[3] = t1 - t3;
  } else if (R == 2) {
    C2<T> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  } else if (R == 3) {
    C2<T> s = v[1] + v[2], d = v[1] - v[2];
    C2<T> a = v[0];
    v[0] = a + s;
    C2<T> m = a + scale(s, T(-0.5));
    C2<T> n = imul(d, sgn * T(kSin60));
    v[1] = m + n;
    v[2] = m - n;
  } else if (R == 5) {
    C2<T> a = v[0];
    C2<T> s1 = v[1] + v[4], d1 = v[1] - v[4];
    C2<T> s2 = v[2] + v[3], d2 = v[2] - v[3];
    v[0] = a + s1 + s2;
    C2<T> m1 = a + scale(s1, T(kCos72)) + scale(s2, T(kCos144));
    C2<T> m2 = a + scale(s1, T(kCos144)) + scale(s2, T(kCos72));
    C2<T> p1 = imul(scale(d1, T(kSin72)) + scale(d2, T(kSin144)), sgn);
    C2<T> p2 = imul(scale(d1, T(kSin144)) - scale(d2, T(kSin72)), sgn);
    v[1] = m1 + p1;
    v[4] = m1 - p1;
    v[2] = m2 + p2;
    v[3] = m2 - p2;
  }
}

// Cooperative in-place Stockham autosort FFT of `nlines` lines of length
// d.n held in shared memory.  Element e of line l lives at
// data[l*line_stride + e*elem_stride].  `tw` holds the forward twiddle
// table exp(-2 pi i m / n), m = 0..n-1 (conjugated for backward).
// Every thread of the block must call this (it synchronises internally);
// the call ends with a __syncthreads().
//
// Stage s (radix R, Ns = product of earlier radices), butterfly j of a line:
//   v[r] = x[j + r n/R] * w^(r * (j mod Ns) * n/(Ns R)),  DFT_R(v),
//   y[(j / Ns) Ns R + (j mod Ns) + r Ns] = v[r].
template <typename T, int MAXB>
__device__ void fft_lines(C2<T>* data, int nlines, int line_stride, int elem_stride,
                          const FftDesc& d, const C2<T>* tw, bool backward) {
  const int n = d.n;
  const T sgn = backward ? T(1) : T(-1);
  int Ns = 1;
  for (int s = 0; s < d.nstages; ++s) {
    const int R = d.radix[s];
    const int nbf = n / R;
    const int tw_stride = n / (Ns * R);
    int lines_per_chunk = (int)(blockDim.x * MAXB) / nbf;
    if (lines_per_chunk < 1) lines_per_chunk = 1;
    for (int l0 = 0; l0 < nlines; l0 += lines_per_chunk) {
      const int lc = min(lines_per_chunk, nlines - l0);
      const int total = lc * nbf;
      C2<T> v[MAXB][kMaxRadix];
#pragma unroll
      for (int k = 0; k < MAXB; ++k) {
        const int t = threadIdx.x + k * blockDim.x;
        if (t < total) {
          const int l = l0 + t / nbf;
          const int j = t - (t / nbf) * nbf;
          const C2<T>* line = data + (size_t)l * line_stride;
#pragma unroll
          for (int r = 0; r < kMaxRadix; ++r)
            if (r < R) v[k][r] = line[(j + r * nbf) * elem_stride];
          if (Ns > 1) {
            const int kk = j % Ns;
#pragma unroll
            for (int r = 1; r < kMaxRadix; ++r) {
              if (r < R) {
                C2<T> w = tw[r * kk * tw_stride];
                if (backward) w.im = -w.im;
                v[k][r] = cmul(v[k][r], w);
              }
            }
          }
          dft_small(v[k], R, sgn);
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < MAXB; ++k) {
        const int t = threadIdx.x + k * blockDim.x;
        if (t < total) {
          const int l = l0 + t / nbf;
          const int j = t - (t / nbf) * nbf;
          const int kk = j % Ns;
          const int base = (j / Ns) * Ns * R + kk;
          C2<T>* line = data + (size_t)l * line_stride;
#pragma unroll
          for (int r = 0; r < kMaxRadix; ++r)
            if (r < R) line[(base + r * Ns) * elem_stride] = v[k][r];
        }
      }
      __syncthreads();
    }
    Ns *= R;
  }
}

// Host: factor n into radices 4, 2, 3, 5 (returns false for other primes).
bool make_fft_desc(int n, FftDesc* d);

}  // namespace qeb
