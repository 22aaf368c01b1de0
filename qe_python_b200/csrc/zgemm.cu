// Complex GEMMs of the nonlocal projector and Davidson subspace contractions.
//
//   C = alpha * op(A) * B + beta * C,   op(A) = A ("N") or A^H ("C")
//
// All matrices are column-major with explicit leading dimensions.  The
// plain form runs in FP64 (complex128) on the FP64 pipes: a register-tiled
// SIMT kernel (64 x 64 block tile, 4 x 4 complex micro tile per thread,
// 16-deep K tiles double-buffered in shared memory).  Contractions over the
// long plane-wave dimension (calbec beta^H psi, Davidson V^H HV) split K
// across blocks; the partial tiles go to caller scratch and a second kernel
// reduces them in a fixed order, so results are deterministic.
//
// Reference calls replaced: projector_overlaps (ZGEMM ConjTrans/NoTrans,
// qepy_pw/_native_fft.pyx:694-731), add_projector_product (ZGEMM beta=1,
// :782-836), the Davidson reduced-matrix and Ritz products
// (qepy_pw/diagonalization.py:658-726) and coupling @ overlaps (:348).
#include <mutex>

#include "qeb_common.cuh"
#include "../../include/qe_b200.h"

using qeb::C2;

namespace {

constexpr int BM = 64, BN = 64, BK = 16, THREADS = 256;

template <typename T>
struct Tile {
  C2<T> a[2][BK][BM];
  C2<T> b[2][BK][BN];
};

template <typename T, bool CONJ_A>
__device__ __forceinline__ void load_tiles(const C2<T>* __restrict__ A, int64_t lda,
                                           const C2<T>* __restrict__ B, int64_t ldb, int M,
                                           int N, int k0, int k1, int m0, int n0,
                                           C2<T> (&ra)[4], C2<T> (&rb)[4]) {
  const int t = threadIdx.x;
  const C2<T> zero = qeb::mk<T>(0, 0);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (CONJ_A) {
      // op(A)(m, k) = conj(A[k + m*lda]), contiguous along k
      const int k = t % BK, m = t / BK + 16 * r;
      const int gk = k0 + k, gm = m0 + m;
      C2<T> v = zero;
      if (gk < k1 && gm < M) {
        v = A[gk + (int64_t)gm * lda];
        v.im = -v.im;
      }
      ra[r] = v;
    } else {
      // op(A)(m, k) = A[m + k*lda], contiguous along m
      const int m = t % BM, k = t / BM + 4 * r;
      const int gk = k0 + k, gm = m0 + m;
      ra[r] = (gk < k1 && gm < M) ? A[gm + (int64_t)gk * lda] : zero;
    }
    const int k = t % BK, n = t / BK + 16 * r;
    const int gk = k0 + k, gn = n0 + n;
    rb[r] = (gk < k1 && gn < N) ? B[gk + (int64_t)gn * ldb] : zero;
  }
}

template <typename T, bool CONJ_A>
__device__ __forceinline__ void store_tiles(Tile<T>& s, int buf, const C2<T> (&ra)[4],
                                            const C2<T> (&rb)[4]) {
  const int t = threadIdx.x;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (CONJ_A) {
      s.a[buf][t % BK][t / BK + 16 * r] = ra[r];
    } else {
      s.a[buf][t / BM + 4 * r][t % BM] = ra[r];
    }
    s.b[buf][t % BK][t / BK + 16 * r] = rb[r];
  }
}

// One block computes a BM x BN tile of op(A) B over K range [kbeg, kend).
// split == 0: C = alpha*acc + beta*C.  split > 0: write acc to the partial
// buffer P (slice blockIdx.z, ldp = M).
template <typename T, bool CONJ_A>
__global__ void __launch_bounds__(THREADS) gemm_kernel(int M, int N, int K, int kchunk,
                                                       C2<T> alpha, const C2<T>* __restrict__ A,
                                                       int64_t lda, const C2<T>* __restrict__ B,
                                                       int64_t ldb, C2<T> beta, C2<T>* C,
                                                       int64_t ldc, C2<T>* __restrict__ P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Tile<T>& s = *reinterpret_cast<Tile<T>*>(smem_raw);
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kbeg = blockIdx.z * kchunk;
  const int kend = min(K, kbeg + kchunk);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  C2<T> acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = qeb::mk<T>(0, 0);
  C2<T> ra[4], rb[4];
  int buf = 0;
  if (kbeg < kend) {
    load_tiles<T, CONJ_A>(A, lda, B, ldb, M, N, kbeg, kend, m0, n0, ra, rb);
    store_tiles<T, CONJ_A>(s, 0, ra, rb);
  }
  __syncthreads();
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    const bool more = k0 + BK < kend;
    if (more) load_tiles<T, CONJ_A>(A, lda, B, ldb, M, N, k0 + BK, kend, m0, n0, ra, rb);
#pragma unroll 4
    for (int kk = 0; kk < BK; ++kk) {
      C2<T> av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = s.a[buf][kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = s.b[buf][kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].re = fma(av[i].re, bv[j].re, acc[i][j].re);
          acc[i][j].re = fma(-av[i].im, bv[j].im, acc[i][j].re);
          acc[i][j].im = fma(av[i].re, bv[j].im, acc[i][j].im);
          acc[i][j].im = fma(av[i].im, bv[j].re, acc[i][j].im);
        }
    }
    if (more) store_tiles<T, CONJ_A>(s, buf ^ 1, ra, rb);
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx + 16 * j;
      if (gn >= N) continue;
      if (P != nullptr) {
        P[(int64_t)blockIdx.z * M * N + gm + (int64_t)gn * M] = acc[i][j];
      } else {
        C2<T> v = qeb::cmul(alpha, acc[i][j]);
        C2<T>* c = C + gm + (int64_t)gn * ldc;
        if (beta.re != T(0) || beta.im != T(0)) v = v + qeb::cmul(beta, *c);
        *c = v;
      }
    }
  }
}

// C = alpha * sum_s P[s] + beta * C, slices summed in ascending order.
template <typename T>
__global__ void reduce_partials(int M, int N, int splits, const C2<T>* __restrict__ P,
                                C2<T> alpha, C2<T> beta, C2<T>* C, int64_t ldc) {
  const int64_t total = (int64_t)M * N;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    C2<T> sum = P[i];
    for (int s = 1; s < splits; ++s) sum = sum + P[(int64_t)s * total + i];
    const int64_t m = i % M, n = i / M;
    C2<T> v = qeb::cmul(alpha, sum);
    C2<T>* c = C + m + n * ldc;
    if (beta.re != T(0) || beta.im != T(0)) v = v + qeb::cmul(beta, *c);
    *c = v;
  }
}

// ---------------------------------------------------------------------------
// Skinny products: one side of the output has at most 16 columns.  The tiled
// kernel above wastes most of a 64-wide tile there and reads the large
// operand once per tile column; these kernels stream the large operand once
// from HBM and keep the narrow one in shared memory.  Cases of the hot path:
// calbec and the projector add for a few unconverged bands, the Davidson
// rows of a few correction vectors (new^H [HV, V]) and their Ritz columns.

constexpr int kSkinnyMax = 16;
constexpr int kSkinnyThreads = 256;
constexpr int kSkinnyColumns = kSkinnyThreads / 32;  // large-operand columns per block (OP_C)
constexpr int kSkinnyChunkC = 128;                   // K rows staged per step (OP_C)
constexpr int kSkinnyChunkN = 64;                    // K rows staged per step (OP_N)

int skinny_width(int n) { return n <= 4 ? 4 : (n <= 8 ? 8 : 16); }

// D[mb, ns] = sum_k conj(X[k, mb]) Y[k, ns] over this block's K range, one
// warp per large column mb, Y rows staged [ns][k].  splits == 1: the block
// writes C directly; else the partial slice blockIdx.y of P (Mb x Ns).
// Output mapping: swapped == 0: C[mb, ns] = alpha D + beta C;
//                 swapped == 1: C[ns, mb] = alpha conj(D) + beta C.
template <typename T, int NS>
__global__ void __launch_bounds__(kSkinnyThreads) skinny_c_kernel(
    int Mb, int Ns, int K, int krange, const C2<T>* __restrict__ X, int64_t ldx,
    const C2<T>* __restrict__ Y, int64_t ldy, C2<T> alpha, C2<T> beta, C2<T>* C, int64_t ldc,
    int swapped, C2<T>* __restrict__ P) {
  __shared__ C2<T> ys[NS][kSkinnyChunkC];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mb = blockIdx.x * kSkinnyColumns + warp;
  const int kbeg = blockIdx.y * krange;
  const int kend = min(K, kbeg + krange);
  const C2<T> zero = qeb::mk<T>(0, 0);
  C2<T> acc[NS];
#pragma unroll
  for (int n = 0; n < NS; ++n) acc[n] = zero;
  const C2<T>* xcol = X + (int64_t)(mb < Mb ? mb : 0) * ldx;
  for (int k0 = kbeg; k0 < kend; k0 += kSkinnyChunkC) {
    __syncthreads();
    for (int i = threadIdx.x; i < NS * kSkinnyChunkC; i += kSkinnyThreads) {
      const int n = i / kSkinnyChunkC, kk = i - n * kSkinnyChunkC;
      const int k = k0 + kk;
      ys[n][kk] = (n < Ns && k < kend) ? Y[k + (int64_t)n * ldy] : zero;
    }
    __syncthreads();
    if (mb < Mb) {
      C2<T> xv[kSkinnyChunkC / 32];
#pragma unroll
      for (int j = 0; j < kSkinnyChunkC / 32; ++j) {
        const int k = k0 + lane + 32 * j;
        xv[j] = (k < kend) ? xcol[k] : zero;
      }
#pragma unroll
      for (int j = 0; j < kSkinnyChunkC / 32; ++j) {
        const int kk = lane + 32 * j;
#pragma unroll
        for (int n = 0; n < NS; ++n) {
          const C2<T> y = ys[n][kk];
          // conj(x) * y
          acc[n].re = fma(xv[j].re, y.re, acc[n].re);
          acc[n].re = fma(xv[j].im, y.im, acc[n].re);
          acc[n].im = fma(xv[j].re, y.im, acc[n].im);
          acc[n].im = fma(-xv[j].im, y.re, acc[n].im);
        }
      }
    }
  }
#pragma unroll
  for (int n = 0; n < NS; ++n) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc[n].re += __shfl_xor_sync(0xffffffffu, acc[n].re, off);
      acc[n].im += __shfl_xor_sync(0xffffffffu, acc[n].im, off);
    }
  }
  if (lane != 0 || mb >= Mb) return;
  const bool use_beta = beta.re != T(0) || beta.im != T(0);
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    if (n >= Ns) break;
    if (P != nullptr) {
      P[(int64_t)blockIdx.y * Mb * Ns + mb + (int64_t)n * Mb] = acc[n];
    } else {
      C2<T> d = acc[n];
      if (swapped) d.im = -d.im;
      C2<T>* c = swapped ? C + n + (int64_t)mb * ldc : C + mb + (int64_t)n * ldc;
      C2<T> v = qeb::cmul(alpha, d);
      if (use_beta) v = v + qeb::cmul(beta, *c);
      *c = v;
    }
  }
}

// Sum of the skinny partial slices in ascending order, then the output
// mapping of skinny_c_kernel.
template <typename T>
__global__ void skinny_reduce(int Mb, int Ns, int splits, const C2<T>* __restrict__ P,
                              C2<T> alpha, C2<T> beta, C2<T>* C, int64_t ldc, int swapped) {
  const int64_t total = (int64_t)Mb * Ns;
  const bool use_beta = beta.re != T(0) || beta.im != T(0);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    C2<T> d = P[i];
    for (int s = 1; s < splits; ++s) d = d + P[(int64_t)s * total + i];
    const int64_t mb = i % Mb, n = i / Mb;
    if (swapped) d.im = -d.im;
    C2<T>* c = swapped ? C + n + mb * ldc : C + mb + n * ldc;
    C2<T> v = qeb::cmul(alpha, d);
    if (use_beta) v = v + qeb::cmul(beta, *c);
    *c = v;
  }
}

// C[m, n] = alpha sum_k A[m, k] B[k, n] + beta C[m, n] for N <= NS: one
// thread per row m, B rows staged [k][n] (every lane reads the same entry).
template <typename T, int NS>
__global__ void __launch_bounds__(kSkinnyThreads) skinny_n_kernel(
    int M, int N, int K, C2<T> alpha, const C2<T>* __restrict__ A, int64_t lda,
    const C2<T>* __restrict__ B, int64_t ldb, C2<T> beta, C2<T>* C, int64_t ldc) {
  __shared__ C2<T> bs[kSkinnyChunkN][NS];
  const int m = blockIdx.x * kSkinnyThreads + threadIdx.x;
  const C2<T> zero = qeb::mk<T>(0, 0);
  C2<T> acc[NS];
#pragma unroll
  for (int n = 0; n < NS; ++n) acc[n] = zero;
  const C2<T>* arow = A + (m < M ? m : 0);
  for (int k0 = 0; k0 < K; k0 += kSkinnyChunkN) {
    __syncthreads();
    for (int i = threadIdx.x; i < NS * kSkinnyChunkN; i += kSkinnyThreads) {
      const int n = i / kSkinnyChunkN, kk = i - n * kSkinnyChunkN;
      const int k = k0 + kk;
      bs[kk][n] = (n < N && k < K) ? B[k + (int64_t)n * ldb] : zero;
    }
    __syncthreads();
    if (m < M) {
      const int kn = min(kSkinnyChunkN, K - k0);
#pragma unroll 8
      for (int kk = 0; kk < kn; ++kk) {
        const C2<T> a = arow[(int64_t)(k0 + kk) * lda];
#pragma unroll
        for (int n = 0; n < NS; ++n) {
          const C2<T> b = bs[kk][n];
          acc[n].re = fma(a.re, b.re, acc[n].re);
          acc[n].re = fma(-a.im, b.im, acc[n].re);
          acc[n].im = fma(a.re, b.im, acc[n].im);
          acc[n].im = fma(a.im, b.re, acc[n].im);
        }
      }
    }
  }
  if (m >= M) return;
  const bool use_beta = beta.re != T(0) || beta.im != T(0);
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    if (n >= N) break;
    C2<T>* c = C + m + (int64_t)n * ldc;
    C2<T> v = qeb::cmul(alpha, acc[n]);
    if (use_beta) v = v + qeb::cmul(beta, *c);
    *c = v;
  }
}

int g_sm_count = 0;

int sm_count() {
  if (g_sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  return g_sm_count;
}

// Number of K slices: enough blocks for ~2 waves, each slice >= 256 deep.
int choose_splits(int M, int N, int K) {
  const int tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  const int want = (2 * sm_count() + tiles - 1) / tiles;
  int by_depth = K / 256;
  if (by_depth < 1) by_depth = 1;
  int s = want < by_depth ? want : by_depth;
  if (s > 64) s = 64;
  return s < 1 ? 1 : s;
}

// Skinny OP_C plan: the narrow side (N, else M when N is wide), the large
// side Mb and the number of K slices (about four waves, each >= 1024 deep).
struct SkinnyC {
  bool use = false, swapped = false;
  int mb = 0, ns = 0, splits = 1;
};

SkinnyC skinny_c_plan(int M, int N, int K) {
  SkinnyC p;
  if (N <= kSkinnyMax) {
    p.use = true, p.mb = M, p.ns = N;
  } else if (M <= kSkinnyMax) {
    p.use = true, p.swapped = true, p.mb = N, p.ns = M;
  } else {
    return p;
  }
  const int groups = (p.mb + kSkinnyColumns - 1) / kSkinnyColumns;
  int want = (4 * sm_count() + groups - 1) / groups;
  int by_depth = K / 1024;
  if (by_depth < 1) by_depth = 1;
  int s = want < by_depth ? want : by_depth;
  if (s > 64) s = 64;
  p.splits = s < 1 ? 1 : s;
  return p;
}

template <typename T, int NS>
void launch_skinny_c(const SkinnyC& p, int K, int krange, const C2<T>* X, int64_t ldx,
                     const C2<T>* Y, int64_t ldy, C2<T> al, C2<T> be, C2<T>* C, int64_t ldc,
                     C2<T>* partials, cudaStream_t stream) {
  const dim3 grid((p.mb + kSkinnyColumns - 1) / kSkinnyColumns, p.splits);
  skinny_c_kernel<T, NS><<<grid, kSkinnyThreads, 0, stream>>>(
      p.mb, p.ns, K, krange, X, ldx, Y, ldy, al, be, C, ldc, p.swapped ? 1 : 0, partials);
}

template <typename T>
int gemm_skinny_c(int M, int N, int K, C2<T> al, const C2<T>* A, int64_t lda, const C2<T>* B,
                  int64_t ldb, C2<T> be, C2<T>* C, int64_t ldc, void* scratch,
                  int64_t scratch_bytes, cudaStream_t stream) {
  SkinnyC p = skinny_c_plan(M, N, K);
  const int64_t slice_bytes = (int64_t)p.mb * p.ns * (int64_t)sizeof(C2<T>);
  if (p.splits > 1) {
    const int64_t fit = (scratch == nullptr) ? 0 : scratch_bytes / slice_bytes;
    if (fit < p.splits) p.splits = (int)(fit < 1 ? 1 : fit);
  }
  int krange = (K + p.splits - 1) / p.splits;
  krange = (krange + kSkinnyChunkC - 1) / kSkinnyChunkC * kSkinnyChunkC;
  if (krange < 1) krange = kSkinnyChunkC;
  p.splits = K > 0 ? (K + krange - 1) / krange : 1;
  // large operand X and narrow operand Y of D = X^H Y
  const C2<T>* X = p.swapped ? B : A;
  const C2<T>* Y = p.swapped ? A : B;
  const int64_t ldx = p.swapped ? ldb : lda, ldy = p.swapped ? lda : ldb;
  C2<T>* partials = p.splits > 1 ? static_cast<C2<T>*>(scratch) : nullptr;
  const int width = skinny_width(p.ns);
  if (width == 4)
    launch_skinny_c<T, 4>(p, K, krange, X, ldx, Y, ldy, al, be, C, ldc, partials, stream);
  else if (width == 8)
    launch_skinny_c<T, 8>(p, K, krange, X, ldx, Y, ldy, al, be, C, ldc, partials, stream);
  else
    launch_skinny_c<T, 16>(p, K, krange, X, ldx, Y, ldy, al, be, C, ldc, partials, stream);
  qeb::count_launches(p.splits > 1 ? 2 : 1);
  if (p.splits > 1) {
    const int64_t total = (int64_t)p.mb * p.ns;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 4 * sm_count()) blocks = 4 * sm_count();
    skinny_reduce<T><<<blocks, 256, 0, stream>>>(p.mb, p.ns, p.splits, partials, al, be, C, ldc,
                                                p.swapped ? 1 : 0);
  }
  return qeb::cuda_status(cudaGetLastError(), "zgemm skinny launch");
}

template <typename T>
int gemm_skinny_n(int M, int N, int K, C2<T> al, const C2<T>* A, int64_t lda, const C2<T>* B,
                  int64_t ldb, C2<T> be, C2<T>* C, int64_t ldc, cudaStream_t stream) {
  const dim3 grid((M + kSkinnyThreads - 1) / kSkinnyThreads);
  const int width = skinny_width(N);
  if (width == 4)
    skinny_n_kernel<T, 4><<<grid, kSkinnyThreads, 0, stream>>>(M, N, K, al, A, lda, B, ldb, be, C, ldc);
  else if (width == 8)
    skinny_n_kernel<T, 8><<<grid, kSkinnyThreads, 0, stream>>>(M, N, K, al, A, lda, B, ldb, be, C, ldc);
  else
    skinny_n_kernel<T, 16><<<grid, kSkinnyThreads, 0, stream>>>(M, N, K, al, A, lda, B, ldb, be, C, ldc);
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "zgemm skinny launch");
}

template <typename T>
int gemm(int opa, int M, int N, int K, const double* alpha, const void* A, int64_t lda,
         const void* B, int64_t ldb, const double* beta, void* C, int64_t ldc, void* scratch,
         int64_t scratch_bytes, cudaStream_t stream) {
  if (M < 0 || N < 0 || K < 0 || (opa != QEB_OP_N && opa != QEB_OP_C)) {
    qeb::set_error("zgemm: invalid sizes or op");
    return QEB_EINVAL;
  }
  if (M == 0 || N == 0) return QEB_OK;
  const int64_t a_rows = (opa == QEB_OP_N) ? M : K;
  if (lda < (a_rows > 0 ? a_rows : 1) || ldb < (K > 0 ? K : 1) || ldc < M) {
    qeb::set_error("zgemm: leading dimension too small (lda=%lld ldb=%lld ldc=%lld)",
                   (long long)lda, (long long)ldb, (long long)ldc);
    return QEB_EINVAL;
  }
  if (C == nullptr || (K > 0 && (A == nullptr || B == nullptr))) {
    qeb::set_error("zgemm: null operand");
    return QEB_EINVAL;
  }
  const C2<T> al = qeb::mk<T>((T)alpha[0], (T)alpha[1]);
  const C2<T> be = qeb::mk<T>((T)beta[0], (T)beta[1]);
  if (K > 0 && opa == QEB_OP_C && (N <= kSkinnyMax || M <= kSkinnyMax))
    return gemm_skinny_c<T>(M, N, K, al, static_cast<const C2<T>*>(A), lda,
                            static_cast<const C2<T>*>(B), ldb, be, static_cast<C2<T>*>(C), ldc,
                            scratch, scratch_bytes, stream);
  if (K > 0 && opa == QEB_OP_N && N <= kSkinnyMax)
    return gemm_skinny_n<T>(M, N, K, al, static_cast<const C2<T>*>(A), lda,
                            static_cast<const C2<T>*>(B), ldb, be, static_cast<C2<T>*>(C), ldc,
                            stream);
  const size_t smem = sizeof(Tile<T>);
  static bool configured[2] = {false, false};
  if (!configured[opa]) {
    cudaFuncSetAttribute(gemm_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    cudaFuncSetAttribute(gemm_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    configured[opa] = true;
  }
  int splits = (opa == QEB_OP_C) ? choose_splits(M, N, K) : 1;
  const int64_t slice_bytes = (int64_t)M * N * (int64_t)sizeof(C2<T>);
  if (splits > 1) {
    const int64_t fit = (scratch == nullptr) ? 0 : scratch_bytes / slice_bytes;
    if (fit < splits) splits = (int)(fit < 1 ? 1 : fit);
  }
  int kchunk = K;
  if (splits > 1) {
    kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + BK - 1) / BK * BK;
    splits = (K + kchunk - 1) / kchunk;
  }
  if (K == 0) kchunk = 1;
  const dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, splits);
  C2<T>* partials = (splits > 1) ? static_cast<C2<T>*>(scratch) : nullptr;
  if (opa == QEB_OP_C) {
    gemm_kernel<T, true><<<grid, THREADS, smem, stream>>>(
        M, N, K, kchunk, al, static_cast<const C2<T>*>(A), lda, static_cast<const C2<T>*>(B),
        ldb, be, static_cast<C2<T>*>(C), ldc, partials);
  } else {
    gemm_kernel<T, false><<<grid, THREADS, smem, stream>>>(
        M, N, K, kchunk, al, static_cast<const C2<T>*>(A), lda, static_cast<const C2<T>*>(B),
        ldb, be, static_cast<C2<T>*>(C), ldc, partials);
  }
  qeb::count_launches(splits > 1 ? 2 : 1);
  if (splits > 1) {
    const int64_t total = (int64_t)M * N;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 4 * sm_count()) blocks = 4 * sm_count();
    reduce_partials<T><<<blocks, 256, 0, stream>>>(M, N, splits, partials, al, be,
                                                   static_cast<C2<T>*>(C), ldc);
  }
  return qeb::cuda_status(cudaGetLastError(), "zgemm launch");
}

}  // namespace

extern "C" int64_t qeb_zgemm_scratch_bytes(int opa, int M, int N, int K, int precision) {
  if (opa != QEB_OP_C || M <= 0 || N <= 0 || K <= 0) return 0;
  const int64_t elem = (precision == QEB_F64) ? 16 : 8;
  if (N <= kSkinnyMax || M <= kSkinnyMax) {
    const SkinnyC p = skinny_c_plan(M, N, K);
    return p.splits > 1 ? (int64_t)p.splits * p.mb * p.ns * elem : 0;
  }
  const int splits = choose_splits(M, N, K);
  return splits > 1 ? (int64_t)splits * M * N * elem : 0;
}

extern "C" int qeb_zgemm(int opa, int M, int N, int K, const double* alpha, const void* A,
                         int64_t lda, const void* B, int64_t ldb, const double* beta, void* C,
                         int64_t ldc, void* scratch, int64_t scratch_bytes, void* stream) {
  return gemm<double>(opa, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, scratch, scratch_bytes,
                      static_cast<cudaStream_t>(stream));
}

extern "C" int qeb_cgemm(int opa, int M, int N, int K, const double* alpha, const void* A,
                         int64_t lda, const void* B, int64_t ldb, const double* beta, void* C,
                         int64_t ldc, void* scratch, int64_t scratch_bytes, void* stream) {
  return gemm<float>(opa, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, scratch, scratch_bytes,
                     static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the split-K product C = alpha A^H B + beta C.
//
// For callers that must not allocate device memory themselves, for example a
// host code that runs inside a memory pool it does not own, a process whose
// allocator is reserved for other data, or a driver that forbids cudaMalloc
// between set-up and shutdown.  Instead of caller scratch, the partial K
// tiles live in the fixed array below, which every GPU that loads this
// library holds until the process exits.
namespace {

constexpr int64_t kStaticPartialBytes = 16ll << 20;  // 16 MiB per device
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_static_partials[kStaticPartialBytes];

std::mutex g_static_mutex;
void* g_static_address[kMaxDevices] = {nullptr};

// Device address of g_static_partials on the current device.  The host-side
// symbol is only a stand-in, so the address is looked up once per device
// (with that device current) and cached for the life of the process; the
// cache assumes the primary context of each device throughout (a
// cudaDeviceReset or another current context leaves it stale).
int static_partials(void** out) {
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) return qeb::cuda_status(err, "zgemm_static_scratch: cudaGetDevice");
  if (device < 0 || device >= kMaxDevices) {
    qeb::set_error("zgemm_static_scratch: device index %d above %d", device, kMaxDevices);
    return QEB_EUNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (g_static_address[device] == nullptr) {
    void* address = nullptr;
    err = cudaGetSymbolAddress(&address, g_static_partials);
    if (err != cudaSuccess) return qeb::cuda_status(err, "zgemm_static_scratch: cudaGetSymbolAddress");
    g_static_address[device] = address;
  }
  *out = g_static_address[device];
  return QEB_OK;
}

}  // namespace

extern "C" int64_t qeb_zgemm_static_scratch_capacity(void) { return kStaticPartialBytes; }

extern "C" int qeb_zgemm_static_scratch(int M, int N, int K, const double* alpha, const void* A,
                                        int64_t lda, const void* B, int64_t ldb,
                                        const double* beta, void* C, int64_t ldc, void* stream) {
  // Two partial slices of M x N complex128 values must fit the array.
  if (M > 0 && N > 0 && (int64_t)M * N * 16 * 2 > kStaticPartialBytes) {
    qeb::set_error(
        "zgemm_static_scratch: M*N = %lld exceeds the %lld complex128 entries the static "
        "partial buffer allows (M*N*16*2 <= %lld bytes)",
        (long long)M * N, (long long)(kStaticPartialBytes / 32), (long long)kStaticPartialBytes);
    return QEB_EUNSUPPORTED;
  }
  void* scratch = nullptr;
  const int rc = static_partials(&scratch);
  if (rc != QEB_OK) return rc;
  return gemm<double>(QEB_OP_C, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, scratch,
                      kStaticPartialBytes, static_cast<cudaStream_t>(stream));
}
