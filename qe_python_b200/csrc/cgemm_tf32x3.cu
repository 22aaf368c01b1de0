// Split-TF32 complex GEMM that reads complex64 operands directly.
//
//   C = alpha * op(A) B + beta * C,  op(A) = A^H (QEB_OP_C) or A (QEB_OP_N)
//
// A, B and C are column-major complex64 matrices.  Unlike qeb_tf32_gemm,
// nothing is packed beforehand: each pipeline stage TMA-loads the raw FP32
// words of one 128-row by 16-complex slab of A and of B into shared memory,
// and the worker warps split every value x into hi = tf32(x) and
// lo = tf32(x - hi) in place, in the 128-byte-swizzled K-major layout that
// tcgen05.mma reads.  The complex product is carried by real products over
// (re, im) pairs interleaved along K:
//   OP_C  Re(conj(a) b) = [a_re, a_im].[b_re, b_im]
//         Im(conj(a) b) = [a_re, a_im].[b_im, -b_re]       (B1 = swap-negated B)
//   OP_N  Re(a b)       = [a_re, -a_im].[b_re, b_im]      (A0, A transposed by
//         Im(a b)       = [a_im, a_re].[b_re, b_im]        the workers)
// and each real product is hi*hi + hi*lo + lo*hi, three tcgen05.mma.kind::tf32.
//
// Two-level accumulation: the tensor cores add each MMA's products into the
// FP32 accumulator with an error that grows with the number of additions
// (measured: 7e-6 relative after 384 MMAs into one accumulator, 2e-4 after
// 12 000), so each stage's 12 MMAs per accumulator start a fresh tensor-memory
// accumulator (two buffers of Re and Im, 512 columns) and the worker warps add
// it into FP32 registers with round-to-nearest.  The result is as accurate
// as an FP32 FMA GEMM.
//
// One CTA = 320 threads computes a 128 x 128 output tile over a K range:
//   warp 0 lane 0 : TMA producer, two stages
//   warp 1 lane 0 : MMA issuer; warp 1 owns the tensor-memory allocation
//   warps 2-9     : workers: split the next stage, drain the previous
//                   stage's accumulator into registers, then store C
// Worker warp w reads tensor-memory lanes 32 (w % 4) .. +31 (its rows) and
// columns 64 ((w - 2) / 4) .. +63 of Re and of Im.  K is split across CTAs
// (grid.z) into caller scratch when the output has few tiles; a second kernel
// sums the slices in a fixed order.  Every wait is bounded; on timeout the
// CTA records an error code in the device word read by qeb_tf32_gemm_error
// and unwinds.
//
// Requirements (else QEB_STATUS_EUNSUPPORTED, and the caller uses the packed
// path): A and B 16-byte aligned with even leading dimensions (TMA rows must
// start on 16-byte boundaries).
#include <cuda.h>
#include <cuda_runtime.h>

#include "qeb_common.cuh"
#include "tcgen05.cuh"
#include "../../include/qe_b200.h"

namespace {

using namespace qeb::tc;

constexpr int BM = 128, BN = 128;
constexpr int BKF = 32;      // FP32 words along K per stage (16 complex values)
constexpr int TILE = 16384;  // bytes of one 128-row x 32-word tile
constexpr int STAGES = 2;
// Stages ahead whose tiles the producer prefetches into L2, so that the
// loads of the two-stage ring read L2 rather than HBM.
constexpr int kPrefetch = 2;
constexpr int WORKERS = 8;                 // worker warps (2 .. 9)
constexpr int WORKER_THREADS = 32 * WORKERS;
constexpr int THREADS = 64 + WORKER_THREADS;
constexpr int ACC_COLS = 2 * BN;           // Re and Im of one accumulator buffer
constexpr int TMEM_COLS = 2 * ACC_COLS;    // two buffers
constexpr uint32_t kIdesc = idesc_tf32(BM, BN);
// OP_C: Re and Im share A, so one M128 N256 product over [B; B1] (the two
// K-major tiles adjacent in shared memory, 256 rows at the same 1024-byte
// group stride) writes the Re and Im columns of an accumulator buffer at
// once: 12 KB of operands per 128 x 256 x 8 products instead of 16 KB for
// two N128 ones.
constexpr uint32_t kIdescReIm = idesc_tf32(BM, 2 * BN);

// Tile slots of one stage.  OP_C: 0 A (raw, then hi), 1 A lo, 2 B (raw, then
// hi), 3 B1 hi, 4 B lo, 5 B1 lo ([B; B1] hi and lo each 256 contiguous
// rows).  OP_N: 0 A raw (16 x 256 words, row-major, unswizzled), 1 B (raw,
// then hi), 2 B lo, 3 A0 hi, 4 A0 lo, 5 A1 hi, 6 A1 lo.
template <int OP>
struct Slots {
  static constexpr bool kC = OP == QEB_OP_C;
  static constexpr int tiles = kC ? 6 : 7;
  static constexpr int stage_bytes = tiles * TILE;
  static constexpr int raw_a = 0, raw_b = kC ? 2 : 1;
  static constexpr int a_re_hi = kC ? 0 : 3, a_re_lo = kC ? 1 : 4;
  static constexpr int a_im_hi = kC ? 0 : 5, a_im_lo = kC ? 1 : 6;
  static constexpr int b_re_hi = kC ? 2 : 1, b_re_lo = kC ? 4 : 2;
  static constexpr int b_im_hi = kC ? 3 : 1, b_im_lo = kC ? 5 : 2;
  static_assert(!kC || (b_im_hi == b_re_hi + 1 && b_im_lo == b_re_lo + 1),
                "[B; B1] contiguous for the N256 product");
};

template <int OP>
constexpr size_t smem_bytes() {
  return (size_t)STAGES * Slots<OP>::stage_bytes + 1024 /*alignment*/ + 256 /*barriers*/;
}

struct Maps {
  CUtensorMap a, b;
};

__device__ __forceinline__ float4 hi4(float4 v) {
  return make_float4(tf32_round(v.x), tf32_round(v.y), tf32_round(v.z), tf32_round(v.w));
}
__device__ __forceinline__ float4 lo4(float4 v, float4 h) {
  return make_float4(tf32_round(v.x - h.x), tf32_round(v.y - h.y), tf32_round(v.z - h.z),
                     tf32_round(v.w - h.w));
}

// Split one K-major tile in place (hi) with its lo part into another slot.
// The split is elementwise, so the 128-byte swizzle needs no attention.
__device__ __forceinline__ void split_tile(unsigned char* tile, unsigned char* lo, int ct,
                                           unsigned char* swap_hi, unsigned char* swap_lo) {
  float4* t = reinterpret_cast<float4*>(tile);
  float4* l = reinterpret_cast<float4*>(lo);
#pragma unroll 2
  for (int c = ct; c < TILE / 16; c += WORKER_THREADS) {
    const float4 v = t[c];
    const float4 h = hi4(v), w = lo4(v, h);
    t[c] = h;
    l[c] = w;
    if (swap_hi != nullptr) {  // (re, im) -> (im, -re)
      reinterpret_cast<float4*>(swap_hi)[c] = make_float4(h.y, -h.x, h.w, -h.z);
      reinterpret_cast<float4*>(swap_lo)[c] = make_float4(w.y, -w.x, w.w, -w.z);
    }
  }
}

// OP_N: transpose the raw M-major slab of A (16 K rows x 128 complex) into
// the K-major swizzled tiles A0 = [re, -im] and A1 = [im, re], hi and lo.
__device__ __forceinline__ void transpose_a(const unsigned char* raw, unsigned char* a0h,
                                            unsigned char* a0l, unsigned char* a1h,
                                            unsigned char* a1l, int ct) {
  const float2* x = reinterpret_cast<const float2*>(raw);
#pragma unroll 2
  for (int it = ct; it < BM * 8; it += WORKER_THREADS) {
    const int m = it & (BM - 1), kp = it >> 7;  // kp: pair of K values 2kp, 2kp+1
    const float2 x0 = x[(2 * kp) * BM + m];
    const float2 x1 = x[(2 * kp + 1) * BM + m];
    const float4 r0 = make_float4(x0.x, -x0.y, x1.x, -x1.y);
    const float4 r1 = make_float4(x0.y, x0.x, x1.y, x1.x);
    const float4 h0 = hi4(r0), h1 = hi4(r1);
    const int off = m * 128 + ((kp ^ (m & 7)) << 4);
    *reinterpret_cast<float4*>(a0h + off) = h0;
    *reinterpret_cast<float4*>(a0l + off) = lo4(r0, h0);
    *reinterpret_cast<float4*>(a1h + off) = h1;
    *reinterpret_cast<float4*>(a1l + off) = lo4(r1, h1);
  }
}

// Worker side of one stage's accumulator buffer: wait until its MMAs are
// done, add Re (columns [0, 64) of this warp's half) and Im into registers,
// release the buffer.  False on a timed-out wait.
__device__ __forceinline__ bool drain_accumulator(float (&acc)[BN], uint64_t* acc_full,
                                                  uint64_t* acc_empty, int i, uint32_t lane_base,
                                                  int lane) {
  const int b = i & 1;
  if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[b], (i >> 1) & 1))) return false;
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t t = lane_base + b * ACC_COLS;
#pragma unroll
  for (int part = 0; part < 4; ++part) {  // Re 0-31, Re 32-63, Im 0-31, Im 32-63
    float v[32];
    tmem_ld32(t + (part >> 1) * BN + (part & 1) * 32, v);
    tmem_wait_ld();
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[part * 32 + j] += v[j];
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncwarp();
  if (lane == 0) mbar_arrive(&acc_empty[b]);
  return true;
}

template <int OP, bool TAIL = false>
__global__ void __launch_bounds__(THREADS, 1) cgemm_tf32x3_kernel(
    const __grid_constant__ Maps maps, int M, int N, int kb_per_split, int kb_total, float2 alpha,
    float2 beta, float2* C, int64_t ldc, float2* split, int* error, int skip_m, int skip_n,
    int m_off, int n_off, int tail_tiles) {
  // TAIL == false: grid (M tiles, N tiles, K slices); the tiles of column
  // skip_n from row skip_m on belong to a tail launch and return at once.
  // TAIL: grid (tail tiles, 1, K slices) over rows m_off + x of column
  // n_off; the K slices go to compact BM x BN partial tiles.
  if (!TAIL && (int)blockIdx.y == skip_n && (int)blockIdx.x >= skip_m) return;
  using S = Slots<OP>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * S::stage_bytes);
  uint64_t* conv = full + STAGES;       // stage split by the workers
  uint64_t* empty = conv + STAGES;      // stage consumed by the MMAs
  uint64_t* acc_full = empty + STAGES;  // accumulator buffer written by the MMAs
  uint64_t* acc_empty = acc_full + 2;   // accumulator buffer drained by the workers
  uint64_t* done = acc_empty + 2;       // every MMA issued has completed
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  volatile int* abort_v = abort_flag;

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int m0 = ((int)blockIdx.x + (TAIL ? m_off : 0)) * BM;
  const int n0 = ((int)blockIdx.y + (TAIL ? n_off : 0)) * BN;
  const int kb0 = blockIdx.z * kb_per_split;
  const int nk = max(0, min(kb_total, kb0 + kb_per_split) - kb0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&conv[s], WORKERS);  // one arrival per worker warp
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], WORKERS);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      for (int i = 0; i < nk; ++i) {
        const int s = i % STAGES;
        if (i >= STAGES && !mbar_wait(&empty[s], ((i / STAGES) - 1) & 1)) {
          atomicExch(error, 11);
          *abort_v = 1;
          break;
        }
        if (*abort_v) break;
        unsigned char* st = base + s * S::stage_bytes;
        mbar_expect_tx(&full[s], 2 * TILE);
        const int kb = kb0 + i;
        if (OP == QEB_OP_C) {
          tma_load_2d(st + S::raw_a * TILE, &maps.a, &full[s], kb * BKF, m0);
        } else {
          tma_load_2d(st + S::raw_a * TILE, &maps.a, &full[s], 2 * m0, kb * (BKF / 2));
        }
        tma_load_2d(st + S::raw_b * TILE, &maps.b, &full[s], kb * BKF, n0);
        if (i + kPrefetch < nk) {  // the tiles of stage i + kPrefetch into L2
          const int kp = kb + kPrefetch;
          if (OP == QEB_OP_C)
            tma_prefetch_2d(&maps.a, kp * BKF, m0);
          else
            tma_prefetch_2d(&maps.a, 2 * m0, kp * (BKF / 2));
          tma_prefetch_2d(&maps.b, kp * BKF, n0);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      for (int i = 0; i < nk; ++i) {
        const int s = i % STAGES, b = i & 1;
        // the stage is split, and this accumulator buffer was drained (i - 2)
        if (!mbar_wait(&conv[s], (i / STAGES) & 1) ||
            (i >= 2 && !mbar_wait(&acc_empty[b], ((i >> 1) - 1) & 1))) {
          atomicExch(error, 12);
          *abort_v = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t st = smem_u32(base + s * S::stage_bytes);
        const uint32_t t_re = tmem + b * ACC_COLS, t_im = t_re + BN;
#pragma unroll
        for (int kk = 0; kk < BKF / 8; ++kk) {
          const uint32_t off = kk * 32;  // 8 tf32 words along K
          const uint32_t acc = kk > 0 ? 1u : 0u;
          const uint64_t arh = smem_desc_sw128(st + S::a_re_hi * TILE + off);
          const uint64_t arl = smem_desc_sw128(st + S::a_re_lo * TILE + off);
          const uint64_t aih = smem_desc_sw128(st + S::a_im_hi * TILE + off);
          const uint64_t ail = smem_desc_sw128(st + S::a_im_lo * TILE + off);
          const uint64_t brh = smem_desc_sw128(st + S::b_re_hi * TILE + off);
          const uint64_t brl = smem_desc_sw128(st + S::b_re_lo * TILE + off);
          const uint64_t bih = smem_desc_sw128(st + S::b_im_hi * TILE + off);
          const uint64_t bil = smem_desc_sw128(st + S::b_im_lo * TILE + off);
          if constexpr (OP == QEB_OP_C) {
            // [B; B1] from the B slot: Re columns t_re .. +127, Im t_im .. +127
            mma_tf32(t_re, arh, brh, kIdescReIm, acc);
            mma_tf32(t_re, arh, brl, kIdescReIm, 1u);
            mma_tf32(t_re, arl, brh, kIdescReIm, 1u);
            (void)aih, (void)ail, (void)bih, (void)bil;
          } else {
            mma_tf32(t_re, arh, brh, kIdesc, acc);
            mma_tf32(t_re, arh, brl, kIdesc, 1u);
            mma_tf32(t_re, arl, brh, kIdesc, 1u);
            mma_tf32(t_im, aih, bih, kIdesc, acc);
            mma_tf32(t_im, aih, bil, kIdesc, 1u);
            mma_tf32(t_im, ail, bih, kIdesc, 1u);
          }
        }
        mma_commit(&empty[s]);     // the stage may be reloaded
        mma_commit(&acc_full[b]);  // the accumulator buffer may be drained
      }
      // tensor memory is freed below only after every MMA issued completed
      mma_commit(done);
      if (!mbar_wait(done, 0)) atomicExch(error, 14);
    }
  } else {
    const int ct = threadIdx.x - 64;          // 0 .. WORKER_THREADS - 1
    const int quarter = warp & 3;             // tensor-memory lane window
    const int half = (warp - 2) >> 2;         // column half of Re and Im
    const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16) + half * (BN / 2);
    float acc[BN];                            // Re [0, 64), Im [64, 128) of this row
#pragma unroll
    for (int j = 0; j < BN; ++j) acc[j] = 0.0f;
    bool ok = true;
    for (int i = 0; i < nk && ok; ++i) {
      const int s = i % STAGES;
      if (!__all_sync(0xffffffffu, mbar_wait(&full[s], (i / STAGES) & 1)) || *abort_v) {
        ok = false;
        break;
      }
      unsigned char* st = base + s * S::stage_bytes;
      if (OP == QEB_OP_C) {
        split_tile(st + S::raw_a * TILE, st + S::a_re_lo * TILE, ct, nullptr, nullptr);
        split_tile(st + S::raw_b * TILE, st + S::b_re_lo * TILE, ct, st + S::b_im_hi * TILE,
                   st + S::b_im_lo * TILE);
      } else {
        transpose_a(st + S::raw_a * TILE, st + S::a_re_hi * TILE, st + S::a_re_lo * TILE,
                    st + S::a_im_hi * TILE, st + S::a_im_lo * TILE, ct);
        split_tile(st + S::raw_b * TILE, st + S::b_re_lo * TILE, ct, nullptr, nullptr);
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&conv[s]);
      if (i > 0 && !drain_accumulator(acc, acc_full, acc_empty, i - 1, lane_base, lane)) ok = false;
    }
    if (ok && nk > 0 && !drain_accumulator(acc, acc_full, acc_empty, nk - 1, lane_base, lane))
      ok = false;
    if (!ok && lane == 0) {
      atomicExch(error, 13);
      *abort_v = 1;
    }
    const bool aborted = !__all_sync(0xffffffffu, ok) || *abort_v;
    const int row = m0 + quarter * 32 + lane;
    if (!aborted && row < M) {
      const int cbase = n0 + half * (BN / 2);
      if (split != nullptr) {
        // partial slice of this K range: full M x N slices, or compact
        // BM x BN tiles for a tail launch
        const int64_t cstride = TAIL ? BM : M;
        float2* sbase = TAIL
            ? split + ((int64_t)blockIdx.z * tail_tiles + blockIdx.x) * (BM * BN) + (row - m0) -
                  (int64_t)n0 * BM
            : split + (int64_t)blockIdx.z * M * N + row;
#pragma unroll
        for (int j = 0; j < BN / 2; ++j) {
          const int col = cbase + j;
          if (col < N) sbase[(int64_t)col * cstride] = make_float2(acc[j], acc[BN / 2 + j]);
        }
      } else {
        const bool use_beta = beta.x != 0.0f || beta.y != 0.0f;
        float2* crow = C + row;
        // 8 columns at a time: their C loads are all issued before the
        // first store, so the read-modify-write does not wait on one load
        // per column
#pragma unroll
        for (int j0 = 0; j0 < BN / 2; j0 += 8) {
          float2 old[8];
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int col = cbase + j0 + jj;
            old[jj] = make_float2(0.f, 0.f);
            if (use_beta && col < N) old[jj] = crow[(int64_t)col * ldc];
          }
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int col = cbase + j0 + jj;
            const float re = acc[j0 + jj], im = acc[BN / 2 + j0 + jj];
            const float vx = alpha.x * re - alpha.y * im + beta.x * old[jj].x - beta.y * old[jj].y;
            const float vy = alpha.x * im + alpha.y * re + beta.x * old[jj].y + beta.y * old[jj].x;
            if (col < N) crow[(int64_t)col * ldc] = make_float2(vx, vy);
          }
        }
      }
    }
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
}

// C = alpha * sum_k P_k + beta * C over the split slices, in slice order.
__global__ void reduce_slices(int M, int N, int splits, const float2* __restrict__ P, float2 alpha,
                              float2 beta, float2* C, int64_t ldc) {
  const int64_t total = (int64_t)M * N;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    float2 s = make_float2(0.0f, 0.0f);
    for (int k = 0; k < splits; ++k) {
      const float2 p = P[(int64_t)k * total + i];
      s.x += p.x;
      s.y += p.y;
    }
    const int64_t m = i % M, n = i / M;
    float2* c = C + m + n * ldc;
    float2 v = make_float2(alpha.x * s.x - alpha.y * s.y, alpha.x * s.y + alpha.y * s.x);
    if (beta.x != 0.0f || beta.y != 0.0f) {
      const float2 o = *c;
      v.x += beta.x * o.x - beta.y * o.y;
      v.y += beta.x * o.y + beta.y * o.x;
    }
    *c = v;
  }
}

// C = alpha * sum_s P[s] + beta * C over the ntiles tail tiles (rows m_off ..
// m_off + ntiles - 1 of tile column n_off): compact partial tiles
// P[(s * ntiles + t) * BM * BN + r + c * BM], slices summed in ascending order.
__global__ void reduce_tail(int M, int N, int splits, int m_off, int n_off, int ntiles,
                            const float2* __restrict__ P, float2 alpha, float2 beta, float2* C,
                            int64_t ldc) {
  const int64_t per_tile = (int64_t)BM * BN;
  const int64_t total = (int64_t)ntiles * per_tile;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int lt = (int)(i / per_tile);
    const int64_t e = i - lt * per_tile;
    const int m = (m_off + lt) * BM + (int)(e % BM);
    const int n = n_off * BN + (int)(e / BM);
    if (m >= M || n >= N) continue;
    float2 s = make_float2(0.0f, 0.0f);
    for (int k = 0; k < splits; ++k) {
      const float2 p = P[((int64_t)k * ntiles + lt) * per_tile + e];
      s.x += p.x;
      s.y += p.y;
    }
    float2* c = C + m + (int64_t)n * ldc;
    float2 v = make_float2(alpha.x * s.x - alpha.y * s.y, alpha.x * s.y + alpha.y * s.x);
    if (beta.x != 0.0f || beta.y != 0.0f) {
      const float2 o = *c;
      v.x += beta.x * o.x - beta.y * o.y;
      v.y += beta.x * o.y + beta.y * o.x;
    }
    *c = v;
  }
}

int encode_map(qeb::EncodeTiled enc, CUtensorMap* map, const void* ptr, uint64_t inner,
               uint64_t outer, int64_t ld_bytes, uint32_t box_inner, uint32_t box_outer,
               bool swizzle) {
  const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  const cuuint64_t strides[1] = {(cuuint64_t)ld_bytes};
  const cuuint32_t box[2] = {box_inner, box_outer};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(ptr), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   swizzle ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    qeb::set_error("cgemm_tf32x3: cuTensorMapEncodeTiled failed (%d) for %llu x %llu words",
                   (int)r, (unsigned long long)inner, (unsigned long long)outer);
    return QEB_ECUDA;
  }
  return QEB_OK;
}

int sm_count() {
  static int count = 0;
  if (count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (count <= 0) count = 148;
  }
  return count;
}

// K slices per output tile: as many as fill two whole waves of CTAs (one CTA
// per SM), or one whole wave when two would leave slices shorter than 64
// K tiles; rounding up to one wave instead left a second wave of a few CTAs
// (for 8 tiles, 152 CTAs on 148 SMs), and measured two-wave splits were
// 25-30 % faster on the Davidson overlaps (K = 80 725).
int choose_splits(int M, int N, int K) {
  const int tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  const int kblocks = (2 * K + BKF - 1) / BKF;
  int s = (2 * sm_count()) / tiles;
  if (s > 0 && kblocks / s < 64) s = sm_count() / tiles;
  if (s > kblocks / 4) s = kblocks / 4;  // at least four stages per slice
  if (s > 64) s = 64;
  return s < 1 ? 1 : s;
}

// Split of a partial last wave: an unsplit product of several waves whose
// last wave holds rem <= sm/2 output tiles runs its full waves as usual and
// the rem tail tiles with their K range split over about one wave of CTAs
// (reduced afterwards), instead of leaving most SMs idle for a whole wave.
// Returns the tail's slice count (0: no tail split) and its scratch bytes.
int tail_splits(int M, int N, int K, int64_t* bytes) {
  const int mt = (M + BM - 1) / BM;
  const int tiles = mt * ((N + BN - 1) / BN);
  const int sm = sm_count();
  const int kblocks = (2 * K + BKF - 1) / BKF;
  *bytes = 0;
  if (tiles <= sm) return 0;
  const int rem = tiles % sm;
  if (rem == 0 || rem > sm / 2 || rem > mt) return 0;  // the tail: part of the last tile column
  int ts = sm / rem;
  if (ts > kblocks / 4) ts = kblocks / 4;
  if (ts > 64) ts = 64;
  if (ts < 2) return 0;
  *bytes = (int64_t)ts * rem * BM * BN * (int64_t)sizeof(float2);
  return ts;
}

template <int OP>
int launch(const Maps& maps, int M, int N, int K, float2 al, float2 be, float2* C, int64_t ldc,
           void* scratch, int64_t scratch_bytes, int requested_splits, int* err, cudaStream_t s) {
  cudaError_t e = qeb::raise_smem_limit(cgemm_tf32x3_kernel<OP>, smem_bytes<OP>());
  if (e == cudaSuccess) e = qeb::raise_smem_limit(cgemm_tf32x3_kernel<OP, true>, smem_bytes<OP>());
  if (e != cudaSuccess) return qeb::cuda_status(e, "cgemm_tf32x3 shared-memory limit");
  const int kblocks = (2 * K + BKF - 1) / BKF;
  int splits = requested_splits > 0 ? (requested_splits < kblocks ? requested_splits : kblocks)
                                    : choose_splits(M, N, K);
  if (splits == 1) {
    int64_t tail_bytes = 0;
    int ts = tail_splits(M, N, K, &tail_bytes);
    if (ts > 1 && scratch != nullptr && scratch_bytes >= tail_bytes) {
      const int mt = (M + BM - 1) / BM, nt = (N + BN - 1) / BN;
      const int rem = (mt * nt) % sm_count();
      float2* part = static_cast<float2*>(scratch);
      // every tile but the tail (the last rem rows of the last tile column), unsplit
      cgemm_tf32x3_kernel<OP><<<dim3(mt, nt, 1), THREADS, smem_bytes<OP>(), s>>>(
          maps, M, N, kblocks, kblocks, al, be, C, ldc, nullptr, err, mt - rem, nt - 1, 0, 0, 0);
      const int per_t = (kblocks + ts - 1) / ts;
      ts = (kblocks + per_t - 1) / per_t;
      cgemm_tf32x3_kernel<OP, true><<<dim3(rem, 1, ts), THREADS, smem_bytes<OP>(), s>>>(
          maps, M, N, per_t, kblocks, al, be, C, ldc, part, err, 0, -1, mt - rem, nt - 1, rem);
      int blocks = (int)(((int64_t)rem * BM * BN + 255) / 256);
      if (blocks > 4 * sm_count()) blocks = 4 * sm_count();
      reduce_tail<<<blocks, 256, 0, s>>>(M, N, ts, mt - rem, nt - 1, rem, part, al, be, C, ldc);
      qeb::count_launches(3);
      return qeb::cuda_status(cudaGetLastError(), "cgemm_tf32x3 launch");
    }
  }
  const int64_t slice = (int64_t)M * N * 8;
  if (splits > 1 && (scratch == nullptr || scratch_bytes < splits * slice)) {
    const int64_t fit = scratch == nullptr ? 0 : scratch_bytes / slice;
    splits = fit > 1 ? (int)(fit < splits ? fit : splits) : 1;
  }
  const int per = (kblocks + splits - 1) / splits;
  splits = (kblocks + per - 1) / per;
  float2* part = splits > 1 ? static_cast<float2*>(scratch) : nullptr;
  const dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, splits);
  cgemm_tf32x3_kernel<OP><<<grid, THREADS, smem_bytes<OP>(), s>>>(maps, M, N, per, kblocks, al,
                                                                  be, C, ldc, part, err, 0, -1,
                                                                  0, 0, 0);
  qeb::count_launches(1);
  if (splits > 1) {
    int blocks = (int)(((int64_t)M * N + 255) / 256);
    if (blocks > 4 * sm_count()) blocks = 4 * sm_count();
    reduce_slices<<<blocks, 256, 0, s>>>(M, N, splits, part, al, be, C, ldc);
    qeb::count_launches(1);
  }
  return qeb::cuda_status(cudaGetLastError(), "cgemm_tf32x3 launch");
}

}  // namespace

extern "C" int qeb_cgemm_tf32x3_default_splits(int op_a, int M, int N, int K) {
  (void)op_a;
  if (M <= 0 || N <= 0 || K <= 0) return 1;
  return choose_splits(M, N, K);
}

extern "C" int64_t qeb_cgemm_tf32x3_scratch_bytes(int op_a, int M, int N, int K) {
  (void)op_a;
  if (M <= 0 || N <= 0 || K <= 0) return 0;
  const int s = choose_splits(M, N, K);
  if (s > 1) return (int64_t)s * M * N * 8;
  int64_t tail_bytes = 0;
  tail_splits(M, N, K, &tail_bytes);
  return tail_bytes;
}

extern "C" int qeb_cgemm_tf32x3(int op_a, int M, int N, int K, const double* alpha, const void* A,
                                int64_t lda, const void* B, int64_t ldb, const double* beta,
                                void* C, int64_t ldc, void* scratch, int64_t scratch_bytes,
                                void* stream) {
  return qeb_cgemm_tf32x3_ex(op_a, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, scratch,
                             scratch_bytes, 0, stream);
}

extern "C" int qeb_cgemm_tf32x3_ex(int op_a, int M, int N, int K, const double* alpha,
                                   const void* A, int64_t lda, const void* B, int64_t ldb,
                                   const double* beta, void* C, int64_t ldc, void* scratch,
                                   int64_t scratch_bytes, int splits, void* stream) {
  if ((op_a != QEB_OP_N && op_a != QEB_OP_C) || M < 0 || N < 0 || K < 0 || alpha == nullptr ||
      beta == nullptr || ldc < (M > 0 ? M : 1) || ldb < (K > 0 ? K : 1) ||
      lda < (op_a == QEB_OP_N ? (M > 0 ? M : 1) : (K > 0 ? K : 1))) {
    qeb::set_error("cgemm_tf32x3: invalid arguments (op=%d M=%d N=%d K=%d)", op_a, M, N, K);
    return QEB_EINVAL;
  }
  if (M == 0 || N == 0) return QEB_OK;
  if (K == 0) {
    qeb::set_error("cgemm_tf32x3: K = 0 (scale C by beta instead)");
    return QEB_EUNSUPPORTED;
  }
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) % 16 != 0 || lda % 2 != 0 ||
      ldb % 2 != 0) {
    qeb::set_error("cgemm_tf32x3: A and B need 16-byte aligned columns (even leading dimension)");
    return QEB_EUNSUPPORTED;
  }
  if ((int64_t)2 * K > 0x7fffffff || (int64_t)2 * M > 0x7fffffff || (N + BN - 1) / BN > 65535) {
    qeb::set_error("cgemm_tf32x3: matrix too large for one launch");
    return QEB_EUNSUPPORTED;
  }
  qeb::EncodeTiled enc;
  int rc = qeb::tensor_map_encoder(&enc);
  if (rc) return rc;
  int* err = nullptr;
  if ((rc = qeb::tensor_error_word(&err))) return rc;
  Maps maps;
  if (op_a == QEB_OP_C) {
    rc = encode_map(enc, &maps.a, A, 2 * (uint64_t)K, M, lda * 8, BKF, BM, true);
  } else {
    rc = encode_map(enc, &maps.a, A, 2 * (uint64_t)M, K, lda * 8, 2 * BM, BKF / 2, false);
  }
  if (rc == QEB_OK) rc = encode_map(enc, &maps.b, B, 2 * (uint64_t)K, N, ldb * 8, BKF, BN, true);
  if (rc) return rc;
  const float2 al = make_float2((float)alpha[0], (float)alpha[1]);
  const float2 be = make_float2((float)beta[0], (float)beta[1]);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float2* c = static_cast<float2*>(C);
  return op_a == QEB_OP_C
             ? launch<QEB_OP_C>(maps, M, N, K, al, be, c, ldc, scratch, scratch_bytes, splits, err, s)
             : launch<QEB_OP_N>(maps, M, N, K, al, be, c, ldc, scratch, scratch_bytes, splits, err, s);
}
