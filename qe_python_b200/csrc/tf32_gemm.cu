// Split-TF32 complex GEMM on the 5th-generation tensor cores (tcgen05).
//
//   C = alpha * (A B0^T + i A B1^T) + beta * C        (complex64 C, FP32 accumulate)
//
// A (M x Kp), B0 and B1 (N x Kp) are real FP32 operands, K-major, packed
// from complex matrices with each complex value stored as two consecutive
// reals along K (Kp = 2K, zero padded to a multiple of 32):
//   becp = beta^H psi      : A = beta columns [re, im],  B0 = psi [re, im],
//                            B1 = psi [im, -re]          (Re, Im of conj(a) b)
//   H psi += beta coupled  : A = beta rows [re, im],     B0 = coupled [re, -im],
//                            B1 = coupled [im, re]       (Re, Im of a b)
// Every operand is split into hi = tf32(x) and lo = tf32(x - hi); each real
// product is hi*hi + hi*lo + lo*hi ("split TF32", three tcgen05.mma.kind::tf32
// per product) accumulated in FP32 in tensor memory: Re in TMEM columns
// [0, BN), Im in [BN, 2 BN).
//
// One CTA = 128 threads computes a 128 x 64 tile over a K range:
//   warp 0 lane 0 : TMA producer (cp.async.bulk.tensor, 128B swizzle), 3 stages
//   warp 1 lane 0 : MMA issuer (tcgen05.mma, commit to the stage's empty barrier)
//   warps 0-3     : epilogue, tcgen05.ld of the two accumulators, complex store
// K is split across CTAs (grid.z) into caller scratch when the output tile
// count is small; a reduction kernel sums the slices in a fixed order.
// Every mbarrier wait is bounded: on timeout the CTA records an error code,
// stops issuing, drains what it issued and frees its tensor memory.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "qeb_common.cuh"
#include "tcgen05.cuh"
#include "../../include/qe_b200.h"

using qeb::C2;

namespace {

using namespace qeb::tc;

constexpr int BM = 128, BN = 64, BK = 32;  // BK: fp32 elements = 128 bytes
constexpr int STAGES = 3;
constexpr int A_TILE_BYTES = BM * BK * 4;  // 16 KiB
constexpr int B_TILE_BYTES = BN * BK * 4;  // 8 KiB
constexpr int STAGE_BYTES = 2 * A_TILE_BYTES + 4 * B_TILE_BYTES;  // 64 KiB
constexpr int TMEM_COLS = 2 * BN;  // Re and Im accumulators
constexpr int THREADS = 128;
constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;

// Instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N = BN.
constexpr uint32_t kIdesc = idesc_tf32(BM, BN);

struct Maps {
  CUtensorMap a_hi, a_lo, b0_hi, b0_lo, b1_hi, b1_lo;
};

// split == nullptr: C = alpha*acc + beta*C.  Otherwise write the slice's
// partial (re, im) to split + blockIdx.z * M * N, M-contiguous.
__global__ void __launch_bounds__(THREADS, 1) tf32x3_gemm_kernel(
    const __grid_constant__ Maps maps, int M, int N, int ktiles_per_split, int ktiles_total,
    float2 alpha, float2 beta, float2* C, int64_t ldc, float2* split, int* error) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kt0 = blockIdx.z * ktiles_per_split;
  const int kt1 = min(ktiles_total, kt0 + ktiles_per_split);
  const int nk = max(0, kt1 - kt0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // TMA producer
    for (int i = 0; i < nk; ++i) {
      const int s = i % STAGES;
      if (i >= STAGES && !mbar_wait(&empty[s], ((i / STAGES) - 1) & 1)) {
        atomicExch(error, 1);
        *reinterpret_cast<volatile int*>(abort_flag) = 1;
        break;
      }
      if (*reinterpret_cast<volatile int*>(abort_flag)) break;
      unsigned char* st = base + s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      const int kc = (kt0 + i) * BK;
      tma_load_2d(st, &maps.a_hi, &full[s], kc, m0);
      tma_load_2d(st + A_TILE_BYTES, &maps.a_lo, &full[s], kc, m0);
      unsigned char* bt = st + 2 * A_TILE_BYTES;
      tma_load_2d(bt, &maps.b0_hi, &full[s], kc, n0);
      tma_load_2d(bt + B_TILE_BYTES, &maps.b0_lo, &full[s], kc, n0);
      tma_load_2d(bt + 2 * B_TILE_BYTES, &maps.b1_hi, &full[s], kc, n0);
      tma_load_2d(bt + 3 * B_TILE_BYTES, &maps.b1_lo, &full[s], kc, n0);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t t_re = tmem, t_im = tmem + BN;
    int issued = 0;
    for (int i = 0; i < nk; ++i) {
      const int s = i % STAGES;
      if (!mbar_wait(&full[s], (i / STAGES) & 1)) {
        atomicExch(error, 2);
        *reinterpret_cast<volatile int*>(abort_flag) = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t st = smem_u32(base + s * STAGE_BYTES);
      const uint32_t a_hi = st, a_lo = st + A_TILE_BYTES;
      const uint32_t b0_hi = st + 2 * A_TILE_BYTES, b0_lo = b0_hi + B_TILE_BYTES;
      const uint32_t b1_hi = b0_hi + 2 * B_TILE_BYTES, b1_lo = b0_hi + 3 * B_TILE_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 8; ++kk) {
        const uint32_t off = kk * 32;  // 8 tf32 = 32 bytes along K
        const uint32_t acc = (i > 0 || kk > 0) ? 1u : 0u;
        mma_tf32(t_re, smem_desc_sw128(a_hi + off), smem_desc_sw128(b0_hi + off), kIdesc, acc);
        mma_tf32(t_re, smem_desc_sw128(a_hi + off), smem_desc_sw128(b0_lo + off), kIdesc, 1u);
        mma_tf32(t_re, smem_desc_sw128(a_lo + off), smem_desc_sw128(b0_hi + off), kIdesc, 1u);
        mma_tf32(t_im, smem_desc_sw128(a_hi + off), smem_desc_sw128(b1_hi + off), kIdesc, acc);
        mma_tf32(t_im, smem_desc_sw128(a_hi + off), smem_desc_sw128(b1_lo + off), kIdesc, 1u);
        mma_tf32(t_im, smem_desc_sw128(a_lo + off), smem_desc_sw128(b1_hi + off), kIdesc, 1u);
      }
      mma_commit(&empty[s]);
      ++issued;
    }
    mma_commit(done);  // arrives once every MMA issued above has completed
    (void)issued;
  }
  __syncwarp();
  // Epilogue: all four warps wait for the accumulators.
  const bool ok = mbar_wait(done, 0);
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (!ok) atomicExch(error, 3);
  const bool aborted = !ok || *reinterpret_cast<volatile int*>(abort_flag);
  const int row = m0 + warp * 32 + lane;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  for (int c0 = 0; c0 < BN; c0 += 32) {
    float re[32], im[32];
    if (nk > 0) {
      tmem_ld32(lane_base + c0, re);
      tmem_ld32(lane_base + BN + c0, im);
      tmem_wait_ld();
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) re[j] = im[j] = 0.0f;
    }
    if (aborted || row >= M) continue;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int col = n0 + c0 + j;
      if (col >= N) break;
      if (split != nullptr) {
        split[(int64_t)blockIdx.z * M * N + row + (int64_t)col * M] = make_float2(re[j], im[j]);
      } else {
        float2* c = C + row + (int64_t)col * ldc;
        float2 v = make_float2(alpha.x * re[j] - alpha.y * im[j], alpha.x * im[j] + alpha.y * re[j]);
        if (beta.x != 0.0f || beta.y != 0.0f) {
          const float2 o = *c;
          v.x += beta.x * o.x - beta.y * o.y;
          v.y += beta.x * o.y + beta.y * o.x;
        }
        *c = v;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
}

__global__ void reduce_split(int M, int N, int splits, const float2* __restrict__ P, float2 alpha,
                             float2 beta, float2* C, int64_t ldc) {
  const int64_t total = (int64_t)M * N;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    float2 s = P[i];
    for (int k = 1; k < splits; ++k) {
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

// ---------------------------------------------------------------------------
// Packing: complex source -> K-major hi/lo FP32 planes with interleaved
// (re, im) along K, rows padded to kp (multiple of 32) with zeros.

// layout: QEB_PACK_RAW [re, im]; QEB_PACK_SWAPNEG [im, -re];
// QEB_PACK_NEGIM [re, -im]; QEB_PACK_SWAP [im, re].
// transposed == 0: src column r (K contiguous complex values) -> dst row r.
// transposed == 1: src row r of a column-major rows x K matrix -> dst row r.
template <typename S>
__global__ void pack_kernel(int rows, int K, int kp, const S* __restrict__ src, int64_t ld,
                            int layout, int transposed, float* __restrict__ hi,
                            float* __restrict__ lo, int64_t ldp) {
  const int64_t total = (int64_t)rows * (kp / 2);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r, k;
    if (transposed) {  // consecutive threads walk rows: coalesced source reads
      r = i % rows;
      k = i / rows;
    } else {           // consecutive threads walk K: coalesced both ways
      k = i % (kp / 2);
      r = i / (kp / 2);
    }
    float a = 0.0f, b = 0.0f;
    if (k < K) {
      const S v = transposed ? src[r + k * ld] : src[k + r * ld];
      const float re = (float)v.re, im = (float)v.im;
      if (layout == QEB_PACK_RAW) { a = re; b = im; }
      else if (layout == QEB_PACK_SWAPNEG) { a = im; b = -re; }
      else if (layout == QEB_PACK_NEGIM) { a = re; b = -im; }
      else { a = im; b = re; }
    }
    const float ah = tf32_round(a), bh = tf32_round(b);
    float2* dh = reinterpret_cast<float2*>(hi + r * ldp) + k;
    float2* dl = reinterpret_cast<float2*>(lo + r * ldp) + k;
    *dh = make_float2(ah, bh);
    *dl = make_float2(tf32_round(a - ah), tf32_round(b - bh));
  }
}

// ---------------------------------------------------------------------------
// Host

using qeb::EncodeTiled;

int encode(EncodeTiled enc, CUtensorMap* map, const float* ptr, int rows, int kp, int64_t ldp,
           int box_rows) {
  if (reinterpret_cast<uintptr_t>(ptr) % 16 != 0 || (ldp * 4) % 16 != 0 || kp % BK != 0) {
    qeb::set_error("tf32 gemm: packed operand must be 16-byte aligned with kp %% 32 == 0");
    return QEB_EINVAL;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ldp * 4};
  const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ptr), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    qeb::set_error("cuTensorMapEncodeTiled failed (%d) for a %d x %d operand", (int)r, rows, kp);
    return QEB_ECUDA;
  }
  return QEB_OK;
}

int g_sms = 0;

int sms() {
  if (g_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  return g_sms;
}

int tf32_splits(int M, int N, int kp) {
  const int tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  const int ktiles = kp / BK;
  int s = (sms() + tiles - 1) / tiles;  // about one wave of CTAs
  const int by_depth = ktiles / 8;       // at least 8 K tiles per slice
  if (s > by_depth) s = by_depth;
  if (s > 64) s = 64;
  // at most 32 K tiles per tensor-memory accumulator: its FP32 additions
  // lose accuracy with the chain length (see cgemm_tf32x3.cu)
  const int by_chain = (ktiles + 31) / 32;
  if (s < by_chain) s = by_chain;
  return s < 1 ? 1 : s;
}

}  // namespace

namespace qeb {

namespace {
std::mutex g_encode_mutex;
EncodeTiled g_encode = nullptr;
std::mutex g_err_mutex;
int* g_err[64] = {nullptr};
}  // namespace

int tensor_map_encoder(EncodeTiled* out) {
  std::lock_guard<std::mutex> lock(g_encode_mutex);
  if (g_encode == nullptr) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (err != cudaSuccess || fn == nullptr || q != cudaDriverEntryPointSuccess) {
      set_error("cuTensorMapEncodeTiled is unavailable from the driver");
      return QEB_ECUDA;
    }
    g_encode = reinterpret_cast<EncodeTiled>(fn);
  }
  *out = g_encode;
  return QEB_OK;
}

int tensor_error_word(int** out) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return QEB_EUNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_err_mutex);
  if (g_err[dev] == nullptr) {
    cudaError_t e = cudaMalloc(&g_err[dev], sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(g_err[dev], 0, sizeof(int));
    if (e != cudaSuccess) return cuda_status(e, "tensor-core GEMM error word");
  }
  *out = g_err[dev];
  return QEB_OK;
}

}  // namespace qeb

extern "C" int qeb_tf32_pack(int precision, int layout, int transposed, int rows, int K,
                             const void* src, int64_t ld, void* hi, void* lo, int64_t ldp,
                             void* stream) {
  if (rows < 0 || K < 0 || ldp < 2 * (int64_t)((K + 15) / 16 * 16) ||
      (rows > 0 && K > 0 && (src == nullptr || hi == nullptr || lo == nullptr)) ||
      layout < QEB_PACK_RAW || layout > QEB_PACK_SWAP) {
    qeb::set_error("tf32_pack: invalid arguments");
    return QEB_EINVAL;
  }
  if (rows == 0) return QEB_OK;
  const int kp = (int)((2 * (int64_t)K + BK - 1) / BK * BK);
  if (ldp < kp) {
    qeb::set_error("tf32_pack: packed row stride %lld below %d", (long long)ldp, kp);
    return QEB_EINVAL;
  }
  const int64_t work = (int64_t)rows * (kp / 2);
  if (work == 0) return QEB_OK;  // K = 0: nothing to pack
  int blocks = (int)((work + 255) / 256);
  if (blocks > sms() * 16) blocks = sms() * 16;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == QEB_F64) {
    pack_kernel<C2<double>><<<blocks, 256, 0, s>>>(rows, K, kp, static_cast<const C2<double>*>(src),
                                                   ld, layout, transposed, static_cast<float*>(hi),
                                                   static_cast<float*>(lo), ldp);
  } else {
    pack_kernel<C2<float>><<<blocks, 256, 0, s>>>(rows, K, kp, static_cast<const C2<float>*>(src), ld,
                                                  layout, transposed, static_cast<float*>(hi),
                                                  static_cast<float*>(lo), ldp);
  }
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "tf32_pack");
}

extern "C" int64_t qeb_tf32_gemm_scratch_bytes(int M, int N, int kp) {
  if (M <= 0 || N <= 0 || kp <= 0) return 0;
  const int s = tf32_splits(M, N, kp);
  return s > 1 ? (int64_t)s * M * N * 8 : 0;
}

extern "C" int qeb_tf32_gemm(int M, int N, int kp, const void* a_hi, const void* a_lo,
                             int64_t lda, const void* b0_hi, const void* b0_lo,
                             const void* b1_hi, const void* b1_lo, int64_t ldb,
                             const double* alpha, const double* beta, void* C, int64_t ldc,
                             void* scratch, int64_t scratch_bytes, void* stream) {
  if (M < 0 || N < 0 || kp < 0 || kp % BK != 0 || ldc < M || lda < kp || ldb < kp) {
    qeb::set_error("tf32_gemm: invalid sizes (M=%d N=%d kp=%d)", M, N, kp);
    return QEB_EINVAL;
  }
  if (M == 0 || N == 0) return QEB_OK;
  if (M > 65535 * BM || N > 65535 * BN) {
    qeb::set_error("tf32_gemm: output too large for one launch");
    return QEB_EUNSUPPORTED;
  }
  EncodeTiled enc;
  int rc = qeb::tensor_map_encoder(&enc);
  if (rc) return rc;
  int* err = nullptr;
  if ((rc = qeb::tensor_error_word(&err))) return rc;
  Maps maps;
  if ((rc = encode(enc, &maps.a_hi, (const float*)a_hi, M, kp, lda, BM)) ||
      (rc = encode(enc, &maps.a_lo, (const float*)a_lo, M, kp, lda, BM)) ||
      (rc = encode(enc, &maps.b0_hi, (const float*)b0_hi, N, kp, ldb, BN)) ||
      (rc = encode(enc, &maps.b0_lo, (const float*)b0_lo, N, kp, ldb, BN)) ||
      (rc = encode(enc, &maps.b1_hi, (const float*)b1_hi, N, kp, ldb, BN)) ||
      (rc = encode(enc, &maps.b1_lo, (const float*)b1_lo, N, kp, ldb, BN)))
    return rc;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(tf32x3_gemm_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
    if (e != cudaSuccess) return qeb::cuda_status(e, "tf32 gemm smem attribute");
    configured = true;
  }
  const int ktiles = kp / BK;
  int splits = tf32_splits(M, N, kp);
  const int64_t slice = (int64_t)M * N * 8;
  if (splits > 1 && (scratch == nullptr || scratch_bytes < splits * slice)) {
    const int64_t fit = scratch == nullptr ? 0 : scratch_bytes / slice;
    splits = fit > 1 ? (int)fit : 1;
  }
  const int per = (ktiles + splits - 1) / splits;
  splits = (ktiles + per - 1) / per;
  const float2 al = make_float2((float)alpha[0], (float)alpha[1]);
  const float2 be = make_float2((float)beta[0], (float)beta[1]);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, splits);
  float2* part = splits > 1 ? static_cast<float2*>(scratch) : nullptr;
  tf32x3_gemm_kernel<<<grid, THREADS, SMEM_BYTES, s>>>(maps, M, N, per, ktiles, al, be,
                                                      static_cast<float2*>(C), ldc, part, err);
  qeb::count_launches(1);
  if (splits > 1) {
    int blocks = (int)(((int64_t)M * N + 255) / 256);
    if (blocks > 4 * sms()) blocks = 4 * sms();
    reduce_split<<<blocks, 256, 0, s>>>(M, N, splits, part, al, be, static_cast<float2*>(C), ldc);
    qeb::count_launches(1);
  }
  return qeb::cuda_status(cudaGetLastError(), "tf32_gemm launch");
}

// Reads and clears the device error word of the tensor-core GEMMs' bounded waits
// (0 = no timeout since the last call).  Synchronises the device.
extern "C" int qeb_tf32_gemm_error(int* out) {
  int* err = nullptr;
  int rc = qeb::tensor_error_word(&err);
  if (rc) return rc;
  int value = 0;
  cudaError_t e = cudaMemcpy(&value, err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && value != 0) e = cudaMemset(err, 0, sizeof(int));
  if (e != cudaSuccess) return qeb::cuda_status(e, "tf32 gemm error word read");
  *out = value;
  return QEB_OK;
}
