// Four-step register FFT versions of the local H|psi> passes (sm_100a).
//
// Same operator and HBM layout as the generic kernels of local_hpsi.cu
// (qepy_pw/_native_fft.pyx qepy_apply_serial_spatial :58-135), with every
// line transform done by one warp-resident line group (fft4.cuh): the index
// arithmetic is compile time, each line needs one shared-memory exchange and
// only warp-level synchronisation, and block-wide barriers separate the
// stages (scatter, row transforms, column transforms, gather).
//   pass A : z transforms of the occupied sticks          (grid: sticks/32 x bands)
//   pass B : per (z, band) plane: inverse x transforms of the active rows,
//            per column inverse y transform . V . forward y transform (in
//            registers), forward x transforms, gather the sticks
//   pass C : forward z transforms, gather, 1/N and the kinetic term
// Used when the line length has a listed factorisation n = N1 * N2 (pass B:
// nx == ny); other grids take the generic Stockham kernels.
#include <atomic>
#include <mutex>

#include "fft4.cuh"
#include "local_plan.cuh"
#include "../../include/qe_b200.h"

using qeb::C2;

namespace qeb {
// The device word of bounded waits that gave up (tf32_gemm.cu).
int tensor_error_word(int** out);
}  // namespace qeb

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSticksPerBlock = 32;

// n, N1, N2 of every four-step variant (index = position in this list).
#define QEB_FOUR_SIZES(X) \
  X(16, 4, 4)             \
  X(24, 4, 6)             \
  X(32, 4, 8)             \
  X(36, 6, 6)             \
  X(48, 6, 8)             \
  X(64, 8, 8)             \
  X(72, 8, 9)             \
  X(90, 9, 10)            \
  X(96, 8, 12)            \
  X(108, 9, 12)           \
  X(128, 8, 16)           \
  X(135, 9, 15)           \
  X(144, 12, 12)          \
  X(180, 12, 15)

constexpr int kFourLengths[] = {
#define QEB_LEN(n, a, b) n,
    QEB_FOUR_SIZES(QEB_LEN)
#undef QEB_LEN
};
constexpr int kFourCount = sizeof(kFourLengths) / sizeof(int);

template <class F>
struct GroupIds {
  int lig, gid, ngroups;
  unsigned mask;
  bool valid;
  __device__ GroupIds() {
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int gw = lane / F::G;
    lig = lane - gw * F::G;
    valid = gw < F::per_warp;
    gid = warp * F::per_warp + gw;
    ngroups = kWarps * F::per_warp;
    mask = (F::G == 32 ? 0xffffffffu : ((1u << F::G) - 1u)) << (gw * F::G);
  }
};

// Line stride of the z passes.  Each line doubles as its own four-step
// exchange buffer (its values are in registers by then), so it holds
// F::scratch values; the stride is odd so that the transposed copies between
// the lines and the stick buffer hit distinct banks.  Without a separate
// exchange buffer a block needs about half the shared memory, and eight
// blocks fit on an SM instead of six.
template <class F>
constexpr int line_stride() {
  return (F::scratch > F::n ? F::scratch : F::n) | 1;
}

// Line rounds of the z passes.  When the line groups fill the warp, the
// groups of a warp take lines lead + gw (lead = the warp's first group id)
// in rounds that every lane runs, and synchronise with the full mask (no
// run-time membership check).  A round's line then stays below
// kSticksPerBlock: the round starts at a multiple of per_warp below nsl <=
// kSticksPerBlock, and per_warp divides 32.  Otherwise each group runs its
// own rounds over lines gid, gid + ngroups, ...
template <class F>
struct ZRounds {
  static constexpr bool kFull = F::G * F::per_warp == 32;
  static_assert(!kFull || kSticksPerBlock % F::per_warp == 0, "rounds stay inside the block");
  // every lane of a group holds a value of the N1 (N2) role; resolved at
  // compile time only with full-warp rounds (with partial warps, ptxas 12.9
  // failed register allocation on the compile-time form)
  static constexpr bool kWhole1 = kFull && F::N1 == F::G;
  static constexpr bool kWhole2 = kFull && F::N2 == F::G;
  int start, offset;
  unsigned mask;
  __device__ explicit ZRounds(const GroupIds<F>& g) {
    const int gw = g.gid % F::per_warp;
    start = kFull ? g.gid - gw : g.gid;
    offset = kFull ? gw : 0;
    mask = kFull ? 0xffffffffu : g.mask;
  }
};

template <typename T, class F>
constexpr size_t ac_smem() {
  return sizeof(C2<T>) * ((size_t)kSticksPerBlock * line_stride<F>() + F::n);
}

template <typename T, class F>
size_t b_smem(const qeb_local_plan* p) {
  return sizeof(C2<T>) * ((size_t)p->nay * p->nx_pad + F::n +
                          (size_t)kWarps * F::per_warp * F::scratch) +
         sizeof(int) * F::n;
}

// ---------------------------------------------------------------------------
template <typename T, class F>
__device__ __forceinline__ void pass_a_body(
    const C2<T>* __restrict__ psi, int64_t ld, int nst,
    const int32_t* __restrict__ entry_g, const int32_t* __restrict__ entry_z,
    const int32_t* __restrict__ entry_stick, const int32_t* __restrict__ stick_off,
    const C2<T>* __restrict__ tw_z, C2<T>* __restrict__ sticks, uint32_t zmask, int block_x,
    int64_t band) {
  constexpr int nz = F::n;
  constexpr int nz_pad = line_stride<F>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* lines = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* tw = lines + kSticksPerBlock * nz_pad;
  const int s0 = block_x * kSticksPerBlock;
  const int nsl = min(kSticksPerBlock, nst - s0);
  for (int i = threadIdx.x; i < nz; i += kThreads) tw[i] = tw_z[i];
  for (int i = threadIdx.x; i < kSticksPerBlock * nz_pad; i += kThreads) lines[i] = qeb::mk<T>(0, 0);
  __syncthreads();
  const int e0 = stick_off[s0], e1 = stick_off[s0 + nsl];
  const C2<T>* col = psi + band * ld;
  for (int e = e0 + threadIdx.x; e < e1; e += kThreads)
    lines[(entry_stick[e] - s0) * nz_pad + entry_z[e]] = col[entry_g[e]];
  __syncthreads();
  const GroupIds<F> g;
  const ZRounds<F> zr(g);
  if (g.valid) {
    for (int base = zr.start; base < nsl; base += g.ngroups) {
      // a line past nsl (full-warp rounds only) is a zeroed line of the block
      C2<T>* line = lines + (base + zr.offset) * nz_pad;
      C2<T> v[F::R];
      if (ZRounds<F>::kWhole2 || g.lig < F::N2) {
        // blocks of z that hold no entry are zero: no load
#pragma unroll
        for (int i = 0; i < F::N1; ++i)
          v[i] = ((zmask >> i) & 1u) ? line[g.lig + F::N2 * i] : qeb::mk<T>(0, 0);
      }
      __syncwarp(zr.mask);  // the line becomes the exchange buffer
      qeb::four_inverse<T, F>(v, g.lig, line, tw, zr.mask);
      if (ZRounds<F>::kWhole1 || g.lig < F::N1) {
#pragma unroll
        for (int p = 0; p < F::N2; ++p) line[g.lig + F::N1 * p] = v[p];
      }
      __syncwarp(zr.mask);
    }
  }
  __syncthreads();
  C2<T>* out = sticks + band * (int64_t)nz * nst;
  for (int i = threadIdx.x; i < nz * nsl; i += kThreads) {
    const int z = i / nsl, sl = i - z * nsl;
    out[(int64_t)z * nst + s0 + sl] = lines[sl * nz_pad + z];
  }
}

template <typename T, class F>
__device__ __forceinline__ void pass_c_body(
    const C2<T>* __restrict__ sticks, int nst, const int32_t* __restrict__ entry_g,
    const int32_t* __restrict__ entry_z, const int32_t* __restrict__ entry_stick,
    const int32_t* __restrict__ stick_off, const C2<T>* __restrict__ tw_z,
    const C2<T>* __restrict__ psi, int64_t ld, const T* __restrict__ kinetic, T inv_n,
    C2<T>* __restrict__ out, int64_t ldo, uint32_t zmask, int block_x, int64_t band) {
  constexpr int nz = F::n;
  constexpr int nz_pad = line_stride<F>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* lines = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* tw = lines + kSticksPerBlock * nz_pad;
  const int s0 = block_x * kSticksPerBlock;
  const int nsl = min(kSticksPerBlock, nst - s0);
  for (int i = threadIdx.x; i < nz; i += kThreads) tw[i] = tw_z[i];
  const C2<T>* in = sticks + band * (int64_t)nz * nst;
  for (int i = threadIdx.x; i < nz * nsl; i += kThreads) {
    const int z = i / nsl, sl = i - z * nsl;
    lines[sl * nz_pad + z] = in[(int64_t)z * nst + s0 + sl];
  }
  __syncthreads();
  const GroupIds<F> g;
  const ZRounds<F> zr(g);
  if (g.valid) {
    for (int base = zr.start; base < nsl; base += g.ngroups) {
      // a line past nsl (full-warp rounds only) is a line of the block that
      // nothing gathers from
      C2<T>* line = lines + (base + zr.offset) * nz_pad;
      C2<T> v[F::R];
      if (ZRounds<F>::kWhole1 || g.lig < F::N1) {
#pragma unroll
        for (int p = 0; p < F::N2; ++p) v[p] = line[g.lig + F::N1 * p];
      }
      __syncwarp(zr.mask);  // the line becomes the exchange buffer
      qeb::four_forward<T, F>(v, g.lig, line, tw, zr.mask);
      if (ZRounds<F>::kWhole2 || g.lig < F::N2) {
        // only the z of entries are gathered below
#pragma unroll
        for (int i = 0; i < F::N1; ++i)
          if ((zmask >> i) & 1u) line[g.lig + F::N2 * i] = v[i];
      }
      __syncwarp(zr.mask);
    }
  }
  __syncthreads();
  const int e0 = stick_off[s0], e1 = stick_off[s0 + nsl];
  const C2<T>* colp = psi + band * ld;
  C2<T>* dst = out + band * ldo;
  for (int e = e0 + threadIdx.x; e < e1; e += kThreads) {
    const int gidx = entry_g[e];
    C2<T> v = qeb::scale(lines[(entry_stick[e] - s0) * nz_pad + entry_z[e]], inv_n);
    if (kinetic != nullptr) {
      const T t = kinetic[gidx];
      const C2<T> pv = colp[gidx];
      v.re += t * pv.re;
      v.im += t * pv.im;
    }
    dst[gidx] = v;
  }
}

// Spacing, in lines, between the rows (or columns) that the line groups of
// one warp transform at the same time in pass B.  Consecutive rows of the
// plane start 2 (FP32) or 4 (FP64) banks apart (row stride nx_pad odd).
// Shared memory serves 8-byte accesses half a warp at a time (16-byte ones
// a quarter), so for 64-point FP32 lines the two line groups of one half
// warp, reading rows r and r + 1, hit the same banks: every row read, row
// write and column read took twice the minimum of wavefronts.  With the
// groups of a warp 8 rows apart (16 banks) they hit disjoint banks.  s comes
// from a count of the wavefronts of those accesses for every four-step
// length, per half (quarter) warp; s divides the 8 warps of a block.
template <typename T, class F>
constexpr int plane_spread() {
  constexpr int n = F::n;
  if (sizeof(T) == 4)
    return (n == 32 || n == 48 || n == 64 || n == 96) ? 8
           : (n == 16 || n == 24 || n == 90)            ? 4
           : (n == 108 || n == 135)                     ? 2
                                                        : 1;
  return (n == 16 || n == 24 || n == 96 || n == 108 || n == 144) ? 4 : 1;
}

// Blocks per SM that the plane pass keeps resident (its launch bound): the
// register-limited count of the unconstrained build of each variant, so the
// bound caps registers at the same occupancy, raised where a tighter cap
// measured faster on B200 (FP32 135-point lines: 3 blocks instead of 2,
// 3.79 -> 3.46 ms for 256 bands; FP64 64-point lines: 3 instead of 2).  A
// bound below the natural count spilled (FP32 64-point lines at 5 blocks).
template <typename T, class F>
constexpr int b_min_blocks() {
  constexpr int n = F::n;
  if (sizeof(T) == 4)
    return n <= 16 ? 8 : (n == 24 || n == 36) ? 6 : n <= 90 ? 4 : n == 128 ? 2 : 3;
  return n <= 16 ? 4 : n == 24 ? 3 : n == 36 ? 4 : n == 64 ? 3 : n <= 96 ? 2 : 1;
}

// MODE 0: local potential; MODE 1: density accumulation.
template <typename T, class F, int MODE>
__device__ __forceinline__ void pass_b_body(
    C2<T>* __restrict__ sticks, int nst, int nz, int nay, int nx_pad,
    const int32_t* __restrict__ stick_pos, const int32_t* __restrict__ y_to_ay,
    const C2<T>* __restrict__ tw_xy, const T* __restrict__ potential,
    const double* __restrict__ weights, double* __restrict__ density, int z, int64_t band) {
  constexpr int n = F::n;  // nx == ny
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* plane = reinterpret_cast<C2<T>*>(smem_raw);  // [nay][nx_pad]
  C2<T>* tw = plane + (size_t)nay * nx_pad;
  C2<T>* xbuf = tw + n;
  int* yay = reinterpret_cast<int*>(xbuf + kWarps * F::per_warp * F::scratch);
  for (int i = threadIdx.x; i < n; i += kThreads) {
    tw[i] = tw_xy[i];
    yay[i] = y_to_ay[i];
  }
  for (int i = threadIdx.x; i < nay * nx_pad; i += kThreads) plane[i] = qeb::mk<T>(0, 0);
  __syncthreads();
  C2<T>* srow = sticks + (band * nz + z) * (int64_t)nst;
  for (int s = threadIdx.x; s < nst; s += kThreads) plane[stick_pos[s]] = srow[s];
  __syncthreads();
  const GroupIds<F> g;
  C2<T>* x = xbuf + g.gid * F::scratch;
  qeb::LaneTwiddles<T, F> lw;
  lw.load(g.lig, tw);
  // the first row / column of this group: a permutation of the group ids
  // that puts the groups of one warp plane_spread lines apart
  constexpr int spread = plane_spread<T, F>();
  static_assert(kWarps % spread == 0, "the spread must divide the warps of a block");
  const int warp = threadIdx.x / 32;
  const int gw = g.gid - warp * F::per_warp;  // the group's index within its warp
  const int lead = (warp / spread) * (spread * F::per_warp) + warp % spread;
  const int first = lead + gw * spread;
  // When the line groups fill the warp, every lane runs the same number of
  // line rounds (a group past the end transforms but loads and stores
  // nothing) and the warp synchronises with the full mask, which needs no
  // run-time membership check; otherwise each group runs its own rounds.
  constexpr bool kFull = F::G * F::per_warp == 32;
  const unsigned mask = kFull ? 0xffffffffu : g.mask;
  const int start = kFull ? lead : first;
  // inverse transforms along x of the active rows (D1 in, D2 out, in place)
  if (kFull || g.valid) {
    for (int base = start; base < nay; base += g.ngroups) {
      const int r = kFull ? base + gw * spread : base;
      const bool on = !kFull || r < nay;  // per-group rounds stop at nay
      C2<T>* row = plane + r * nx_pad;
      C2<T> v[F::R];
      if (F::N2 == F::G || g.lig < F::N2) {
#pragma unroll
        for (int i = 0; i < F::N1; ++i) v[i] = on ? row[g.lig + F::N2 * i] : qeb::mk<T>(0, 0);
      }
      qeb::four_inverse<T, F>(v, g.lig, x, lw, mask);
      if (on && (F::N1 == F::G || g.lig < F::N1)) {
#pragma unroll
        for (int p = 0; p < F::N2; ++p) row[g.lig + F::N1 * p] = v[p];
      }
      __syncwarp(mask);
    }
  }
  __syncthreads();
  // columns: inverse y transform, V (or |psi|^2), forward y transform
  double w = 0.0;
  if (MODE == 1) w = weights[band];
  if (kFull || g.valid) {
    for (int base = start; base < n; base += g.ngroups) {
      const int col = kFull ? base + gw * spread : base;
      const bool on = !kFull || col < n;
      C2<T> v[F::R];
      if (F::N2 == F::G || g.lig < F::N2) {
#pragma unroll
        for (int i = 0; i < F::N1; ++i) {
          const int ay = yay[g.lig + F::N2 * i];
          v[i] = (on && ay >= 0) ? plane[ay * nx_pad + col] : qeb::mk<T>(0, 0);
        }
      }
      qeb::four_inverse<T, F>(v, g.lig, x, lw, mask);
      if (MODE == 0) {
        if (on && (F::N1 == F::G || g.lig < F::N1)) {
          const T* vcol = potential + ((int64_t)z * n + col) * n;
#pragma unroll
          for (int p = 0; p < F::N2; ++p) v[p] = qeb::scale(v[p], __ldg(vcol + g.lig + F::N1 * p));
        }
        qeb::four_forward<T, F>(v, g.lig, x, lw, mask);
        if (on && (F::N2 == F::G || g.lig < F::N2)) {
#pragma unroll
          for (int i = 0; i < F::N1; ++i) {
            const int ay = yay[g.lig + F::N2 * i];
            if (ay >= 0) plane[ay * nx_pad + col] = v[i];
          }
        }
      } else {
        if (on && (F::N1 == F::G || g.lig < F::N1)) {
#pragma unroll
          for (int p = 0; p < F::N2; ++p) {
            const int y = g.lig + F::N1 * p;
            const double m = (double)v[p].re * v[p].re + (double)v[p].im * v[p].im;
            atomicAdd(density + ((int64_t)col * n + y) * nz + z, w * m);
          }
        }
      }
      __syncwarp(mask);
    }
  }
  if (MODE == 1) return;
  __syncthreads();
  // forward transforms along x of the active rows (D2 in, D1 out, in place)
  if (kFull || g.valid) {
    for (int base = start; base < nay; base += g.ngroups) {
      const int r = kFull ? base + gw * spread : base;
      const bool on = !kFull || r < nay;  // per-group rounds stop at nay
      C2<T>* row = plane + r * nx_pad;
      C2<T> v[F::R];
      if (F::N1 == F::G || g.lig < F::N1) {
#pragma unroll
        for (int p = 0; p < F::N2; ++p) v[p] = on ? row[g.lig + F::N1 * p] : qeb::mk<T>(0, 0);
      }
      qeb::four_forward<T, F>(v, g.lig, x, lw, mask);
      if (on && (F::N2 == F::G || g.lig < F::N2)) {
#pragma unroll
        for (int i = 0; i < F::N1; ++i) row[g.lig + F::N2 * i] = v[i];
      }
      __syncwarp(mask);
    }
  }
  __syncthreads();
  for (int s = threadIdx.x; s < nst; s += kThreads) srow[s] = plane[stick_pos[s]];
}

// The pruned plane pass (MODE 0 only): the plane holds the 2 K N2 slots of
// the rows y in [0, K N2) and [n - K N2, n), and with every stick inside
// them, the D1 blocks K <= i < N1 - K of a line (x or y = j + N2 i) are zero
// on input to the inverse transforms and unread after the forward ones.  So
// the first DFT of an inverse transform neither loads nor adds them, the
// last DFT of a forward transform does not store them, and a column's
// values sit at compile-time offsets from its lane's first slot (no row
// table).  Each step adds or multiplies the same values as pass_b_body, so
// the output is the same bit for bit.
template <class F>
constexpr bool prunable() {
  return F::N1 == 8 && F::N2 == 8;
}
constexpr int kPruneK = 2;
// Bands of one z plane per block of the pruned pass: the table and register
// twiddles are loaded once for them (measured on the 64^3 microbenchmark,
// 256 bands: one band 0.225 ms, two 0.212 ms, four 0.213 ms).
constexpr int kPrunedBands = 2;

template <typename T, class F, int K>
size_t b_pruned_smem(const qeb_local_plan* p) {
  return sizeof(C2<T>) *
         ((size_t)2 * K * F::N2 * p->nx_pad + F::n + (size_t)kWarps * F::per_warp * F::scratch);
}

template <typename T, class F, int K>
__device__ __forceinline__ void pass_b_pruned_body(
    C2<T>* __restrict__ sticks, int nst, int nz, int nay, int nx_pad,
    const int32_t* __restrict__ slot_pos, const int32_t* __restrict__ ay_to_slot,
    const C2<T>* __restrict__ tw_xy, const T* __restrict__ potential, int z, int64_t band0,
    int bands) {
  constexpr int n = F::n, N1 = F::N1, N2 = F::N2;
  constexpr int half = K * N2, slots = 2 * half, gap = n - slots;
  static_assert(F::G * F::per_warp == 32 && 2 * K < N1, "pruned plane: full-warp groups");
  // D1 blocks that are zero on input and unread on output
  constexpr unsigned kZero = ((1u << (N1 - K)) - 1u) & ~((1u << K) - 1u);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* plane = reinterpret_cast<C2<T>*>(smem_raw);  // [slots][nx_pad]
  C2<T>* tw = plane + slots * nx_pad;
  C2<T>* xbuf = tw + n;
  for (int i = threadIdx.x; i < n; i += kThreads) tw[i] = tw_xy[i];
  __syncthreads();
  const GroupIds<F> g;
  C2<T>* x = xbuf + g.gid * F::scratch;
  qeb::LaneTwiddles<T, F> lw;  // loaded once for the block's bands
  lw.load(g.lig, tw);
  constexpr int spread = plane_spread<T, F>();
  const int warp = threadIdx.x / 32;
  const int gw = g.gid - warp * F::per_warp;
  const int lead = (warp / spread) * (spread * F::per_warp) + warp % spread;
  constexpr unsigned mask = 0xffffffffu;
  // slot offset of D1 block i (y = j + N2 i) from the lane's slot j
  auto slot_off = [](int i) { return N2 * i - (i < K ? 0 : gap); };
  for (int b = 0; b < bands; ++b) {
    const int64_t band = band0 + b;
    if (b > 0) __syncthreads();  // the previous band's gather has read the plane
    // zero the kept columns of every slot: the inverse row transforms read
    // only those, and write every column of every slot
    for (int i = threadIdx.x; i < slots * slots; i += kThreads) {
      const int r = i / slots, c = i - r * slots;
      plane[r * nx_pad + (c < half ? c : c + gap)] = qeb::mk<T>(0, 0);
    }
    __syncthreads();
    C2<T>* srow = sticks + (band * nz + z) * (int64_t)nst;
    for (int s = threadIdx.x; s < nst; s += kThreads) plane[slot_pos[s]] = srow[s];
    __syncthreads();
    // inverse transforms along x of every slot (a slot without sticks
    // transforms zeros: its row becomes zero in every column)
    for (int base = lead; base < slots; base += g.ngroups) {
      const int r = base + gw * spread;
      const bool on = r < slots;
      C2<T>* row = plane + (on ? r : 0) * nx_pad;
      C2<T> v[F::R];
#pragma unroll
      for (int i = 0; i < N1; ++i)
        if (!((kZero >> i) & 1u)) v[i] = on ? row[g.lig + N2 * i] : qeb::mk<T>(0, 0);
      qeb::four_inverse<T, F, kZero>(v, g.lig, x, lw, mask);
      if (on) {
#pragma unroll
        for (int p = 0; p < N2; ++p) row[g.lig + N1 * p] = v[p];
      }
      __syncwarp(mask);
    }
    __syncthreads();
    // columns: inverse y transform, V, forward y transform
    for (int base = lead; base < n; base += g.ngroups) {
      const int col = base + gw * spread;
      const bool on = col < n;
      C2<T>* c0 = plane + g.lig * nx_pad + (on ? col : 0);
      C2<T> v[F::R];
#pragma unroll
      for (int i = 0; i < N1; ++i)
        if (!((kZero >> i) & 1u)) v[i] = on ? c0[slot_off(i) * nx_pad] : qeb::mk<T>(0, 0);
      qeb::four_inverse<T, F, kZero>(v, g.lig, x, lw, mask);
      if (on) {
        const T* vcol = potential + ((int64_t)z * n + col) * n;
#pragma unroll
        for (int p = 0; p < N2; ++p) v[p] = qeb::scale(v[p], __ldg(vcol + g.lig + N1 * p));
      }
      qeb::four_forward<T, F>(v, g.lig, x, lw, mask);
      if (on) {
#pragma unroll
        for (int i = 0; i < N1; ++i)
          if (!((kZero >> i) & 1u)) c0[slot_off(i) * nx_pad] = v[i];
      }
      __syncwarp(mask);
    }
    __syncthreads();
    // forward transforms along x of the active rows
    for (int base = lead; base < nay; base += g.ngroups) {
      const int r = base + gw * spread;
      const bool on = r < nay;
      C2<T>* row = plane + (on ? __ldg(ay_to_slot + r) : 0) * nx_pad;
      C2<T> v[F::R];
#pragma unroll
      for (int p = 0; p < N2; ++p) v[p] = on ? row[g.lig + N1 * p] : qeb::mk<T>(0, 0);
      qeb::four_forward<T, F>(v, g.lig, x, lw, mask);
      if (on) {
#pragma unroll
        for (int i = 0; i < N1; ++i)
          if (!((kZero >> i) & 1u)) row[g.lig + N2 * i] = v[i];
      }
      __syncwarp(mask);
    }
    __syncthreads();
    for (int s = threadIdx.x; s < nst; s += kThreads) srow[s] = plane[slot_pos[s]];
  }
}

// ---------------------------------------------------------------------------
// Launch wrappers: one plan (grid.x, grid.y = blocks, bands) or a batch of
// k points on the same grid (grid.z = k; blocks past a k point's sticks or
// bands return at once).

template <typename T, class F>
__global__ void __launch_bounds__(kThreads) four_pass_a(
    const C2<T>* __restrict__ psi, int64_t ld, int nst,
    const int32_t* __restrict__ entry_g, const int32_t* __restrict__ entry_z,
    const int32_t* __restrict__ entry_stick, const int32_t* __restrict__ stick_off,
    const C2<T>* __restrict__ tw_z, C2<T>* __restrict__ sticks, uint32_t zmask) {
  pass_a_body<T, F>(psi, ld, nst, entry_g, entry_z, entry_stick, stick_off, tw_z, sticks, zmask,
                    blockIdx.x, blockIdx.y);
}

template <typename T, class F>
__global__ void __launch_bounds__(kThreads) four_pass_c(
    const C2<T>* __restrict__ sticks, int nst, const int32_t* __restrict__ entry_g,
    const int32_t* __restrict__ entry_z, const int32_t* __restrict__ entry_stick,
    const int32_t* __restrict__ stick_off, const C2<T>* __restrict__ tw_z,
    const C2<T>* __restrict__ psi, int64_t ld, const T* __restrict__ kinetic, T inv_n,
    C2<T>* __restrict__ out, int64_t ldo, uint32_t zmask) {
  pass_c_body<T, F>(sticks, nst, entry_g, entry_z, entry_stick, stick_off, tw_z, psi, ld,
                    kinetic, inv_n, out, ldo, zmask, blockIdx.x, blockIdx.y);
}

template <typename T, class F, int MODE>
__global__ void __launch_bounds__(kThreads, (b_min_blocks<T, F>())) four_pass_b(
    C2<T>* __restrict__ sticks, int nst, int nz, int nay, int nx_pad,
    const int32_t* __restrict__ stick_pos, const int32_t* __restrict__ y_to_ay,
    const C2<T>* __restrict__ tw_xy, const T* __restrict__ potential,
    const double* __restrict__ weights, double* __restrict__ density) {
  pass_b_body<T, F, MODE>(sticks, nst, nz, nay, nx_pad, stick_pos, y_to_ay, tw_xy, potential,
                          weights, density, blockIdx.x, blockIdx.y);
}

template <typename T>
struct KDesc {
  const C2<T>* psi;
  C2<T>* out;
  const T* kinetic;
  C2<T>* sticks;
  const int32_t* entry_g;
  const int32_t* entry_z;
  const int32_t* entry_stick;
  const int32_t* stick_off;
  const int32_t* stick_pos;
  const int32_t* y_to_ay;
  const int32_t* slot_pos;
  const int32_t* ay_to_slot;
  int64_t ld, ldo;
  int nst, nay, nb;
  uint32_t zmask;
};

template <typename T>
struct KBatch {
  KDesc<T> k[QEB_MAX_KBATCH];
};

template <typename T, class F>
__global__ void __launch_bounds__(kThreads) four_pass_a_multi(const __grid_constant__ KBatch<T> kb,
                                                              const C2<T>* tw_z) {
  const KDesc<T>& d = kb.k[blockIdx.z];
  if ((int)blockIdx.x * kSticksPerBlock >= d.nst || (int)blockIdx.y >= d.nb) return;
  pass_a_body<T, F>(d.psi, d.ld, d.nst, d.entry_g, d.entry_z, d.entry_stick, d.stick_off,
                    tw_z, d.sticks, d.zmask, blockIdx.x, blockIdx.y);
}

template <typename T, class F>
__global__ void __launch_bounds__(kThreads, (b_min_blocks<T, F>())) four_pass_b_multi(const __grid_constant__ KBatch<T> kb,
                                                              int nz, int nx_pad,
                                                              const C2<T>* tw_xy,
                                                              const T* potential) {
  const KDesc<T>& d = kb.k[blockIdx.z];
  if ((int)blockIdx.y >= d.nb) return;
  pass_b_body<T, F, 0>(d.sticks, d.nst, nz, d.nay, nx_pad, d.stick_pos, d.y_to_ay, tw_xy,
                       potential, nullptr, nullptr, blockIdx.x, blockIdx.y);
}

template <typename T, class F, int K>
__global__ void __launch_bounds__(kThreads, (b_min_blocks<T, F>())) four_pass_b_pruned_multi(
    const __grid_constant__ KBatch<T> kb, int nz, int nx_pad, const C2<T>* tw_xy,
    const T* potential) {
  const KDesc<T>& d = kb.k[blockIdx.z];
  const int band0 = kPrunedBands * (int)blockIdx.y;
  if (band0 >= d.nb) return;
  pass_b_pruned_body<T, F, K>(d.sticks, d.nst, nz, d.nay, nx_pad, d.slot_pos, d.ay_to_slot,
                              tw_xy, potential, blockIdx.x, band0,
                              min(kPrunedBands, d.nb - band0));
}

template <typename T, class F>
__global__ void __launch_bounds__(kThreads) four_pass_c_multi(const __grid_constant__ KBatch<T> kb,
                                                              const C2<T>* tw_z, T inv_n) {
  const KDesc<T>& d = kb.k[blockIdx.z];
  if ((int)blockIdx.x * kSticksPerBlock >= d.nst || (int)blockIdx.y >= d.nb) return;
  pass_c_body<T, F>(d.sticks, d.nst, d.entry_g, d.entry_z, d.entry_stick, d.stick_off,
                    tw_z, d.psi, d.ld, d.kinetic, inv_n, d.out, d.ldo, d.zmask, blockIdx.x,
                    blockIdx.y);
}

// ---------------------------------------------------------------------------
// Persistent form: the three passes of every k point in one cooperative
// launch of as many blocks as fit on the GPU at once; each block takes work
// items (a stick block or a z plane of one band of one k point) in turn, and
// a grid barrier separates the passes.  Same bodies, same arithmetic as the
// three launches.

constexpr long long kBarrierLimit = 1ll << 24;  // polls before a barrier gives up

// Grid barrier over `nblocks` co-resident blocks on two words of global
// memory (arrival count, generation), bounded: false when the wait gave up,
// which the caller records.  The last block to arrive resets the count and
// advances the generation; the others wait for the generation to change.
__device__ __forceinline__ bool grid_barrier(unsigned int* words, unsigned int nblocks) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned int* generation = words + 1;
    const unsigned int g = *generation;
    __threadfence();  // this block's writes before its arrival
    if (atomicAdd(words, 1u) == nblocks - 1) {
      words[0] = 0u;
      __threadfence();
      atomicAdd(words + 1, 1u);
    } else {
      long long polls = 0;
      while (*generation == g) {
        if (++polls > kBarrierLimit) {
          ok = 0;
          break;
        }
      }
    }
    __threadfence();  // the other blocks' writes before this block reads
  }
  __syncthreads();
  return ok != 0;
}

template <typename T, class F>
__global__ void __launch_bounds__(kThreads) four_passes_persistent(
    const __grid_constant__ KBatch<T> kb, int nk, int sblocks, int max_nb, int nx_pad,
    const C2<T>* tw_z, const C2<T>* tw_xy, const T* potential, T inv_n, unsigned int* barrier,
    int* error) {
  constexpr int nz = F::n;  // cubic grids only: one four-step type for z and the planes
  const int64_t per_k_ac = (int64_t)max_nb * sblocks;
  const int64_t items_ac = (int64_t)nk * per_k_ac;
  for (int64_t it = blockIdx.x; it < items_ac; it += gridDim.x) {
    const int k = (int)(it / per_k_ac);
    const int64_t r = it - k * per_k_ac;
    const int band = (int)(r / sblocks), bx = (int)(r - (int64_t)band * sblocks);
    const KDesc<T>& d = kb.k[k];
    if (bx * kSticksPerBlock >= d.nst || band >= d.nb) continue;
    __syncthreads();  // shared memory of the previous item
    pass_a_body<T, F>(d.psi, d.ld, d.nst, d.entry_g, d.entry_z, d.entry_stick, d.stick_off,
                      tw_z, d.sticks, d.zmask, bx, band);
  }
  if (!grid_barrier(barrier, gridDim.x) && threadIdx.x == 0) atomicExch(error, 21);
  const int64_t per_k_b = (int64_t)max_nb * nz;
  const int64_t items_b = (int64_t)nk * per_k_b;
  for (int64_t it = blockIdx.x; it < items_b; it += gridDim.x) {
    const int k = (int)(it / per_k_b);
    const int64_t r = it - k * per_k_b;
    const int band = (int)(r / nz), z = (int)(r - (int64_t)band * nz);
    const KDesc<T>& d = kb.k[k];
    if (band >= d.nb) continue;
    __syncthreads();
    pass_b_body<T, F, 0>(d.sticks, d.nst, nz, d.nay, nx_pad, d.stick_pos, d.y_to_ay, tw_xy,
                         potential, nullptr, nullptr, z, band);
  }
  if (!grid_barrier(barrier, gridDim.x) && threadIdx.x == 0) atomicExch(error, 21);
  for (int64_t it = blockIdx.x; it < items_ac; it += gridDim.x) {
    const int k = (int)(it / per_k_ac);
    const int64_t r = it - k * per_k_ac;
    const int band = (int)(r / sblocks), bx = (int)(r - (int64_t)band * sblocks);
    const KDesc<T>& d = kb.k[k];
    if (bx * kSticksPerBlock >= d.nst || band >= d.nb) continue;
    __syncthreads();
    pass_c_body<T, F>(d.sticks, d.nst, d.entry_g, d.entry_z, d.entry_stick, d.stick_off, tw_z,
                      d.psi, d.ld, d.kinetic, inv_n, d.out, d.ldo, d.zmask, bx, band);
  }
}

std::atomic<int> g_persistent{0};

template <typename T>
const C2<T>* tw_at(const qeb_local_plan* p, int which) {
  const C2<T>* base = static_cast<const C2<T>*>(p->tw);
  return which == 0 ? base : (which == 1 ? base + p->nx : base + p->nx + p->ny);
}

// Calls `fn.template operator()<F>()` with the four-step type of variant v.
template <class Fn>
int with_variant(int v, Fn&& fn) {
  int index = 0;
#define QEB_CASE(n, a, b)                                    \
  if (v == index) return fn.template operator()<qeb::Four<a, b>>(); \
  ++index;
  QEB_FOUR_SIZES(QEB_CASE)
#undef QEB_CASE
  qeb::set_error("four-step variant %d does not exist", v);
  return QEB_EUNSUPPORTED;
}

template <typename T>
struct SetLimits {
  const qeb_local_plan* p;
  template <class F>
  int operator()() const {
    cudaError_t err = cudaSuccess;
    if (p->fast_z >= 0 && F::n == p->nz) {
      const int s = (int)ac_smem<T, F>();
      err = qeb::raise_smem_limit(four_pass_a<T, F>, s);
      if (err == cudaSuccess)
        err = qeb::raise_smem_limit(four_pass_c<T, F>, s);
      if (err == cudaSuccess)
        err = qeb::raise_smem_limit(four_pass_a_multi<T, F>, s);
      if (err == cudaSuccess)
        err = qeb::raise_smem_limit(four_pass_c_multi<T, F>, s);
    }
    if (err == cudaSuccess && p->fast_xy >= 0 && F::n == p->nx) {
      const size_t s = b_smem<T, F>(p);
      if (s > 227 * 1024) {
        qeb::set_error("four-step pass B needs %zu bytes of shared memory", s);
        return QEB_EUNSUPPORTED;
      }
      err = qeb::raise_smem_limit(four_pass_b<T, F, 0>, s);
      if (err == cudaSuccess)
        err = qeb::raise_smem_limit(four_pass_b<T, F, 1>, s);
      if (err == cudaSuccess)
        err = qeb::raise_smem_limit(four_pass_b_multi<T, F>, s);
      if constexpr (prunable<F>()) {
        if (err == cudaSuccess && p->prune_k == kPruneK)
          err = qeb::raise_smem_limit(four_pass_b_pruned_multi<T, F, kPruneK>,
                                      b_pruned_smem<T, F, kPruneK>(p));
      }
      // the persistent launch takes the larger of the two footprints of
      // whichever plans share it: allow a block's shared memory less 1 KB
      // for the barrier's static word (dynamic + static may not pass 227 KB)
      if (err == cudaSuccess && p->fast_z == p->fast_xy)
        err = qeb::raise_smem_limit(four_passes_persistent<T, F>, 226 * 1024);
    }
    return qeb::cuda_status(err, "four-step shared memory attribute");
  }
};

template <typename T>
struct PassA {
  const qeb_local_plan* p; C2<T>* sticks; const C2<T>* psi; int64_t ld; int64_t nb; cudaStream_t s;
  template <class F>
  int operator()() const {
    const dim3 grid((p->nst + kSticksPerBlock - 1) / kSticksPerBlock, (unsigned)nb);
    four_pass_a<T, F><<<grid, kThreads, ac_smem<T, F>(), s>>>(
        psi, ld, p->nst, p->entry_g, p->entry_z, p->entry_stick, p->stick_off,
        tw_at<T>(p, 2), sticks, p->zmask);
    return QEB_OK;
  }
};

template <typename T>
struct PassC {
  const qeb_local_plan* p; const C2<T>* sticks; const C2<T>* psi; int64_t ld; int64_t nb;
  const T* kinetic; C2<T>* out; int64_t ldo; cudaStream_t s;
  template <class F>
  int operator()() const {
    const dim3 grid((p->nst + kSticksPerBlock - 1) / kSticksPerBlock, (unsigned)nb);
    const T inv_n = T(1.0 / ((double)p->nx * p->ny * p->nz));
    four_pass_c<T, F><<<grid, kThreads, ac_smem<T, F>(), s>>>(
        sticks, p->nst, p->entry_g, p->entry_z, p->entry_stick, p->stick_off,
        tw_at<T>(p, 2), psi, ld, kinetic, inv_n, out, ldo, p->zmask);
    return QEB_OK;
  }
};

template <typename T, int MODE>
struct PassB {
  const qeb_local_plan* p; C2<T>* sticks; int64_t nb; const T* potential;
  const double* weights; double* density; cudaStream_t s;
  template <class F>
  int operator()() const {
    const dim3 grid(p->nz, (unsigned)nb);
    four_pass_b<T, F, MODE><<<grid, kThreads, b_smem<T, F>(p), s>>>(
        sticks, p->nst, p->nz, p->nay, p->nx_pad, p->stick_pos, p->y_to_ay, tw_at<T>(p, 0),
        potential, weights, density);
    return QEB_OK;
  }
};

template <typename T>
struct PassAMulti {
  const KBatch<T>* kb; const qeb_local_plan* p0; int nk; int sblocks; int nb; cudaStream_t s;
  template <class F>
  int operator()() const {
    const dim3 grid(sblocks, (unsigned)nb, (unsigned)nk);
    four_pass_a_multi<T, F><<<grid, kThreads, ac_smem<T, F>(), s>>>(*kb,
                                                                             tw_at<T>(p0, 2));
    return QEB_OK;
  }
};

template <typename T>
struct PassBMulti {
  const KBatch<T>* kb; const qeb_local_plan* p0; int nk; int nb; size_t smem; const T* potential;
  cudaStream_t s;
  template <class F>
  int operator()() const {
    const dim3 grid(p0->nz, (unsigned)nb, (unsigned)nk);
    four_pass_b_multi<T, F><<<grid, kThreads, smem, s>>>(*kb, p0->nz, p0->nx_pad, tw_at<T>(p0, 0),
                                                        potential);
    return QEB_OK;
  }
};

template <typename T>
struct PassBPrunedMulti {
  const KBatch<T>* kb; const qeb_local_plan* p0; int nk; int nb; const T* potential;
  cudaStream_t s;
  template <class F>
  int operator()() const {
    if constexpr (prunable<F>()) {
      const dim3 grid(p0->nz, (unsigned)((nb + kPrunedBands - 1) / kPrunedBands),
                      (unsigned)nk);
      four_pass_b_pruned_multi<T, F, kPruneK><<<grid, kThreads,
                                                b_pruned_smem<T, F, kPruneK>(p0), s>>>(
          *kb, p0->nz, p0->nx_pad, tw_at<T>(p0, 0), potential);
      return QEB_OK;
    } else {
      qeb::set_error("four-step variant of length %d has no pruned plane pass", F::n);
      return QEB_EUNSUPPORTED;
    }
  }
};

template <typename T>
struct PassCMulti {
  const KBatch<T>* kb; const qeb_local_plan* p0; int nk; int sblocks; int nb; cudaStream_t s;
  template <class F>
  int operator()() const {
    const dim3 grid(sblocks, (unsigned)nb, (unsigned)nk);
    const T inv_n = T(1.0 / ((double)p0->nx * p0->ny * p0->nz));
    four_pass_c_multi<T, F><<<grid, kThreads, ac_smem<T, F>(), s>>>(
        *kb, tw_at<T>(p0, 2), inv_n);
    return QEB_OK;
  }
};

template <typename T>
struct PersistentLaunch {
  const KBatch<T>* kb; int nk; int sblocks; int nb; int nx_pad; const C2<T>* tw_z;
  const C2<T>* tw_xy; const T* potential; T inv_n; size_t smem_b; unsigned int* barrier;
  cudaStream_t s;
  template <class F>
  int operator()() const {
    const size_t ac = ac_smem<T, F>();
    const size_t smem = ac > smem_b ? ac : smem_b;
    int per_sm = 0, device = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, four_passes_persistent<T, F>, kThreads, smem);
    if (e == cudaSuccess) e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return qeb::cuda_status(e, "persistent passes: occupancy");
    if (per_sm < 1) {
      qeb::set_error("persistent passes: a block of %zu bytes of shared memory does not fit", smem);
      return QEB_EUNSUPPORTED;
    }
    int* error = nullptr;
    int rc = qeb::tensor_error_word(&error);
    if (rc) return rc;
    e = cudaMemsetAsync(barrier, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return qeb::cuda_status(e, "persistent passes: barrier reset");
    KBatch<T> batch = *kb;
    int nk_ = nk, sblocks_ = sblocks, nb_ = nb, nx_pad_ = nx_pad;
    const C2<T>* tw_z_ = tw_z;
    const C2<T>* tw_xy_ = tw_xy;
    const T* potential_ = potential;
    T inv_n_ = inv_n;
    unsigned int* barrier_ = barrier;
    void* args[] = {&batch, &nk_, &sblocks_, &nb_, &nx_pad_, &tw_z_, &tw_xy_, &potential_,
                    &inv_n_, &barrier_, &error};
    // cooperative: every block of the grid is resident at once, which the
    // grid barrier needs
    e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(four_passes_persistent<T, F>),
                                    dim3(per_sm * sms), dim3(kThreads), args, smem, s);
    qeb::count_launches(1);
    return qeb::cuda_status(e, "persistent passes launch");
  }
};

// Largest pass-B shared memory over the batch (the plane holds nay rows).
template <typename T>
struct BSmem {
  const qeb_local_plan* p;
  size_t* out;
  template <class F>
  int operator()() const {
    *out = b_smem<T, F>(p);
    return QEB_OK;
  }
};

template <typename T>
int apply_multi_t(int nk, const qeb_local_plan* const* plans, void* const* sticks,
                  const void* const* psi, const int64_t* ld, const int64_t* nb,
                  const void* potential, const void* const* kinetic, void* const* out,
                  const int64_t* ldo, cudaStream_t s, cudaEvent_t* ev, unsigned int* barrier) {
  KBatch<T> kb;
  bool pruned = true;  // every plan on the pruned plane
  int max_nb = 0, max_blocks = 0;
  size_t smem_b = 0;
  for (int k = 0; k < nk; ++k) {
    const qeb_local_plan* p = plans[k];
    KDesc<T>& d = kb.k[k];
    d.psi = static_cast<const C2<T>*>(psi[k]);
    d.out = static_cast<C2<T>*>(out[k]);
    d.kinetic = static_cast<const T*>(kinetic[k]);
    d.sticks = static_cast<C2<T>*>(sticks[k]);
    d.entry_g = p->entry_g;
    d.entry_z = p->entry_z;
    d.entry_stick = p->entry_stick;
    d.stick_off = p->stick_off;
    d.stick_pos = p->stick_pos;
    d.y_to_ay = p->y_to_ay;
    d.slot_pos = p->slot_pos;
    d.ay_to_slot = p->ay_to_slot;
    pruned = pruned && p->prune_k == kPruneK;
    d.ld = ld[k];
    d.ldo = ldo[k];
    d.nst = p->nst;
    d.nay = p->nay;
    d.nb = (int)nb[k];
    d.zmask = p->zmask;
    max_nb = max(max_nb, d.nb);
    max_blocks = max(max_blocks, (p->nst + kSticksPerBlock - 1) / kSticksPerBlock);
    size_t sb = 0;
    int rc = with_variant(p->fast_xy, BSmem<T>{p, &sb});
    if (rc) return rc;
    smem_b = sb > smem_b ? sb : smem_b;
  }
  if (max_nb == 0) return QEB_OK;
  const qeb_local_plan* p0 = plans[0];
  int rc;
  if (g_persistent.load() && ev == nullptr && barrier != nullptr && p0->fast_z == p0->fast_xy) {
    const T inv_n = T(1.0 / ((double)p0->nx * p0->ny * p0->nz));
    return with_variant(p0->fast_z,
                        PersistentLaunch<T>{&kb, nk, max_blocks, max_nb, p0->nx_pad,
                                            tw_at<T>(p0, 2), tw_at<T>(p0, 0),
                                            static_cast<const T*>(potential), inv_n, smem_b,
                                            barrier, s});
  }
  if (ev) cudaEventRecord(ev[0], s);
  if ((rc = with_variant(p0->fast_z, PassAMulti<T>{&kb, p0, nk, max_blocks, max_nb, s}))) return rc;
  if (ev) cudaEventRecord(ev[1], s);
  if (pruned) {
    if ((rc = with_variant(p0->fast_xy, PassBPrunedMulti<T>{&kb, p0, nk, max_nb,
                                                            static_cast<const T*>(potential), s})))
      return rc;
  } else if ((rc = with_variant(p0->fast_xy, PassBMulti<T>{&kb, p0, nk, max_nb, smem_b,
                                                           static_cast<const T*>(potential), s}))) {
    return rc;
  }
  if (ev) cudaEventRecord(ev[2], s);
  if ((rc = with_variant(p0->fast_z, PassCMulti<T>{&kb, p0, nk, max_blocks, max_nb, s}))) return rc;
  if (ev) cudaEventRecord(ev[3], s);
  qeb::count_launches(3);
  return qeb::cuda_status(cudaGetLastError(), "four-step apply_local_multi launch");
}

template <typename T>
int density_t(const qeb_local_plan* p, C2<T>* sticks, const C2<T>* psi, int64_t ld, int64_t nb,
              const double* weights, double* density, cudaStream_t s) {
  int rc;
  if ((rc = with_variant(p->fast_z, PassA<T>{p, sticks, psi, ld, nb, s}))) return rc;
  if ((rc = with_variant(p->fast_xy, PassB<T, 1>{p, sticks, nb, nullptr, weights, density, s})))
    return rc;
  qeb::count_launches(2);
  return qeb::cuda_status(cudaGetLastError(), "four-step accumulate_density launch");
}

std::mutex g_tw_mutex;
bool g_tw_ready[64] = {false};

}  // namespace

namespace qeb {

int four_variant(int n) {
  for (int i = 0; i < kFourCount; ++i)
    if (kFourLengths[i] == n) return i;
  return -1;
}

bool four_split(int variant, int* n1, int* n2) {
  int index = 0;
#define QEB_SPLIT(n, a, b) \
  if (variant == index) {  \
    *n1 = a;               \
    *n2 = b;               \
    return true;           \
  }                        \
  ++index;
  QEB_FOUR_SIZES(QEB_SPLIT)
#undef QEB_SPLIT
  return false;
}

int prune_k_of(int variant) {
  int index = 0, k = 0;
#define QEB_PRUNE(n, a, b)                                             \
  if (variant == index) k = prunable<qeb::Four<a, b>>() ? kPruneK : 0; \
  ++index;
  QEB_FOUR_SIZES(QEB_PRUNE)
#undef QEB_PRUNE
  return k;
}

int init_small_dft_twiddles() {
  int device = 0;
  cudaGetDevice(&device);
  if (device < 0 || device >= 64) return QEB_EUNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  if (g_tw_ready[device]) return QEB_OK;
  double2 t64[kSmallTwTotal];
  float2 t32[kSmallTwTotal];
  const int sizes[] = {6, 8, 9, 10, 12, 15, 16};
  const long double two_pi = 6.283185307179586476925286766559005768L;
  int off = 0;
  for (int n : sizes) {
    for (int m = 0; m < n; ++m) {
      const long double a = two_pi * (long double)m / (long double)n;
      t64[off + m] = make_double2((double)cosl(a), (double)(-sinl(a)));
      t32[off + m] = make_float2((float)cosl(a), (float)(-sinl(a)));
    }
    off += n;
  }
  cudaError_t err = cudaMemcpyToSymbol(c_small_tw64, t64, sizeof(t64));
  if (err == cudaSuccess) err = cudaMemcpyToSymbol(c_small_tw32, t32, sizeof(t32));
  if (err != cudaSuccess) return cuda_status(err, "small DFT twiddle upload");
  g_tw_ready[device] = true;
  return QEB_OK;
}

int fast_smem_limits(const qeb_local_plan* p) {
  int rc = init_small_dft_twiddles();
  if (rc) return rc;
  for (int v : {p->fast_z, p->fast_xy}) {
    if (v < 0) continue;
    rc = (p->precision == QEB_F64) ? with_variant(v, SetLimits<double>{p})
                                   : with_variant(v, SetLimits<float>{p});
    if (rc) return rc;
  }
  return QEB_OK;
}

int fast_apply_multi(int nk, const qeb_local_plan* const* plans, void* const* sticks,
                     const void* const* psi, const int64_t* ld, const int64_t* nb,
                     const void* potential, const void* const* kinetic, void* const* out,
                     const int64_t* ldo, cudaStream_t stream, unsigned int* barrier) {
  if (plans[0]->precision == QEB_F64)
    return apply_multi_t<double>(nk, plans, sticks, psi, ld, nb, potential, kinetic, out, ldo,
                                 stream, nullptr, barrier);
  return apply_multi_t<float>(nk, plans, sticks, psi, ld, nb, potential, kinetic, out, ldo,
                              stream, nullptr, barrier);
}

// One plan runs through the batched kernels with a batch of one, so a k point
// gives the same bits alone and inside a batch.
int fast_apply(const qeb_local_plan* p, void* sticks, const void* psi, int64_t ld, int64_t nb,
               const void* potential, const void* kinetic, void* out, int64_t ldo,
               cudaStream_t stream, cudaEvent_t* events, unsigned int* barrier) {
  const qeb_local_plan* plans[1] = {p};
  void* st[1] = {sticks};
  const void* ps[1] = {psi};
  const void* kin[1] = {kinetic};
  void* o[1] = {out};
  const int64_t lds[1] = {ld}, nbs[1] = {nb}, ldos[1] = {ldo};
  if (p->precision == QEB_F64)
    return apply_multi_t<double>(1, plans, st, ps, lds, nbs, potential, kin, o, ldos, stream,
                                 events, barrier);
  return apply_multi_t<float>(1, plans, st, ps, lds, nbs, potential, kin, o, ldos, stream, events,
                              barrier);
}

int fast_density(const qeb_local_plan* p, void* sticks, const void* psi, int64_t ld, int64_t nb,
                 const double* weights, double* density, cudaStream_t stream) {
  if (p->precision == QEB_F64)
    return density_t<double>(p, static_cast<C2<double>*>(sticks),
                             static_cast<const C2<double>*>(psi), ld, nb, weights, density, stream);
  return density_t<float>(p, static_cast<C2<float>*>(sticks), static_cast<const C2<float>*>(psi),
                          ld, nb, weights, density, stream);
}

}  // namespace qeb

extern "C" int qeb_set_persistent_passes(int enabled) {
  g_persistent.store(enabled ? 1 : 0);
  return QEB_OK;
}

extern "C" int qeb_persistent_passes(void) { return g_persistent.load(); }
