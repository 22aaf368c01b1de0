// Band-batched local H|psi> and density accumulation on the FFT grid.
//
// Restates, for one GPU, the operator of qepy_pw/_native_fft.pyx
// qepy_apply_serial_spatial (:58-135) and apply_serial (:2338-2455):
//   Hpsi[g, b] = FFT^-( V(r) * FFT^+(psi[:, b]) )[slot_g] / N_r + T_g psi[g, b]
// factorised the way QE/FFTXlib (and the reference's spatial path) do it:
//   pass A : per occupied (x, y) stick, gather psi(G) and inverse-FFT along z;
//   pass B : per (z plane, band) inverse 2-D FFT, multiply by V(x, y, z),
//            forward 2-D FFT, keep only the stick columns;
//   pass C : per stick forward FFT along z, gather, scale by 1/N_r and add the
//            kinetic term.
// Inside pass B the 2-D transform is pruned: the x transforms run only on the
// "active" y rows (those containing sticks), the y transforms on every x
// column; both directions keep the plane in shared memory.
//
// HBM layout:
//   psi, out : column-major (npw, nbands), leading dimension ld (complex T)
//   V        : native (nz, nx, ny) real T      (reference "native layout")
//   sticks   : scratch (nbands, nz, nst) complex T
//   density  : C-order (nx, ny, nz) float64 (reference serial layout)
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "local_plan.cuh"
#include "qeb_common.cuh"
#include "../../include/qe_b200.h"

using qeb::C2;
using qeb::FftDesc;

namespace {

constexpr int kThreads = 256;
constexpr int kSticksPerBlock = 32;  // pass A/C
constexpr int kRowBatch = 16;        // pass B column batch

inline int odd_pad(int n) { return (n % 2 == 0) ? n + 1 : n; }

template <typename T>
size_t pass_b_smem(const qeb_local_plan* p) {
  return sizeof(C2<T>) * ((size_t)p->nay * p->nx_pad + (size_t)kRowBatch * p->ny_pad +
                          (size_t)p->nx + p->ny);
}

template <typename T>
size_t pass_ac_smem(const qeb_local_plan* p) {
  return sizeof(C2<T>) * ((size_t)kSticksPerBlock * p->nz_pad + p->nz);
}

// ---------------------------------------------------------------------------
// Pass A: scatter psi(G) into z lines of the occupied sticks, inverse FFT.
template <typename T>
__global__ void __launch_bounds__(kThreads) pass_a_kernel(
    const C2<T>* __restrict__ psi, int64_t ld, int nst, int nz, int nz_pad, FftDesc fz,
    const int32_t* __restrict__ entry_g, const int32_t* __restrict__ entry_z,
    const int32_t* __restrict__ entry_stick, const int32_t* __restrict__ stick_off,
    const C2<T>* __restrict__ tw_z, C2<T>* __restrict__ sticks) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* lines = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* tw = lines + kSticksPerBlock * nz_pad;
  const int s0 = blockIdx.x * kSticksPerBlock;
  const int nsl = min(kSticksPerBlock, nst - s0);
  const int64_t band = blockIdx.y;
  for (int i = threadIdx.x; i < nz; i += blockDim.x) tw[i] = tw_z[i];
  for (int i = threadIdx.x; i < kSticksPerBlock * nz_pad; i += blockDim.x) lines[i] = qeb::mk<T>(0, 0);
  __syncthreads();
  const int e0 = stick_off[s0], e1 = stick_off[s0 + nsl];
  const C2<T>* col = psi + band * ld;
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    lines[(entry_stick[e] - s0) * nz_pad + entry_z[e]] = col[entry_g[e]];
  }
  __syncthreads();
  qeb::fft_lines<T, 2>(lines, nsl, nz_pad, 1, fz, tw, true);
  C2<T>* out = sticks + band * (int64_t)nz * nst;
  for (int i = threadIdx.x; i < nz * nsl; i += blockDim.x) {
    const int z = i / nsl, sl = i - z * nsl;
    out[(int64_t)z * nst + s0 + sl] = lines[sl * nz_pad + z];
  }
}

// ---------------------------------------------------------------------------
// Pass C: forward FFT of the stick lines along z, gather, 1/N and T*psi.
template <typename T>
__global__ void __launch_bounds__(kThreads) pass_c_kernel(
    const C2<T>* __restrict__ sticks, int nst, int nz, int nz_pad, FftDesc fz,
    const int32_t* __restrict__ entry_g, const int32_t* __restrict__ entry_z,
    const int32_t* __restrict__ entry_stick, const int32_t* __restrict__ stick_off,
    const C2<T>* __restrict__ tw_z, const C2<T>* __restrict__ psi, int64_t ld,
    const T* __restrict__ kinetic, T inv_n, C2<T>* __restrict__ out, int64_t ldo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* lines = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* tw = lines + kSticksPerBlock * nz_pad;
  const int s0 = blockIdx.x * kSticksPerBlock;
  const int nsl = min(kSticksPerBlock, nst - s0);
  const int64_t band = blockIdx.y;
  for (int i = threadIdx.x; i < nz; i += blockDim.x) tw[i] = tw_z[i];
  const C2<T>* in = sticks + band * (int64_t)nz * nst;
  for (int i = threadIdx.x; i < nz * nsl; i += blockDim.x) {
    const int z = i / nsl, sl = i - z * nsl;
    lines[sl * nz_pad + z] = in[(int64_t)z * nst + s0 + sl];
  }
  __syncthreads();
  qeb::fft_lines<T, 2>(lines, nsl, nz_pad, 1, fz, tw, false);
  const int e0 = stick_off[s0], e1 = stick_off[s0 + nsl];
  const C2<T>* col = psi + band * ld;
  C2<T>* dst = out + band * ldo;
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int g = entry_g[e];
    C2<T> v = qeb::scale(lines[(entry_stick[e] - s0) * nz_pad + entry_z[e]], inv_n);
    if (kinetic != nullptr) {
      const T t = kinetic[g];
      const C2<T> p = col[g];
      v.re += t * p.re;
      v.im += t * p.im;
    }
    dst[g] = v;
  }
}

// ---------------------------------------------------------------------------
// Pass B: one (z plane, band) per block; 2-D FFT^+ . V . FFT^- in shared memory.
// mode 0: local potential (sticks rewritten in place);
// mode 1: density, rho[(x*ny+y)*nz+z] += w_b |psi_b(r)|^2 (sticks untouched).
template <typename T, int MODE>
__global__ void __launch_bounds__(kThreads) pass_b_kernel(
    C2<T>* __restrict__ sticks, int nst, int nx, int ny, int nz, int nay, int nx_pad,
    int ny_pad, FftDesc fx, FftDesc fy, const int32_t* __restrict__ stick_pos,
    const int32_t* __restrict__ ay_to_y, const int32_t* __restrict__ y_to_ay,
    const C2<T>* __restrict__ tw_x, const C2<T>* __restrict__ tw_y,
    const T* __restrict__ potential, const double* __restrict__ weights,
    double* __restrict__ density) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* plane = reinterpret_cast<C2<T>*>(smem_raw);  // [nay][nx_pad]
  C2<T>* cols = plane + (size_t)nay * nx_pad;           // [kRowBatch][ny_pad]
  C2<T>* twx = cols + (size_t)kRowBatch * ny_pad;
  C2<T>* twy = twx + nx;
  const int z = blockIdx.x;
  const int64_t band = blockIdx.y;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) twx[i] = tw_x[i];
  for (int i = threadIdx.x; i < ny; i += blockDim.x) twy[i] = tw_y[i];
  for (int i = threadIdx.x; i < nay * nx_pad; i += blockDim.x) plane[i] = qeb::mk<T>(0, 0);
  __syncthreads();
  C2<T>* srow = sticks + (band * nz + z) * (int64_t)nst;
  for (int s = threadIdx.x; s < nst; s += blockDim.x) plane[stick_pos[s]] = srow[s];
  __syncthreads();
  // inverse transform along x of the active rows
  qeb::fft_lines<T, 2>(plane, nay, nx_pad, 1, fx, twx, true);
  double w = 0.0;
  if (MODE == 1) w = weights[band];
  for (int x0 = 0; x0 < nx; x0 += kRowBatch) {
    const int nb = min(kRowBatch, nx - x0);
    for (int i = threadIdx.x; i < nb * ny; i += blockDim.x) {
      const int r = i / ny, y = i - r * ny;
      const int ay = y_to_ay[y];
      cols[r * ny_pad + y] = (ay >= 0) ? plane[ay * nx_pad + x0 + r] : qeb::mk<T>(0, 0);
    }
    __syncthreads();
    qeb::fft_lines<T, 2>(cols, nb, ny_pad, 1, fy, twy, true);
    if (MODE == 0) {
      const T* vrow = potential + ((int64_t)z * nx + x0) * ny;
      for (int i = threadIdx.x; i < nb * ny; i += blockDim.x) {
        const int r = i / ny, y = i - r * ny;
        cols[r * ny_pad + y] = qeb::scale(cols[r * ny_pad + y], vrow[(int64_t)r * ny + y]);
      }
      __syncthreads();
      qeb::fft_lines<T, 2>(cols, nb, ny_pad, 1, fy, twy, false);
      for (int i = threadIdx.x; i < nb * nay; i += blockDim.x) {
        const int r = i / nay, ay = i - r * nay;
        plane[ay * nx_pad + x0 + r] = cols[r * ny_pad + ay_to_y[ay]];
      }
      __syncthreads();
    } else {
      for (int i = threadIdx.x; i < nb * ny; i += blockDim.x) {
        const int r = i / ny, y = i - r * ny;
        const C2<T> v = cols[r * ny_pad + y];
        const double m = (double)v.re * (double)v.re + (double)v.im * (double)v.im;
        atomicAdd(density + ((int64_t)(x0 + r) * ny + y) * nz + z, w * m);
      }
      __syncthreads();
    }
  }
  if (MODE == 0) {
    qeb::fft_lines<T, 2>(plane, nay, nx_pad, 1, fx, twx, false);
    for (int s = threadIdx.x; s < nst; s += blockDim.x) srow[s] = plane[stick_pos[s]];
  }
}

template <typename T>
int set_smem_limits(const qeb_local_plan* p) {
  const size_t b = pass_b_smem<T>(p), ac = pass_ac_smem<T>(p);
  cudaError_t err;
  err = qeb::raise_smem_limit(pass_b_kernel<T, 0>, b);
  if (err != cudaSuccess) return qeb::cuda_status(err, "pass B smem attribute");
  err = qeb::raise_smem_limit(pass_b_kernel<T, 1>, b);
  if (err != cudaSuccess) return qeb::cuda_status(err, "pass B (density) smem attribute");
  err = qeb::raise_smem_limit(pass_a_kernel<T>, ac);
  if (err != cudaSuccess) return qeb::cuda_status(err, "pass A smem attribute");
  err = qeb::raise_smem_limit(pass_c_kernel<T>, ac);
  if (err != cudaSuccess) return qeb::cuda_status(err, "pass C smem attribute");
  return QEB_OK;
}

template <typename T>
const C2<T>* tw_ptr(const qeb_local_plan* p, int which) {
  const C2<T>* base = static_cast<const C2<T>*>(p->tw);
  if (which == 0) return base;
  if (which == 1) return base + p->nx;
  return base + p->nx + p->ny;
}

// Scratch of one apply: the stick buffer (nbands x nz x nst values), rounded
// up to 256 bytes, then the 256-byte word block of the persistent launch's
// grid barrier (local_fast.cu).
static int64_t stick_region_bytes(const qeb_local_plan* p, int64_t nbands) {
  const int64_t elem = (p->precision == QEB_F64) ? 16 : 8;
  return (nbands * (int64_t)p->nz * p->nst * elem + 255) / 256 * 256;
}

template <typename T>
int launch_apply(const qeb_local_plan* p, C2<T>* sticks, const C2<T>* psi, int64_t ld,
                 int64_t nb, const T* potential, const T* kinetic, C2<T>* out, int64_t ldo,
                 cudaStream_t stream, cudaEvent_t* events = nullptr) {
  if (nb == 0) return QEB_OK;
  if (nb > 65535) {
    qeb::set_error("apply_local: at most 65535 bands per call (got %lld)", (long long)nb);
    return QEB_EINVAL;
  }
  if (p->fast_xy >= 0 && p->fast_z >= 0)
    return qeb::fast_apply(p, sticks, psi, ld, nb, potential, kinetic, out, ldo, stream, events,
                           reinterpret_cast<unsigned int*>(reinterpret_cast<unsigned char*>(sticks) +
                                                           stick_region_bytes(p, nb)));
  const dim3 grid_ac((p->nst + kSticksPerBlock - 1) / kSticksPerBlock, (unsigned)nb);
  const dim3 grid_b(p->nz, (unsigned)nb);
  if (events) cudaEventRecord(events[0], stream);
  pass_a_kernel<T><<<grid_ac, kThreads, pass_ac_smem<T>(p), stream>>>(
      psi, ld, p->nst, p->nz, p->nz_pad, p->fz, p->entry_g, p->entry_z, p->entry_stick,
      p->stick_off, tw_ptr<T>(p, 2), sticks);
  if (events) cudaEventRecord(events[1], stream);
  pass_b_kernel<T, 0><<<grid_b, kThreads, pass_b_smem<T>(p), stream>>>(
      sticks, p->nst, p->nx, p->ny, p->nz, p->nay, p->nx_pad, p->ny_pad, p->fx, p->fy,
      p->stick_pos, p->ay_to_y, p->y_to_ay, tw_ptr<T>(p, 0), tw_ptr<T>(p, 1), potential,
      nullptr, nullptr);
  if (events) cudaEventRecord(events[2], stream);
  const T inv_n = T(1.0 / ((double)p->nx * p->ny * p->nz));
  pass_c_kernel<T><<<grid_ac, kThreads, pass_ac_smem<T>(p), stream>>>(
      sticks, p->nst, p->nz, p->nz_pad, p->fz, p->entry_g, p->entry_z, p->entry_stick,
      p->stick_off, tw_ptr<T>(p, 2), psi, ld, kinetic, inv_n, out, ldo);
  if (events) cudaEventRecord(events[3], stream);
  qeb::count_launches(3);
  return qeb::cuda_status(cudaGetLastError(), "apply_local launch");
}

template <typename T>
int launch_density(const qeb_local_plan* p, C2<T>* sticks, const C2<T>* psi, int64_t ld,
                   int64_t nb, const double* weights, double* density, cudaStream_t stream) {
  if (nb == 0) return QEB_OK;
  if (nb > 65535) {
    qeb::set_error("accumulate_density: at most 65535 bands per call (got %lld)", (long long)nb);
    return QEB_EINVAL;
  }
  if (p->fast_xy >= 0 && p->fast_z >= 0)
    return qeb::fast_density(p, sticks, psi, ld, nb, weights, density, stream);
  const dim3 grid_ac((p->nst + kSticksPerBlock - 1) / kSticksPerBlock, (unsigned)nb);
  const dim3 grid_b(p->nz, (unsigned)nb);
  pass_a_kernel<T><<<grid_ac, kThreads, pass_ac_smem<T>(p), stream>>>(
      psi, ld, p->nst, p->nz, p->nz_pad, p->fz, p->entry_g, p->entry_z, p->entry_stick,
      p->stick_off, tw_ptr<T>(p, 2), sticks);
  pass_b_kernel<T, 1><<<grid_b, kThreads, pass_b_smem<T>(p), stream>>>(
      sticks, p->nst, p->nx, p->ny, p->nz, p->nay, p->nx_pad, p->ny_pad, p->fx, p->fy,
      p->stick_pos, p->ay_to_y, p->y_to_ay, tw_ptr<T>(p, 0), tw_ptr<T>(p, 1), nullptr,
      weights, density);
  qeb::count_launches(2);
  return qeb::cuda_status(cudaGetLastError(), "accumulate_density launch");
}

template <typename T>
void fill_twiddles(std::vector<C2<T>>& out, int n) {
  // exp(-2 pi i m / n) evaluated in long double and rounded once.
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < n; ++m) {
    const long double a = two_pi * (long double)m / (long double)n;
    out.push_back(qeb::mk<T>((T)cosl(a), (T)(-sinl(a))));
  }
}

void free_plan(qeb_local_plan* p) {
  if (p == nullptr) return;
  cudaFree(p->entry_g);
  cudaFree(p->entry_z);
  cudaFree(p->entry_stick);
  cudaFree(p->stick_off);
  cudaFree(p->stick_pos);
  cudaFree(p->ay_to_y);
  cudaFree(p->y_to_ay);
  cudaFree(p->slot_pos);
  cudaFree(p->ay_to_slot);
  cudaFree(p->tw);
  delete p;
}

template <typename V>
int upload(V** dst, const std::vector<V>& src) {
  const size_t bytes = std::max<size_t>(1, src.size()) * sizeof(V);
  cudaError_t err = cudaMalloc((void**)dst, bytes);
  if (err != cudaSuccess) return qeb::cuda_status(err, "plan allocation");
  if (!src.empty()) {
    err = cudaMemcpy(*dst, src.data(), src.size() * sizeof(V), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return qeb::cuda_status(err, "plan upload");
  }
  return QEB_OK;
}

}  // namespace

extern "C" int qeb_local_plan_create(qeb_local_plan** out, int nx, int ny, int nz, int64_t npw,
                                     const int64_t* z_major_slots, int precision) {
  if (out == nullptr) {
    qeb::set_error("local_plan_create: null output pointer");
    return QEB_EINVAL;
  }
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1 || npw < 1 || z_major_slots == nullptr) {
    qeb::set_error("local_plan_create: invalid grid (%d,%d,%d) or basis size %lld", nx, ny, nz,
                   (long long)npw);
    return QEB_EINVAL;
  }
  if (precision != QEB_F64 && precision != QEB_F32) {
    qeb::set_error("local_plan_create: unknown precision %d", precision);
    return QEB_EINVAL;
  }
  if (npw > INT32_MAX) {
    qeb::set_error("local_plan_create: basis too large");
    return QEB_EINVAL;
  }
  qeb_local_plan* p = new (std::nothrow) qeb_local_plan();
  if (p == nullptr) {
    qeb::set_error("local_plan_create: host allocation failed");
    return QEB_ECUDA;
  }
  std::memset(p, 0, sizeof(*p));
  p->nx = nx;
  p->ny = ny;
  p->nz = nz;
  p->npw = npw;
  p->precision = precision;
  cudaGetDevice(&p->device);
  if (!qeb::make_fft_desc(nx, &p->fx) || !qeb::make_fft_desc(ny, &p->fy) ||
      !qeb::make_fft_desc(nz, &p->fz)) {
    qeb::set_error("local_plan_create: grid (%d,%d,%d) is not 2-3-5 smooth", nx, ny, nz);
    delete p;
    return QEB_EUNSUPPORTED;
  }
  const int64_t plane = (int64_t)nx * ny;
  const int64_t total = plane * nz;
  // Derive sticks from the z-major slots z*nx*ny + x*ny + y
  // (qepy_pw/basis.py:530-541): sticks are the sorted unique xy slots.
  std::vector<int64_t> xy(npw);
  std::vector<int32_t> zs(npw);
  for (int64_t g = 0; g < npw; ++g) {
    const int64_t slot = z_major_slots[g];
    if (slot < 0 || slot >= total) {
      qeb::set_error("local_plan_create: slot %lld of row %lld outside the grid", (long long)slot,
                     (long long)g);
      delete p;
      return QEB_EINVAL;
    }
    zs[g] = (int32_t)(slot / plane);
    xy[g] = slot % plane;
  }
  std::vector<int64_t> sticks(xy);
  std::sort(sticks.begin(), sticks.end());
  sticks.erase(std::unique(sticks.begin(), sticks.end()), sticks.end());
  const int nst = (int)sticks.size();
  p->nst = nst;
  std::vector<int32_t> stick_of(npw);
  std::vector<int32_t> count(nst + 1, 0);
  for (int64_t g = 0; g < npw; ++g) {
    stick_of[g] = (int32_t)(std::lower_bound(sticks.begin(), sticks.end(), xy[g]) - sticks.begin());
    count[stick_of[g] + 1]++;
  }
  for (int s = 0; s < nst; ++s) count[s + 1] += count[s];
  std::vector<int32_t> stick_off(count);
  std::vector<int32_t> entry_g(npw), entry_z(npw), entry_stick(npw);
  {
    std::vector<int32_t> cursor(count.begin(), count.end() - 1);
    for (int64_t g = 0; g < npw; ++g) {
      const int s = stick_of[g];
      const int e = cursor[s]++;
      entry_g[e] = (int32_t)g;
      entry_z[e] = zs[g];
      entry_stick[e] = s;
    }
  }
  // Detect duplicate (x, y, z) slots: two plane waves cannot share a grid point.
  for (int s = 0; s < nst; ++s) {
    std::vector<int32_t> zl(entry_z.begin() + stick_off[s], entry_z.begin() + stick_off[s + 1]);
    std::sort(zl.begin(), zl.end());
    if (std::adjacent_find(zl.begin(), zl.end()) != zl.end()) {
      qeb::set_error("local_plan_create: two plane waves map to one grid point");
      delete p;
      return QEB_EINVAL;
    }
  }
  // Active y rows.
  std::vector<int32_t> y_to_ay(ny, -1), ay_to_y;
  for (int s = 0; s < nst; ++s) y_to_ay[sticks[s] % ny] = 1;
  for (int y = 0; y < ny; ++y) {
    if (y_to_ay[y] >= 0) {
      y_to_ay[y] = (int32_t)ay_to_y.size();
      ay_to_y.push_back(y);
    }
  }
  p->nay = (int)ay_to_y.size();
  p->nx_pad = odd_pad(nx);
  p->ny_pad = odd_pad(ny);
  p->nz_pad = odd_pad(nz);
  // Four-step kernels when both the plane (nx == ny) and the z lines have a
  // listed factorisation; QEB_FORCE_GENERIC=1 selects the Stockham kernels.
  const char* force_generic = std::getenv("QEB_FORCE_GENERIC");
  p->fast_xy = (nx == ny) ? qeb::four_variant(nx) : -1;
  p->fast_z = qeb::four_variant(nz);
  if (p->fast_xy < 0 || p->fast_z < 0 || (force_generic && force_generic[0] == '1')) {
    p->fast_xy = -1;
    p->fast_z = -1;
  }
  std::vector<int32_t> stick_pos(nst);
  for (int s = 0; s < nst; ++s) {
    const int x = (int)(sticks[s] / ny), y = (int)(sticks[s] % ny);
    stick_pos[s] = y_to_ay[y] * p->nx_pad + x;
  }
  p->zmask = 0xffffffffu;
  int n1 = 0, n2 = 0;
  if (p->fast_z >= 0 && qeb::four_split(p->fast_z, &n1, &n2)) {
    uint32_t m = 0;
    for (int64_t e = 0; e < npw; ++e) m |= 1u << (entry_z[e] / n2);
    p->zmask = m;
  }
  // Pruned plane: every stick's x and y within the 2 K N2 kept rows.
  p->prune_k = 0;
  std::vector<int32_t> slot_pos, ay_to_slot;
  const char* prune_env = std::getenv("QEB_PRUNE_PLANE");
  const int prune_k = p->fast_xy >= 0 ? qeb::prune_k_of(p->fast_xy) : 0;
  if (prune_k > 0 && !(prune_env && prune_env[0] == '0') &&
      qeb::four_split(p->fast_xy, &n1, &n2)) {
    const int half = prune_k * n2, gap = nx - 2 * half;
    auto kept = [&](int c) { return c < half || c >= nx - half; };
    bool fits = 2 * prune_k < n1;
    for (int s = 0; s < nst && fits; ++s)
      fits = kept((int)(sticks[s] / ny)) && kept((int)(sticks[s] % ny));
    if (fits) {
      auto slot = [&](int y) { return y < half ? y : y - gap; };
      slot_pos.resize(nst);
      for (int s = 0; s < nst; ++s) {
        const int x = (int)(sticks[s] / ny), y = (int)(sticks[s] % ny);
        slot_pos[s] = slot(y) * p->nx_pad + x;
      }
      for (int y : ay_to_y) ay_to_slot.push_back(slot(y));
      p->prune_k = prune_k;
    }
  }
  int rc = QEB_OK;
  if (p->prune_k > 0 &&
      ((rc = upload(&p->slot_pos, slot_pos)) || (rc = upload(&p->ay_to_slot, ay_to_slot)))) {
    free_plan(p);
    return rc;
  }
  if ((rc = upload(&p->entry_g, entry_g)) || (rc = upload(&p->entry_z, entry_z)) ||
      (rc = upload(&p->entry_stick, entry_stick)) || (rc = upload(&p->stick_off, stick_off)) ||
      (rc = upload(&p->stick_pos, stick_pos)) || (rc = upload(&p->ay_to_y, ay_to_y)) ||
      (rc = upload(&p->y_to_ay, y_to_ay))) {
    free_plan(p);
    return rc;
  }
  if (precision == QEB_F64) {
    std::vector<C2<double>> tw;
    fill_twiddles(tw, nx);
    fill_twiddles(tw, ny);
    fill_twiddles(tw, nz);
    rc = upload(reinterpret_cast<C2<double>**>(&p->tw), tw);
    if (rc == QEB_OK) rc = set_smem_limits<double>(p);
    if (rc == QEB_OK && pass_b_smem<double>(p) > 227 * 1024) {
      qeb::set_error("local_plan_create: FP64 plane of %d x %d active rows exceeds shared memory",
                     p->nay, nx);
      rc = QEB_EUNSUPPORTED;
    }
  } else {
    std::vector<C2<float>> tw;
    fill_twiddles(tw, nx);
    fill_twiddles(tw, ny);
    fill_twiddles(tw, nz);
    rc = upload(reinterpret_cast<C2<float>**>(&p->tw), tw);
    if (rc == QEB_OK) rc = set_smem_limits<float>(p);
  }
  if (rc == QEB_OK && p->fast_xy >= 0) rc = qeb::fast_smem_limits(p);
  if (rc != QEB_OK) {
    free_plan(p);
    return rc;
  }
  *out = p;
  return QEB_OK;
}

extern "C" int qeb_local_plan_destroy(qeb_local_plan* plan) {
  free_plan(plan);
  return QEB_OK;
}

extern "C" int qeb_local_plan_info(const qeb_local_plan* p, int64_t* info, int n) {
  if (p == nullptr || info == nullptr || n < 8) {
    qeb::set_error("local_plan_info: invalid arguments");
    return QEB_EINVAL;
  }
  info[0] = p->nx;
  info[1] = p->ny;
  info[2] = p->nz;
  info[3] = p->npw;
  info[4] = p->nst;
  info[5] = p->nay;
  info[6] = p->precision;
  info[7] = p->device;
  if (n >= 9) info[8] = p->prune_k;
  return QEB_OK;
}

extern "C" int64_t qeb_local_scratch_bytes(const qeb_local_plan* p, int64_t nbands) {
  if (p == nullptr || nbands < 0) return -1;
  return stick_region_bytes(p, nbands) + 256;
}

static int check_call(const qeb_local_plan* p, const void* scratch, int64_t scratch_bytes,
                      const void* psi, int64_t ld, int64_t nb, const char* who) {
  if (p == nullptr) {
    qeb::set_error("%s: null plan", who);
    return QEB_ENOPLAN;
  }
  if (nb < 0 || ld < p->npw) {
    qeb::set_error("%s: leading dimension %lld below basis size %lld or negative band count", who,
                   (long long)ld, (long long)p->npw);
    return QEB_EINVAL;
  }
  if (nb > 0 && (psi == nullptr || scratch == nullptr)) {
    qeb::set_error("%s: null operand", who);
    return QEB_EINVAL;
  }
  if (scratch_bytes < qeb_local_scratch_bytes(p, nb)) {
    qeb::set_error("%s: scratch of %lld bytes is below the %lld required", who,
                   (long long)scratch_bytes, (long long)qeb_local_scratch_bytes(p, nb));
    return QEB_ESCRATCH;
  }
  // complex values are accessed as one 8-byte (complex64) or 16-byte
  // (complex128) word, so operands must be aligned to their element size
  const uintptr_t align = (p->precision == QEB_F64) ? 16 : 8;
  if ((reinterpret_cast<uintptr_t>(scratch) | reinterpret_cast<uintptr_t>(psi)) % align != 0) {
    qeb::set_error("%s: operands must be %d-byte aligned", who, (int)align);
    return QEB_EINVAL;
  }
  return QEB_OK;
}

extern "C" int qeb_apply_local(const qeb_local_plan* p, void* scratch, int64_t scratch_bytes,
                               const void* psi, int64_t ld, int64_t nbands,
                               const void* potential_native, const void* kinetic, void* out,
                               int64_t ldo, void* stream) {
  int rc = check_call(p, scratch, scratch_bytes, psi, ld, nbands, "apply_local");
  if (rc) return rc;
  if (nbands > 0 && (potential_native == nullptr || out == nullptr || ldo < p->npw)) {
    qeb::set_error("apply_local: null potential/output or short output leading dimension");
    return QEB_EINVAL;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == QEB_F64) {
    return launch_apply<double>(p, static_cast<C2<double>*>(scratch),
                                static_cast<const C2<double>*>(psi), ld, nbands,
                                static_cast<const double*>(potential_native),
                                static_cast<const double*>(kinetic),
                                static_cast<C2<double>*>(out), ldo, s);
  }
  return launch_apply<float>(p, static_cast<C2<float>*>(scratch),
                             static_cast<const C2<float>*>(psi), ld, nbands,
                             static_cast<const float*>(potential_native),
                             static_cast<const float*>(kinetic), static_cast<C2<float>*>(out),
                             ldo, s);
}

static int64_t round_up_256(int64_t n) { return (n + 255) / 256 * 256; }

extern "C" int64_t qeb_local_multi_scratch_bytes(int nk, const qeb_local_plan* const* plans,
                                                 const int64_t* nbands) {
  if (nk < 1 || plans == nullptr || nbands == nullptr) return -1;
  int64_t total = 0;
  for (int k = 0; k < nk; ++k) {
    const int64_t b = qeb_local_scratch_bytes(plans[k], nbands[k]);
    if (b < 0) return -1;
    total += round_up_256(b);
  }
  return total;
}

extern "C" int qeb_apply_local_multi(int nk, const qeb_local_plan* const* plans, void* scratch,
                                     int64_t scratch_bytes, const void* const* psi,
                                     const int64_t* ld_psi, const int64_t* nbands,
                                     const void* potential_native, const void* const* kinetic,
                                     void* const* out, const int64_t* ld_out, void* stream) {
  if (nk < 1 || nk > QEB_MAX_KBATCH || plans == nullptr || psi == nullptr || ld_psi == nullptr ||
      nbands == nullptr || kinetic == nullptr || out == nullptr || ld_out == nullptr) {
    qeb::set_error("apply_local_multi: 1..%d k points with non-null argument arrays",
                   QEB_MAX_KBATCH);
    return QEB_EINVAL;
  }
  const int64_t need = qeb_local_multi_scratch_bytes(nk, plans, nbands);
  if (need < 0 || scratch_bytes < need) {
    qeb::set_error("apply_local_multi: scratch of %lld bytes is below the %lld required",
                   (long long)scratch_bytes, (long long)need);
    return need < 0 ? QEB_EINVAL : QEB_ESCRATCH;
  }
  const qeb_local_plan* p0 = plans[0];
  bool fused = p0 != nullptr && p0->fast_xy >= 0 && p0->fast_z >= 0;
  void* sticks[QEB_MAX_KBATCH];
  unsigned char* cursor = static_cast<unsigned char*>(scratch);
  for (int k = 0; k < nk; ++k) {
    const qeb_local_plan* p = plans[k];
    int rc = check_call(p, cursor, qeb_local_scratch_bytes(p, nbands[k]), psi[k], ld_psi[k],
                        nbands[k], "apply_local_multi");
    if (rc) return rc;
    if (nbands[k] > 0 && (potential_native == nullptr || out[k] == nullptr || ld_out[k] < p->npw)) {
      qeb::set_error("apply_local_multi: null potential/output or short output leading dimension");
      return QEB_EINVAL;
    }
    if (nbands[k] > 65535) {
      qeb::set_error("apply_local_multi: at most 65535 bands per k point");
      return QEB_EINVAL;
    }
    if (p->nx != p0->nx || p->ny != p0->ny || p->nz != p0->nz || p->precision != p0->precision ||
        p->device != p0->device) {
      qeb::set_error("apply_local_multi: every k point must use the same grid, precision and device");
      return QEB_EINVAL;
    }
    fused = fused && p->fast_xy == p0->fast_xy && p->fast_z == p0->fast_z &&
            p->nx_pad == p0->nx_pad && p->nz_pad == p0->nz_pad;
    sticks[k] = cursor;
    cursor += round_up_256(qeb_local_scratch_bytes(p, nbands[k]));
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (fused)
    return qeb::fast_apply_multi(nk, plans, sticks, psi, ld_psi, nbands, potential_native, kinetic,
                                 out, ld_out, s,
                                 reinterpret_cast<unsigned int*>(
                                     static_cast<unsigned char*>(sticks[0]) +
                                     stick_region_bytes(plans[0], nbands[0])));
  // grids without a four-step variant: one launch sequence per k point
  for (int k = 0; k < nk; ++k) {
    const int rc = qeb_apply_local(plans[k], sticks[k],
                                   qeb_local_scratch_bytes(plans[k], nbands[k]), psi[k],
                                   ld_psi[k], nbands[k], potential_native, kinetic[k], out[k],
                                   ld_out[k], stream);
    if (rc) return rc;
  }
  return QEB_OK;
}

extern "C" int qeb_accumulate_density(const qeb_local_plan* p, void* scratch,
                                      int64_t scratch_bytes, const void* psi, int64_t ld,
                                      int64_t nbands, const double* weights, double* density,
                                      void* stream) {
  int rc = check_call(p, scratch, scratch_bytes, psi, ld, nbands, "accumulate_density");
  if (rc) return rc;
  if (nbands > 0 && (weights == nullptr || density == nullptr)) {
    qeb::set_error("accumulate_density: null weights or density");
    return QEB_EINVAL;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == QEB_F64) {
    return launch_density<double>(p, static_cast<C2<double>*>(scratch),
                                  static_cast<const C2<double>*>(psi), ld, nbands, weights,
                                  density, s);
  }
  return launch_density<float>(p, static_cast<C2<float>*>(scratch),
                               static_cast<const C2<float>*>(psi), ld, nbands, weights, density,
                               s);
}

// Same operator as qeb_apply_local, with CUDA events recorded on `stream`
// around each pass; waits for them and returns the three pass durations in
// milliseconds (pass_ms[0..2] = A, B, C).  Used by the benchmark to time
// the kernels inside its measured loop.
extern "C" int qeb_apply_local_profiled(const qeb_local_plan* p, void* scratch,
                                        int64_t scratch_bytes, const void* psi, int64_t ld,
                                        int64_t nbands, const void* potential_native,
                                        const void* kinetic, void* out, int64_t ldo,
                                        void* stream, float* pass_ms) {
  int rc = check_call(p, scratch, scratch_bytes, psi, ld, nbands, "apply_local_profiled");
  if (rc) return rc;
  if (pass_ms == nullptr || (nbands > 0 && (potential_native == nullptr || out == nullptr))) {
    qeb::set_error("apply_local_profiled: null output");
    return QEB_EINVAL;
  }
  cudaEvent_t ev[4];
  for (int i = 0; i < 4; ++i) {
    cudaError_t err = cudaEventCreate(&ev[i]);
    if (err != cudaSuccess) {
      for (int j = 0; j < i; ++j) cudaEventDestroy(ev[j]);
      return qeb::cuda_status(err, "apply_local_profiled events");
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == QEB_F64) {
    rc = launch_apply<double>(p, static_cast<C2<double>*>(scratch),
                              static_cast<const C2<double>*>(psi), ld, nbands,
                              static_cast<const double*>(potential_native),
                              static_cast<const double*>(kinetic), static_cast<C2<double>*>(out),
                              ldo, s, ev);
  } else {
    rc = launch_apply<float>(p, static_cast<C2<float>*>(scratch),
                             static_cast<const C2<float>*>(psi), ld, nbands,
                             static_cast<const float*>(potential_native),
                             static_cast<const float*>(kinetic), static_cast<C2<float>*>(out),
                             ldo, s, ev);
  }
  if (rc == QEB_OK && nbands > 0) {
    cudaError_t err = cudaEventSynchronize(ev[3]);
    for (int i = 0; i < 3 && err == cudaSuccess; ++i) err = cudaEventElapsedTime(&pass_ms[i], ev[i], ev[i + 1]);
    rc = qeb::cuda_status(err, "apply_local_profiled timing");
  } else if (rc == QEB_OK) {
    pass_ms[0] = pass_ms[1] = pass_ms[2] = 0.0f;
  }
  for (int i = 0; i < 4; ++i) cudaEventDestroy(ev[i]);
  return rc;
}
