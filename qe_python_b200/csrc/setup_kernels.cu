// Per-k-point projector construction and density symmetrisation on the GPU.
//
// qeb_projector_basis: the species projector columns
//   beta_lm(k+G) = (-i)^l Y_lm(k+G) beta_l(|k+G|)
// with beta_l(q) from a dq-spaced radial table by QE's four-point Lagrange
// interpolation and the real harmonics of QE's ylmr2 for l <= 2
// (qepy_pw/upf.py:483-556, _native_fft.pyx:1556-1600, 1603-1661,
// 1702-1791).  One thread per plane wave writes every channel of its row.
//
// qeb_symmetrize_density: the real-space average of a density over the
// space-group operations (qepy_pw/symmetry.py:28-238): for every grid point
// the operations' transformed points are gathered in the operations' order,
// summed in FP64 and divided by the number of operations.  The transformed
// coordinate along axis b is (offset_b + sum_a coeff_ab i_a) mod n_b with
// integer offsets and coefficients prepared on the host (the translation
// times n_b, and M_ab n_b / n_a).  The whole grid (nx ny nz doubles) stays
// in L2 on the benchmark cells, so the gathers are L2 reads.
//
// qeb_random_trials: the random starting wavefunctions of the first SCF
// iteration, amp e^(2 pi i phase) / (1 + 2 T(k+G)) with T the basis's
// kinetic table (Ha) and amp, phase the QE randy stream's pairs (qepy_pw/pw/scf.py:853-870), from the stream's
// integer values (qeb_qe_random_draws): each draw is value / 714025 in
// IEEE double, as on the host.
#include <cuda_runtime.h>
#include <cuComplex.h>

#include "qeb_common.cuh"
#include "../../include/qe_b200.h"

namespace {

constexpr int kMaxOps = 96;
constexpr int kMaxChannels = 64;

struct SymTerms {
  int nops;
  int offset[kMaxOps][3];      // [op][b]
  int coeff[kMaxOps][3][3];    // [op][a][b]
};

__global__ void symmetrize_kernel(int nx, int ny, int nz, const __grid_constant__ SymTerms t,
                                  const double* __restrict__ in, double* __restrict__ out) {
  const int64_t total = (int64_t)nx * ny * nz;
  const int n[3] = {nx, ny, nz};
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int iz = (int)(p % nz);
    const int iy = (int)((p / nz) % ny);
    const int ix = (int)(p / ((int64_t)nz * ny));
    const int i[3] = {ix, iy, iz};
    double sum = 0.0;
    for (int op = 0; op < t.nops; ++op) {
      int target[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        int64_t v = t.offset[op][b];
#pragma unroll
        for (int a = 0; a < 3; ++a) v += (int64_t)t.coeff[op][a][b] * i[a];
        v %= n[b];
        if (v < 0) v += n[b];
        target[b] = (int)v;
      }
      sum += in[((int64_t)target[0] * ny + target[1]) * nz + target[2]];
    }
    out[p] = sum / (double)t.nops;
  }
}

struct Channels {
  int count;
  int radial[kMaxChannels];  // radial-table column of the channel
  int l[kMaxChannels];
  int m[kMaxChannels];       // QE ylmr2 order within l
};

// QE's four-point Lagrange interpolation of a dq table at q.
__device__ __forceinline__ double lagrange4(const double* table, int64_t rows, int column,
                                            int columns, double q, double inv_dq) {
  const double scaled = q * inv_dq;
  int64_t lower = (int64_t)floor(scaled);
  if (lower < 0) lower = 0;
  if (lower > rows - 4) lower = rows - 4;
  const double f = scaled - (double)lower;
  const double u = 1.0 - f, v = 2.0 - f, w = 3.0 - f;
  const double* t = table + lower * columns + column;
  return t[0] * u * v * w / 6.0 + t[columns] * f * v * w / 2.0 -
         t[2 * columns] * f * u * w / 2.0 + t[3 * columns] * f * u * v / 6.0;
}

// Real spherical harmonics of QE's ylmr2 for l <= 2 at the unit vector
// (x, y, z); m indexes QE's order within l.
__device__ __forceinline__ double real_harmonic(int l, int m, double x, double y, double z) {
  const double pi = 3.14159265358979323846;
  if (l == 0) return 1.0 / sqrt(4.0 * pi);
  if (l == 1) {
    const double c = sqrt(3.0 / (4.0 * pi));
    return m == 0 ? c * z : (m == 1 ? -c * x : -c * y);
  }
  const double c = sqrt(5.0 / (4.0 * pi));
  switch (m) {
    case 0: return c * 0.5 * (3.0 * z * z - 1.0);
    case 1: return -c * sqrt(3.0) * z * x;
    case 2: return -c * sqrt(3.0) * z * y;
    case 3: return c * 0.5 * sqrt(3.0) * (x * x - y * y);
    default: return c * sqrt(3.0) * x * y;
  }
}

__global__ void projector_basis_kernel(int64_t npw, const double* __restrict__ kg,
                                       const double* __restrict__ table, int64_t rows,
                                       int columns, double inv_dq,
                                       const __grid_constant__ Channels ch, double2* beta,
                                       int64_t ldb) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < npw;
       g += (int64_t)gridDim.x * blockDim.x) {
    const double kx = kg[g], ky = kg[npw + g], kz = kg[2 * npw + g];
    const double q = sqrt(kx * kx + ky * ky + kz * kz);
    double x = 0.0, y = 0.0, z = 1.0;
    if (q > 1.0e-14) {
      const double inv = 1.0 / q;
      x = kx * inv, y = ky * inv, z = kz * inv;
    }
    for (int c = 0; c < ch.count; ++c) {
      const double value =
          lagrange4(table, rows, ch.radial[c], columns, q, inv_dq) * real_harmonic(ch.l[c], ch.m[c], x, y, z);
      // (-i)^l: 1, -i, -1
      double2 out;
      if (ch.l[c] == 0) out = make_double2(value, 0.0);
      else if (ch.l[c] == 1) out = make_double2(0.0, -value);
      else out = make_double2(-value, 0.0);
      beta[g + c * ldb] = out;
    }
  }
}

template <typename Out>
__device__ __forceinline__ void store_trial(Out* out, int64_t at, double re, double im);

template <>
__device__ __forceinline__ void store_trial<double2>(double2* out, int64_t at, double re,
                                                     double im) {
  out[at] = make_double2(re, im);
}

template <>
__device__ __forceinline__ void store_trial<float2>(float2* out, int64_t at, double re,
                                                    double im) {
  out[at] = make_float2((float)re, (float)im);
}

// One thread per (plane wave, band) entry, plane waves fastest, so the two
// int32 inputs and the output are read and written coalesced.
template <typename Out>
__global__ void random_trials_kernel(int64_t npw, int64_t bands, const int32_t* __restrict__ first,
                                     const int32_t* __restrict__ second,
                                     const double* __restrict__ kinetic, Out* __restrict__ out,
                                     int64_t ldo) {
  const double two_pi = 6.283185307179586;
  const int64_t total = npw * bands;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = e / npw;
    const int64_t g = e - b * npw;
    const double amp = (double)first[e] / 714025.0;
    const double phase = (double)second[e] / 714025.0;
    double s, c;
    sincos(two_pi * phase, &s, &c);
    const double den = 1.0 + 2.0 * kinetic[g];
    store_trial(out, g + b * ldo, (amp * c) / den, (amp * s) / den);
  }
}

// Grid-stride launches: at most 8 blocks per SM of a 148-SM B200.
int grid_blocks(int64_t total, int threads) {
  const int64_t want = (total + threads - 1) / threads;
  const int64_t cap = 8 * 148;
  return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace

extern "C" int qeb_symmetrize_density(int nx, int ny, int nz, int nops, const int* offsets,
                                      const int* coefficients, const void* density_in,
                                      void* density_out, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || nops < 1 || offsets == nullptr || coefficients == nullptr ||
      density_in == nullptr || density_out == nullptr) {
    qeb::set_error("symmetrize_density: invalid arguments");
    return QEB_EINVAL;
  }
  if (nops > kMaxOps) {
    qeb::set_error("symmetrize_density: %d operations exceed the %d supported", nops, kMaxOps);
    return QEB_EUNSUPPORTED;
  }
  if (density_in == density_out) {
    qeb::set_error("symmetrize_density: input and output must differ");
    return QEB_EINVAL;
  }
  SymTerms t;
  t.nops = nops;
  for (int op = 0; op < nops; ++op)
    for (int b = 0; b < 3; ++b) {
      t.offset[op][b] = offsets[op * 3 + b];
      for (int a = 0; a < 3; ++a) t.coeff[op][a][b] = coefficients[(op * 3 + a) * 3 + b];
    }
  const int64_t total = (int64_t)nx * ny * nz;
  symmetrize_kernel<<<grid_blocks(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      nx, ny, nz, t, static_cast<const double*>(density_in), static_cast<double*>(density_out));
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "symmetrize_density launch");
}

extern "C" int qeb_projector_basis(int64_t npw, const void* kg, const void* table, int64_t rows,
                                   int columns, double dq, int channels,
                                   const int* channel_radial, const int* channel_l,
                                   const int* channel_m, void* beta, int64_t ldb, void* stream) {
  if (npw < 0 || rows < 4 || columns < 1 || dq <= 0.0 || channels < 0 || ldb < npw ||
      (npw > 0 && (kg == nullptr || table == nullptr || beta == nullptr))) {
    qeb::set_error("projector_basis: invalid arguments");
    return QEB_EINVAL;
  }
  if (channels > kMaxChannels) {
    qeb::set_error("projector_basis: %d channels exceed the %d supported", channels, kMaxChannels);
    return QEB_EUNSUPPORTED;
  }
  Channels ch;
  ch.count = channels;
  for (int c = 0; c < channels; ++c) {
    if (channel_radial[c] < 0 || channel_radial[c] >= columns || channel_l[c] < 0 ||
        channel_l[c] > 2 || channel_m[c] < 0 || channel_m[c] > 2 * channel_l[c]) {
      qeb::set_error("projector_basis: channel %d has an invalid (radial, l, m)", c);
      return QEB_EINVAL;
    }
    ch.radial[c] = channel_radial[c];
    ch.l[c] = channel_l[c];
    ch.m[c] = channel_m[c];
  }
  if (npw == 0 || channels == 0) return QEB_OK;
  projector_basis_kernel<<<grid_blocks(npw, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
      npw, static_cast<const double*>(kg), static_cast<const double*>(table), rows, columns,
      1.0 / dq, ch, static_cast<double2*>(beta), ldb);
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "projector_basis launch");
}

extern "C" int qeb_random_trials(int64_t npw, int64_t bands, const void* first,
                                 const void* second, const void* kinetic, void* out, int64_t ldo,
                                 int out_complex64, void* stream) {
  if (npw < 0 || bands < 0 || ldo < npw ||
      (npw * bands > 0 && (first == nullptr || second == nullptr || kinetic == nullptr ||
                           out == nullptr))) {
    qeb::set_error("random_trials: invalid arguments");
    return QEB_EINVAL;
  }
  if (npw == 0 || bands == 0) return QEB_OK;
  const int blocks = grid_blocks(npw * bands, 256);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (out_complex64)
    random_trials_kernel<float2><<<blocks, 256, 0, s>>>(
        npw, bands, static_cast<const int32_t*>(first), static_cast<const int32_t*>(second),
        static_cast<const double*>(kinetic), static_cast<float2*>(out), ldo);
  else
    random_trials_kernel<double2><<<blocks, 256, 0, s>>>(
        npw, bands, static_cast<const int32_t*>(first), static_cast<const int32_t*>(second),
        static_cast<const double*>(kinetic), static_cast<double2*>(out), ldo);
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "random_trials launch");
}
