// Davidson column kernels: QE g_psi preconditioner, column norms, inner
// products, normalisation and residual formation.
//
// Reference: qepy_pw/_native_fft.pyx qe_precondition (:852-899),
// column_squared_norms (:1153-1190), subtract_band_energies (:1193-1234),
// column_inner_products (:1237-1291), column_diagonal_expectations
// (:1294-1343), normalize_selected_columns (:1495-1530).
// Column reductions accumulate in FP64 whatever the vector precision, one
// block per column with a fixed-order tree, so they are deterministic.
#include "qeb_common.cuh"
#include "../../include/qe_b200.h"

using qeb::C2;

namespace {

constexpr int kReduceThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* shared) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (lane == 0) shared[warp] = v;
  __syncthreads();
  double total = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) total += shared[w];
  }
  __syncthreads();
  return total;
}

// mode 0: sum |v|^2; mode 1: sum diag |v|^2; mode 2: sum conj(l) r (complex)
template <typename T, int MODE>
__global__ void __launch_bounds__(kReduceThreads) column_reduce(
    int64_t rows, const C2<T>* __restrict__ left, int64_t ldl, const C2<T>* __restrict__ right,
    int64_t ldr, const double* __restrict__ diag, double* __restrict__ out) {
  __shared__ double shared[2][32];
  const int64_t col = blockIdx.x;
  const C2<T>* l = left + col * ldl;
  double re = 0.0, im = 0.0;
  if (MODE == 2) {
    const C2<T>* r = right + col * ldr;
    for (int64_t g = threadIdx.x; g < rows; g += blockDim.x) {
      const C2<T> a = l[g], b = r[g];
      re += (double)a.re * b.re + (double)a.im * b.im;
      im += (double)a.re * b.im - (double)a.im * b.re;
    }
  } else {
    for (int64_t g = threadIdx.x; g < rows; g += blockDim.x) {
      const C2<T> a = l[g];
      const double m = (double)a.re * a.re + (double)a.im * a.im;
      re += (MODE == 1) ? diag[g] * m : m;
    }
  }
  re = block_sum(re, shared[0]);
  if (MODE == 2) im = block_sum(im, shared[1]);
  if (threadIdx.x == 0) {
    if (MODE == 2) {
      out[2 * col] = re;
      out[2 * col + 1] = im;
    } else {
      out[col] = re;
    }
  }
}

// x = 2 (H_GG - e_b) [Ry], d = (1 + x + sqrt(1 + (x - 1)^2)) / 2, out = 2 r / d
template <typename T>
__global__ void precondition_kernel(int64_t rows, int64_t cols, const C2<T>* __restrict__ r,
                                    int64_t ldr, const double* __restrict__ e,
                                    const double* __restrict__ diag, C2<T>* __restrict__ out,
                                    int64_t ldo) {
  const int64_t total = rows * cols;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / rows, g = i - b * rows;
    const double x = 2.0 * (diag[g] - e[b]);
    const double d = 0.5 * (1.0 + x + sqrt(1.0 + (x - 1.0) * (x - 1.0)));
    const double s = 2.0 / d;
    const C2<T> v = r[g + b * ldr];
    out[g + b * ldo] = qeb::mk<T>((T)(s * (double)v.re), (T)(s * (double)v.im));
  }
}

// out[:, j] = v[:, sel[j]] / sqrt(norms2[sel[j]])
template <typename T>
__global__ void normalize_kernel(int64_t rows, int64_t cols, const C2<T>* __restrict__ v,
                                 int64_t ldv, const double* __restrict__ norms2,
                                 const int64_t* __restrict__ sel, C2<T>* __restrict__ out,
                                 int64_t ldo) {
  const int64_t total = rows * cols;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = i / rows, g = i - j * rows;
    const int64_t src = sel ? sel[j] : j;
    const double s = 1.0 / sqrt(norms2[src]);
    const C2<T> a = v[g + src * ldv];
    out[g + j * ldo] = qeb::mk<T>((T)(s * (double)a.re), (T)(s * (double)a.im));
  }
}

// r[:, b] -= e[b] v[:, b]
template <typename T>
__global__ void subtract_kernel(int64_t rows, int64_t cols, C2<T>* __restrict__ r, int64_t ldr,
                                const C2<T>* __restrict__ v, int64_t ldv,
                                const double* __restrict__ e) {
  const int64_t total = rows * cols;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / rows, g = i - b * rows;
    const C2<T> a = v[g + b * ldv];
    C2<T>& t = r[g + b * ldr];
    const T eb = (T)e[b];
    t.re -= eb * a.re;
    t.im -= eb * a.im;
  }
}

int grid_for(int64_t total) {
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  return (int)(blocks < 1 ? 1 : blocks);
}

bool bad(int64_t rows, int64_t cols, int64_t ld) { return rows < 0 || cols < 0 || ld < rows; }

}  // namespace

#define QEB_DISPATCH(prec, call_f64, call_f32)                      \
  do {                                                              \
    if ((prec) == QEB_F64) {                                        \
      call_f64;                                                     \
    } else if ((prec) == QEB_F32) {                                 \
      call_f32;                                                     \
    } else {                                                        \
      qeb::set_error("unknown precision %d", (int)(prec));          \
      return QEB_EINVAL;                                            \
    }                                                               \
  } while (0)

extern "C" int qeb_column_squared_norms(int precision, int64_t rows, int64_t cols,
                                        const void* v, int64_t ld, double* out, void* stream) {
  if (bad(rows, cols, ld) || (cols > 0 && (v == nullptr || out == nullptr))) {
    qeb::set_error("column_squared_norms: invalid arguments");
    return QEB_EINVAL;
  }
  if (cols == 0) return QEB_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  QEB_DISPATCH(precision,
               (column_reduce<double, 0><<<(unsigned)cols, kReduceThreads, 0, s>>>(
                   rows, static_cast<const C2<double>*>(v), ld, nullptr, 0, nullptr, out)),
               (column_reduce<float, 0><<<(unsigned)cols, kReduceThreads, 0, s>>>(
                   rows, static_cast<const C2<float>*>(v), ld, nullptr, 0, nullptr, out)));
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "column_squared_norms");
}

extern "C" int qeb_column_diagonal_expectations(int precision, int64_t rows, int64_t cols,
                                                const void* v, int64_t ld, const double* diag,
                                                double* out, void* stream) {
  if (bad(rows, cols, ld) || (cols > 0 && (v == nullptr || out == nullptr || diag == nullptr))) {
    qeb::set_error("column_diagonal_expectations: invalid arguments");
    return QEB_EINVAL;
  }
  if (cols == 0) return QEB_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  QEB_DISPATCH(precision,
               (column_reduce<double, 1><<<(unsigned)cols, kReduceThreads, 0, s>>>(
                   rows, static_cast<const C2<double>*>(v), ld, nullptr, 0, diag, out)),
               (column_reduce<float, 1><<<(unsigned)cols, kReduceThreads, 0, s>>>(
                   rows, static_cast<const C2<float>*>(v), ld, nullptr, 0, diag, out)));
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "column_diagonal_expectations");
}

extern "C" int qeb_column_inner_products(int precision, int64_t rows, int64_t cols,
                                         const void* left, int64_t ldl, const void* right,
                                         int64_t ldr, double* out_complex, void* stream) {
  if (bad(rows, cols, ldl) || ldr < rows ||
      (cols > 0 && (left == nullptr || right == nullptr || out_complex == nullptr))) {
    qeb::set_error("column_inner_products: invalid arguments");
    return QEB_EINVAL;
  }
  if (cols == 0) return QEB_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  QEB_DISPATCH(precision,
               (column_reduce<double, 2><<<(unsigned)cols, kReduceThreads, 0, s>>>(
                   rows, static_cast<const C2<double>*>(left), ldl,
                   static_cast<const C2<double>*>(right), ldr, nullptr, out_complex)),
               (column_reduce<float, 2><<<(unsigned)cols, kReduceThreads, 0, s>>>(
                   rows, static_cast<const C2<float>*>(left), ldl,
                   static_cast<const C2<float>*>(right), ldr, nullptr, out_complex)));
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "column_inner_products");
}

extern "C" int qeb_precondition(int precision, int64_t rows, int64_t cols, const void* residuals,
                                int64_t ldr, const double* eigenvalues, const double* diagonal,
                                void* out, int64_t ldo, void* stream) {
  if (bad(rows, cols, ldr) || ldo < rows ||
      (cols > 0 && (!residuals || !eigenvalues || !diagonal || !out))) {
    qeb::set_error("precondition: invalid arguments");
    return QEB_EINVAL;
  }
  if (cols == 0 || rows == 0) return QEB_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = grid_for(rows * cols);
  QEB_DISPATCH(precision,
               (precondition_kernel<double><<<blocks, 256, 0, s>>>(
                   rows, cols, static_cast<const C2<double>*>(residuals), ldr, eigenvalues,
                   diagonal, static_cast<C2<double>*>(out), ldo)),
               (precondition_kernel<float><<<blocks, 256, 0, s>>>(
                   rows, cols, static_cast<const C2<float>*>(residuals), ldr, eigenvalues,
                   diagonal, static_cast<C2<float>*>(out), ldo)));
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "precondition");
}

extern "C" int qeb_normalize_columns(int precision, int64_t rows, int64_t cols, const void* v,
                                     int64_t ldv, const double* norms2, const int64_t* selected,
                                     void* out, int64_t ldo, void* stream) {
  if (rows < 0 || cols < 0 || ldo < rows || ldv < rows ||
      (cols > 0 && (!v || !norms2 || !out))) {
    qeb::set_error("normalize_columns: invalid arguments");
    return QEB_EINVAL;
  }
  if (cols == 0 || rows == 0) return QEB_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = grid_for(rows * cols);
  QEB_DISPATCH(precision,
               (normalize_kernel<double><<<blocks, 256, 0, s>>>(
                   rows, cols, static_cast<const C2<double>*>(v), ldv, norms2, selected,
                   static_cast<C2<double>*>(out), ldo)),
               (normalize_kernel<float><<<blocks, 256, 0, s>>>(
                   rows, cols, static_cast<const C2<float>*>(v), ldv, norms2, selected,
                   static_cast<C2<float>*>(out), ldo)));
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "normalize_columns");
}

extern "C" int qeb_subtract_band_energies(int precision, int64_t rows, int64_t cols,
                                          void* residual, int64_t ldr, const void* v,
                                          int64_t ldv, const double* energies, void* stream) {
  if (bad(rows, cols, ldr) || ldv < rows || (cols > 0 && (!residual || !v || !energies))) {
    qeb::set_error("subtract_band_energies: invalid arguments");
    return QEB_EINVAL;
  }
  if (cols == 0 || rows == 0) return QEB_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = grid_for(rows * cols);
  QEB_DISPATCH(precision,
               (subtract_kernel<double><<<blocks, 256, 0, s>>>(
                   rows, cols, static_cast<C2<double>*>(residual), ldr,
                   static_cast<const C2<double>*>(v), ldv, energies)),
               (subtract_kernel<float><<<blocks, 256, 0, s>>>(
                   rows, cols, static_cast<C2<float>*>(residual), ldr,
                   static_cast<const C2<float>*>(v), ldv, energies)));
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "subtract_band_energies");
}

namespace {

// diag[g] += m * Re sum_i coupled[g, i] conj(beta[g, i])
template <typename T>
__global__ void projector_diagonal_kernel(int64_t rows, int64_t channels,
                                          const C2<T>* __restrict__ coupled, int64_t ldc,
                                          const C2<T>* __restrict__ beta, int64_t ldb,
                                          double multiplicity, double* __restrict__ diag) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < rows;
       g += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int64_t i = 0; i < channels; ++i) {
      const C2<T> c = coupled[g + i * ldc], b = beta[g + i * ldb];
      acc += (double)c.re * b.re + (double)c.im * b.im;
    }
    diag[g] += multiplicity * acc;
  }
}

}  // namespace

extern "C" int qeb_accumulate_projector_diagonal(int precision, int64_t rows, int64_t channels,
                                                 const void* coupled, int64_t ldc,
                                                 const void* beta, int64_t ldb,
                                                 double multiplicity, double* diagonal,
                                                 void* stream) {
  if (rows < 0 || channels < 0 || ldc < rows || ldb < rows ||
      (rows > 0 && channels > 0 && (!coupled || !beta || !diagonal))) {
    qeb::set_error("accumulate_projector_diagonal: invalid arguments");
    return QEB_EINVAL;
  }
  if (rows == 0 || channels == 0) return QEB_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = grid_for(rows);
  QEB_DISPATCH(precision,
               (projector_diagonal_kernel<double><<<blocks, 256, 0, s>>>(
                   rows, channels, static_cast<const C2<double>*>(coupled), ldc,
                   static_cast<const C2<double>*>(beta), ldb, multiplicity, diagonal)),
               (projector_diagonal_kernel<float><<<blocks, 256, 0, s>>>(
                   rows, channels, static_cast<const C2<float>*>(coupled), ldc,
                   static_cast<const C2<float>*>(beta), ldb, multiplicity, diagonal)));
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "accumulate_projector_diagonal");
}
