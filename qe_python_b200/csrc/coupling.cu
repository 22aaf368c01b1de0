// Block-diagonal projector coupling: coupled = D becp.
//
// D (P x P) is block diagonal, one block per atom (0.5 D_Ry of the species,
// qepy_pw/upf.py:541-556; the reference forms coupling @ overlaps as a dense
// product, qepy_pw/diagonalization.py:348).  Each output entry sums over its
// own block only:  out[p, b] = sum_{q in block(p)} D_blk[p - s, q - s] becp[q, b].
// Blocks: start[k], size[k], offset[k] into `values` (row-major blocks);
// row_block[p] = k.  Memory-bound: reads becp once, writes out once.
#include "qeb_common.cuh"
#include "../../include/qe_b200.h"

using qeb::C2;

namespace {

template <typename T>
__global__ void block_coupling_kernel(int P, int nb, const int32_t* __restrict__ row_block,
                                      const int32_t* __restrict__ start,
                                      const int32_t* __restrict__ size,
                                      const int64_t* __restrict__ offset,
                                      const C2<T>* __restrict__ values,
                                      const C2<T>* __restrict__ becp, int64_t ldb,
                                      C2<T>* __restrict__ out, int64_t ldo) {
  const int64_t total = (int64_t)P * nb;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(i % P);
    const int64_t b = i / P;
    const int k = row_block[p];
    const int s = start[k], n = size[k];
    const C2<T>* row = values + offset[k] + (int64_t)(p - s) * n;
    const C2<T>* col = becp + b * ldb + s;
    C2<T> acc = qeb::mk<T>(0, 0);
    for (int q = 0; q < n; ++q) acc = acc + qeb::cmul(row[q], col[q]);
    out[p + b * ldo] = acc;
  }
}

}  // namespace

extern "C" int qeb_block_coupling(int precision, int P, int nb, int nblocks,
                                  const int32_t* row_block, const int32_t* start,
                                  const int32_t* size, const int64_t* offset, const void* values,
                                  const void* becp, int64_t ldb, void* out, int64_t ldo,
                                  void* stream) {
  if (P < 0 || nb < 0 || nblocks < 0 || ldb < P || ldo < P ||
      (P > 0 && nb > 0 && (!row_block || !start || !size || !offset || !values || !becp || !out))) {
    qeb::set_error("block_coupling: invalid arguments");
    return QEB_EINVAL;
  }
  if (P == 0 || nb == 0) return QEB_OK;
  const int64_t total = (int64_t)P * nb;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == QEB_F64) {
    block_coupling_kernel<double><<<blocks, 256, 0, s>>>(
        P, nb, row_block, start, size, offset, static_cast<const C2<double>*>(values),
        static_cast<const C2<double>*>(becp), ldb, static_cast<C2<double>*>(out), ldo);
  } else if (precision == QEB_F32) {
    block_coupling_kernel<float><<<blocks, 256, 0, s>>>(
        P, nb, row_block, start, size, offset, static_cast<const C2<float>*>(values),
        static_cast<const C2<float>*>(becp), ldb, static_cast<C2<float>*>(out), ldo);
  } else {
    qeb::set_error("block_coupling: unknown precision %d", precision);
    return QEB_EINVAL;
  }
  qeb::count_launches(1);
  return qeb::cuda_status(cudaGetLastError(), "block_coupling");
}
