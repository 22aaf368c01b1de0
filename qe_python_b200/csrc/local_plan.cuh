// Plan object of the local H|psi> operator, shared by the generic
// (local_hpsi.cu) and the register four-step (local_fast.cu) kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "qeb_common.cuh"

// k points one batched local apply handles (qeb_apply_local_multi).
#define QEB_MAX_KBATCH 16

struct qeb_local_plan {
  int nx, ny, nz;
  int64_t npw;
  int nst;       // occupied (x, y) sticks
  int nay;       // active y rows
  int nx_pad;    // shared-memory row stride of the active-row plane
  int ny_pad;    // shared-memory stride of the column lines
  int nz_pad;    // shared-memory stride of the stick lines
  int precision; // QEB_F64 or QEB_F32
  int device;
  qeb::FftDesc fx, fy, fz;
  int fast_xy;   // four-step variant of nx (== ny), or -1: generic pass B
  int fast_z;    // four-step variant of nz, or -1: generic passes A and C
  // Four-step z lines: bit i set when the block of N2 consecutive points
  // [N2 i, N2 i + N2) (the values one lane holds in the D1 distribution,
  // z = j + N2 i) contains an entry's z.  The other blocks are zero on input
  // to pass A and unread on output of pass C: those passes skip their
  // shared-memory loads and stores.  (The same skip for the plane rows of
  // pass B measured 7 % slower on the 64^3 grid: 0.271 -> 0.292 ms.)
  uint32_t zmask;
  // Pruned plane of pass B (the potential apply; 64-point four-step planes,
  // n = N1 N2 with N1 = N2 = 8): when every stick's x and y lie in
  // [0, K N2) or [n - K N2, n) (K = prune_k, 2K < N1), the plane keeps only
  // the 2 K N2 rows ("slots") of those y, and the inverse line transforms
  // skip the blocks [N2 i, N2 i + N2), K <= i < N1 - K, that are zero on
  // input (the forward ones do not store them).  0: the plane of the nay
  // active rows.  QEB_PRUNE_PLANE=0 keeps every plan on the active-row plane.
  int prune_k;
  // device arrays (plan-owned)
  int32_t* entry_g;      // npw: plane-wave row, CSR-ordered by (stick, z)
  int32_t* entry_z;      // npw: z slot
  int32_t* entry_stick;  // npw: stick index
  int32_t* stick_off;    // nst + 1
  int32_t* stick_pos;    // nst: ay * nx_pad + x (shared-memory plane position)
  int32_t* ay_to_y;      // nay
  int32_t* y_to_ay;      // ny (-1 when the row holds no stick)
  int32_t* slot_pos;     // nst: slot(y) * nx_pad + x (pruned plane), or null
  int32_t* ay_to_slot;   // nay: slot of active row ay (pruned plane), or null
  void* tw;              // forward twiddles: nx, then ny, then nz entries (complex T)
};

namespace qeb {

// Four-step variant index of a line length (-1 when only the generic
// Stockham engine handles it).
int four_variant(int n);
// N1 and N2 of a four-step variant (false when it does not exist).
bool four_split(int variant, int* n1, int* n2);
// The K of the pruned plane pass of a four-step variant, or 0 when it has
// none.
int prune_k_of(int variant);

// Launchers of the four-step kernels (local_fast.cu).  Each returns QEB_OK
// or an error status; events may be null.
int fast_smem_limits(const qeb_local_plan* p);
// ``barrier``: two words of the caller's scratch for the grid barrier of the
// persistent launch (qeb_set_persistent_passes); unused otherwise.
int fast_apply(const qeb_local_plan* p, void* sticks, const void* psi, int64_t ld, int64_t nb,
               const void* potential, const void* kinetic, void* out, int64_t ldo,
               cudaStream_t stream, cudaEvent_t* events, unsigned int* barrier);
int fast_density(const qeb_local_plan* p, void* sticks, const void* psi, int64_t ld, int64_t nb,
                 const double* weights, double* density, cudaStream_t stream);
// The three passes once for nk <= QEB_MAX_KBATCH plans on one grid (same
// four-step variants, precision and device): grid.z = k point.
int fast_apply_multi(int nk, const qeb_local_plan* const* plans, void* const* sticks,
                     const void* const* psi, const int64_t* ld, const int64_t* nb,
                     const void* potential, const void* const* kinetic, void* const* out,
                     const int64_t* ldo, cudaStream_t stream, unsigned int* barrier);

}  // namespace qeb
