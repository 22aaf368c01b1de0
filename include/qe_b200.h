/*
 * qe_b200 — C ABI of the B200 Kohn–Sham H|psi> / Davidson hot path.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream handle
 * (passed as void*; NULL = legacy default stream) and returns an int status:
 * 0 on success, negative on failure (see QEB_E* below; qeb_last_error()
 * returns a message for the calling thread).  Nothing throws across the ABI.
 * Device pointers are caller-owned; no call keeps a device allocation alive
 * beyond its plan object.  Complex values are interleaved (re, im) pairs
 * (complex128 = 16 bytes, complex64 = 8 bytes).  Matrices are column-major
 * ("Fortran order") with an explicit leading dimension, as qepy-pw's
 * Davidson stores them (qepy_pw/diagonalization.py:632-635).
 *
 * Each declaration names the reference interface it replaces, as
 * path:line inside the sjhong6230/QE_python (qepy-pw 1.0.2) tree.
 */
#ifndef QE_B200_H
#define QE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QEB_ABI_VERSION 1

/* precisions of a local plan */
#define QEB_F64 0 /* complex128 psi, float64 V(r) and kinetic */
#define QEB_F32 1 /* complex64 psi, float32 V(r) and kinetic */

/* status codes */
#define QEB_STATUS_OK 0
#define QEB_STATUS_EINVAL -1      /* bad shape, pointer, stride or alignment */
#define QEB_STATUS_EUNSUPPORTED -2 /* size outside what the kernels handle */
#define QEB_STATUS_ECUDA -3       /* CUDA runtime or launch error */
#define QEB_STATUS_ESCRATCH -4    /* caller scratch smaller than required */
#define QEB_STATUS_ENOPLAN -5     /* null plan */

/* Message of the last failed call on this thread. */
const char* qeb_last_error(void);
/* QEB_ABI_VERSION of the loaded library. */
int qeb_version(void);
/* Kernels launched by this library since it was loaded (all threads). */
int64_t qeb_launch_count(void);

/* Host routine: QE's randy stream as band-major (amplitude, phase) pairs
 * for the random starting wavefunctions; first/second are column-major
 * (plane_waves, bands); table (97 entries), current and seed are updated.
 * Replaces qe_random_pairs (qepy_pw/_native_fft.pyx:1411-1444). */
int qeb_qe_random_pairs(int64_t plane_waves, int64_t bands, int64_t* table, int64_t* current,
                        int64_t* seed, double* first, double* second);

/* The same stream as its integer values (each draw times 714025), for a
 * division on the device (qeb_random_trials); host code, same arguments
 * and state update as qeb_qe_random_pairs.  Replaces the draw of
 * qepy_pw/pw/scf.py:855-860 (_QERandom.pairs_by_band, :493-510). */
int qeb_qe_random_draws(int64_t plane_waves, int64_t bands, int64_t* table, int64_t* current,
                        int64_t* seed, int32_t* first, int32_t* second);

/* ------------------------------------------------------------------------
 * Local potential operator on the FFT grid (sticks / planes).
 * ---------------------------------------------------------------------- */
typedef struct qeb_local_plan qeb_local_plan;

/* Build the device index maps of one plane-wave basis on an (nx, ny, nz)
 * grid from its z-major slots z*nx*ny + x*ny + y (host int64 array, npw).
 * Replaces the per-k serial maps of LocalPotentialWorkspace.__init__
 * (qepy_pw/basis.py:510-555: z_major_slots, serial_stick_positions) and the
 * FFTW plan pair NativeFFTWPlan (qepy_pw/_native_fft.pyx:1973-2086).
 * The grid lengths must be 2-3-5 smooth (qepy_pw/basis.py:27-37). */
int qeb_local_plan_create(qeb_local_plan** plan, int nx, int ny, int nz, int64_t npw,
                          const int64_t* z_major_slots, int precision);
int qeb_local_plan_destroy(qeb_local_plan* plan);
/* info[0..7] = nx, ny, nz, npw, sticks, active y rows, precision, device;
 * with n >= 9, info[8] = K of the pruned plane pass (0: active-row plane). */
int qeb_local_plan_info(const qeb_local_plan* plan, int64_t* info, int n);
/* Bytes of caller scratch needed for nbands (the stick buffer
 * nbands*nz*sticks complex values); the role of the grid scratch argument
 * of apply_serial_spatial (qepy_pw/_native_fft.pyx:2458-2471). */
int64_t qeb_local_scratch_bytes(const qeb_local_plan* plan, int64_t nbands);

/* out[:, b] = FFT^-( V . FFT^+(psi[:, b]) )[slots] / N_r + kinetic * psi[:, b]
 * for b < nbands.  potential is the native (nz, nx, ny) real grid; kinetic
 * may be NULL.  Replaces apply_serial_spatial / apply_serial
 * (qepy_pw/_native_fft.pyx:2458-2534, 2338-2455; operator at :58-135). */
int qeb_apply_local(const qeb_local_plan* plan, void* scratch, int64_t scratch_bytes,
                    const void* psi, int64_t ld_psi, int64_t nbands,
                    const void* potential_native, const void* kinetic, void* out,
                    int64_t ld_out, void* stream);
/* qeb_apply_local with CUDA events around its three passes on `stream`;
 * waits for completion and stores the pass durations (ms) in pass_ms[0..2].
 * Benchmark instrumentation; no reference counterpart. */
int qeb_apply_local_profiled(const qeb_local_plan* plan, void* scratch, int64_t scratch_bytes,
                             const void* psi, int64_t ld_psi, int64_t nbands,
                             const void* potential_native, const void* kinetic, void* out,
                             int64_t ld_out, void* stream, float* pass_ms);

/* qeb_apply_local for nk <= 16 k points on one grid in one launch per pass
 * (grid.z = k point): plans[k], psi[k] (ld_psi[k], nbands[k] columns),
 * kinetic[k] (may be NULL), out[k] (ld_out[k]); one potential.  The k points'
 * stick buffers are carved from one scratch of qeb_local_multi_scratch_bytes()
 * bytes.  Chosen-form batching of the per-k apply_serial_spatial calls of
 * qepy_pw/pw/scf.py:3396-3411 (no counterpart in the reference).  Grids
 * without a four-step factorisation run one launch sequence per k point. */
int64_t qeb_local_multi_scratch_bytes(int nk, const qeb_local_plan* const* plans,
                                      const int64_t* nbands);
int qeb_apply_local_multi(int nk, const qeb_local_plan* const* plans, void* scratch,
                          int64_t scratch_bytes, const void* const* psi, const int64_t* ld_psi,
                          const int64_t* nbands, const void* potential_native,
                          const void* const* kinetic, void* const* out, const int64_t* ld_out,
                          void* stream);

/* Process-wide choice of how the four-step passes run (qeb_apply_local and
 * qeb_apply_local_multi on cubic grids): 0 (default) three launches, one
 * per pass; 1 one persistent cooperative launch that runs the three passes
 * of every k point with a grid barrier between them (the barrier's words
 * are the last 256 bytes of the caller's scratch; a barrier that gives up
 * after about a second records code 21 in qeb_tf32_gemm_error).  The same
 * arithmetic either way.  qeb_persistent_passes() returns the choice. */
int qeb_set_persistent_passes(int enabled);
int qeb_persistent_passes(void);

/* density[(x*ny + y)*nz + z] += sum_b weights[b] |FFT^+(psi[:, b])(x,y,z)|^2
 * (float64 accumulation; weights is a device float64 array of nbands).
 * Replaces accumulate_density_serial(_spatial)
 * (qepy_pw/_native_fft.pyx:2537-2648; operator at :137-193). */
int qeb_accumulate_density(const qeb_local_plan* plan, void* scratch, int64_t scratch_bytes,
                           const void* psi, int64_t ld_psi, int64_t nbands,
                           const double* weights, double* density, void* stream);

/* ------------------------------------------------------------------------
 * Complex GEMM: C = alpha * op(A) * B + beta * C, column-major.
 * op(A) = A (QEB_OP_N; A is M x K) or A^H (QEB_OP_C; A is K x M).
 * alpha, beta: host pointers to {re, im} doubles.  With QEB_OP_C the long
 * K dimension is split across blocks when `scratch` holds at least
 * qeb_zgemm_scratch_bytes(); partial tiles are reduced in a fixed order.
 * qeb_zgemm: complex128; qeb_cgemm: complex64 with FP32 FMA.
 * Replace projector_overlaps (ZGEMM ConjTrans, qepy_pw/_native_fft.pyx
 * :694-731), add_projector_product (ZGEMM beta=1, :782-836), the Davidson
 * reduced matrices V^H HV, V^H V and Ritz products V c, HV c
 * (qepy_pw/diagonalization.py:658-726) and coupling @ overlaps (:348).
 * ---------------------------------------------------------------------- */
#define QEB_OP_N 0
#define QEB_OP_C 1
int64_t qeb_zgemm_scratch_bytes(int opa, int M, int N, int K, int precision);
int qeb_zgemm(int opa, int M, int N, int K, const double* alpha, const void* A, int64_t lda,
              const void* B, int64_t ldb, const double* beta, void* C, int64_t ldc,
              void* scratch, int64_t scratch_bytes, void* stream);
int qeb_cgemm(int opa, int M, int N, int K, const double* alpha, const void* A, int64_t lda,
              const void* B, int64_t ldb, const double* beta, void* C, int64_t ldc,
              void* scratch, int64_t scratch_bytes, void* stream);

/* Allocation-free C = alpha * A^H * B + beta * C (complex128, A is K x M).
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc themselves (code running inside a device memory pool it does
 * not own, or a host program whose allocator is reserved for its own data).
 * The split-K partial tiles live in a 16 MiB file-scope __device__ array
 * that every GPU loading this library holds until the process exits
 * (qeb_zgemm_static_scratch_capacity() returns its size); the call itself
 * allocates nothing.  It rejects M*N > capacity/32 (two complex128 partial
 * slices must fit) with QEB_STATUS_EUNSUPPORTED.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) with that
 * device current; make that first call before any stream capture.  The
 * address is cached per device index for the life of the process, so it
 * assumes the runtime's primary context throughout: after cudaDeviceReset,
 * or with another context made current, the cached address is stale and
 * this entry point must not be called.  All
 * calls share the one array and each call overwrites every partial entry it
 * reads, so nothing needs clearing between calls; calls that overlap on the
 * GPU (different streams, or different host threads) race on the array and
 * must be serialised by the caller. */
int64_t qeb_zgemm_static_scratch_capacity(void);
int qeb_zgemm_static_scratch(int M, int N, int K, const double* alpha, const void* A,
                             int64_t lda, const void* B, int64_t ldb, const double* beta,
                             void* C, int64_t ldc, void* stream);

/* Species projector columns beta[g + c ldb] = (-i)^l Y_lm(k+G) beta_l(|k+G|)
 * (complex128, column-major) for npw plane waves: kg is (npw, 3) float64
 * column-major (k+G in bohr^-1), table is (rows, columns) float64 row-major
 * with row r at q = r dq; channel c uses table column channel_radial[c],
 * angular momentum channel_l[c] <= 2 and QE ylmr2 index channel_m[c].
 * All pointers but the channel arrays (host) are device pointers.
 * Replaces qe_cubic_interpolate + low_l_real_harmonics +
 * assemble_low_l_projectors (qepy_pw/_native_fft.pyx:1556-1600, 1603-1661,
 * 1702-1791) as called by projector_basis (qepy_pw/upf.py:483-556). */
int qeb_projector_basis(int64_t npw, const void* kg, const void* table, int64_t rows,
                        int columns, double dq, int channels, const int* channel_radial,
                        const int* channel_l, const int* channel_m, void* beta, int64_t ldb,
                        void* stream);

/* density_out[p] = (1/nops) sum_op density_in[op(p)] on an (nx, ny, nz)
 * C-order float64 grid (device pointers, in != out): op maps grid point
 * (i0, i1, i2) to ((offsets[3 op + b] + sum_a coefficients[9 op + 3 a + b]
 * i_a) mod n_b)_b, summed in operation order.  Host arrays offsets (nops x
 * 3) and coefficients (nops x 3 x 3); nops <= 96.  Replaces
 * DensitySymmetrizer.apply (qepy_pw/symmetry.py:28-238). */
int qeb_symmetrize_density(int nx, int ny, int nz, int nops, const int* offsets,
                           const int* coefficients, const void* density_in, void* density_out,
                           void* stream);

/* Random starting wavefunctions: out[g + b ldo] = amp e^(2 pi i phase) /
 * (1 + 2 kinetic[g]) with amp = first[g + b npw] / 714025 and phase =
 * second[g + b npw] / 714025 (IEEE double), stored as complex128, or
 * complex64 when out_complex64 != 0.  Device arrays: first/second int32
 * (npw x bands, column-major), kinetic float64 (npw).  Replaces
 * qepy_pw/pw/scf.py:861-869. */
int qeb_random_trials(int64_t npw, int64_t bands, const void* first, const void* second,
                      const void* kinetic, void* out, int64_t ldo, int out_complex64,
                      void* stream);

/* out = D becp for a block-diagonal D (P x P): block k covers rows/columns
 * [start[k], start[k] + size[k]) with its size x size entries row-major at
 * values + offset[k]; row_block[p] is the block of row p.  All arrays are
 * device arrays; becp/out are column-major (P, nb).  Replaces the dense
 * coupling @ overlaps product (qepy_pw/diagonalization.py:348). */
int qeb_block_coupling(int precision, int P, int nb, int nblocks, const int32_t* row_block,
                       const int32_t* start, const int32_t* size, const int64_t* offset,
                       const void* values, const void* becp, int64_t ldb, void* out,
                       int64_t ldo, void* stream);

/* ------------------------------------------------------------------------
 * Split-TF32 complex GEMM on tcgen05 tensor cores (the chosen form of the
 * projector and subspace contractions; replaces the same ZGEMM calls as
 * qeb_zgemm, in FP32 precision).
 *
 * qeb_tf32_pack turns a complex matrix into two K-major FP32 planes
 * hi = tf32(x), lo = tf32(x - hi), rows of kp = roundup(2K, 32) reals with
 * each complex value as two consecutive reals, transformed by `layout`:
 *   RAW [re, im], SWAPNEG [im, -re], NEGIM [re, -im], SWAP [im, re].
 * transposed = 0: source column r (K contiguous values, leading dim ld) is
 * packed row r; transposed = 1: source row r of a column-major rows x K
 * matrix is packed row r.  precision: QEB_F64 or QEB_F32 source.
 *
 * qeb_tf32_gemm: C = alpha (A B0^T + i A B1^T) + beta C with A (M x kp) and
 * B0, B1 (N x kp) packed operands (row strides lda, ldb floats), C complex64
 * column-major.  Each real product is hi.hi + hi.lo + lo.hi on
 * tcgen05.mma.kind::tf32 with FP32 accumulation in tensor memory.  With
 * scratch of qeb_tf32_gemm_scratch_bytes() the K range is split over CTAs.
 *   beta^H psi  : A = pack(beta, RAW), B0 = pack(psi, RAW), B1 = pack(psi, SWAPNEG)
 *   beta coupled: A = pack(beta, RAW, transposed), B0 = pack(c, NEGIM), B1 = pack(c, SWAP)
 * All waits inside the kernel are bounded; qeb_tf32_gemm_error() returns a
 * non-zero code (and clears it) if any timed out.
 * ---------------------------------------------------------------------- */
#define QEB_PACK_RAW 0
#define QEB_PACK_SWAPNEG 1
#define QEB_PACK_NEGIM 2
#define QEB_PACK_SWAP 3
int qeb_tf32_pack(int precision, int layout, int transposed, int rows, int K, const void* src,
                  int64_t ld, void* hi, void* lo, int64_t ldp, void* stream);
int64_t qeb_tf32_gemm_scratch_bytes(int M, int N, int kp);
int qeb_tf32_gemm(int M, int N, int kp, const void* a_hi, const void* a_lo, int64_t lda,
                  const void* b0_hi, const void* b0_lo, const void* b1_hi, const void* b1_lo,
                  int64_t ldb, const double* alpha, const double* beta, void* C, int64_t ldc,
                  void* scratch, int64_t scratch_bytes, void* stream);
int qeb_tf32_gemm_error(int* out);

/* ------------------------------------------------------------------------
 * Split-TF32 complex GEMM on unpacked complex64 operands (the chosen form of
 * projector_overlaps / add_projector_product, _native_fft.pyx:694-731 and
 * :782-836, and of the Davidson subspace GEMMs, diagonalization.py:658-726).
 *   C = alpha op(A) B + beta C,  op = QEB_OP_C (A^H, A is K x M) or QEB_OP_N
 * A, B, C column-major complex64.  hi/lo splitting happens in shared memory
 * inside the kernel; no packed copies.  A and B must be 16-byte aligned with
 * even leading dimensions, else QEB_STATUS_EUNSUPPORTED (the caller then uses
 * the packed path).  K = 0 is QEB_STATUS_EUNSUPPORTED (scale C instead).
 * scratch: qeb_cgemm_tf32x3_scratch_bytes() for a split K range (less or
 * none lowers the split).  Bounded waits report through
 * qeb_tf32_gemm_error().
 * ---------------------------------------------------------------------- */
int64_t qeb_cgemm_tf32x3_scratch_bytes(int op_a, int M, int N, int K);
int qeb_cgemm_tf32x3(int op_a, int M, int N, int K, const double* alpha, const void* A,
                     int64_t lda, const void* B, int64_t ldb, const double* beta, void* C,
                     int64_t ldc, void* scratch, int64_t scratch_bytes, void* stream);
/* The same with the K split chosen by the caller (splits <= 0: the built-in
 * choice, qeb_cgemm_tf32x3_default_splits); a split needs splits*M*N*8 bytes
 * of scratch, less lowers it. */
int qeb_cgemm_tf32x3_default_splits(int op_a, int M, int N, int K);
int qeb_cgemm_tf32x3_ex(int op_a, int M, int N, int K, const double* alpha, const void* A,
                        int64_t lda, const void* B, int64_t ldb, const double* beta, void* C,
                        int64_t ldc, void* scratch, int64_t scratch_bytes, int splits,
                        void* stream);

/* ------------------------------------------------------------------------
 * Davidson column kernels (precision QEB_F64 / QEB_F32 selects the vector
 * type; reductions accumulate in FP64; eigenvalues, diagonals and norms
 * are device float64 arrays).
 * ---------------------------------------------------------------------- */
/* out[b] = sum_g |v[g,b]|^2 — column_squared_norms (qepy_pw/_native_fft.pyx:1153-1190) */
int qeb_column_squared_norms(int precision, int64_t rows, int64_t cols, const void* v,
                             int64_t ld, double* out, void* stream);
/* out[b] = sum_g diag[g] |v[g,b]|^2 — column_diagonal_expectations (:1294-1343) */
int qeb_column_diagonal_expectations(int precision, int64_t rows, int64_t cols, const void* v,
                                     int64_t ld, const double* diag, double* out, void* stream);
/* out[b] = sum_g conj(l[g,b]) r[g,b] as {re, im} — column_inner_products (:1237-1291) */
int qeb_column_inner_products(int precision, int64_t rows, int64_t cols, const void* left,
                              int64_t ldl, const void* right, int64_t ldr, double* out_complex,
                              void* stream);
/* QE g_psi: x = 2(diag_g - e_b), d = (1 + x + sqrt(1 + (x-1)^2))/2,
 * out = 2 r / d — qe_precondition (:852-899) */
int qeb_precondition(int precision, int64_t rows, int64_t cols, const void* residuals,
                     int64_t ldr, const double* eigenvalues, const double* diagonal, void* out,
                     int64_t ldo, void* stream);
/* out[:, j] = v[:, sel[j]] / sqrt(norms2[sel[j]]) (sel may be NULL = identity)
 * — normalize_selected_columns (:1495-1530) */
int qeb_normalize_columns(int precision, int64_t rows, int64_t cols, const void* v, int64_t ldv,
                          const double* norms2, const int64_t* selected, void* out, int64_t ldo,
                          void* stream);
/* residual[:, b] -= energies[b] v[:, b] — subtract_band_energies (:1193-1234) */
int qeb_subtract_band_energies(int precision, int64_t rows, int64_t cols, void* residual,
                               int64_t ldr, const void* v, int64_t ldv, const double* energies,
                               void* stream);

/* diag[g] += multiplicity * Re sum_i coupled[g,i] conj(beta[g,i]) (coupled = beta D)
 * — accumulate_projector_diagonal (qepy_pw/_native_fft.pyx:734-779) */
int qeb_accumulate_projector_diagonal(int precision, int64_t rows, int64_t channels,
                                      const void* coupled, int64_t ldc, const void* beta,
                                      int64_t ldb, double multiplicity, double* diagonal,
                                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QE_B200_H */
