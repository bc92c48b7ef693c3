/* sdpx_b200: B200 (sm_100a) implementation of the SDPX interior-point hot path.
 *
 * Two C-ABI levels, both exported by libsdpx_b200.so:
 *
 *  1. The solver ABI of the reference (yongjunx23-del/SDPX.rs, include/sdpx.h, ABI 4): the same
 *     entry points, struct layouts, return codes and status codes, so a C caller of libsdpx
 *     relinks against this library unchanged.  Each declaration cites the reference line it
 *     replaces.  The hot path (NT scaling, Schur assembly, dense Cholesky, solves, refinement,
 *     step lengths) runs on the GPU; setup (copying, Ruiz equilibration) runs on the host.
 *
 *  2. Kernel-level entry points (sdpxg_*) for a host that keeps its own interior-point driver
 *     (the Rust solver's KKTSolver / DirectLDLSolver / Cone seams).  They take host pointers,
 *     run one hot-path operation on the context's stream and return when it is complete.
 *
 * Conventions shared with the reference (include/sdpx.h:8-17): inputs are copied; indices are
 * zero based, sorted and unique within each CSC column; P is upper triangular; PSD entries use
 * the upper triangle in column order with off-diagonal entries scaled by sqrt(2).
 * Return codes: 0 OK, 1 invalid input, 2 unsupported, 3 busy, 4 poisoned, 5 internal error
 * (the reference's "panic": an exception caught at the boundary), 6 insufficient output
 * capacity, 7 no solved result.  The last error message is thread-local.
 *
 * Supported subset: precision_bits 53 (binary64), PSD triangle cones of order <= 64 and
 * nonnegative orthants, sampled blocks with dim = 1, kkt_form 0 (auto) or 2 (condensed).  Other
 * inputs return 2 (unsupported) with a message.
 */
#ifndef SDPX_B200_H
#define SDPX_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define SDPX_ABI_VERSION 4u
#define SDPX_PREPROCESS_RUIZ 1u
#define SDPX_PREPROCESS_PRESOLVE 2u
#define SDPX_PREPROCESS_CHORDAL 4u
#define SDPX_PREPROCESS_ALL 7u

/* ---- solver ABI: layouts identical to the reference (include/sdpx.h:25-81) ---- */
typedef struct sdpx_handle sdpx_handle;
/* include/sdpx.h:26 -- kind 0 = f64 array, 1 = decimal strings */
typedef struct {
  uint32_t kind;
  uint32_t reserved;
  uint64_t count;
  const double *f64;
  const char *const *decimal;
} sdpx_scalars;
/* include/sdpx.h:27 */
typedef struct {
  uint64_t rows, cols, nnz;
  const uint64_t *colptr, *rowval;
  sdpx_scalars values;
} sdpx_csc;
/* include/sdpx.h:39 -- kind 3 = PSD triangle (dim = matrix order) */
typedef struct {
  uint32_t kind, reserved;
  uint64_t dim;
  sdpx_scalars alpha;
} sdpx_cone;
/* include/sdpx.h:47-50 */
typedef struct {
  uint64_t row_start, column_start, dim, basis_rows, basis_cols;
  sdpx_scalars basis, weights;
} sdpx_sampled_block;
/* include/sdpx.h:51-66 (88 bytes on 64-bit) */
typedef struct {
  uint32_t abi_version, struct_size, precision_bits, max_iter;
  uint32_t verbose, preprocessing_flags, max_threads, kkt_form;
  uint32_t reserved_0;
  double time_limit;
  const char *tol_gap_abs, *tol_gap_rel, *tol_feas, *tol_infeas_abs, *tol_infeas_rel;
} sdpx_settings;
/* include/sdpx.h:67-75 (112 bytes on 64-bit) */
typedef struct {
  uint32_t abi_version, struct_size, status, iterations;
  uint32_t working_bits, backend_threads, cone_threads, kkt_form;
  uint32_t reserved_0;
  uint64_t n, m;
  double solve_time, objective, dual_objective, primal_residual, dual_residual, gap_abs, gap_rel;
} sdpx_info;

/* include/sdpx.h:82 (ffi/src/lib.rs:586-593) */
int32_t sdpx_default_settings_v4(sdpx_settings *out);
#define sdpx_default_settings sdpx_default_settings_v4
/* include/sdpx.h:86 (ffi/src/lib.rs:720-723): always 1, one GPU per handle */
int32_t sdpx_mpi_world_size(void);
/* include/sdpx.h:87 (ffi/src/lib.rs:594-607) */
int32_t sdpx_prepare(const sdpx_csc *P, const sdpx_scalars *q, const sdpx_csc *A,
                     const sdpx_scalars *b, const sdpx_cone *cones, uint64_t cone_count,
                     const sdpx_settings *settings, sdpx_handle **out);
/* include/sdpx.h:90 (ffi/src/lib.rs:608-658): factor-authoritative sampled blocks.  Blocks with
 * dim = 1 (columns weight_k svec(q_k q_k')) run on the GPU's Gram form with the given basis and
 * weights (scaled by the equilibration); matrix-valued blocks (dim > 1) return 2. */
int32_t sdpx_prepare_sampled(const sdpx_csc *P, const sdpx_scalars *q, const sdpx_csc *A_linear,
                             const sdpx_scalars *b, const sdpx_cone *cones, uint64_t cone_count,
                             const sdpx_settings *settings, const sdpx_sampled_block *blocks,
                             uint64_t block_count, sdpx_handle **out);
/* include/sdpx.h:91 (ffi/src/lib.rs:660-663) */
int32_t sdpx_solve(sdpx_handle *handle);
/* include/sdpx.h:97 (ffi/src/lib.rs:664-670) */
int32_t sdpx_update(sdpx_handle *handle, const sdpx_scalars *q, const sdpx_scalars *b);
/* include/sdpx.h:98 (ffi/src/lib.rs:671-680) */
int32_t sdpx_get_info(sdpx_handle *handle, sdpx_info *out);
/* include/sdpx.h:103 (ffi/src/lib.rs:689-703) */
int32_t sdpx_get_solver_name(sdpx_handle *handle, char *out, uint64_t capacity,
                             uint64_t *required);
/* include/sdpx.h:109 (ffi/src/lib.rs:722-735): x[n], z[m], s[m], 6 summary scalars */
int32_t sdpx_result_f64(sdpx_handle *handle, double *out, uint64_t capacity, uint64_t *required);
/* include/sdpx.h:110 (ffi/src/lib.rs:736-752) */
int32_t sdpx_result_decimal(sdpx_handle *handle, char *out, uint64_t capacity,
                            uint64_t *required);
/* include/sdpx.h:113 (ffi/src/lib.rs:753-768) */
uint64_t sdpx_last_error(char *out, uint64_t capacity);
/* include/sdpx.h:114 (ffi/src/lib.rs:769-786) */
int32_t sdpx_destroy(sdpx_handle *handle);

/* ---- B200 extensions of the solver ABI ---- */
/* Per-phase wall times (seconds) of the last solve, in the order scale, assemble, factor,
 * kkt_solve, step, residual, other; and counters (factorizations, kkt solves, outer and inner
 * refinement steps).  Counterpart of the reference's SDPX_PROFILE phase receipt
 * (src/receipt.rs:104-160).  times needs 7 doubles, counts 4 uint64. */
int32_t sdpx_b200_phase_times(sdpx_handle *handle, double *times, uint64_t *counts);
/* KKT solves of the last solve whose two-level refinement ran on the device (one CUDA graph with
 * WHILE nodes driven by control kernels, one host read per solve: the default when graphs are on)
 * and those driven from the host (a host read per refinement step: graphs off, kernel timing on,
 * or ir_max_iter > 64).  Both run the same kernels in the same order. */
int32_t sdpx_b200_kkt_paths(sdpx_handle *handle, uint64_t *device_driven, uint64_t *host_driven);
/* Enable (on != 0) or disable CUDA-event timing of the device phases of later solves and reset
 * the totals.  Events are recorded on the handle's stream around each phase: NT scaling,
 * Schur assembly, factorisation, triangular solves, cone congruences, step lengths, the
 * Schur matvec and the inverse of the factor, in that order (no counterpart in the reference, which has no device). */
int32_t sdpx_b200_set_kernel_timing(sdpx_handle *handle, int32_t on);
/* Totals since the last reset: ms[9] milliseconds and counts[9] timed regions per phase (the
 * seven above, then the explicit inverse of the factor, then the split-precision products and
 * block assembly of the split form). */
int32_t sdpx_b200_kernel_times(sdpx_handle *handle, double *ms, uint64_t *counts);
/* Number of CUDA kernels this library has launched in this process (all handles). */
uint64_t sdpx_b200_launch_count(void);
/* Number of device memory blocks this library has obtained in this process (from its cache of
 * released blocks or from cudaMalloc; all handles).  A call that allocates nothing leaves it
 * unchanged.  No counterpart in the reference (it has no device memory). */
uint64_t sdpx_b200_device_allocations(void);
/* Measurement of the INT8 tensor-core GEMM (k_i8_mod_gemm, used by the exact RNS products and
 * the split-precision products): on != 0 times every later launch with CUDA events on its stream
 * (synchronising the host: measurement runs only) and resets the totals.  No counterpart in the
 * reference (it has no device). */
int32_t sdpx_b200_set_i8_timing(int32_t on);
/* Totals since the last sdpx_b200_set_i8_timing: milliseconds, INT8 operations executed (2 per
 * multiply-add over the padded tiles), algorithmic INT8 operations (2 m n k per digit pair and
 * modulus), launches. */
int32_t sdpx_b200_i8_times(double *ms, double *ops, double *alg_ops, uint64_t *launches);
/* Tile configuration of the INT8 tensor-core GEMM: -1 (default) autotuned -- the first launch of
 * each shape class (digit count, power-of-two classes of the padded extents, K range and moduli)
 * times every configuration on the real operands with CUDA events and keeps the fastest; results
 * do not depend on the choice (exact integer arithmetic) -- or 0 / 1 / 2 to force a configuration
 * (0: 128 x 256 tiles for single-digit and 128 x 128 for two-digit residues, one CTA per SM;
 * 1: half-width tiles with a deeper stage ring; 2: two CTAs per SM with two-stage rings, 128 x 256
 * and 128 x 64 tiles).  SDPX_B200_AUTOTUNE=0 keeps configuration 0.  No counterpart in the
 * reference (it tunes CPU tile sizes by constant). */
int32_t sdpx_b200_i8_config(int32_t variant);
/* The autotuner's table as text (one line per shape class), in the sdpx_result_decimal style:
 * required receives the bytes needed including the terminating zero. */
int32_t sdpx_b200_i8_tuning(char *out, uint64_t capacity, uint64_t *required);
/* Bytes this library has copied host-to-device and device-to-host in this process (all
 * handles): the host-device traffic of prepare, solve and result reads. */
int32_t sdpx_b200_transfer_bytes(uint64_t *h2d, uint64_t *d2h);
/* Re-prepare an existing handle with another problem (any dimensions, cones and settings, the
 * same validation as sdpx_prepare) and keep its device state: buffers are reused and grow only,
 * so a worker that solves a stream of independent instances allocates and frees nothing per
 * instance (cudaFree would synchronise the device and stall the other workers' solves).  The
 * previous result is invalidated.  No counterpart in the reference (it has no batching). */
int32_t sdpx_b200_reprepare(sdpx_handle *handle, const sdpx_csc *P, const sdpx_scalars *q,
                            const sdpx_csc *A, const sdpx_scalars *b, const sdpx_cone *cones,
                            uint64_t cone_count, const sdpx_settings *settings);
/* Gradients of a loss L(x, z, s) of the solution with respect to the data: given dl_dx (n) and
 * optionally dl_dz, dl_ds (m; NULL = zero), writes dq (n), db (m) and, when dA is not NULL, dA
 * (nnz values on the sparsity pattern of the A passed to prepare, in its CSC order).  One solve
 * of the KKT system [P A'; A -Hs] re-factored on the device at the NT scaling of the solution
 * moved onto the central path at relative mu 1e-9 in the equilibrated coordinates (per PSD block
 * in the eigenbasis of S - Z; per orthant row the smaller of s_i, z_i at 1e-9 of the larger):
 * dq = -u, db = v, dA = -(z u' + v x') with [u; v] = K^-1 [dl_dx; dl_dz - Hs dl_ds].  Requires
 * a Solved or AlmostSolved result (else 7).  The reference has no differentiation; this is the
 * adjoint of its own KKT system. */
int32_t sdpx_b200_adjoint(sdpx_handle *handle, const double *dl_dx, const double *dl_dz,
                          const double *dl_ds, double *dq, double *db, double *dA, uint64_t nnz);
/* Capture the KKT solve's straight runs as CUDA graphs and replay them (on != 0, the default
 * unless SDPX_B200_GRAPHS=0) or launch them eagerly (on == 0); results are bitwise the same.
 * Capture pays off over the many solves of one problem; a handle re-prepared for every small
 * instance of a batch is better off eager.  No counterpart in the reference. */
int32_t sdpx_b200_set_graphs(sdpx_handle *handle, int32_t on);
/* Factorisation form of later solves: 0 plain (one FP64 dataflow Cholesky of the Schur
 * complement and its explicit inverse; the default unless SDPX_B200_FORM=split), 1 split
 * precision (Schur dimension >= 1024: the two diagonal halves factored and inverted in FP64
 * with the same pivot rule, the off-diagonal block, the trailing Schur update and the inverse's
 * off-diagonal block as Ozaki-II products on the INT8 tensor cores; refinement against the
 * unshifted FP64 Schur complement as before).  Replaces the f64 dgemm/dsyrk trailing updates
 * of DenseBlockSolver::tiled_potrf (kkt/ldl/dense_block.rs:515-594). */
int32_t sdpx_b200_set_form(sdpx_handle *handle, uint32_t form);
/* Schur forms chosen at prepare: PSD blocks whose every constraint column is rank one
 * (sigma u u', stored as the factor U and used in the Gram form S = (sigma sigma') o (U' Ginv U)^2,
 * like the reference's sampled Gram update, sampled/mod.rs:1973-2025) and blocks kept in the
 * ordinary dense-column form.  Setting SDPX_B200_GRAM=0 before prepare forces the ordinary form. */
int32_t sdpx_b200_schur_forms(sdpx_handle *handle, uint32_t *gram_blocks, uint32_t *ordinary_blocks);

/* ---- kernel-level ABI (sdpxg_*): one hot-path operation per call ---- */
typedef struct sdpxg_ctx sdpxg_ctx;
/* Create a context on CUDA device `device` (flags must be 0). */
int32_t sdpxg_ctx_create(int32_t device, uint32_t flags, sdpxg_ctx **out);
int32_t sdpxg_ctx_destroy(sdpxg_ctx *ctx);
/* Upload an already equilibrated problem: P (n x n upper CSC, may be NULL), A (m x n CSC) whose
 * rows stack the svec rows of `block_count` PSD blocks of the given orders.  Replaces the data
 * that CondensedKKTSolver::new reads (kkt/condensed/mod.rs:1279-1347). */
int32_t sdpxg_problem_upload(sdpxg_ctx *ctx, const sdpx_csc *P, const sdpx_csc *A,
                             const uint64_t *psd_orders, uint64_t block_count);
/* sdpxg_problem_upload with factor-authoritative sampled blocks (dim = 1; the layout of
 * sdpx_prepare_sampled): their columns are weight_k svec(q_k q_k') materialised into A, and the
 * Schur complement and operator use the given basis and weights exactly.  Replaces
 * CondensedKKTSolver::set_sampled_operator (kkt/mod.rs:34-135, solver/sampled/mod.rs:180). */
int32_t sdpxg_problem_upload_sampled(sdpxg_ctx *ctx, const sdpx_csc *P, const sdpx_csc *A_linear,
                                     const uint64_t *psd_orders, uint64_t block_count,
                                     const sdpx_sampled_block *blocks, uint64_t nblocks);
/* Set the scaling of every PSD block from R and R^-1 (n_j x n_j column-major per block, stacked in
 * cone order); G^-1 = R^-T R^-1 is formed on the device.  Only the Schur assembly and the cone
 * operators read it (lambda is not set).  Replaces the condensed KKT's sync of R / R^-1 from the
 * cones (kkt/condensed/kkt.rs:1077-1180) and SampledSchurWorkspace::update_with_pool's Rinv
 * (solver/sampled/mod.rs:1836-1867). */
int32_t sdpxg_set_scaling(sdpxg_ctx *ctx, const double *R, const double *Rinv);
/* NT scaling of every PSD block at (s, z) (m-length svec vectors).  Writes lambda (sum of
 * orders) when out_lambda is not NULL.  *status: 0 ok, else SDPXG_ST bits.
 * Replaces PSDTriangleCone::update_scaling (cones/psdtrianglecone.rs:311-439). */
int32_t sdpxg_nt_scale(sdpxg_ctx *ctx, const double *s, const double *z, double *out_lambda,
                       uint32_t *status);
/* Identity scaling of every block (core/solver.rs:1212 reset_scaling). */
int32_t sdpxg_identity_scaling(sdpxg_ctx *ctx);
/* Assemble the condensed Schur complement P + A' Hs^-1 A of the current scaling.  Optional
 * out_schur receives the dense n x n matrix (column-major).  Replaces
 * CondensedKKTSolver::assemble (kkt/condensed/mod.rs:1962-2147). */
int32_t sdpxg_schur_assemble(sdpxg_ctx *ctx, double *out_schur);
/* Factor Schur + shift*I with the dynamic pivot rule (dynamic != 0: pivots <= eps become
 * delta).  *status != 0 on a failed pivot.  Replaces DenseBlockSolver::refactor /
 * factor_with_shift (kkt/ldl/dense_block.rs:95-365, kkt/direct/solver.rs:758-877). */
int32_t sdpxg_factor(sdpxg_ctx *ctx, double shift, uint32_t dynamic, double eps, double delta,
                     uint32_t *status);
/* Factorisation form of this context's sdpxg_factor (0 plain, 1 split precision; see
 * sdpx_b200_set_form).  Same seam: DenseBlockSolver::refactor (kkt/ldl/dense_block.rs:95-365). */
int32_t sdpxg_set_factor_form(sdpxg_ctx *ctx, uint32_t form);
/* C = alpha op(A) op(B) + beta C in binary64 through split-precision products on the INT8 tensor
 * cores (Ozaki scheme II: rows of op(A) and columns of op(B) scaled by powers of two to integers
 * of b = 55..57 bits, residues modulo 16 coprime moduli <= 256, one tcgen05 kind::i8 GEMM per
 * modulus, Garner reconstruction in FP64).  DEVICE pointers, column-major, k <= 65536; returns
 * when C is complete; *status = SDPXG_ST_NONFINITE bit for non-finite inputs.  Replaces the f64
 * dgemm of the reference's BLAS provider on the dense factorisation's trailing updates
 * (algebra/dense/blas/traits.rs XgemmScalar, used by kkt/ldl/dense_block.rs:515-594). */
int32_t sdpxg_split_dgemm_device(sdpxg_ctx *ctx, char ta, char tb, uint64_t m, uint64_t n, uint64_t k,
                                 double alpha, const double *d_A, uint64_t lda, const double *d_B,
                                 uint64_t ldb, double beta, double *d_C, uint64_t ldc, uint32_t *status);
/* Solve the factored reduced system for ncols right-hand sides (n-length columns), refined
 * against the unshifted Schur complement.  Replaces DirectLDLSolver::solve
 * (kkt/ldl/dense_block.rs:795-850 with kkt/direct/solver.rs:1046-1125). */
int32_t sdpxg_solve_many(sdpxg_ctx *ctx, const double *rhs, double *out, uint32_t ncols);
/* No counterpart in the reference (it has no device memory to manage).  The refined reduced
 * solve of sdpxg_solve_many for callers that cannot allocate device memory at call time (a
 * host that owns all device memory through its own pool, or a latency-bound loop where a
 * cudaMalloc could synchronise the device): d_rhs and d_out are DEVICE pointers to n x ncols
 * column-major arrays, and all per-call scratch sits in one static device array of the library
 * (about 0.17 MB on every GPU that loads it).  It calls no cudaMalloc or cudaFree.  n above 4096
 * returns 2; host pointers, or no current factorization (sdpxg_factor not called since the last
 * upload or assembly), return 1.  The solve runs on the context's own stream, which is not
 * ordered after the caller's streams: the writes to d_rhs must be complete before the call (for
 * instance, synchronise the stream that produced them); d_out is complete when the call
 * returns.  The caller's current device is restored on return.  The first call on a device
 * looks up the array's address: make it before any stream capture.  Calls that overlap on the
 * GPU share the array and race. */
int32_t sdpxg_solve_noalloc(sdpxg_ctx *ctx, const double *d_rhs, double *d_out, uint32_t ncols);
/* Full condensed KKT solve [P A'; A -Hs][x; z] = [bx; bz] with the outer refinement on the
 * original operator.  Replaces CondensedKKTSolver::solve (kkt/condensed/kkt.rs:275-318). */
int32_t sdpxg_kkt_solve(sdpxg_ctx *ctx, const double *bx, const double *bz, double *x, double *z);
/* e = b - [P A'; A -Hs][x; z]; returns ||e||_inf in *norm.  Replaces residual_inner
 * (kkt/condensed/mod.rs:2631-2871). */
int32_t sdpxg_residual(sdpxg_ctx *ctx, const double *bx, const double *bz, const double *x,
                       const double *z, double *ex, double *ez, double *norm);
/* Largest alpha <= amax keeping z + alpha dz and s + alpha ds in the PSD cones, from the current
 * NT scaling; mode 1 only tests whether amax is admissible (out = amax or 0).  Replaces
 * PSDTriangleCone::step_length (cones/psdtrianglecone.rs:475-576, 1168-1231). */
int32_t sdpxg_step_length(sdpxg_ctx *ctx, const double *dz, const double *ds, double amax,
                          uint32_t mode, double *out_alpha, uint32_t *status);
/* Exact product C = op(A) op(B) of MpFloat<limbs> matrices (the reference's in-memory layout:
 * limbs u64 least significant first, i32 kind = sign * MPFR kind (2 zero, 3 regular), i32
 * exponent; 8 * limbs + 8 bytes per element), column-major with leading dimensions lda / ldb;
 * C is m x n column-major (ldc = m).  Every entry is the exact dot product rounded once to
 * 64 * limbs bits, ties to even -- bitwise MpFloat::dot_fma.  ta, tb are 'N' or 'T'; upper_only
 * computes the entries i <= j and writes zeros below.  limbs 1..16.  Non-finite operands
 * return 2 with *status = SDPXG_ST_NONFINITE.  Replaces rns_blas::gemm
 * (crates/solver/src/algebra/dense/blas/rns_blas.rs:2134-2417): the residue products run on
 * the INT8 tensor cores (primes below 2^15 as two signed-byte digits, tcgen05.mma kind::i8)
 * or, after sdpxg_rns_set_form(ctx, 1), as exact FP64 products modulo primes below 2^21; both
 * forms give the same bits. */
int32_t sdpxg_rns_gemm(sdpxg_ctx *ctx, uint32_t limbs, char ta, char tb, uint64_t m, uint64_t n,
                       uint64_t k, const void *A, uint64_t lda, const void *B, uint64_t ldb,
                       uint32_t upper_only, void *C, uint32_t *status);
/* sdpxg_rns_gemm on DEVICE buffers (A, B and C in device memory, same layouts): no host copies of
 * the operands or the result, for callers that keep MpFloat matrices resident (a factorisation's
 * trailing updates).  Runs on the context's stream and returns when C is complete; the operands
 * must be complete before the call.  Same rns_blas::gemm contract
 * (crates/solver/src/algebra/dense/blas/rns_blas.rs:2134-2417). */
int32_t sdpxg_rns_gemm_device(sdpxg_ctx *ctx, uint32_t limbs, char ta, char tb, uint64_t m,
                              uint64_t n, uint64_t k, const void *d_A, uint64_t lda,
                              const void *d_B, uint64_t ldb, uint32_t upper_only, void *d_C,
                              uint32_t *status);
/* Exact congruence C = op(A) X op(A)' of MpFloat<limbs> matrices (op(A) m x k, X k x k, host
 * buffers in the layout of sdpxg_rns_gemm; C m x m column-major): every entry is the exact sum
 * over all (a, b) of op(A)(i, a) X(a, b) op(A)(j, b), rounded once to 64 * limbs bits, ties to
 * even.  Two products per prime on the INT8 tensor cores (T = X op(A)', C = op(A) T) and one
 * CRT.  upper_only writes zeros below the diagonal.  Replaces rns_blas::congruence
 * (crates/solver/src/algebra/dense/blas/rns_blas.rs:3563-3736), the exact congruence behind the
 * MPFR PSD transforms (congruence_exact_sym). */
int32_t sdpxg_rns_congruence(sdpxg_ctx *ctx, uint32_t limbs, char ta, uint64_t m, uint64_t k,
                             const void *A, uint64_t lda, const void *X, uint64_t ldx,
                             uint32_t upper_only, void *C, uint32_t *status);
/* Exact C = A' diag(d) A (m x m) of MpFloat<limbs> arrays: A k x m column-major (leading
 * dimension lda), d k entries; every entry is the exact sum over r of A(r, i) d(r) A(r, j),
 * rounded once to 64 * limbs bits, ties to even.  One product per prime on the INT8 tensor cores
 * (left operand the residues of A's columns, right operand those residues times d's) and one CRT.
 * upper_only writes zeros below the diagonal.  Replaces rns_blas::diag_congruence
 * (crates/solver/src/algebra/dense/blas/rns_blas.rs:2990-3194). */
int32_t sdpxg_rns_diag_congruence(sdpxg_ctx *ctx, uint32_t limbs, uint64_t m, uint64_t k, const void *A,
                                  uint64_t lda, const void *d, uint32_t upper_only, void *C, uint32_t *status);
/* Exact weighted quadratic forms v[k] = sum_{i <= j} c_ij x_t Q(i, k) Q(j, k), k < kmax, with x an
 * svec of order h (t = j (j + 1) / 2 + i), c_ii = 1 and c_ij = sqrt2 (the caller's working-precision
 * constant, one MpFloat<limbs>), Q h x kmax column-major (abs_q: |Q|); each v[k] the exact sum
 * rounded once.  Replaces rns_blas::svec_quadratic (rns_blas.rs:4025-4174), the sampled adjoint's
 * exact form. */
int32_t sdpxg_rns_svec_quadratic(sdpxg_ctx *ctx, uint32_t limbs, uint64_t h, uint64_t kmax, const void *Q,
                                 uint32_t abs_q, const void *x, const void *sqrt2, void *out, uint32_t *status);
/* Exact bilinear forms out[s] = Q(:, a)' X Q(:, b) for the pairs s = (pairs[2s], pairs[2s+1]), X
 * symmetric of order h packed upper without svec factors (entry (i, j), i <= j, at
 * j (j + 1) / 2 + i), Q h x columns column-major; each the exact sum rounded once.  Replaces
 * rns_blas::symmetric_bilinear (rns_blas.rs:4175-4277). */
int32_t sdpxg_rns_symmetric_bilinear(sdpxg_ctx *ctx, uint32_t limbs, uint64_t h, uint64_t columns, const void *Q,
                                     const void *X, uint64_t npairs, const uint64_t *pairs, void *out,
                                     uint32_t *status);
/* Upper triangle of sum_b Z_b' Y_b (m x m) with Z_b = diag(d_b) Y_b rounded entrywise: block b has
 * width widths[b] and counts[b] sorted global columns (below m), its factor Y_b widths[b] x counts[b]
 * column-major; y, d and columns concatenate the blocks in order.  Every entry of the sum over all
 * blocks and rows is exact and rounded once (zeros below the diagonal).  Replaces
 * rns_blas::gemm_blocks_upper (rns_blas.rs:2656-2923); the blocks are stacked into dense operands
 * (sum of widths times m entries at most 2^28). */
int32_t sdpxg_rns_gemm_blocks_upper(sdpxg_ctx *ctx, uint32_t limbs, uint64_t m, uint64_t nblocks,
                                    const uint64_t *widths, const uint64_t *counts, const void *y, const void *d,
                                    const uint64_t *columns, void *C, uint32_t *status);
/* NT scaling of PSD blocks at MPFR width: the reference's PSDTriangleCone::update_scaling
 * (crates/solver/src/solver/cones/psdtrianglecone.rs:311-439) for MpFloat<limbs> (1..8), blocks of
 * order orders[b] <= 64 with their svec s and z concatenated (tri(n_b) entries each).  Per block:
 * L1 = chol(mat(s)), L2 = chol(mat(z)) (exact-dot Cholesky), the right singular vectors V of
 * L2' L1 by one-sided Jacobi in MpFloat arithmetic (singular values descending), and lambda (n_b),
 * Lambda^-1/2 (n_b), R = L1 V Lambda^-1/2, Rinv = Lambda^1/2 V' L1^-1 and G = R R' (upper, zeros
 * below) as n_b x n_b column-major, concatenated.  block_status[b]: 0, 1 (s or z not interior) or
 * 2 (Jacobi sweeps exhausted); a failed block's outputs are zeros.  Replaces the MPFR right SVD (algebra/dense/blas/mpfr_svd.rs,
 * mpfr_dqds.rs) behind update_scaling: V may differ in column signs, lambda, G and the
 * congruences agree. */
int32_t sdpxg_mp_nt_scale(sdpxg_ctx *ctx, uint32_t limbs, uint64_t nblocks, const uint64_t *orders,
                          const void *s, const void *z, void *lambda, void *lisqrt, void *R, void *Rinv,
                          void *G, int32_t *block_status, uint32_t *status);
/* Step-length bounds of PSD blocks at MPFR width: the reference's step_component /
 * step_length_psd_component for precisions above 64 bits (crates/solver/src/solver/cones/
 * psdtrianglecone.rs:1041-1072, 1180-1390) for MpFloat<limbs> (1..8).  Per block of order
 * orders[b] <= 64: the direction's svec d (concatenated), the scaling matrix Rx (R for a dual
 * direction, primal = 0; Rinv for a primal one, primal = 1; n_b x n_b column-major, concatenated)
 * and Lambda^-1/2 (concatenated).  Delta = Lambda^-1/2 W-congruence(mat(d)) Lambda^-1/2 with the
 * congruence exact (rounded once per entry); gamma = lambda_min(Delta) from its binary64 copy
 * (the reference's Householder/Sturm bisection, bitwise) under the a priori bound or an exact
 * Cholesky certificate of I + alpha_c Delta, else from an MpFloat Jacobi eigensolver; alpha[b] =
 * min(-1/gamma, alpha_max) for gamma < 0, else alpha_max (one MpFloat each).  path[b]: 0 a priori
 * bound, 1 certified, 2 MpFloat eigensolver, 3 eigensolver not converged (alpha 0). */
int32_t sdpxg_mp_step_length(sdpxg_ctx *ctx, uint32_t limbs, uint64_t nblocks, const uint64_t *orders,
                             uint32_t primal, const void *d, const void *Rx, const void *lisqrt,
                             const void *alpha_max, void *alpha, int32_t *path, uint32_t *status);
/* The reference's dense MPFR LDL' (ArrowLDLSolver::try_dense -> ldl_rec, kkt/ldl/arrow.rs:2609-2620,
 * 255-420, with ldl_dots leaves 156-242 and solve_unit_lower_t 430-470) of the n x n MpFloat<limbs>
 * matrix A (host, column-major, leading dimension lda; its lower triangle is read): L (n x n,
 * ld n) receives the unit lower factor in its lower triangle (the strict upper triangle holds A's
 * upper triangle, as the reference leaves it), dinv (n) receives D^-1.  Blocks up to 128 are
 * factored by exact dots rounded once (left-looking), larger ones are halved with their trailing
 * update A22 -= W21 L21' as one exact product per entry (INT8 tensor-core RNS) rounded once and
 * then subtracted; every other operation rounds once (round to nearest, ties to even).  reg:
 * NULL or two MpFloat values (eps, delta) of the pivot rule (a pivot below eps becomes delta).
 * limbs 1..8.  A zero pivot sets SDPXG_ST_PIVOT_FAIL in *status (return 0); an exact dot whose
 * exponent spread exceeds the device accumulator returns 2. */
int32_t sdpxg_mp_ldl(sdpxg_ctx *ctx, uint32_t limbs, uint64_t n, const void *A, uint64_t lda,
                     const void *reg, void *L, void *dinv, uint32_t *status);
/* The reference's exact Cholesky XpotrfScalar::xpotrf for MpFloat<limbs> (algebra/dense/blas/
 * mpfr.rs:726-789), in place on the host n x n matrix A (column-major, ld lda), uplo 'L' (lower
 * triangle stored) or 'U': left-looking, every dot exact and rounded once, the differences, the
 * square roots and the divisions rounded once (round to nearest, ties to even).  *info = 0, or
 * j + 1 when pivot j is not positive (A then holds the factor up to it), as LAPACK's potrf.
 * limbs 1..8. */
int32_t sdpxg_mp_potrf(sdpxg_ctx *ctx, uint32_t limbs, char uplo, uint64_t n, void *A, uint64_t lda,
                       int32_t *info, uint32_t *status);
/* sdpxg_mp_ldl in place on device memory: d_A (n x n, ld lda) is overwritten with L, d_dinv (n)
 * receives D^-1, d_reg NULL or (eps, delta) in device memory. */
int32_t sdpxg_mp_ldl_device(sdpxg_ctx *ctx, uint32_t limbs, uint64_t n, void *d_A, uint64_t lda,
                            const void *d_reg, void *d_dinv, uint32_t *status);
/* Residue arithmetic of the exact products of this context: 0 = INT8 tensor cores (default),
 * 1 = FP64 CUDA cores.  The reference computes its per-prime products with FP64 dgemm
 * (rns_blas.rs:447-580); the result bits do not depend on the form. */
int32_t sdpxg_rns_set_form(sdpxg_ctx *ctx, uint32_t form);
/* y = op(x) per PSD block: op 0 W, 1 W', 2 W^-1, 3 W^-T, 4 Hs = W'W, 5 Hs^-1.
 * Replaces mul_W / mul_Winv / PsdBlock::apply (cones/psdtrianglecone.rs:860-917,
 * kkt/condensed/psd.rs:1968-2027). */
int32_t sdpxg_cone_apply(sdpxg_ctx *ctx, uint32_t op, const double *x, double *y);

#ifdef __cplusplus
}
#endif
#endif /* SDPX_B200_H */
