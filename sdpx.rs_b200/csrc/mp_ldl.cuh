// Kernels of the MPFR dense LDL' on the GPU (the reference's ArrowLDLSolver dense leaf,
// crates/solver/src/solver/kkt/ldl/arrow.rs:156-470), on MpFloat<N> arrays in device memory
// (column-major, element size 8N + 8).  The recursion that drives them, with its exact products,
// lives beside the RNS product (rns.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace sdpxg {

constexpr int kMpRecBase = 128;  // arrow.rs:63 REC_BASE: blocks up to this order take exact dots
constexpr int kMpMaxLimbs = 8;   // up to 512-bit values on the device

// Left-looking exact-dot LDL' of the order-`size` diagonal block at (off, off) of A (lower
// triangle read and overwritten with the unit lower L), D^-1 into dinv[0..size); W is a
// 2 size^2 scratch (row-major W and a row-major copy of the block).  reg: NULL or (eps, delta) as two MpFloat values (the pivot rule).
void mp_launch_ldl_dots(unsigned char* A, long lda, int off, int size, int N, unsigned char* W,
                        unsigned char* dinv, const unsigned char* reg, uint32_t* status, cudaStream_t st);
// The reference's exact Cholesky xpotrf (mpfr.rs:726-789) of the n x n triangle of A (lower
// or upper storage, ld lda) in place; *info (device int): 0, or j + 1 when pivot j is not
// positive.  One CTA, left-looking, exact dots.
void mp_launch_potrf(unsigned char* A, long lda, int n, bool lower, int N, int* info, uint32_t* status,
                     cudaStream_t st);
// X L' = B for the m rows of B (m x k, ld ldb) with L unit lower k x k (ld ldl), k <= 128:
// each row by exact dots (arrow.rs:437-447).
void mp_launch_solve_lt(const unsigned char* L, long ldl, int k, unsigned char* B, long ldb, int m, int N,
                        uint32_t* status, cudaStream_t st);
// B -= P (m x n blocks, rounded once per entry).
void mp_launch_sub_block(unsigned char* B, long ldb, const unsigned char* P, long ldp, int m, int n, int N,
                         uint32_t* status, cudaStream_t st);
// W = A (m x n block, ld m), then A(:, j) *= d[j] (rounded): L21 = W21 D1^-1.
void mp_launch_copy_scale_cols(unsigned char* A, long lda, unsigned char* W, const unsigned char* d, int m, int n,
                               int N, uint32_t* status, cudaStream_t st);
// A(b, a) -= C(a, b) for b >= a (the Schur update of the lower triangle from the upper product).
void mp_launch_sub_upper_t(unsigned char* A, long lda, const unsigned char* C, long ldc, int n, int N,
                           uint32_t* status, cudaStream_t st);

// Stacked operands of the exact block product sum (gemm_blocks_upper): nb blocks, block b with
// rows [r0[b], r0[b+1]) of the W x m outputs, factor y_b at element yoff[b] of y (w_b x qn[b],
// column-major), scales d at rows r0[b].., sorted global columns cols[coff[b] ..]; Y = y_b and
// Z = d_b y_b (rounded) at those columns, zeros elsewhere.  All arrays on the device.
void mp_launch_stack_blocks(int nb, const long* r0, const long* yoff, const long* coff, const int* qn,
                            const unsigned char* y, const unsigned char* d, const unsigned long long* cols, long W,
                            int m, int N, unsigned char* Z, unsigned char* Y, uint32_t* status, cudaStream_t st);

// MPFR NT scaling of PSD blocks (mp_nt.cu): block b of order n (<= 64) reads its svec at element
// `svec` of s and z, writes R, Rinv and G (upper) as n x n column-major at element `mat`, lambda and
// Lambda^-1/2 at element `vec`; work holds 5 * sum n^2 elements, wvec 2 * sum n; frac (one
// element) receives the working-precision 1/sqrt 2.  bstatus[b]: 0, SDPXG_ST_CHOL_FAIL or SDPXG_ST_SVD_UNCONVERGED.
struct MpNtBlock {
  int n;
  long svec, mat, vec;
};
void mp_launch_nt_scale(const MpNtBlock* blocks, int nblk, int N, const unsigned char* s, const unsigned char* z,
                        unsigned char* frac, unsigned char* work, unsigned char* wvec, unsigned char* lam,
                        unsigned char* lisqrt, unsigned char* R, unsigned char* Rinv, unsigned char* G, int* bstatus,
                        uint32_t* status, cudaStream_t st);

// MPFR step-length bound of PSD blocks (mp_step.cu): block b of order n reads the exact
// congruence Y of its direction (n x n at element `mat`) and Lambda^-1/2 (at element `vec`); consts
// holds two elements: [0] the working-precision 1/sqrt 2 (mp_launch_step_smat), [1] alpha_max.  work:
// 2 sum n^2 elements, fwork: sum (n^2 + 2n) doubles.  alpha[b] (one element each) and path[b]
// (0 a priori FP64 bound, 1 certified by the exact Cholesky, 2 MpFloat eigensolver, 3 that did not
// converge: alpha 0).
struct MpStepBlock {
  int n;
  long svec, mat, vec;
};
// X_b = mat(d_b) (d's svec at element `svec`, X at element `mat`, full symmetric) after computing
// consts[0] = the working-precision 1/sqrt 2.
void mp_launch_step_smat(const MpStepBlock* blocks, int nblk, int N, const unsigned char* d, unsigned char* consts,
                         unsigned char* X, uint32_t* status, cudaStream_t st);
void mp_launch_step_bound(const MpStepBlock* blocks, int nblk, int N, const unsigned char* Y,
                          const unsigned char* lisqrt, unsigned char* consts, unsigned char* work, double* fwork,
                          unsigned char* alpha, int* path, uint32_t* status, cudaStream_t st);

}  // namespace sdpxg
