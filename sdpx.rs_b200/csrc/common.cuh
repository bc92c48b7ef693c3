// Shared definitions for the sm_100a SDPX hot-path kernels.
//
// Layout conventions (all device buffers in HBM, float64):
//  * PSD vectors use the reference's triangle convention: upper triangle, column order,
//    off-diagonal entries scaled by sqrt(2); entry (i, j), i <= j, sits at j(j+1)/2 + i
//    (include/sdpx.h:32-33 of the reference).
//  * Per-block n x n matrices (R, Rinv, Ginv, ...) are column-major with leading dimension n,
//    packed one after another at BlockDesc::mat_off.
//  * The Schur complement and its factor are dense column-major m x m.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define SDPXG_NMAX 64               // largest PSD block order handled by the CTA kernels
// Shared-memory leading dimension: 68 = 4 (mod 16), so the 16 lanes of a half-warp reading an
// m8n8k4 f64 fragment (rows r + 4-column k, or 4-row k + columns r) hit 16 distinct 8-byte
// bank pairs, and a column read is conflict-free.
#define SDPXG_LD 68
#define SDPXG_THREADS 256         // dense tile kernels (their thread maps assume 256)
#define SDPXG_CONE_THREADS 1024   // one CTA per PSD block
#define SDPXG_NT_SVD_THREADS 512  // the NT scaling's Jacobi launch (8 warps iterate, 128 registers)
#define SDPXG_RSQRT2 0.70710678118654752440
#define SDPXG_SQRT2 1.41421356237309504880
#define SDPXG_CHOL_SCRATCH (3 * SDPXG_NMAX)  // doubles of shared scratch for cta_cholesky_lower

// Device status bits reported by the kernels (read back by the host after each phase).
enum SdpxgStatus : uint32_t {
  SDPXG_ST_OK = 0,
  SDPXG_ST_CHOL_FAIL = 1u,        // Cholesky of s or z failed (not interior)
  SDPXG_ST_SVD_UNCONVERGED = 2u,  // Jacobi sweeps hit their bound
  SDPXG_ST_NONFINITE = 4u,        // a non-finite value was produced
  SDPXG_ST_PIVOT_FAIL = 8u,       // clearly negative or non-finite Schur pivot
  SDPXG_ST_EIG_FAIL = 16u,        // eigenvalue bisection did not converge
  SDPXG_ST_SYNC_TIMEOUT = 32u,    // a bounded inter-CTA wait gave up (no progress)
  SDPXG_ST_EXACT_SPREAD = 64u,    // an exact dot's terms spread beyond the device accumulator
};

// Device-resident control of one refined KKT solve: the stopping rules of the two-level
// stationary refinement (kkt/refinement.rs:118-191) evaluated by one-thread control kernels that
// drive the WHILE nodes of the solve's CUDA graph; the host reads it once per solve.
struct RefineCtl {
  double normb, norme, tol;      // reduced-system level (inner)
  double onormb, onorme, otol;   // original-operator level (outer)
  int it, oit;                   // accepted steps at each level
  int ok;                        // cleared by the first failed check
  int accept, oaccept;           // the last candidate is kept
  int cont, ocont;               // the loop goes on (its residual is carried over)
  int inner_steps, outer_steps;  // refinement steps run (trace counters)
  int guard;                     // loop-body executions: a hard bound on every loop
};
struct RefineParams {
  double abstol, reltol, stop_ratio;
  int max_iter, guard_max;
};

// One reduction of a batched launch (k_reduce_batch): op over x (and y) of length n.
struct RedReq {
  int op;
  long n;
  const double* x;
  const double* y;
};
constexpr int kRedBatchMax = 12;
struct RedBatch {
  RedReq r[kRedBatchMax];
};

// One vector update of a batched launch (k_lincomb_batch): out = a x + b y + c w over n entries
// (a null operand is left out), with the arithmetic of k_lincomb.
struct LinReq {
  long n;
  double a, b, c;
  const double* x;
  const double* y;
  const double* w;
  double* out;
};
constexpr int kLinBatchMax = 6;
struct LinBatch {
  LinReq r[kLinBatchMax];
};

struct BlockDesc {
  int n;         // block order
  int svec_off;  // first row of the block in the stacked cone vector
  int mat_off;   // offset of the block's n*n matrices
  int vec_off;   // offset of the block's length-n vectors (lambda, Lambda^-1/2)
};

// A matrix-valued sampled block (dim D > 1): its PSD block j, D, basis rows h, basis columns c,
// and the offsets of its basis Q (h x c), of V = R^-1 U (n x Dc) and of K = V'V (Dc x Dc).
struct MsDesc {
  int j, D, h, c;
  long q_off, v_off, k_off;
};

__device__ __forceinline__ int tri_idx(int i, int j) {  // i <= j
  return j * (j + 1) / 2 + i;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ------------------------------------------------------------------------------------
// CTA-level helpers on n x n shared-memory matrices with leading dimension SDPXG_LD.
// Callers place __syncthreads() between dependent calls.
// ------------------------------------------------------------------------------------
#define SM(A, i, j) (A)[(i) + (j) * SDPXG_LD]

// Shared matrices are 64 x 64 (leading dimension SDPXG_LD) whatever the block order n; the
// entries outside n x n are kept at zero so the tensor-core products below can run on whole
// 8 x 8 x 4 fragments.  Loads write the zero padding; products of padded inputs keep it.
__device__ __forceinline__ void cta_zero_mat(double* M) {
  for (int e = threadIdx.x; e < SDPXG_LD * SDPXG_NMAX; e += blockDim.x) M[e] = 0.0;
}

// M = smat(v): symmetric matrix from an svec (zero padded to 64 x 64).  Column j of the upper
// triangle is contiguous in the svec (v[j(j+1)/2 + i], i <= j): one warp per column reads it
// coalesced and writes both triangles.
__device__ __forceinline__ void cta_load_smat(double* M, const double* __restrict__ v, int n) {
  for (int e = threadIdx.x; e < SDPXG_NMAX * SDPXG_NMAX; e += blockDim.x) {
    const int i = e % SDPXG_NMAX, j = e / SDPXG_NMAX;
    if (i >= n || j >= n) SM(M, i, j) = 0.0;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int j = warp; j < n; j += nwarps) {
    const double* col = v + j * (j + 1) / 2;
    for (int i = lane; i <= j; i += 32) {
      double x = col[i];
      if (i != j) x *= SDPXG_RSQRT2;
      SM(M, i, j) = x;
      SM(M, j, i) = x;
    }
  }
}

// v = svec(sym(M)): off-diagonal (M_ij + M_ji) / sqrt(2).
__device__ __forceinline__ void cta_store_svec(double* __restrict__ v, const double* M, int n) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;
    if (i > j) continue;
    v[tri_idx(i, j)] = (i == j) ? SM(M, i, j) : (SM(M, i, j) + SM(M, j, i)) * SDPXG_RSQRT2;
  }
}

__device__ __forceinline__ void cta_load_mat(double* M, const double* __restrict__ g, int n) {
  for (int e = threadIdx.x; e < SDPXG_NMAX * SDPXG_NMAX; e += blockDim.x) {
    int i = e % SDPXG_NMAX, j = e / SDPXG_NMAX;
    SM(M, i, j) = (i < n && j < n) ? g[i + j * n] : 0.0;
  }
}

__device__ __forceinline__ void cta_store_mat(double* __restrict__ g, const double* M, int n) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) g[e] = SM(M, e % n, e / n);
}

// One FP64 tensor-core MMA: D(8x8) = A(8x4) B(4x8) + C.  Fragments (PTX mma.m8n8k4 .f64):
// lane l holds A[l/4][l%4], B[l%4][l/4] and C/D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// C = op(A) op(B) on zero-padded shared matrices, one 8 x 8 output tile per warp at a time.
// K runs to n rounded up to 4, never further: C is written only up to n rounded up to 8, and
// a later product that reads C as an operand must not reach its unwritten columns (another
// kernel's leftovers there, NaN included, would enter through 0 x NaN).  Full groups of four
// k-steps load their fragments before their four MMAs, so the shared-memory latency overlaps
// the accumulation chain; the remaining k-steps follow one by one.  C must not alias A or B.
template <bool TA, bool TB>
__device__ __forceinline__ void cta_gemm_mma(double* C, const double* A, const double* B, int n) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int tiles = (n + 7) >> 3, ksteps = (n + 3) >> 2, kfull = ksteps & ~3;
  const int r = lane >> 2, q = lane & 3;
  for (int t = warp; t < tiles * tiles; t += nwarps) {
    const int ti = (t % tiles) << 3, tj = (t / tiles) << 3;
    double d0 = 0.0, d1 = 0.0;
    for (int ks0 = 0; ks0 < kfull; ks0 += 4) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int k = ((ks0 + u) << 2) + q;
        a[u] = TA ? SM(A, k, ti + r) : SM(A, ti + r, k);
        b[u] = TB ? SM(B, tj + r, k) : SM(B, k, tj + r);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) dmma_m8n8k4(d0, d1, a[u], b[u]);
    }
    for (int ks = kfull; ks < ksteps; ++ks) {
      const int k = (ks << 2) + q;
      dmma_m8n8k4(d0, d1, TA ? SM(A, k, ti + r) : SM(A, ti + r, k),
                  TB ? SM(B, tj + r, k) : SM(B, k, tj + r));
    }
    SM(C, ti + r, tj + 2 * q) = d0;
    SM(C, ti + r, tj + 2 * q + 1) = d1;
  }
}

// C = op(A) * op(B); ta/tb select the transpose.  C must not alias A or B.
__device__ __forceinline__ void cta_gemm(double* C, const double* A, bool ta, const double* B,
                                         bool tb, int n) {
  if (ta) {
    if (tb) cta_gemm_mma<true, true>(C, A, B, n);
    else cta_gemm_mma<true, false>(C, A, B, n);
  } else {
    if (tb) cta_gemm_mma<false, true>(C, A, B, n);
    else cta_gemm_mma<false, false>(C, A, B, n);
  }
}

// In-place lower Cholesky A = L L' (lower triangle of A used), the shared-memory form for CTAs of
// fewer than 256 threads.  The update is lagged so one barrier per column suffices: the trailing matrix is updated with the unscaled
// column divided by the pivot, and columns are scaled at the end.  The thread that
// finishes the next diagonal entry computes its reciprocal once and publishes it for the
// next step (0 marks a pivot that is not positive and finite: the reciprocal of a finite
// positive double is never 0).  Step k visits only the trailing (n-k-1)^2 square.
// cta_cholesky_lower2 factors two matrices of the same order at once (one barrier per
// column for both, the same arithmetic per entry); a failed matrix stops being updated and
// reports false, the other one carries on.
// `piv` is SDPXG_CHOL_SCRATCH doubles of shared memory per matrix: pivots, reciprocals, roots.
__device__ inline void cta_cholesky_lower2_smem(double* A, double* B, int n, double* pivA,
                                                double* pivB, bool* okA, bool* okB) {
  double* pinvA = pivA + SDPXG_NMAX;
  double* pinvB = pivB + SDPXG_NMAX;
  const bool two = (B != nullptr);
  if (threadIdx.x == 0 && n > 0) {
    const double a = SM(A, 0, 0);
    pivA[0] = a;
    pinvA[0] = (a > 0.0 && isfinite(a)) ? 1.0 / a : 0.0;
    if (two) {
      const double b = SM(B, 0, 0);
      pivB[0] = b;
      pinvB[0] = (b > 0.0 && isfinite(b)) ? 1.0 / b : 0.0;
    }
  }
  bool liveA = true, liveB = two;
  for (int k = 0; k < n; ++k) {
    __syncthreads();
    const double dA = pinvA[k];  // written in step k - 1, not touched in step k
    const double dB = two ? pinvB[k] : 0.0;
    liveA = liveA && dA != 0.0;
    liveB = liveB && dB != 0.0;
    if (!liveA && !liveB) break;
    const int w = n - k - 1, tot = w * w;
    const int lim = two ? 2 * tot : tot;
    for (int e = threadIdx.x; e < lim; e += blockDim.x) {
      const bool second = e >= tot;
      const int r = second ? e - tot : e;
      const int i = k + 1 + r % w, j = k + 1 + r / w;
      if (i < j || (second ? !liveB : !liveA)) continue;
      double* X = second ? B : A;
      const double v = SM(X, i, j) - SM(X, i, k) * SM(X, j, k) * (second ? dB : dA);
      SM(X, i, j) = v;
      if (i == k + 1 && j == k + 1) {  // the next pivot is final now
        double* pv = second ? pivB : pivA;
        pv[k + 1] = v;
        pv[SDPXG_NMAX + k + 1] = (v > 0.0 && isfinite(v)) ? 1.0 / v : 0.0;
      }
    }
  }
  __syncthreads();
  *okA = liveA;
  *okB = liveB;
  double* rootA = pinvA + SDPXG_NMAX;
  double* rootB = pinvB + SDPXG_NMAX;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    if (liveA) rootA[j] = sqrt(pivA[j]);
    if (liveB) rootB[j] = sqrt(pivB[j]);
  }
  __syncthreads();
  const int lim = two ? 2 * n * n : n * n;
  for (int e = threadIdx.x; e < lim; e += blockDim.x) {
    const bool second = e >= n * n;
    if (second ? !liveB : !liveA) continue;
    const int r = second ? e - n * n : e;
    const int i = r % n, j = r / n;
    double* X = second ? B : A;
    const double* root = second ? rootB : rootA;
    if (i > j) SM(X, i, j) /= root[j];
    else if (i == j) SM(X, i, j) = root[j];
    else SM(X, i, j) = 0.0;
  }
  __syncthreads();
}

// 1/v for a positive v: the hardware approximation refined by two Newton-Raphson steps
// y <- y + y (1 - v y) (each doubles the correct bits; the result is within a few units in the
// last place of 1/v).  Outside [2^-1000, 2^1000], where the approximation flushes, the IEEE
// division.  Used on the critical path of the blocked CTA Cholesky factorisation.
__device__ __forceinline__ double recip_newton(double v) {
  if (!(v >= 0x1p-1000 && v <= 0x1p1000)) return 1.0 / v;
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(v));
  double e = fma(-v, y, 1.0);
  y = fma(y, e, y);
  e = fma(-v, y, 1.0);
  return fma(y, e, y);
}

// Blocked right-looking form (blockDim.x >= 256): panels of 8 columns.  Warp 0 factors A's
// panel and warp 1 B's, in registers (lane l holds panel rows kb + l and kb + 32 + l; the pivot
// and the entries of the updating rows come by shuffles; L(r,c) = a(r,c) / sqrt(pivot), the
// reciprocal by recip_newton); then every warp takes 8 x 8 tiles of the trailing lower triangle
// of both matrices, A22 -= L21 L21' on the FP64 tensor cores (two m8n8k4 steps).  Two barriers
// per panel instead of one per column.  A pivot that is not positive and finite stops that
// matrix (false); the other carries on.  Entries above the diagonal end as zeros.
__device__ inline void cta_cholesky_lower2_panel(double* A, double* B, int n, bool* okA, bool* okB) {
  __shared__ int live[2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const bool two = (B != nullptr);
  if (threadIdx.x == 0) {
    live[0] = 1;
    live[1] = two ? 1 : 0;
  }
  __syncthreads();
  for (int kb = 0; kb < n; kb += 8) {
    const int w = min(8, n - kb);
    if (warp < 2 && live[warp]) {  // panel of one matrix in one warp
      double* X = warp == 0 ? A : B;
      const int r0 = kb + lane, r1 = kb + 32 + lane;
      double P0[8], P1[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        P0[c] = (c < w && r0 < n) ? SM(X, r0, kb + c) : 0.0;
        P1[c] = (c < w && r1 < n) ? SM(X, r1, kb + c) : 0.0;
      }
      bool ok = true;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < w && ok) {
          const double piv = __shfl_sync(0xffffffffu, P0[c], c);
          ok = piv > 0.0 && isfinite(piv);
          if (ok) {
            const double d = sqrt(piv), rd = recip_newton(d);
            P0[c] = lane < c ? 0.0 : (lane == c ? d : P0[c] * rd);
            P1[c] *= rd;
#pragma unroll
            for (int c2 = c + 1; c2 < 8; ++c2) {
              const double l = __shfl_sync(0xffffffffu, P0[c], c2);  // L(kb + c2, kb + c)
              P0[c2] = fma(-P0[c], l, P0[c2]);
              P1[c2] = fma(-P1[c], l, P1[c2]);
            }
          }
        }
      }
      if (ok) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          if (c < w && r0 < n) SM(X, r0, kb + c) = P0[c];
          if (c < w && r1 < n) SM(X, r1, kb + c) = P1[c];
        }
      } else if (lane == 0) {
        live[warp] = 0;
      }
    }
    __syncthreads();
    const int t0 = kb + 8;
    if (t0 < n) {  // trailing update of the lower tiles on DMMA
      const int nt = (n - t0 + 7) >> 3, per = nt * (nt + 1) / 2;
      const int r = lane >> 2, q = lane & 3;
      for (int e = warp; e < 2 * per; e += nwarps) {
        const int mtx = e >= per ? 1 : 0;
        if (!live[mtx]) continue;
        double* X = mtx ? B : A;
        int u = mtx ? e - per : e, ti = 0;
        while (u > ti) {  // u -> (ti, tj), tj <= ti
          u -= ti + 1;
          ++ti;
        }
        const int row = t0 + 8 * ti, col = t0 + 8 * u;
        double d0 = SM(X, row + r, col + 2 * q), d1 = SM(X, row + r, col + 2 * q + 1);
#pragma unroll
        for (int k4 = 0; k4 < 8; k4 += 4) {
          const double a = -SM(X, row + r, kb + k4 + q), b = SM(X, col + r, kb + k4 + q);
          dmma_m8n8k4(d0, d1, a, b);
        }
        SM(X, row + r, col + 2 * q) = d0;
        SM(X, row + r, col + 2 * q + 1) = d1;
      }
    }
    __syncthreads();
  }
  *okA = live[0] != 0;
  *okB = two && live[1] != 0;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;
    if (i < j) {
      if (*okA) SM(A, i, j) = 0.0;
      if (two && *okB) SM(B, i, j) = 0.0;
    }
  }
  __syncthreads();
}

__device__ inline void cta_cholesky_lower2(double* A, double* B, int n, double* pivA, double* pivB,
                                           bool* okA, bool* okB) {
  if (blockDim.x >= 256) cta_cholesky_lower2_panel(A, B, n, okA, okB);
  else cta_cholesky_lower2_smem(A, B, n, pivA, pivB, okA, okB);
}

__device__ inline bool cta_cholesky_lower(double* A, int n, double* piv) {
  bool ok, unused;
  cta_cholesky_lower2(A, nullptr, n, piv, piv, &ok, &unused);
  return ok;
}

// Solve L' X = B in place of B (L lower, n x n), one column per thread.
// B := L^-T B for the lower triangular L (n x n, n <= 64): blocked back substitution, 8 rows at
// a time from the bottom.  Each block of rows is solved against its 8 x 8 diagonal block, one
// thread per column of B (x_i = (b_i - sum_k L(k,i) x_k) / L(i,i), the reciprocals formed first,
// in parallel); the rows above then take B(0:ib, :) -= L(ib:ib+8, 0:ib)' X on the FP64 tensor
// cores, one warp per 8 x 8 tile (two m8n8k4 steps).  Two barriers per block of rows.
// blockDim.x >= 64; `rd` is n doubles of shared memory.
__device__ __forceinline__ void cta_trsm_lower_t_blocked(const double* L, double* B, int n, double* rd) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) rd[i] = 1.0 / SM(L, i, i);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int r = lane >> 2, q = lane & 3, nt = (n + 7) >> 3;
  for (int ib = (nt - 1) * 8; ib >= 0; ib -= 8) {
    const int ie = min(ib + 8, n);
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      for (int i = ie - 1; i >= ib; --i) {
        double acc = SM(B, i, j);
        for (int k = i + 1; k < ie; ++k) acc = fma(-SM(L, k, i), SM(B, k, j), acc);
        SM(B, i, j) = acc * rd[i];
      }
    }
    __syncthreads();
    for (int t = warp; t < (ib >> 3) * nt; t += nwarps) {  // tiles above the block
      const int ti = (t % (ib >> 3)) << 3, tj = (t / (ib >> 3)) << 3;
      double d0 = SM(B, ti + r, tj + 2 * q), d1 = SM(B, ti + r, tj + 2 * q + 1);
#pragma unroll
      for (int k4 = 0; k4 < 8; k4 += 4)
        dmma_m8n8k4(d0, d1, -SM(L, ib + k4 + q, ti + r), SM(B, ib + k4 + q, tj + r));
      SM(B, ti + r, tj + 2 * q) = d0;
      SM(B, ti + r, tj + 2 * q + 1) = d1;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void cta_trsm_lower_t(const double* L, double* B, int n) {
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    for (int i = n - 1; i >= 0; --i) {
      double acc = SM(B, i, j);
      for (int k = i + 1; k < n; ++k) acc = fma(-SM(L, k, i), SM(B, k, j), acc);
      SM(B, i, j) = acc / SM(L, i, i);
    }
  }
}
