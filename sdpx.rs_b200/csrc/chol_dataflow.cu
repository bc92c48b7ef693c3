// Persistent dataflow Cholesky of the dense Schur complement, H = U'U (upper, 64 x 64 tiles).
//
// The reference factors the reduced KKT matrix with a right-looking tiled Cholesky
// (dense_block.rs:515-594: potrf on the diagonal tile, trsm on the tile row, syrk/gemm on the
// trailing tiles, dynamic pivot rule potrf_dynamic 334-365).  At the sizes of the condensed
// system (m of a few thousand) that chain is latency-bound: every diagonal tile waits for the
// previous step's trailing update.  Here the whole factorization is ONE launch:
//
//  * the critical path -- GEMM(k-1, k, k), POTRF(k), TRSM(k, k+1) for every k -- is ONE work
//    item, the chain (ticket 0): a single CTA keeps the diagonal tile, U_kk^-1 and U(k, k+1) in
//    shared memory from one step to the next, so the path carries no tile reloads and no hand-
//    offs between CTAs; it waits only for the other CTAs' trailing updates of its next tiles;
//  * the remaining tile tasks TRSM(k, j > k+1) and GEMM(k, i, j) are listed on the host step by
//    step (rows k+1, k+2 first: they feed the chain's next steps);
//  * each CTA takes the next item with an atomic ticket and waits for the item's inputs on
//    per-tile progress words in global memory (acquire/release at GPU scope).  The item with
//    the smallest unfinished ticket always has all inputs ready, and a ticket is only taken by
//    a running CTA, so the schedule cannot deadlock whatever the residency;
//  * every wait is bounded: past the limit the CTA sets SDPXG_ST_SYNC_TIMEOUT and the shared
//    error word, and every CTA leaves at its next wait;
//  * all tile products run on the FP64 tensor cores (mma.sync m8n8k4 f64) from shared-memory
//    tiles staged through L2 (the 2000 x 2000 matrix stays L2-resident);
//  * the diagonal tile is factored in 8 x 8 panels: one warp factors the panel's diagonal
//    block with the dynamic pivot rule and inverts it in registers (each lane redundantly,
//    so the 64-pivot chain carries no shuffles), the other
//    warps apply it to the panel row and update the trailing blocks with DMMA; the tile's
//    inverse U_kk^-1 (used by TRSM and by the explicit inverse of the factor) is formed by
//    block back-substitution, one warp per block column.
#include "common.cuh"

#define DF_NB 64
#define DF_LD 68          // 68 = 4 mod 16: the fragment reads of a half-warp hit distinct banks
#define DF_THREADS 256    // 8 warps: one 8-column block of a 64 x 64 output tile each
#define DF_SPIN_LIMIT (1 << 22)
#define DFS(A, i, j) (A)[(i) + (j) * DF_LD]

enum : unsigned { DF_POTRF = 0u, DF_TRSM = 1u, DF_GEMM = 2u, DF_CHAIN = 3u };

__device__ __forceinline__ int df_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.global.acquire.gpu.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void df_st_release(int* p, int v) {
  asm volatile("st.global.release.gpu.b32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Thread 0 only: wait until *flag >= target.  1 = ready, 0 = another CTA raised the error
// word, -1 = the poll limit was reached.
__device__ int df_wait(const int* flag, int target, const int* err) {
  unsigned ns = 32;
  for (int it = 0; it < DF_SPIN_LIMIT; ++it) {
    if (df_ld_acquire(flag) >= target) return 1;
    if (df_ld_acquire(err) != 0) return 0;
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  return -1;
}

// 64 x 64 tile from global (column-major, leading dimension ld) into shared memory, through
// L2 only (the data was written by other SMs).  Rows >= nr and columns >= nc read as zero.
__device__ __forceinline__ void df_load_tile(double* S, const double* __restrict__ G, long ld,
                                             int nr, int nc, bool vec2) {
  for (int e = threadIdx.x; e < DF_NB * DF_NB / 2; e += DF_THREADS) {
    const int c = e >> 5, r = (e & 31) * 2;
    double v0 = 0.0, v1 = 0.0;
    if (c < nc) {
      const double* p = G + (long)c * ld + r;
      if (vec2 && r + 1 < nr) {
        const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
        v0 = v.x;
        v1 = v.y;
      } else {
        if (r < nr) v0 = __ldcg(p);
        if (r + 1 < nr) v1 = __ldcg(p + 1);
      }
    }
    *reinterpret_cast<double2*>(&DFS(S, r, c)) = make_double2(v0, v1);
  }
}

// acc (this warp's 8-column block w of a 64 x 64 output) += sign * A' B over K = 64.
// Fragments (m8n8k4 f64): lane l holds A[l/4][l%4], B[l%4][l/4], C[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void df_atb(const double* As, const double* Bs, double (&acc)[8][2],
                                       double sign) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int q = lane & 3, r = lane >> 2;
#pragma unroll 4
  for (int ks = 0; ks < DF_NB / 4; ++ks) {
    const int kk = ks * 4 + q;
    const double b = DFS(Bs, kk, 8 * w + r);
#pragma unroll
    for (int R = 0; R < 8; ++R) dmma_m8n8k4(acc[R][0], acc[R][1], sign * DFS(As, kk, 8 * R + r), b);
  }
}

// Dynamic pivot rule of the reduced KKT factorization: a pivot within eps of zero becomes
// delta unless it is clearly negative; non-finite or non-positive pivots fail.  The original
// diagonal (shared memory) is read only on the rare small-pivot branch, off the common path.
__device__ __forceinline__ double df_pivot(double d, const double* diag, int nb, double eps,
                                           double delta, int dynamic, bool& fail) {
  if (!isfinite(d)) {
    fail = true;
    return 1.0;
  }
  if (dynamic && d <= eps) {
    if (d < -64.0 * 2.220446049250313e-16 * nb * fabs(*diag)) fail = true;
    else d = delta;
  }
  if (!(d > 0.0)) {
    fail = true;
    return 1.0;
  }
  return d;
}

// Factor the diagonal tile in A (upper triangle valid, lower zero, padded diagonal 1) in
// place: A <- U.  X <- U^-1 (upper).  Wd: 8 x (8 x 8) inverse diagonal blocks; Sc: 8 x 64
// scratch.  Returns true when every pivot was accepted (CTA uniform).
// Warp 0: factor the 8 x 8 diagonal block of panel p in registers and invert it.  Every lane
// factors the whole block (packed upper triangle, static indices, no shuffles on the pivot
// chain); lane c < 8 then writes column c of U_pp and of W = U_pp^-1.  One rsqrt per pivot:
// 1/sqrt(d) and sqrt(d) = d / sqrt(d).
__device__ __forceinline__ void df_panel_factor(double* A, double* Wd, int p, int nb,
                                                const double* sdiag, double eps, double delta,
                                                int dynamic, int* s_fail) {
  const int lane = threadIdx.x & 31;
  const int c = lane & 7;
  const bool own = lane < 8;
  double u[36], rd[8];
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int i = 0; i <= j; ++i) u[j * (j + 1) / 2 + i] = DFS(A, 8 * p + i, 8 * p + j);
  bool fail = false;
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
    double d = u[kk * (kk + 3) / 2];
    if (8 * p + kk < nb) d = df_pivot(d, sdiag + 8 * p + kk, nb, eps, delta, dynamic, fail);
    const double ri = rsqrt(d);
    rd[kk] = ri;
    u[kk * (kk + 3) / 2] = d * ri;
#pragma unroll
    for (int j = kk + 1; j < 8; ++j) u[j * (j + 1) / 2 + kk] *= ri;  // row kk of U
#pragma unroll
    for (int j = kk + 1; j < 8; ++j)
#pragma unroll
      for (int i = kk + 1; i <= j; ++i)
        u[j * (j + 1) / 2 + i] -= u[i * (i + 1) / 2 + kk] * u[j * (j + 1) / 2 + kk];
  }
  if (fail && lane == 0) *s_fail = 1;
  // column c of W = U_pp^-1: w_c = 1/U_cc, w_i = -(sum_{l>i} U_il w_l) / U_ii for i < c
  double wv[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) wv[l] = (l == c) ? rd[l] : 0.0;
#pragma unroll
  for (int i = 6; i >= 0; --i) {
    double sacc = 0.0;
#pragma unroll
    for (int l = i + 1; l < 8; ++l) sacc = fma(u[l * (l + 1) / 2 + i], wv[l], sacc);
    if (i < c) wv[i] = -sacc * rd[i];
  }
  if (own) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (j == c) {
#pragma unroll
        for (int i = 0; i <= j; ++i) DFS(A, 8 * p + i, 8 * p + j) = u[j * (j + 1) / 2 + i];
      }
#pragma unroll
    for (int i = 0; i < 8; ++i) Wd[p * 64 + i + 8 * c] = wv[i];  // column-major 8 x 8
  }
}

// A[I, J] -= U[P, I]' U[P, J] for one 8 x 8 block (one warp).
__device__ __forceinline__ void df_block_update(double* A, int p, int I, int J) {
  const int lane = threadIdx.x & 31, q = lane & 3, r = lane >> 2;
  double c0 = DFS(A, 8 * I + r, 8 * J + 2 * q), c1 = DFS(A, 8 * I + r, 8 * J + 2 * q + 1);
#pragma unroll
  for (int ks = 0; ks < 2; ++ks) {
    const int kk = ks * 4 + q;
    dmma_m8n8k4(c0, c1, -DFS(A, 8 * p + kk, 8 * I + r), DFS(A, 8 * p + kk, 8 * J + r));
  }
  DFS(A, 8 * I + r, 8 * J + 2 * q) = c0;
  DFS(A, 8 * I + r, 8 * J + 2 * q + 1) = c1;
}

// Factor the diagonal tile in A (upper triangle valid, lower zero, padded diagonal 1) in
// place: A <- U.  X <- U^-1 (upper).  Wd: 8 x (8 x 8) inverse diagonal blocks; Sc: 8 x 64
// scratch.  Returns true when every pivot was accepted (CTA uniform).
// Panels of 8 columns with one panel of look-ahead: once panel p's row U[P, J] is formed, warp
// 0 updates diagonal block p+1 itself and factors panel p+1 while warps 1..7 apply the rest of
// panel p's trailing update -- two barriers per panel, the register factorisation overlapped
// with the tensor-core updates.
__device__ bool df_potrf_tile(double* A, double* X, double* Wd, double* Sc, int nb,
                              const double* sdiag, double eps, double delta, int dynamic,
                              int* s_fail) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, q = lane & 3, r = lane >> 2;
  if (w == 0) df_panel_factor(A, Wd, 0, nb, sdiag, eps, delta, dynamic, s_fail);
  __syncthreads();
  for (int p = 0; p < 8; ++p) {
    // panel row: U[P, J] = W_pp' A[P, J], one block column per warp
    if (w < 7 - p) {
      const int J = p + 1 + w;
      double c0 = 0.0, c1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const int kk = ks * 4 + q;
        dmma_m8n8k4(c0, c1, Wd[p * 64 + kk + 8 * r], DFS(A, 8 * p + kk, 8 * J + r));
      }
      DFS(A, 8 * p + r, 8 * J + 2 * q) = c0;
      DFS(A, 8 * p + r, 8 * J + 2 * q + 1) = c1;
    }
    __syncthreads();
    if (p == 7) break;
    if (w == 0) {
      // look-ahead: the next diagonal block is final after this update; factor it
      df_block_update(A, p, p + 1, p + 1);
      __syncwarp();
      df_panel_factor(A, Wd, p + 1, nb, sdiag, eps, delta, dynamic, s_fail);
    } else {
      // the rest of panel p's trailing update: A[I, J] for p < I <= J, (I, J) != (p+1, p+1)
      const int nrem = 7 - p, cnt = nrem * (nrem + 1) / 2;
      for (int t = w; t < cnt; t += DF_THREADS / 32 - 1) {  // t = 0 is (p+1, p+1): warp 0's
        int I = p + 1, tt = t;
        while (tt >= 8 - I) {
          tt -= 8 - I;
          ++I;
        }
        df_block_update(A, p, I, I + tt);
      }
    }
    __syncthreads();
  }
  // X = U^-1 by block back-substitution; warp w owns block column w:
  // X[w, w] = W_ww, X[P, w] = -W_PP sum_{P < R <= w} U[P, R] X[R, w] for P = w-1 .. 0
  {
    const int qb = w;
    double* sc = Sc + w * 64;
    for (int e = lane; e < 64; e += 32) DFS(X, 8 * qb + (e & 7), 8 * qb + (e >> 3)) = Wd[qb * 64 + e];
    __syncwarp();
    for (int P = qb - 1; P >= 0; --P) {
      double c0 = 0.0, c1 = 0.0;
      for (int R = P + 1; R <= qb; ++R) {
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          const int kk = ks * 4 + q;
          dmma_m8n8k4(c0, c1, DFS(A, 8 * P + r, 8 * R + kk), DFS(X, 8 * R + kk, 8 * qb + r));
        }
      }
      sc[r + 8 * (2 * q)] = c0;
      sc[r + 8 * (2 * q + 1)] = c1;
      __syncwarp();
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const int kk = ks * 4 + q;
        dmma_m8n8k4(d0, d1, -Wd[P * 64 + r + 8 * kk], sc[kk + 8 * r]);
      }
      DFS(X, 8 * P + r, 8 * qb + 2 * q) = d0;
      DFS(X, 8 * P + r, 8 * qb + 2 * q + 1) = d1;
      __syncwarp();
    }
  }
  __syncthreads();
  return *s_fail == 0;
}

// Thread 0 waits, the CTA learns the outcome: true = go on.
__device__ __forceinline__ bool df_cta_wait(const int* flag, int target, const int* err,
                                            uint32_t* status, int* err_w, int* s_go) {
  if (threadIdx.x == 0) {
    const int ok = df_wait(flag, target, err);
    if (ok < 0) {
      atomicOr(status, SDPXG_ST_SYNC_TIMEOUT);
      atomicExch(err_w, 1);
    }
    *s_go = (ok == 1);
  }
  __syncthreads();
  return *s_go != 0;
}

// The critical path of the factorization, step k = 0 .. nt-1, in one CTA:
//   diagonal tile: wait for the updates of steps < k-1 (upd[k][k] = k-1), load it, apply
//   step k-1's update with U(k-1, k) still in Cs, factor it (POTRF with the dynamic pivot rule)
//   and publish U_kk and U_kk^-1 (fin[k][k]);  then TRSM(k, k+1): wait for the updates of steps
//   < k of tile (k, k+1), U(k, k+1) = U_kk^-T H(k, k+1) into Cs, publish it (fin[k][k+1]).
// False when a wait gave up or a pivot failed (the error word is raised either way).
__device__ bool df_chain(double* __restrict__ F, int m, int nt, int* upd, int* fin, int* err,
                         double eps, double delta, int dynamic, const double* __restrict__ diag0,
                         double* __restrict__ Dinv, uint32_t* __restrict__ status, double* As,
                         double* Bs, double* Cs, double* Wd, double* Sc, double* s_diag, int* s_go,
                         int* s_fail, bool vec2) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, q = lane & 3, r = lane >> 2;
  for (int k = 0; k < nt; ++k) {
    const int k0 = k * DF_NB, nb = min(DF_NB, m - k0);
    if (k > 0 && !df_cta_wait(upd + k * nt + k, k - 1, err, status, err, s_go)) return false;
    // diagonal tile H(k, k) - U(k-1, k)' U(k-1, k), assembled in registers, then into As
    double acc[8][2];
#pragma unroll
    for (int R = 0; R < 8; ++R)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int row = 8 * R + r, col = 8 * w + 2 * q + e;
        acc[R][e] = (row < nb && col < nb) ? __ldcg(F + (k0 + row) + (long)(k0 + col) * m) : 0.0;
      }
    if (k > 0) df_atb(Cs, Cs, acc, -1.0);
    for (int e = threadIdx.x; e < DF_NB; e += DF_THREADS) s_diag[e] = (e < nb) ? diag0[k0 + e] : 1.0;
    __syncthreads();  // every warp is done reading Cs
#pragma unroll
    for (int R = 0; R < 8; ++R)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int row = 8 * R + r, col = 8 * w + 2 * q + e;
        DFS(As, row, col) = (row > col) ? 0.0 : ((row == col && row >= nb) ? 1.0 : acc[R][e]);
      }
    for (int e = threadIdx.x; e < DF_NB * DF_NB; e += DF_THREADS) DFS(Bs, e & 63, e >> 6) = 0.0;
    if (threadIdx.x == 0) *s_fail = 0;
    __syncthreads();
    const bool ok = df_potrf_tile(As, Bs, Wd, Sc, nb, s_diag, eps, delta, dynamic, s_fail);
    double* D = Dinv + (long)k * DF_NB * DF_NB;
    for (int e = threadIdx.x; e < DF_NB * DF_NB; e += DF_THREADS) {
      const int rr = e & 63, cc = e >> 6;
      const bool live = rr <= cc && cc < nb;
      if (live) F[(k0 + rr) + (long)(k0 + cc) * m] = DFS(As, rr, cc);
      D[e] = live ? DFS(Bs, rr, cc) : 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (ok) {
        __threadfence();
        df_st_release(upd + k * nt + k, k);
        df_st_release(fin + k * nt + k, 1);
      } else {  // the dependants of this tile leave at their next wait
        atomicOr(status, SDPXG_ST_PIVOT_FAIL);
        atomicExch(err, 1);
      }
    }
    if (!ok) return false;
    if (k + 1 >= nt) break;
    // TRSM(k, k+1): U(k, k+1) = U_kk^-T H(k, k+1), U_kk^-1 in Bs
    if (!df_cta_wait(upd + k * nt + k + 1, k, err, status, err, s_go)) return false;
    const int j0 = (k + 1) * DF_NB, nc = min(DF_NB, m - j0);
    df_load_tile(Cs, F + k0 + (long)j0 * m, m, DF_NB, nc, vec2);
    __syncthreads();
    double t[8][2] = {};
    df_atb(Bs, Cs, t, 1.0);
    __syncthreads();  // every warp is done reading Cs before it becomes U(k, k+1)
#pragma unroll
    for (int R = 0; R < 8; ++R)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int row = 8 * R + r, col = 8 * w + 2 * q + e;
        const double v = (col < nc) ? t[R][e] : 0.0;
        DFS(Cs, row, col) = v;
        if (col < nc) F[(k0 + row) + (long)(j0 + col) * m] = v;
      }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      df_st_release(fin + k * nt + k + 1, 1);
    }
  }
  return true;
}

// items[t] = type << 30 | k << 20 | i << 10 | j (topological order, built on the host).
// sync = {ticket, error, upd[nt * nt], fin[nt * nt]}, zero at launch:
//   upd[i * nt + j] = trailing updates applied to tile (i, j) (GEMM(k, i, j) sets k + 1);
//   fin[i * nt + j] = 1 once tile (i, j) of U is final (POTRF / TRSM).
extern "C" __global__ void __launch_bounds__(DF_THREADS, 2)
k_chol_dataflow(double* __restrict__ F, int m, int nt, const unsigned* __restrict__ items,
                int nitems, int* __restrict__ sync, double eps, double delta, int dynamic,
                const double* __restrict__ diag0, double* __restrict__ Dinv,
                uint32_t* __restrict__ status) {
  extern __shared__ __align__(16) double df_sm[];
  double* As = df_sm;
  double* Bs = As + DF_NB * DF_LD;
  double* Cs = Bs + DF_NB * DF_LD;  // the chain's U(k, k+1) (and the tile it comes from)
  double* Wd = Cs + DF_NB * DF_LD;
  double* Sc = Wd + 8 * 64;
  __shared__ int s_item, s_go, s_fail;
  __shared__ double s_diag[DF_NB];  // original diagonal of the tile being factored
  int* ticket = sync;
  int* err = sync + 1;
  int* upd = sync + 2;
  int* fin = upd + nt * nt;
  const bool vec2 = (m & 1) == 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, q = lane & 3, r = lane >> 2;

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(ticket, 1);
    __syncthreads();
    const int t = s_item;
    if (t >= nitems) break;
    const unsigned code = items[t];
    const int type = (int)(code >> 30), k = (int)((code >> 20) & 1023u);
    const int i = (int)((code >> 10) & 1023u), j = (int)(code & 1023u);
    if (type == DF_CHAIN) {
      if (!df_chain(F, m, nt, upd, fin, err, eps, delta, dynamic, diag0, Dinv, status, As, Bs, Cs,
                    Wd, Sc, s_diag, &s_go, &s_fail, vec2))
        break;
      continue;
    }
    if (threadIdx.x == 0) {
      int ok;
      if (type == DF_POTRF) {
        ok = df_wait(upd + k * nt + k, k, err);
      } else if (type == DF_TRSM) {
        ok = df_wait(fin + k * nt + k, 1, err);
        if (ok == 1) ok = df_wait(upd + k * nt + j, k, err);
      } else {
        ok = df_wait(fin + k * nt + i, 1, err);
        if (ok == 1) ok = df_wait(fin + k * nt + j, 1, err);
        if (ok == 1) ok = df_wait(upd + i * nt + j, k, err);
      }
      if (ok < 0) {
        atomicOr(status, SDPXG_ST_SYNC_TIMEOUT);
        atomicExch(err, 1);
      }
      s_go = (ok == 1);
      s_fail = 0;
    }
    __syncthreads();
    if (!s_go) break;

    const int k0 = k * DF_NB;
    if (type == DF_POTRF) {
      const int nb = min(DF_NB, m - k0);
      // upper triangle of the tile, lower zero, padded diagonal 1
      df_load_tile(As, F + k0 + (long)k0 * m, m, nb, nb, vec2);
      for (int e = threadIdx.x; e < DF_NB; e += DF_THREADS) s_diag[e] = (e < nb) ? diag0[k0 + e] : 1.0;
      __syncthreads();
      for (int e = threadIdx.x; e < DF_NB * DF_NB; e += DF_THREADS) {
        const int rr = e & 63, cc = e >> 6;
        if (rr > cc) DFS(As, rr, cc) = 0.0;
        else if (rr == cc && rr >= nb) DFS(As, rr, cc) = 1.0;
        DFS(Bs, rr, cc) = 0.0;
      }
      __syncthreads();
      const bool ok = df_potrf_tile(As, Bs, Wd, Sc, nb, s_diag, eps, delta, dynamic, &s_fail);
      double* D = Dinv + (long)k * DF_NB * DF_NB;
      for (int e = threadIdx.x; e < DF_NB * DF_NB; e += DF_THREADS) {
        const int rr = e & 63, cc = e >> 6;
        const bool live = rr <= cc && cc < nb;
        if (live) F[(k0 + rr) + (long)(k0 + cc) * m] = DFS(As, rr, cc);
        D[e] = live ? DFS(Bs, rr, cc) : 0.0;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        if (ok) {
          __threadfence();
          df_st_release(fin + k * nt + k, 1);
        } else {  // the dependants of this tile leave at their next wait
          atomicOr(status, SDPXG_ST_PIVOT_FAIL);
          atomicExch(err, 1);
        }
      }
      if (!ok) break;
    } else if (type == DF_TRSM) {
      // U[k, j] = U_kk^-T H[k, j]
      const int j0 = j * DF_NB, nc = min(DF_NB, m - j0);
      df_load_tile(As, Dinv + (long)k * DF_NB * DF_NB, DF_NB, DF_NB, DF_NB, true);
      df_load_tile(Bs, F + k0 + (long)j0 * m, m, DF_NB, nc, vec2);
      __syncthreads();
      double acc[8][2] = {};
      df_atb(As, Bs, acc, 1.0);
#pragma unroll
      for (int R = 0; R < 8; ++R)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = 8 * w + 2 * q + e;
          if (col < nc) F[(k0 + 8 * R + r) + (long)(j0 + col) * m] = acc[R][e];
        }
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        df_st_release(fin + k * nt + j, 1);
      }
    } else {
      // H[i, j] -= U[k, i]' U[k, j]
      const int i0 = i * DF_NB, j0 = j * DF_NB;
      const int ni = min(DF_NB, m - i0), nc = min(DF_NB, m - j0);
      df_load_tile(As, F + k0 + (long)i0 * m, m, DF_NB, ni, vec2);
      if (i != j) df_load_tile(Bs, F + k0 + (long)j0 * m, m, DF_NB, nc, vec2);
      double acc[8][2];
#pragma unroll
      for (int R = 0; R < 8; ++R)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int row = 8 * R + r, col = 8 * w + 2 * q + e;
          acc[R][e] = (row < ni && col < nc) ? __ldcg(F + (i0 + row) + (long)(j0 + col) * m) : 0.0;
        }
      __syncthreads();
      df_atb(As, i == j ? As : Bs, acc, -1.0);
#pragma unroll
      for (int R = 0; R < 8; ++R)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int row = 8 * R + r, col = 8 * w + 2 * q + e;
          if (row < ni && col < nc) F[(i0 + row) + (long)(j0 + col) * m] = acc[R][e];
        }
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        df_st_release(upd + i * nt + j, k + 1);
      }
    }
  }
}
