// CTA-level dense eigen / singular-value routines for PSD blocks of order <= SDPXG_NMAX.
//
//  * cta_jacobi_left: one-sided (Hestenes) Jacobi with the parallel round-robin ordering,
//    register-resident.  It orthogonalises the columns of M in place.  Relative accuracy of the small singular values is what the NT scaling
//    needs (the reference takes the SVD of L2'L1 directly instead of an eigensolve of the
//    squared matrix, cones/psdtrianglecone.rs:378-386).
//  * cta_tridiagonalize: Householder reduction of a symmetric matrix to tridiagonal form.
//  * sturm_count / bisect_kth: eigenvalues of the tridiagonal by Sturm-sequence bisection
//    (the same method the reference uses for its binary64 lambda_min bound,
//    cones/psdtrianglecone.rs:1250-1290), every loop bounded.
#pragma once
#include "common.cuh"

#define SDPXG_JACOBI_MAX_SWEEPS 60
#define SDPXG_BISECT_MAX 256

// One-sided (Hestenes) Jacobi on the columns of M (n x n, n <= 64, column-major shared memory
// with leading dimension SDPXG_LD): on return M holds M V = U diag(sigma), columns in their
// original order; V itself is not formed.  Returns the number of sweeps, or -1 when the sweep
// bound was hit.  Every thread of the CTA calls it (blockDim.x >= 256).
//
// The matrix stays in registers for the whole iteration.  Warps 0..7 take part: warp w holds
// rows [8w, 8w + 8) of the two columns of every pair, lane j the pair of slot j of the
// round-robin (circle) ordering, which pairs positions j and N-1-j (N = n rounded up to even;
// an odd n gets a zero column that never rotates).  After each round the columns move to their
// next positions with two shuffles per row (tops one slot up, bottoms one slot down, slot 0's
// top fixed), so no column goes back to shared memory inside the sweeps.  A pair's inner
// products ||x||^2, ||y||^2, x'y are the sums of the eight warps' row partials taken in warp
// order, so every warp holds the same bits and takes the same rotation decisions without a
// broadcast; one named barrier per round (the partials are double-buffered in `part`, 1536
// doubles of shared memory).  A pair rotates while |x'y| > 1e-15 sqrt(||x||^2 ||y||^2); the
// angle comes from the half-angle formulas  cos 2t = |h| / r, sin 2t = sign(h) 2 x'y / r,
// r = sqrt(h^2 + 4 (x'y)^2), h = ||y||^2 - ||x||^2,  c = sqrt((1 + cos 2t) / 2),
// s = sin 2t / (2c)  (|t| <= pi/4, so c >= 1/sqrt 2 and nothing cancels; c^2 + s^2 = 1 to
// rounding whatever the accuracy of the angle).  The sweeps stop after one without a rotation,
// or after one in which every pair's cosine was below 1e-10 (the rotations of that sweep leave
// cosines of order 1e-20: one-sided Jacobi converges quadratically).
__device__ inline int cta_jacobi_left(double* M, int n, double* part, int* out) {
  constexpr double kTol2 = 1e-30, kBig2 = 1e-20;
  constexpr unsigned kFull = 0xffffffffu;
  const int warp = threadIdx.x >> 5, j = threadIdx.x & 31;
  if (warp < 8) {
    const int N = n + (n & 1), H = N / 2;
    int itop = j < H ? j : -1, ibot = j < H ? N - 1 - j : -1;
    double x[8], y[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int row = 8 * warp + k;
      x[k] = (row < n && itop >= 0 && itop < n) ? SM(M, row, itop) : 0.0;
      y[k] = (row < n && ibot >= 0 && ibot < n) ? SM(M, row, ibot) : 0.0;
    }
    int sweeps = (n < 2) ? 0 : -1;
    for (int sweep = 0; n >= 2 && sweep < SDPXG_JACOBI_MAX_SWEEPS; ++sweep) {
      bool any_rot = false, any_big = false;
      for (int r = 0; r < N - 1; ++r) {
        double pa = 0.0, pb = 0.0, pg = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          pa = fma(x[k], x[k], pa);
          pb = fma(y[k], y[k], pb);
          pg = fma(x[k], y[k], pg);
        }
        double* buf = part + ((sweep * (N - 1) + r) & 1) * 768;
        buf[warp * 32 + j] = pa;
        buf[256 + warp * 32 + j] = pb;
        buf[512 + warp * 32 + j] = pg;
        asm volatile("bar.sync 1, 256;" ::: "memory");
        double a = buf[j], b = buf[256 + j], g = buf[512 + j];
#pragma unroll
        for (int v = 1; v < 8; ++v) {
          a += buf[v * 32 + j];
          b += buf[256 + v * 32 + j];
          g += buf[512 + v * 32 + j];
        }
        const double gg = g * g, ab = a * b;
        const bool rot = j < H && gg > kTol2 * ab;
        const bool big = j < H && gg > kBig2 * ab;
        if (rot) {
          const double h = b - a;
          const double ir = rsqrt(fma(h, h, 4.0 * gg));
          const double c2 = fabs(h) * ir, s2 = (h < 0.0 ? -2.0 * g : 2.0 * g) * ir;
          const double cc = fma(0.5, c2, 0.5);
          const double ic = rsqrt(cc);
          const double c = cc * ic, s = 0.5 * s2 * ic;
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const double xk = x[k], yk = y[k];
            x[k] = fma(c, xk, -s * yk);
            y[k] = fma(s, xk, c * yk);
          }
        }
        any_rot |= __any_sync(kFull, rot);
        any_big |= __any_sync(kFull, big);
        // next positions: slot j's top from slot j-1 (slot 1's from slot 0's bottom, slot 0's
        // top stays), slot j's bottom from slot j+1 (the last slot's from its own top; with a
        // single slot nothing moves)
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const double up = __shfl_up_sync(kFull, j == 0 ? y[k] : x[k], 1);
          const double dn = __shfl_down_sync(kFull, y[k], 1);
          const double nx = (j == 0) ? x[k] : up;
          y[k] = (j == H - 1) ? (H == 1 ? y[k] : x[k]) : dn;
          x[k] = nx;
        }
        const int up = __shfl_up_sync(kFull, j == 0 ? ibot : itop, 1);
        const int dn = __shfl_down_sync(kFull, ibot, 1);
        if (j < H) {
          const int nt = (j == 0) ? itop : up;
          ibot = (j == H - 1) ? (H == 1 ? ibot : itop) : dn;
          itop = nt;
        }
      }
      if (!any_rot || !any_big) {
        sweeps = sweep + 1;
        break;
      }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int row = 8 * warp + k;
      if (row < n && j < H) {
        if (itop < n) SM(M, row, itop) = x[k];
        if (ibot < n) SM(M, row, ibot) = y[k];
      }
    }
    if (threadIdx.x == 0) *out = sweeps;
  }
  __syncthreads();
  const int res = *out;
  __syncthreads();
  return res;
}

// Householder tridiagonalisation of the symmetric A (destroyed).  d[0..n), e[0..n-1).
// `work` is 2*n doubles of shared memory, `red` 32 doubles (unused: kept for the callers).
// Step k reflects column k below the diagonal, x = A[k+1:n, k] (m <= 63 entries): every warp
// forms |x|^2 and, after the matvec, v'p itself (one warp covers the whole vector, and every
// warp gets the same value from the same butterfly), v and q = p - (v'p) v are formed inline
// from column k (which the step does not modify), so a step needs two barriers: after p = A v
// (one warp per row, reading the row as a column: A stays exactly symmetric) and after the
// rank-2 update.
__device__ inline void cta_tridiagonalize(double* A, int n, double* d, double* e, double* work,
                                          double* red) {
  (void)red;
  double* p = work;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;  // length of the column below the diagonal
    const double* x = &SM(A, k + 1, k);
    double part = 0.0;
    for (int i = lane; i < m; i += 32) part = fma(x[i], x[i], part);
    const double nrm2 = warp_sum(part);
    const double x0 = x[0];
    const double alpha = -copysign(sqrt(nrm2), x0);
    const double vnorm2 = nrm2 - x0 * x0 + (x0 - alpha) * (x0 - alpha);
    if (threadIdx.x == 0) {
      d[k] = SM(A, k, k);
      e[k] = (nrm2 == 0.0) ? 0.0 : alpha;
    }
    if (nrm2 == 0.0 || vnorm2 == 0.0) continue;  // column already reduced (uniform)
    const double vs = rsqrt(vnorm2);
    const double v0 = (x0 - alpha) * vs;
    // p = A_sub v
    for (int i = warp; i < m; i += nwarps) {
      double acc = 0.0;
      for (int j = lane; j < m; j += 32)
        acc = fma(SM(A, k + 1 + j, k + 1 + i), (j == 0) ? v0 : x[j] * vs, acc);
      acc = warp_sum(acc);
      if (lane == 0) p[i] = acc;
    }
    __syncthreads();
    double kp = 0.0;
    for (int i = lane; i < m; i += 32) kp = fma((i == 0) ? v0 : x[i] * vs, p[i], kp);
    const double K = warp_sum(kp);
    // A_sub -= 2 (v q' + q v'), q = p - K v (both triangles from the same two products)
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
      const int i = t % m, j = t / m;
      const double vi = (i == 0) ? v0 : x[i] * vs, vj = (j == 0) ? v0 : x[j] * vs;
      const double qi = p[i] - K * vi, qj = p[j] - K * vj;
      const double u = __dadd_rn(__dmul_rn(vi, qj), __dmul_rn(qi, vj));
      SM(A, k + 1 + i, k + 1 + j) -= 2.0 * u;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (n >= 2) {
      d[n - 2] = SM(A, n - 2, n - 2);
      d[n - 1] = SM(A, n - 1, n - 1);
      e[n - 2] = SM(A, n - 1, n - 2);
    } else if (n == 1) {
      d[0] = SM(A, 0, 0);
    }
  }
  __syncthreads();
}

// Number of eigenvalues of the tridiagonal (d, e) strictly below x.
__device__ __forceinline__ int sturm_count(const double* d, const double* e, int n, double x,
                                           double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += (q < 0.0);
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - e[i - 1] * e[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += (q < 0.0);
  }
  return cnt;
}

__device__ __forceinline__ void gershgorin(const double* d, const double* e, int n, double* lo,
                                           double* hi, double* pivmin) {
  double l = 1e300, h = -1e300, emax = 0.0;
  for (int i = 0; i < n; ++i) {
    double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
    l = fmin(l, d[i] - r);
    h = fmax(h, d[i] + r);
    if (i + 1 < n) emax = fmax(emax, e[i] * e[i]);
  }
  double span = fmax(fabs(l), fabs(h));
  *lo = l - 2.0 * 2.220446049250313e-16 * span - 1e-300;
  *hi = h + 2.0 * 2.220446049250313e-16 * span + 1e-300;
  *pivmin = 2.2250738585072014e-308 * fmax(1.0, emax);
}

// Smallest eigenvalue of the tridiagonal (d, e) by CTA-wide multisection: each round T threads
// evaluate one Sturm count each on an even grid over the current bracket and the bracket
// shrinks to the first grid cell holding an eigenvalue (about T-fold per round).  T = 512: a
// Sturm count is a chain of n dependent divisions, and with more than 16 warps per SM evaluating
// them the rounds become bound by FP64 issue rather than by that chain, so 1024 points cost
// twice as long per round for one more bit.
// Uniform result; `best` is one int of shared memory.  *ok = false if the round bound is hit.
__device__ inline double cta_eig_min(const double* d, const double* e, int n, int* best, bool* ok) {
  double lo, hi, pivmin;
  gershgorin(d, e, n, &lo, &hi, &pivmin);
  const int T = min((int)blockDim.x, 512);
  for (int round = 0; round < 16; ++round) {
    if (!(hi - lo > 2.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + pivmin)) {
      *ok = true;
      return 0.5 * (lo + hi);
    }
    const double step = (hi - lo) / (T + 1);
    if (threadIdx.x == 0) *best = T;
    __syncthreads();
    const double x = lo + step * (threadIdx.x + 1);
    if ((int)threadIdx.x < T && x > lo && x < hi && sturm_count(d, e, n, x, pivmin) >= 1)
      atomicMin(best, (int)threadIdx.x);
    __syncthreads();
    const int t = *best;
    __syncthreads();
    const double nlo = (t == 0) ? lo : lo + step * t;
    const double nhi = (t == T) ? hi : lo + step * (t + 1);
    lo = nlo;
    hi = nhi;
  }
  *ok = false;
  return 0.5 * (lo + hi);
}

// Every eigenvalue of the tridiagonal (d, e), ascending, into eig[0..n): 16-lane groups, one
// eigenvalue per group, multisection with 15 Sturm counts per round (the bracket shrinks
// 16-fold per round), the same convergence test as bisect_kth; no CTA barrier inside.
// Sets the status bit SDPXG_ST_EIG_FAIL for an eigenvalue whose round bound was hit.
__device__ inline void cta_eig_all(const double* d, const double* e, int n, double* eig,
                                   uint32_t* status) {
  double lo0, hi0, pivmin;
  gershgorin(d, e, n, &lo0, &hi0, &pivmin);
  constexpr int P = 16;
  const int grp = threadIdx.x / P, sl = threadIdx.x % P, base = threadIdx.x & 16;
  const unsigned gmask = 0xFFFFu << base;
  for (int k = grp; k < n; k += blockDim.x / P) {
    double lo = lo0, hi = hi0;
    bool conv = false;
    for (int round = 0; round < 64; ++round) {
      if (!(hi - lo > 2.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + pivmin)) {
        conv = true;
        break;
      }
      const double step = (hi - lo) / P;
      const double x = lo + step * (sl + 1);
      const bool above = (sl < P - 1) && x > lo && x < hi && sturm_count(d, e, n, x, pivmin) > k;
      const unsigned bal = (__ballot_sync(gmask, above) >> base) & 0xFFFFu;
      const int c = bal ? __ffs(bal) - 1 : P - 1;  // eigenvalue k lies in cell c
      const double nlo = (c == 0) ? lo : lo + step * c;
      const double nhi = (c == P - 1) ? hi : lo + step * (c + 1);
      lo = nlo;
      hi = nhi;
    }
    if (sl == 0) {
      eig[k] = 0.5 * (lo + hi);
      if (!conv) atomicOr(status, SDPXG_ST_EIG_FAIL);
    }
  }
}

// k-th smallest eigenvalue (k = 0 is the minimum) by bisection; one thread.
// Sets *ok = false when the bound on steps was hit before convergence.
__device__ inline double bisect_kth(const double* d, const double* e, int n, int k, bool* ok) {
  double lo, hi, pivmin;
  gershgorin(d, e, n, &lo, &hi, &pivmin);
  for (int it = 0; it < SDPXG_BISECT_MAX; ++it) {
    double mid = 0.5 * (lo + hi);
    if (!(mid > lo && mid < hi) ||
        hi - lo <= 2.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + pivmin) {
      *ok = true;
      return mid;
    }
    if (sturm_count(d, e, n, mid, pivmin) > k) hi = mid;
    else lo = mid;
  }
  *ok = false;
  return 0.5 * (lo + hi);
}
