// CTA-level dense eigen / singular-value routines for PSD blocks of order <= SDPXG_NMAX.
//
//  * cta_jacobi_svd: one-sided (Hestenes) Jacobi with the parallel round-robin ordering.
//    It orthogonalises the columns of M in place and accumulates the right singular
//    vectors V.  Relative accuracy of the small singular values is what the NT scaling
//    needs (the reference takes the SVD of L2'L1 directly instead of an eigensolve of the
//    squared matrix, cones/psdtrianglecone.rs:378-386).
//  * cta_tridiagonalize: Householder reduction of a symmetric matrix to tridiagonal form.
//  * sturm_count / bisect_kth: eigenvalues of the tridiagonal by Sturm-sequence bisection
//    (the same method the reference uses for its binary64 lambda_min bound,
//    cones/psdtrianglecone.rs:1250-1290), every loop bounded.
#pragma once
#include "common.cuh"

#define SDPXG_JACOBI_MAX_SWEEPS 60
#define SDPXG_JACOBI_TOL 1e-15
#define SDPXG_BISECT_MAX 256

// Returns the number of sweeps used, or -1 when the sweep bound was hit.  V == nullptr skips
// the accumulation of the right singular vectors (the left ones are the normalised columns of
// the result, which is all the NT scaling needs).
// `flag` is one int of shared memory, `nrm` n doubles of shared memory.  The squared column
// norms are recomputed at the start of every sweep and carried through the rotations with the
// exact update a' = a - t g, b' = b + t g, so a rotation needs one warp reduction (g) instead
// of three.
__device__ inline int cta_jacobi_svd(double* M, double* V, int n, int* flag, double* nrm) {
  if (V) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      int i = e % n, j = e / n;
      SM(V, i, j) = (i == j) ? 1.0 : 0.0;
    }
  }
  const int N = n + (n & 1);
  const int nwarps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (n < 2) {
    __syncthreads();
    return 0;
  }
  for (int sweep = 0; sweep < SDPXG_JACOBI_MAX_SWEEPS; ++sweep) {
    __syncthreads();  // the previous sweep's last rotations are visible
    for (int p = warp; p < n; p += nwarps) {
      double a = 0.0;
      for (int k = lane; k < n; k += 32) a = fma(SM(M, k, p), SM(M, k, p), a);
      a = warp_sum(a);
      if (lane == 0) nrm[p] = a;
    }
    if (threadIdx.x == 0) *flag = 0;
    __syncthreads();
    for (int r = 0; r < N - 1; ++r) {
      for (int pi = warp; pi < N / 2; pi += nwarps) {
        int p, q;  // round-robin pairing without integer division: r, pi < N - 1
        if (pi == 0) {
          p = N - 1;
          q = r;
        } else {
          p = r + pi;
          if (p >= N - 1) p -= N - 1;
          q = r - pi + N - 1;
          if (q >= N - 1) q -= N - 1;
        }
        if (p >= n || q >= n) continue;
        const double a = nrm[p], b = nrm[q];
        double g = 0.0;
        double x0 = 0.0, y0 = 0.0, x1 = 0.0, y1 = 0.0;  // n <= 64: two entries per lane
        if (lane < n) {
          x0 = SM(M, lane, p);
          y0 = SM(M, lane, q);
        }
        if (lane + 32 < n) {
          x1 = SM(M, lane + 32, p);
          y1 = SM(M, lane + 32, q);
        }
        g = fma(x1, y1, x0 * y0);
        g = warp_sum(g);
        if (g * g > (SDPXG_JACOBI_TOL * SDPXG_JACOBI_TOL) * (a * b)) {  // |g| > tol sqrt(ab)
          const double zeta = (b - a) / (2.0 * g);
          const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(fma(zeta, zeta, 1.0)));
          const double c = rsqrt(fma(t, t, 1.0));
          const double s = c * t;
          if (lane < n) {
            SM(M, lane, p) = c * x0 - s * y0;
            SM(M, lane, q) = s * x0 + c * y0;
          }
          if (lane + 32 < n) {
            SM(M, lane + 32, p) = c * x1 - s * y1;
            SM(M, lane + 32, q) = s * x1 + c * y1;
          }
          if (V) {
            if (lane < n) {
              const double v0 = SM(V, lane, p), w0 = SM(V, lane, q);
              SM(V, lane, p) = c * v0 - s * w0;
              SM(V, lane, q) = s * v0 + c * w0;
            }
            if (lane + 32 < n) {
              const double v1 = SM(V, lane + 32, p), w1 = SM(V, lane + 32, q);
              SM(V, lane + 32, p) = c * v1 - s * w1;
              SM(V, lane + 32, q) = s * v1 + c * w1;
            }
          }
          if (lane == 0) {
            nrm[p] = a - t * g;
            nrm[q] = b + t * g;
            *flag = 1;
          }
        }
      }
      __syncthreads();
    }
    int more = *flag;
    __syncthreads();
    if (!more) return sweep + 1;
  }
  return -1;
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
