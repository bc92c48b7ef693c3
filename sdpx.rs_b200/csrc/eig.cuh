// CTA-level dense eigen / singular-value routines for PSD blocks of order <= SDPXG_NMAX.
//
//  * cta_jacobi_left: one-sided (Hestenes) Jacobi with the parallel odd-even ordering,
//    register-resident.  It orthogonalises the columns of M in place.  Relative accuracy of
//    the small singular values is what the NT scaling
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

namespace jacobi_detail {

// x'y over the eight rows a lane holds, as a tree (depth 4).
__device__ __forceinline__ double dot8(const double* x, const double* y) {
  const double p0 = fma(x[1], y[1], x[0] * y[0]), p1 = fma(x[3], y[3], x[2] * y[2]);
  const double p2 = fma(x[5], y[5], x[4] * y[4]), p3 = fma(x[7], y[7], x[6] * y[6]);
  return (p0 + p1) + (p2 + p3);
}

// Sum of the eight warps' partials b[0], b[32], ..., b[224] as a tree (the same bits in every
// warp that reads them).
__device__ __forceinline__ double sum8(const double* b) {
  return ((b[0] + b[32]) + (b[64] + b[96])) + ((b[128] + b[160]) + (b[192] + b[224]));
}

// Rotation x' = c x - s y, y' = s x + c y with x'y' = 0 for a pair with ||x||^2 = a, ||y||^2 = b,
// x'y = g, by the half-angle formulas (|theta| <= pi/4):
//   cos 2t = |h| / r, sin 2t = sign(h) 2g / r, r = sqrt(h^2 + 4g^2), h = b - a,
//   c = sqrt((1 + cos 2t) / 2), s = sin 2t / (2c);
// c >= 1/sqrt 2, so nothing cancels, and c^2 + s^2 = 1 to rounding.  tg = (s / c) g, with which
// ||x'||^2 = a - tg and ||y'||^2 = b + tg.
__device__ __forceinline__ void rotation(double a, double b, double g, double& c, double& s, double& tg) {
  const double h = b - a;
  const double ir = rsqrt(fma(h, h, 4.0 * g * g));
  const double c2 = fabs(h) * ir, s2 = (h < 0.0 ? -2.0 * g : 2.0 * g) * ir;
  const double cc = fma(0.5, c2, 0.5);
  const double ic = rsqrt(cc);
  c = cc * ic;
  s = 0.5 * s2 * ic;
  tg = s * ic * g;
}

}  // namespace jacobi_detail

// One-sided (Hestenes) Jacobi on the columns of M (n x n, n <= 64, column-major shared memory
// with leading dimension SDPXG_LD): on return M holds M V = U diag(sigma), columns in their
// original order; V itself is not formed.  Returns the number of sweeps, or -1 when the sweep
// bound was hit.  Every thread of the CTA calls it (blockDim.x >= 256).
//
// The matrix stays in registers for the whole iteration.  Warps 0..7 take part: warp w holds
// rows [8w, 8w + 8), lane j the columns at positions 2j (A) and 2j+1 (B) of a line of
// N = n rounded up to even positions (an odd n gets a zero column that never rotates).  The
// pairs follow the odd-even ordering of Luk and Park: rounds alternate between the pairs
// (2j, 2j+1), which a lane holds itself, and (2j+1, 2j+2), whose second column comes from lane
// j+1 by a warp shuffle; after every rotation the two columns trade places, so in N rounds
// every pair meets once (the moves are those of odd-even transposition sort on a reversed
// line).  Only the across-lane rounds move data (two shuffles per row), and the lane that
// computes a pair's rotation hands (c, s) to its right neighbour.  A pair's inner product is
// the sum of the eight warps' row partials, taken in a fixed tree order, so every warp holds
// the same bits and takes the same decisions without a broadcast; one named barrier per round
// (the partials are double-buffered in `part`, 1536 doubles of shared memory).  Squared column
// norms are summed exactly at the start of every sweep and carried through its rotations
// (a - tg, b + tg).  A pair rotates while |x'y| > 1e-15 sqrt(||x||^2 ||y||^2); the sweeps stop
// after one without a rotation, or after one in which every cosine was below 1e-10 (the
// rotations of that sweep leave cosines of order 1e-20: one-sided Jacobi converges
// quadratically).
__device__ inline int cta_jacobi_left(double* M, int n, double* part, int* out) {
  using namespace jacobi_detail;
  constexpr double kTol2 = 1e-30, kBig2 = 1e-20;
  constexpr unsigned kFull = 0xffffffffu;
  const int warp = threadIdx.x >> 5, j = threadIdx.x & 31;
  if (warp < 8) {
    const int N = n + (n & 1), H = N / 2;
    int iA = j < H ? 2 * j : -1, iB = j < H ? 2 * j + 1 : -1;
    double A[8], B[8], nA = 0.0, nB = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int row = 8 * warp + k;
      A[k] = (row < n && iA >= 0 && iA < n) ? SM(M, row, iA) : 0.0;
      B[k] = (row < n && iB >= 0 && iB < n) ? SM(M, row, iB) : 0.0;
    }
    int sweeps = (n < 2) ? 0 : -1;
    int phase = 0;
    for (int sweep = 0; n >= 2 && sweep < SDPXG_JACOBI_MAX_SWEEPS; ++sweep) {
      bool rotated = false, big = false;
      for (int r = 0; r < N; r += 2) {
        {  // pairs (2j, 2j+1): both columns in this lane
          double* buf = part + phase * 768;
          phase ^= 1;
          buf[warp * 32 + j] = dot8(A, B);
          if (r == 0) {
            buf[256 + warp * 32 + j] = dot8(A, A);
            buf[512 + warp * 32 + j] = dot8(B, B);
          }
          asm volatile("bar.sync 1, 256;" ::: "memory");
          const double g = sum8(buf + j);
          if (r == 0) {
            nA = sum8(buf + 256 + j);
            nB = sum8(buf + 512 + j);
          }
          const double a = nA, b = nB, gg = g * g, ab = a * b;
          const bool rot = j < H && gg > kTol2 * ab;
          rotated |= rot;
          big |= j < H && gg > kBig2 * ab;
          double c = 1.0, s = 0.0, tg = 0.0;
          if (rot) rotation(a, b, g, c, s, tg);
#pragma unroll
          for (int k = 0; k < 8; ++k) {  // rotate and trade places: A <- y', B <- x'
            const double x = A[k], y = B[k];
            A[k] = fma(s, x, c * y);
            B[k] = fma(c, x, -s * y);
          }
          nA = b + tg;
          nB = a - tg;
          const int t = iA;
          iA = iB;
          iB = t;
        }
        {  // pairs (2j+1, 2j+2): this lane's B and lane j+1's A
          double An[8], Bp[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            An[k] = __shfl_down_sync(kFull, A[k], 1);
            Bp[k] = __shfl_up_sync(kFull, B[k], 1);
          }
          const double nAn = __shfl_down_sync(kFull, nA, 1);
          const int iAn = __shfl_down_sync(kFull, iA, 1), iBp = __shfl_up_sync(kFull, iB, 1);
          double* buf = part + phase * 768;
          phase ^= 1;
          buf[warp * 32 + j] = dot8(B, An);
          asm volatile("bar.sync 1, 256;" ::: "memory");
          const double g = sum8(buf + j);
          const bool ex = j + 1 < H;  // pair (2j+1, 2j+2) exists
          const double a = nB, b = nAn, gg = g * g, ab = a * b;
          const bool rot = ex && gg > kTol2 * ab;
          rotated |= rot;
          big |= ex && gg > kBig2 * ab;
          double c = ex ? 1.0 : 0.0, s = ex ? 0.0 : 1.0, tg = 0.0;  // no pair: B stays
          if (rot) rotation(a, b, g, c, s, tg);
          double cl = __shfl_up_sync(kFull, c, 1), sl = __shfl_up_sync(kFull, s, 1);
          const double nAl = __shfl_up_sync(kFull, a - tg, 1);
          const bool recv = j >= 1 && j < H;  // lane j's A is the right column of pair j-1
          if (!recv) {
            cl = 0.0;
            sl = -1.0;
          }
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            B[k] = fma(s, B[k], c * An[k]);   // y' of pair j
            A[k] = fma(cl, Bp[k], -sl * A[k]);  // x' of pair j-1
          }
          if (ex) {
            nB = b + tg;
            iB = iAn;
          }
          if (recv) {
            nA = nAl;
            iA = iBp;
          }
        }
      }
      if (!__any_sync(kFull, rotated) || !__any_sync(kFull, big)) {
        sweeps = sweep + 1;
        break;
      }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int row = 8 * warp + k;
      if (row < n && j < H) {
        if (iA < n) SM(M, row, iA) = A[k];
        if (iB < n) SM(M, row, iB) = B[k];
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
// `work` is 2*n doubles of shared memory, `red` 32 doubles.  blockDim.x is a multiple of 64.
// Step k reflects column k below the diagonal, x = A[k+1:n, k] (m <= 63 entries): warp 0 forms
// |x|^2, the reflector's scale and v = (x - alpha e1) / |x - alpha e1| into shared memory (one
// barrier); p = A v, one warp per row reading the row as a column (A stays exactly symmetric;
// a barrier); warp 0 forms K = v'p and q = p - K v in place of p (a barrier); then the rank-2
// update A -= 2 (v q' + q v'), thread t on row t % 64 of the columns t / 64 + 16 s (a barrier).
__device__ inline void cta_tridiagonalize(double* A, int n, double* d, double* e, double* work,
                                          double* red) {
  double* p = work;
  double* v = work + n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;  // length of the column below the diagonal
    const double* x = &SM(A, k + 1, k);
    if (warp == 0) {
      double part = 0.0;
      for (int i = lane; i < m; i += 32) part = fma(x[i], x[i], part);
      const double nrm2 = warp_sum(part);
      const double x0 = x[0];
      const double alpha = -copysign(sqrt(nrm2), x0);
      const double vnorm2 = nrm2 - x0 * x0 + (x0 - alpha) * (x0 - alpha);
      const bool skip = (nrm2 == 0.0 || vnorm2 == 0.0);  // column already reduced
      const double vs = skip ? 0.0 : rsqrt(vnorm2);
      for (int i = lane; i < m; i += 32) v[i] = (i == 0) ? (x0 - alpha) * vs : x[i] * vs;
      if (lane == 0) {
        d[k] = SM(A, k, k);
        e[k] = (nrm2 == 0.0) ? 0.0 : alpha;
        red[0] = skip ? 0.0 : 1.0;
      }
    }
    __syncthreads();
    if (red[0] == 0.0) {
      __syncthreads();  // red[0] is read by every thread before warp 0 rewrites it
      continue;
    }
    // p = A_sub v
    for (int i = warp; i < m; i += nwarps) {
      double acc = 0.0;
      for (int j = lane; j < m; j += 32) acc = fma(SM(A, k + 1 + j, k + 1 + i), v[j], acc);
      acc = warp_sum(acc);
      if (lane == 0) p[i] = acc;
    }
    __syncthreads();
    if (warp == 0) {  // K = v'p, then p <- q = p - K v in place
      double kp = 0.0;
      for (int i = lane; i < m; i += 32) kp = fma(v[i], p[i], kp);
      const double K = warp_sum(kp);
      for (int i = lane; i < m; i += 32) p[i] = p[i] - K * v[i];
    }
    __syncthreads();
    // A_sub -= 2 (v q' + q v') (both triangles from the same two products)
    const int ri = threadIdx.x & 63, cstride = blockDim.x >> 6;
    if (ri < m) {
      const double vi = v[ri], qi = p[ri];
      for (int j = threadIdx.x >> 6; j < m; j += cstride) {
        const double vj = v[j], qj = p[j];
        const double u = __dadd_rn(__dmul_rn(vi, qj), __dmul_rn(qi, vj));
        SM(A, k + 1 + ri, k + 1 + j) -= 2.0 * u;
      }
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

// Number of eigenvalues of the tridiagonal (d, e) strictly below x.  The quotient of each step
// takes the Newton-refined reciprocal (recip_newton: a few units in the last place), which
// keeps the count that of a matrix within a few ulps of (d, e); |q| >= pivmin throughout.
__device__ __forceinline__ int sturm_count(const double* d, const double* e, int n, double x,
                                           double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += (q < 0.0);
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - e[i - 1] * e[i - 1] * copysign(recip_newton(fabs(q)), q);
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
