// PSD-cone kernels: Nesterov-Todd scaling, W congruences, Jordan products, step lengths
// and interior margins.  One CTA per PSD block (and per right-hand side or side of the
// step); every block of order <= SDPXG_NMAX lives in shared memory for the whole kernel.
//
// Reference functions restated (crates/solver/src/solver/cones/psdtrianglecone.rs):
//   update_scaling 311-439, mul_Wx_scratch 860-917, circ_op 927-938,
//   lambda_inv_circ_op 757-780, affine_ds 455-460, step_length_psd_component 1180-1231,
//   admits 1168-1178, margins ~590-606; and the binary64 factored Hs / Hs^-1 application
//   of kkt/condensed/psd.rs:1968-2002.
#include "eig.cuh"

namespace {

constexpr int kMat = SDPXG_LD * SDPXG_NMAX;  // doubles per shared matrix

}  // namespace

// ---------------------------------------------------------------------------------------
// NT scaling.  L1 = chol(S), L2 = chol(Z), L2'L1 = U diag(lam) V' (psdtrianglecone.rs:311-439).
// The reference forms R = L1 V lam^-1/2 and Rinv = lam^1/2 V' L1^-1.  With M = L2'L1 and
// M V = U lam, the same matrices are
//   R = L2^-T U lam^1/2,   Rinv = lam^-1/2 U' L2'
// (L1 V = L1 M^-1 U lam = L2^-T U lam), which needs only the LEFT singular vectors: the
// normalised columns that one-sided Jacobi leaves in M, so the rotations are not accumulated
// into V.  Both forms have the same
// normwise accuracy (a triangular solve with L1 or with L2 each).  Ginv = Rinv' Rinv.
// Two launches: k_nt_factor (1024 threads: both Cholesky factors in the register-resident CTA
// form, M = L2'L1) leaves M in R's slot and L2 in Rinv's slot of each block; k_nt_svd (512
// threads, room for the register-resident Jacobi) reads them back and writes R, Rinv, Ginv,
// lam and lam^-1/2.  A failed factorisation sets SDPXG_ST_CHOL_FAIL, which the second launch
// reads to leave every block alone (the scaling is rejected as a whole).
// Shared memory of k_nt_factor: 3 matrices + 2 Cholesky scratches; of k_nt_svd: 5 matrices +
// 2n doubles + n ints + 1 int.
// ---------------------------------------------------------------------------------------
extern "C" __global__ void __launch_bounds__(SDPXG_CONE_THREADS)
k_nt_factor(const BlockDesc* __restrict__ blocks, const double* __restrict__ s,
            const double* __restrict__ z, double* __restrict__ R, double* __restrict__ Rinv,
            uint32_t* __restrict__ status) {
  extern __shared__ double smem[];
  const BlockDesc bd = blocks[blockIdx.x];
  const int n = bd.n;
  double* L1 = smem;
  double* L2 = L1 + kMat;
  double* M = L2 + kMat;
  double* piv = M + kMat;
  double* piv2 = piv + SDPXG_CHOL_SCRATCH;
  cta_zero_mat(M);
  cta_load_smat(L1, s + bd.svec_off, n);
  cta_load_smat(L2, z + bd.svec_off, n);
  bool ok1, ok2;
  cta_cholesky_lower2(L1, L2, n, piv, piv2, &ok1, &ok2);  // chol(S), chol(Z) together
  if (!ok1 || !ok2) {
    if (threadIdx.x == 0) atomicOr(status, SDPXG_ST_CHOL_FAIL);
    return;
  }
  cta_gemm(M, L2, true, L1, false, n);  // M = L2' L1
  __syncthreads();
  cta_store_mat(R + bd.mat_off, M, n);
  cta_store_mat(Rinv + bd.mat_off, L2, n);
}

extern "C" __global__ void __launch_bounds__(SDPXG_NT_SVD_THREADS)
k_nt_svd(const BlockDesc* __restrict__ blocks, double* __restrict__ R, double* __restrict__ Rinv,
         double* __restrict__ Ginv, double* __restrict__ lam, double* __restrict__ lisqrt,
         uint32_t* __restrict__ status) {
  extern __shared__ double smem[];
  if (*status & SDPXG_ST_CHOL_FAIL) return;
  const BlockDesc bd = blocks[blockIdx.x];
  const int n = bd.n;
  double* L1 = smem;
  double* L2 = L1 + kMat;
  double* M = L2 + kMat;
  double* V = M + kMat;
  double* X = V + kMat;
  double* sig = X + kMat;
  double* lsort = sig + SDPXG_NMAX;
  int* rank = reinterpret_cast<int*>(lsort + SDPXG_NMAX);
  int* flag = rank + SDPXG_NMAX;

  cta_zero_mat(V);  // V and X are written n x n only: keep their padding zero for the MMAs
  cta_zero_mat(X);
  cta_load_mat(M, R + bd.mat_off, n);
  cta_load_mat(L2, Rinv + bd.mat_off, n);
  __syncthreads();
  int sweeps = cta_jacobi_left(M, n, L1, flag);  // M -> U diag(lam); L1 as scratch
  if (sweeps < 0) {
    if (threadIdx.x == 0) atomicOr(status, SDPXG_ST_SVD_UNCONVERGED);
    return;
  }
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double acc = 0.0;
    for (int k = 0; k < n; ++k) acc = fma(SM(M, k, j), SM(M, k, j), acc);
    sig[j] = sqrt(acc);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    int r = 0;
    for (int k = 0; k < n; ++k) r += (sig[k] > sig[j]) || (sig[k] == sig[j] && k < j);
    rank[j] = r;
    lsort[r] = sig[j];
  }
  __syncthreads();
  bool good = true;
  for (int j = 0; j < n; ++j) good = good && (lsort[j] > 0.0) && isfinite(lsort[j]);
  if (!good) {
    if (threadIdx.x == 0) atomicOr(status, SDPXG_ST_CHOL_FAIL);
    return;
  }
  // X = U with columns in descending singular-value order; V = X as the right-hand side
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;
    const double u = SM(M, i, j) / sig[j];
    SM(X, i, rank[j]) = u;
    SM(V, i, rank[j]) = u;
  }
  __syncthreads();
  cta_trsm_lower_t_blocked(L2, V, n, sig);  // V = L2^-T U (sig is free: lsort holds lambda)
  double* Rg = R + bd.mat_off;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;
    Rg[e] = SM(V, i, j) * sqrt(lsort[j]);
  }
  cta_gemm(L1, X, true, L2, true, n);  // L1 = U' L2'
  __syncthreads();
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;
    SM(L1, i, j) /= sqrt(lsort[i]);  // Rinv = lam^-1/2 U' L2'
  }
  __syncthreads();
  cta_store_mat(Rinv + bd.mat_off, L1, n);
  cta_gemm(M, L1, true, L1, false, n);  // Ginv = Rinv' Rinv
  __syncthreads();
  cta_store_mat(Ginv + bd.mat_off, M, n);
  bool fin = true;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x)
    fin = fin && isfinite(SM(M, e % n, e / n)) && isfinite(SM(L1, e % n, e / n));
  if (!fin) atomicOr(status, SDPXG_ST_NONFINITE);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    lam[bd.vec_off + j] = lsort[j];
    lisqrt[bd.vec_off + j] = 1.0 / sqrt(lsort[j]);
  }
}

// Identity scaling: R = Rinv = Ginv = I, lam = 1 (the default start, core/solver.rs:1212).
extern "C" __global__ void k_identity_scaling(const BlockDesc* __restrict__ blocks,
                                              double* R, double* Rinv, double* Ginv, double* lam,
                                              double* lisqrt) {
  const BlockDesc bd = blocks[blockIdx.x];
  const int n = bd.n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    double v = (e % n == e / n) ? 1.0 : 0.0;
    R[bd.mat_off + e] = v;
    Rinv[bd.mat_off + e] = v;
    Ginv[bd.mat_off + e] = v;
  }
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    lam[bd.vec_off + j] = 1.0;
    lisqrt[bd.vec_off + j] = 1.0;
  }
}

// G^-1 = R^-T R^-1 per block from a given R^-1 (column-major n x n): G^-1(a, b) =
// sum_r R^-1(r, a) R^-1(r, b), summed in r order (exactly symmetric).
extern "C" __global__ void k_ginv_from_rinv(const BlockDesc* __restrict__ blocks, const double* __restrict__ Rinv,
                                            double* __restrict__ Ginv) {
  const BlockDesc bd = blocks[blockIdx.x];
  const int n = bd.n;
  const double* X = Rinv + bd.mat_off;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int a = e % n, b = e / n;
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    double acc = 0.0;
    for (int r = 0; r < n; ++r) acc = fma(X[r + lo * n], X[r + hi * n], acc);
    Ginv[bd.mat_off + e] = acc;
  }
}

// ---------------------------------------------------------------------------------------
// Congruences on svec vectors.  mode:
//   0  W x     = svec(R' X R)          1  W' x     = svec(R X R')
//   2  Winv x  = svec(Rinv' X Rinv)    3  Winv' x  = svec(Rinv X Rinv')
//   4  Hs x    = W'(W x)  (two congruences through R, never the squared G)
//   5  Hs^-1 x = Winv(Winv' x)
// grid = (blocks, columns); column c of x / y starts at c * ld.
// ---------------------------------------------------------------------------------------
__device__ void cta_congruence(double* Y, double* T, const double* X, const double* B,
                               bool outer_t, int n) {
  // outer_t: Y = B X B'  else Y = B' X B
  if (outer_t) {
    cta_gemm(T, X, false, B, true, n);  // T = X B'
    __syncthreads();
    cta_gemm(Y, B, false, T, false, n);  // Y = B T
  } else {
    cta_gemm(T, X, false, B, false, n);  // T = X B
    __syncthreads();
    cta_gemm(Y, B, true, T, false, n);  // Y = B' T
  }
  __syncthreads();
}

extern "C" __global__ void __launch_bounds__(SDPXG_CONE_THREADS)
k_congruence(const BlockDesc* __restrict__ blocks, int mode, const double* __restrict__ R,
             const double* __restrict__ Rinv, const double* __restrict__ x, double* __restrict__ y,
             long ld) {
  extern __shared__ double smem[];
  const BlockDesc bd = blocks[blockIdx.x];
  const int n = bd.n;
  const long coff = (long)blockIdx.y * ld;
  double* B = smem;
  double* X = B + kMat;
  double* T = X + kMat;
  double* Y = T + kMat;
  const bool use_r = (mode == 0 || mode == 1 || mode == 4);
  cta_load_mat(B, (use_r ? R : Rinv) + bd.mat_off, n);
  cta_load_smat(X, x + coff + bd.svec_off, n);
  __syncthreads();
  if (mode <= 3) {
    cta_congruence(Y, T, X, B, mode == 1 || mode == 3, n);
  } else {
    // first stage: W x (R' X R) for Hs, Winv' x (Rinv X Rinv') for Hs^-1
    cta_congruence(Y, T, X, B, mode == 5, n);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      int i = e % n, j = e / n;
      SM(X, i, j) = 0.5 * (SM(Y, i, j) + SM(Y, j, i));
    }
    __syncthreads();
    cta_congruence(Y, T, X, B, mode == 4, n);
  }
  cta_store_svec(y + coff + bd.svec_off, Y, n);
}

// x = svec((Y Z + Z Y) / 2) per block.
extern "C" __global__ void __launch_bounds__(SDPXG_CONE_THREADS)
k_circ_op(const BlockDesc* __restrict__ blocks, const double* __restrict__ yv,
          const double* __restrict__ zv, double* __restrict__ xv) {
  extern __shared__ double smem[];
  const BlockDesc bd = blocks[blockIdx.x];
  const int n = bd.n;
  double* Y = smem;
  double* Z = Y + kMat;
  cta_load_smat(Y, yv + bd.svec_off, n);
  cta_load_smat(Z, zv + bd.svec_off, n);
  __syncthreads();
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;
    if (i > j) continue;
    double a = 0.0, b = 0.0;
    for (int k = 0; k < n; ++k) {
      a = fma(SM(Y, i, k), SM(Z, k, j), a);
      b = fma(SM(Z, i, k), SM(Y, k, j), b);
    }
    double v = 0.5 * (a + b);
    xv[bd.svec_off + tri_idx(i, j)] = (i == j) ? v : v * SDPXG_SQRT2;
  }
}

// x = lambda \ z: X_ij = 2 Z_ij / (lam_i + lam_j) (svec scaling commutes).
extern "C" __global__ void k_lam_inv_circ(const BlockDesc* __restrict__ blocks,
                                          const double* __restrict__ lam,
                                          const double* __restrict__ zv, double* __restrict__ xv) {
  const BlockDesc bd = blocks[blockIdx.x];
  const int n = bd.n;
  for (int e = threadIdx.x; e < n * (n + 1) / 2; e += blockDim.x) {
    int j = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
    while (j * (j + 1) / 2 > e) --j;
    while ((j + 1) * (j + 2) / 2 <= e) ++j;
    int i = e - j * (j + 1) / 2;
    xv[bd.svec_off + e] = 2.0 * zv[bd.svec_off + e] / (lam[bd.vec_off + i] + lam[bd.vec_off + j]);
  }
}

// ds = svec(diag(lam^2)), plus a multiple of the identity: ds += a * I.
extern "C" __global__ void k_affine_ds(const BlockDesc* __restrict__ blocks,
                                       const double* __restrict__ lam, double* __restrict__ ds) {
  const BlockDesc bd = blocks[blockIdx.x];
  const int n = bd.n;
  for (int e = threadIdx.x; e < n * (n + 1) / 2; e += blockDim.x) ds[bd.svec_off + e] = 0.0;
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double l = lam[bd.vec_off + k];
    ds[bd.svec_off + tri_idx(k, k)] = l * l;
  }
}

// v[diag] += a  (scaled_unit_shift, psdtrianglecone.rs:260-266)
extern "C" __global__ void k_shift_unit(const BlockDesc* __restrict__ blocks, double* v, double a) {
  const BlockDesc bd = blocks[blockIdx.x];
  for (int k = threadIdx.x; k < bd.n; k += blockDim.x) v[bd.svec_off + tri_idx(k, k)] += a;
}

// ---------------------------------------------------------------------------------------
// Step length per (block, side).  side 0: dual, Delta = lam^-1/2 (R' dZ R) lam^-1/2;
// side 1: primal, Delta = lam^-1/2 (Rinv dS Rinv') lam^-1/2.
// mode 0: bound  alpha = amax if chol(I + amax Delta) succeeds, else min(-1/lmin, amax);
// mode 1: admission only (out = amax if admitted else 0).
// out[2*block + side].
// ---------------------------------------------------------------------------------------
extern "C" __global__ void __launch_bounds__(SDPXG_CONE_THREADS)
k_step_length(const BlockDesc* __restrict__ blocks, const double* __restrict__ R,
              const double* __restrict__ Rinv, const double* __restrict__ lisqrt,
              const double* __restrict__ dz, const double* __restrict__ ds, double amax, int mode,
              double* __restrict__ out, uint32_t* __restrict__ status) {
  extern __shared__ double smem[];
  const int b = blockIdx.x, side = blockIdx.y;
  const BlockDesc bd = blocks[b];
  const int n = bd.n;
  double* B = smem;
  double* X = B + kMat;
  double* T = X + kMat;
  double* D = T + kMat;
  double* small = D + kMat;  // Cholesky scratch, d[n], e[n], work[2n], red[32]
  double* piv = small;
  double* dd = piv + SDPXG_CHOL_SCRATCH;
  double* ee = dd + SDPXG_NMAX;
  double* work = ee + SDPXG_NMAX;
  double* red = work + 2 * SDPXG_NMAX;
  cta_load_mat(B, (side == 0 ? R : Rinv) + bd.mat_off, n);
  cta_load_smat(X, (side == 0 ? dz : ds) + bd.svec_off, n);
  __syncthreads();
  cta_congruence(D, T, X, B, side == 1, n);
  const double* ls = lisqrt + bd.vec_off;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;
    double v = 0.5 * (SM(D, i, j) + SM(D, j, i));
    SM(X, i, j) = ls[i] * v * ls[j];  // Delta (symmetric)
  }
  __syncthreads();
  double res = amax;
  // admission: chol(I + amax Delta)
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;
    SM(T, i, j) = amax * SM(X, i, j) + (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  bool admitted = (n <= 3 && mode == 0) ? false : cta_cholesky_lower(T, n, piv);
  if (mode == 1) {
    if (threadIdx.x == 0) out[2 * b + side] = admitted ? amax : 0.0;
    return;
  }
  if (!admitted) {
    cta_tridiagonalize(X, n, dd, ee, work, red);
    bool ok = true;
    double g = cta_eig_min(dd, ee, n, reinterpret_cast<int*>(red), &ok);
    if (!ok || !isfinite(g)) {
      if (threadIdx.x == 0) atomicOr(status, SDPXG_ST_EIG_FAIL);
      res = 0.0;
    } else {
      res = (g < 0.0) ? fmin(-1.0 / g, amax) : amax;
    }
  }
  if (threadIdx.x == 0) out[2 * b + side] = res;
}

// Eigenvalue summary of smat(v) per block: out[2b] = lambda_min, out[2b+1] = sum of positive
// eigenvalues.  (margins, psdtrianglecone.rs; also the cone distance of the original-
// coordinate acceptance test, default/original_check.rs:306-340.)
// min_only != 0 (the acceptance test, which reads only max(0, -lambda_min)): out[2b] =
// min(lambda_min, 0) and out[2b+1] = 0.  A block whose Cholesky factorisation succeeds is
// positive definite to working accuracy and gives 0 without an eigensolve; the others take the
// tridiagonal reduction and the multisection for lambda_min alone.
extern "C" __global__ void __launch_bounds__(SDPXG_CONE_THREADS)
k_margins(const BlockDesc* __restrict__ blocks, const double* __restrict__ v, long ld,
          double* __restrict__ out, uint32_t* __restrict__ status, int min_only) {
  extern __shared__ double smem[];
  const int b = blockIdx.x;
  const BlockDesc bd = blocks[b];
  const int n = bd.n;
  double* X = smem;
  double* dd = X + kMat;
  double* ee = dd + SDPXG_NMAX;
  double* work = ee + SDPXG_NMAX;
  double* red = work + 2 * SDPXG_NMAX;
  double* eig = red + 32;
  const double* vb = v + (long)blockIdx.y * ld + bd.svec_off;
  const long o = 2L * ((long)blockIdx.y * gridDim.x + b);
  cta_load_smat(X, vb, n);
  __syncthreads();
  if (min_only) {
    if (cta_cholesky_lower(X, n, dd)) {
      if (threadIdx.x == 0) out[o] = out[o + 1] = 0.0;
      return;
    }
    cta_load_smat(X, vb, n);
    __syncthreads();
    cta_tridiagonalize(X, n, dd, ee, work, red);
    bool ok = true;
    const double g = cta_eig_min(dd, ee, n, reinterpret_cast<int*>(red), &ok);
    if (threadIdx.x == 0) {
      if (!ok || !isfinite(g)) atomicOr(status, SDPXG_ST_EIG_FAIL);
      out[o] = fmin(g, 0.0);
      out[o + 1] = 0.0;
    }
    return;
  }
  cta_tridiagonalize(X, n, dd, ee, work, red);
  cta_eig_all(dd, ee, n, eig, status);
  __syncthreads();
  if (threadIdx.x == 0) {
    double mn = eig[0], pos = 0.0;
    for (int k = 0; k < n; ++k) {
      mn = fmin(mn, eig[k]);
      pos += fmax(eig[k], 0.0);
    }
    out[o] = mn;
    out[o + 1] = pos;
  }
}
