// Dense Cholesky of the Schur complement with the reference's dynamic pivot rule, the
// triangular solves that use it, and the Schur matvec of the inner refinement.
//
// Right-looking tiled factorisation H = U'U (upper), tile NB = 64:
//   k_potrf_diag   factor the diagonal tile with the dynamic pivot rule and store
//                  Dinv = U_kk^-1 (kkt/ldl/dense_block.rs:334-365, 370-388, 515-594)
//   k_trsm_panel   U[k, j] = U_kk^-T H[k, j] for the tiles right of the diagonal
//   k_syrk_update  H[i, j] -= U[k, i]' U[k, j] on the upper trailing tiles
// Solves U'y = b then Ux = y run one launch per tile row using the stored Dinv
// (kkt/ldl/dense_block.rs:604-669 tiled_trsv).
#include "common.cuh"

#define CH_NB 64
#define CH_LD (CH_NB + 1)

// ------------------------------------------------------------------------------------
extern "C" __global__ void __launch_bounds__(SDPXG_THREADS)
k_potrf_diag(double* __restrict__ H, int m, int kb, double eps, double delta, int dynamic,
             const double* __restrict__ diag0, double* __restrict__ Dinv,
             uint32_t* __restrict__ status) {
  __shared__ double A[CH_NB * CH_LD];
  __shared__ double dmod[CH_NB];
  const int k0 = kb * CH_NB;
  const int nb = min(CH_NB, m - k0);
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e % nb, j = e / nb;
    if (i <= j) A[i + j * CH_LD] = H[(k0 + i) + (long)(k0 + j) * m];
  }
  for (int k = 0; k < nb; ++k) {
    __syncthreads();
    double d = A[k + k * CH_LD];
    bool fail = !isfinite(d);
    if (!fail && dynamic && d <= eps) {
      if (d < -64.0 * 2.220446049250313e-16 * nb * fabs(diag0[k0 + k])) fail = true;
      else d = delta;
    }
    if (!fail && !(d > 0.0)) fail = true;
    if (fail) {
      if (threadIdx.x == 0) atomicOr(status, SDPXG_ST_PIVOT_FAIL);
      return;  // uniform: every thread read the same pivot
    }
    if (threadIdx.x == 0) dmod[k] = d;
    const int rem = nb - k - 1;
    const double dinv = 1.0 / d;
    for (int e = threadIdx.x; e < rem * rem; e += blockDim.x) {
      int i = k + 1 + e % rem, j = k + 1 + e / rem;
      if (i > j) continue;
      A[i + j * CH_LD] -= A[k + i * CH_LD] * A[k + j * CH_LD] * dinv;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e % nb, j = e / nb;
    if (i > j) continue;
    double r = sqrt(dmod[i]);
    double u = (i == j) ? r : A[i + j * CH_LD] / r;
    A[i + j * CH_LD] = u;
    H[(k0 + i) + (long)(k0 + j) * m] = u;
  }
  __syncthreads();
  // Dinv = U^-1 (upper), one column per thread; zero below the diagonal.
  double* D = Dinv + (long)kb * CH_NB * CH_NB;
  for (int j = threadIdx.x; j < CH_NB; j += blockDim.x) {
    double x[CH_NB];
    for (int i = 0; i < CH_NB; ++i) x[i] = 0.0;
    if (j < nb) {
      x[j] = 1.0 / A[j + j * CH_LD];
      for (int i = j - 1; i >= 0; --i) {
        double acc = 0.0;
        for (int l = i + 1; l <= j; ++l) acc = fma(A[i + l * CH_LD], x[l], acc);
        x[i] = -acc / A[i + i * CH_LD];
      }
    }
    for (int i = 0; i < CH_NB; ++i) D[i + j * CH_NB] = x[i];
  }
}

// ------------------------------------------------------------------------------------
extern "C" __global__ void __launch_bounds__(SDPXG_THREADS)
k_trsm_panel(double* __restrict__ H, int m, int kb, const double* __restrict__ Dinv) {
  extern __shared__ double sm[];
  double* D = sm;                 // CH_NB x CH_LD
  double* P = D + CH_NB * CH_LD;  // CH_NB x CH_LD
  const int k0 = kb * CH_NB, nb = min(CH_NB, m - k0);
  const int cb = kb + 1 + blockIdx.x;
  const int c0 = cb * CH_NB, nc = min(CH_NB, m - c0);
  const double* Dg = Dinv + (long)kb * CH_NB * CH_NB;
  for (int e = threadIdx.x; e < CH_NB * CH_NB; e += blockDim.x)
    D[(e % CH_NB) + (e / CH_NB) * CH_LD] = Dg[e];
  for (int e = threadIdx.x; e < nb * nc; e += blockDim.x) {
    int i = e % nb, c = e / nb;
    P[i + c * CH_LD] = H[(k0 + i) + (long)(c0 + c) * m];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * nc; e += blockDim.x) {
    int i = e % nb, c = e / nb;
    double acc = 0.0;
    for (int l = 0; l <= i; ++l) acc = fma(D[l + i * CH_LD], P[l + c * CH_LD], acc);
    H[(k0 + i) + (long)(c0 + c) * m] = acc;
  }
}

// ------------------------------------------------------------------------------------
// Trailing update on upper tiles; blockIdx.x enumerates (ib <= jb) over the T x T trailing
// tile grid in column order.
extern "C" __global__ void __launch_bounds__(SDPXG_THREADS)
k_syrk_update(double* __restrict__ H, int m, int kb) {
  extern __shared__ double syrk_sm[];
  double (*Ui)[CH_NB + 2] = reinterpret_cast<double (*)[CH_NB + 2]>(syrk_sm);
  double (*Uj)[CH_NB + 2] = reinterpret_cast<double (*)[CH_NB + 2]>(syrk_sm + CH_NB * (CH_NB + 2));
  const int t = blockIdx.x;
  int jb = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while (jb * (jb + 1) / 2 > t) --jb;
  while ((jb + 1) * (jb + 2) / 2 <= t) ++jb;
  int ib = t - jb * (jb + 1) / 2;
  ib += kb + 1;
  jb += kb + 1;
  const int k0 = kb * CH_NB, nb = min(CH_NB, m - k0);
  const int i0 = ib * CH_NB, ni = min(CH_NB, m - i0);
  const int j0 = jb * CH_NB, nj = min(CH_NB, m - j0);
  for (int e = threadIdx.x; e < CH_NB * CH_NB; e += blockDim.x) {
    int l = e % CH_NB, c = e / CH_NB;
    Ui[l][c] = (l < nb && c < ni) ? H[(k0 + l) + (long)(i0 + c) * m] : 0.0;
    Uj[l][c] = (l < nb && c < nj) ? H[(k0 + l) + (long)(j0 + c) * m] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int l = 0; l < nb; ++l) {
    double x[4], y[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) x[a] = Ui[l][tx + 16 * a];
#pragma unroll
    for (int b = 0; b < 4; ++b) y[b] = Uj[l][ty + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      int r = tx + 16 * a, c = ty + 16 * b;
      if (r < ni && c < nj && (ib < jb || r <= c)) H[(i0 + r) + (long)(j0 + c) * m] -= acc[a][b];
    }
}

// ------------------------------------------------------------------------------------
// Forward step kb of U'y = b (ncols <= 4 right-hand sides, column stride ld).
extern "C" __global__ void __launch_bounds__(SDPXG_THREADS)
k_trsv_fwd(const double* __restrict__ H, int m, int kb, const double* __restrict__ Dinv,
           double* __restrict__ b, double* __restrict__ y, long ld, int ncols) {
  __shared__ double bk[CH_NB * 4];
  __shared__ double yk[CH_NB * 4];
  const int k0 = kb * CH_NB, nb = min(CH_NB, m - k0);
  const int cb = kb + blockIdx.x;
  const double* D = Dinv + (long)kb * CH_NB * CH_NB;
  for (int e = threadIdx.x; e < nb * ncols; e += blockDim.x) {
    int i = e % nb, c = e / nb;
    bk[i + c * CH_NB] = b[(k0 + i) + c * ld];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * ncols; e += blockDim.x) {
    int i = e % nb, c = e / nb;
    double acc = 0.0;
    for (int l = 0; l <= i; ++l) acc = fma(D[l + i * CH_NB], bk[l + c * CH_NB], acc);
    yk[i + c * CH_NB] = acc;
  }
  __syncthreads();
  if (cb == kb) {
    for (int e = threadIdx.x; e < nb * ncols; e += blockDim.x) {
      int i = e % nb, c = e / nb;
      y[(k0 + i) + c * ld] = yk[i + c * CH_NB];
    }
    return;
  }
  const int c0 = cb * CH_NB, nc = min(CH_NB, m - c0);
  for (int e = threadIdx.x; e < nc * ncols; e += blockDim.x) {
    int q = e % nc, c = e / nc;
    const double* col = H + k0 + (long)(c0 + q) * m;
    double acc = 0.0;
    for (int l = 0; l < nb; ++l) acc = fma(col[l], yk[l + c * CH_NB], acc);
    b[(c0 + q) + c * ld] -= acc;
  }
}

// Backward step kb of Ux = y (y updated in place for the rows above).
extern "C" __global__ void __launch_bounds__(SDPXG_THREADS)
k_trsv_bwd(const double* __restrict__ H, int m, int kb, const double* __restrict__ Dinv,
           double* __restrict__ y, double* __restrict__ x, long ld, int ncols) {
  __shared__ double yk[CH_NB * 4];
  __shared__ double xk[CH_NB * 4];
  const int k0 = kb * CH_NB, nb = min(CH_NB, m - k0);
  const int rb = blockIdx.x;
  const double* D = Dinv + (long)kb * CH_NB * CH_NB;
  for (int e = threadIdx.x; e < nb * ncols; e += blockDim.x) {
    int i = e % nb, c = e / nb;
    yk[i + c * CH_NB] = y[(k0 + i) + c * ld];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * ncols; e += blockDim.x) {
    int i = e % nb, c = e / nb;
    double acc = 0.0;
    for (int l = i; l < nb; ++l) acc = fma(D[i + l * CH_NB], yk[l + c * CH_NB], acc);
    xk[i + c * CH_NB] = acc;
  }
  __syncthreads();
  if (rb == kb) {
    for (int e = threadIdx.x; e < nb * ncols; e += blockDim.x) {
      int i = e % nb, c = e / nb;
      x[(k0 + i) + c * ld] = xk[i + c * CH_NB];
    }
    return;
  }
  const int r0 = rb * CH_NB;  // full tile (rb < kb)
  for (int e = threadIdx.x; e < CH_NB * ncols; e += blockDim.x) {
    int r = e % CH_NB, c = e / CH_NB;
    double acc = 0.0;
    for (int l = 0; l < nb; ++l) acc = fma(H[(r0 + r) + (long)(k0 + l) * m], xk[l + c * CH_NB], acc);
    y[(r0 + r) + c * ld] -= acc;
  }
}

// ------------------------------------------------------------------------------------
// Factor preparation: F = Hsave + eps I (copy), diag0 = diag(F).
extern "C" __global__ void k_shifted_copy(const double* __restrict__ Hs, double* __restrict__ F,
                                          int m, double eps, double* __restrict__ diag0) {
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long total = (long)m * m;
  for (; idx < total; idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % m), j = (int)(idx / m);
    double v = Hs[idx];
    if (i == j) {
      v += eps;
      diag0[i] = v;
    }
    F[idx] = v;
  }
}

// Partial sums of e = r - H x over column chunks: part[s][i] for chunk s.
#define SYMV_SPLIT 16
extern "C" __global__ void k_symv_partial(const double* __restrict__ Hs, int m,
                                          const double* __restrict__ x, long ldx,
                                          double* __restrict__ part, long ldp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  const int c = blockIdx.z;
  if (i >= m) return;
  const int chunk = (m + SYMV_SPLIT - 1) / SYMV_SPLIT;
  const int k0 = s * chunk, k1 = min(m, k0 + chunk);
  const double* xc = x + c * ldx;
  double acc = 0.0;
  for (int k = k0; k < k1; ++k) acc = fma(Hs[i + (long)k * m], xc[k], acc);
  part[(long)c * ldp + (long)s * m + i] = acc;
}

extern "C" __global__ void k_symv_finish(int m, const double* __restrict__ part, long ldp,
                                         const double* __restrict__ r, long ldr,
                                         double* __restrict__ e, long lde) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= m) return;
  double acc = 0.0;
  for (int s = 0; s < SYMV_SPLIT; ++s) acc += part[(long)c * ldp + (long)s * m + i];
  e[c * lde + i] = r[c * ldr + i] - acc;
}
