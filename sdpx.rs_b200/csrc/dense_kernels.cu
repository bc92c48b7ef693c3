// Dense Cholesky of the Schur complement with the reference's dynamic pivot rule, the explicit
// inverse of its factor, and the GEMVs that apply it.
//
// Factorisation H + eps I = U'U (upper), right-looking over 64 x 64 tiles
// (kkt/ldl/dense_block.rs:334-365 potrf_dynamic, 370-388 potrf_tile, 515-594 tiled_potrf):
//   k_potrf_diag   factor the diagonal tile with the dynamic pivot rule; store Dinv = U_kk^-1
//   k_trsm_panel   U[k, j] = U_kk^-T H[k, j] for the tiles right of the diagonal
//   k_syrk_update  H[i, j] -= U[k, i]' U[k, j] on the upper trailing tiles
// Inverse X = U^-1, recursive over tile groups: with U = [U11 U12; 0 U22],
//   X12 = -X11 (U12 X22), level by level (k_trinv_level, two batched GEMM phases per level),
// so every level is one wide batched GEMM instead of a serial chain of tiles.
// Solves of an iteration then read X twice: y = X' b (upper, by columns) and x = X y (through
// the stored transpose, by columns) -- coalesced GEMVs (the reference substitutes tile by tile,
// dense_block.rs:604-669; refinement against the unshifted matrix makes the two equivalent).
#include "common.cuh"

#define CH_NB 64
#define CH_LD (CH_NB + 1)
#define TI_LD 68  // k_trinv_level tiles (4 mod 16)

// F = Hsave + eps I (copy), diag0 = diag(F).
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

// out[i] = H[i * stride] + eps: a strided diagonal (the original diagonal of a trailing block).
extern "C" __global__ void k_strided_diag(const double* __restrict__ H, long stride, int n, double eps,
                                          double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = H[(long)i * stride] + eps;
}

// dst(j, i) = src(i, j) for a rows x cols block (column-major, leading dimensions lds, ldd),
// through a 32 x 33 shared tile so both sides are coalesced.  block (32, 8), grid (cols/32,
// rows/32).
extern "C" __global__ void k_transpose_block(const double* __restrict__ src, long lds, int rows, int cols,
                                             double* __restrict__ dst, long ldd) {
  __shared__ double t[32][33];
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  for (int jj = threadIdx.y; jj < 32; jj += 8) {
    const int i = i0 + threadIdx.x, j = j0 + jj;
    if (i < rows && j < cols) t[jj][threadIdx.x] = src[i + (long)j * lds];
  }
  __syncthreads();
  for (int ii = threadIdx.y; ii < 32; ii += 8) {
    const int j = j0 + threadIdx.x, i = i0 + ii;
    if (i < rows && j < cols) dst[j + (long)i * ldd] = t[threadIdx.x][ii];
  }
}

// ------------------------------------------------------------------------------------
// Pivot k of the diagonal tile under the dynamic pivot rule (the reference's LDL pivot
// handling, dense_block.rs): a pivot within eps of zero becomes delta, a clearly negative or
// non-finite one fails.  Written once by the thread that finished the pivot entry:
// info = {1/d, sqrt(d), 1/sqrt(d)}, all 0 on failure (sqrt of an accepted pivot is > 0).
__device__ __forceinline__ void potrf_pivot(double d, const double* diag, int nb, double eps,
                                            double delta, int dynamic, double* info) {
  bool fail = !isfinite(d);
  if (!fail && dynamic && d <= eps) {
    if (d < -64.0 * 2.220446049250313e-16 * nb * fabs(*diag)) fail = true;
    else d = delta;
  }
  if (!fail && !(d > 0.0)) fail = true;
  if (fail) {
    info[0] = info[1] = info[2] = 0.0;
    return;
  }
  const double r = sqrt(d);
  info[0] = 1.0 / d;
  info[1] = r;
  info[2] = 1.0 / r;
}

// Diagonal tile: lagged upper Cholesky with the dynamic pivot rule, then Dinv = U^-1.
// Dynamic shared memory: two CH_NB x CH_LD tiles.
extern "C" __global__ void __launch_bounds__(1024)
k_potrf_diag(double* __restrict__ H, int m, int kb, double eps, double delta, int dynamic,
             const double* __restrict__ diag0, double* __restrict__ Dinv,
             uint32_t* __restrict__ status) {
  extern __shared__ double pd_sm[];
  double* A = pd_sm;
  __shared__ double rowbuf[2][CH_NB];   // row k of the partially eliminated tile
  __shared__ double mrowbuf[2][CH_NB];  // row k of M = L^-1 (unit lower)
  __shared__ double pinfo[2][3];        // pivot k: 1/d, sqrt(d), 1/sqrt(d)
  __shared__ double root[CH_NB];        // sqrt of the accepted pivots
  const int k0 = kb * CH_NB;
  const int nb = min(CH_NB, m - k0);
  // thread (tx, ty) owns rows tx + 32p and columns ty + 32q (p, q < 2) of the tile, in
  // registers: a = upper triangle being eliminated (H = L D L'), mm = lower triangle of
  // M = L^-1, updated with the same elimination multipliers (Gauss elimination applied to I).
  // The divisions and the square root of a pivot are computed once, by the thread that
  // finishes the pivot entry, one step ahead of their use.
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  double a[2][2], mm[2][2];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      int i = tx + 32 * p, j = ty + 32 * q;
      a[p][q] = (i <= j && j < nb) ? H[(k0 + i) + (long)(k0 + j) * m] : 0.0;
      mm[p][q] = (i == j) ? 1.0 : 0.0;
      if (i == 0 && j < nb) rowbuf[0][j] = a[p][q];
      if (i == 0) mrowbuf[0][j] = (j == 0) ? 1.0 : 0.0;
    }
  if (threadIdx.x == 0 && nb > 0) {
    potrf_pivot(a[0][0], diag0 + k0, nb, eps, delta, dynamic, pinfo[0]);
    root[0] = pinfo[0][1];
  }
  for (int k = 0; k < nb; ++k) {
    __syncthreads();
    const double* row = rowbuf[k & 1];
    const double dinv = pinfo[k & 1][0], r = pinfo[k & 1][1], rinv = pinfo[k & 1][2];
    if (r == 0.0) {
      if (threadIdx.x == 0) atomicOr(status, SDPXG_ST_PIVOT_FAIL);
      return;  // uniform: every thread read the same pivot record
    }
    const double* mrow = mrowbuf[k & 1];
    double* next = rowbuf[(k + 1) & 1];
    double* mnext = mrowbuf[(k + 1) & 1];
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int i = tx + 32 * p, j = ty + 32 * q;
        if (i >= nb || j >= nb) continue;
        if (i <= j) {
          if (i == k) A[k + j * CH_LD] = (j == k) ? r : a[p][q] * rinv;  // final row k of U
          if (i > k) {
            a[p][q] -= row[i] * row[j] * dinv;
            if (i == k + 1) {
              next[j] = a[p][q];
              if (j == k + 1) {  // pivot k + 1 is final: publish its record for the next step
                potrf_pivot(a[p][q], diag0 + k0 + k + 1, nb, eps, delta, dynamic,
                            pinfo[(k + 1) & 1]);
                root[k + 1] = pinfo[(k + 1) & 1][1];
              }
            }
          }
        }
        if (i >= j) {  // M entry (i, c = j): row i -= l_ik * row k, for c <= k
          if (i > k && j <= k) mm[p][q] -= (row[i] * dinv) * mrow[j];
          if (i == k + 1 && j <= k + 1) mnext[j] = mm[p][q];
        }
      }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e % nb, j = e / nb;
    if (i <= j) H[(k0 + i) + (long)(k0 + j) * m] = A[i + j * CH_LD];
  }
  // Dinv = U^-1 = L^-T D^-1/2: Dinv[c][i] = M[i][c] / sqrt(d_i) (upper, zero elsewhere)
  double* D = Dinv + (long)kb * CH_NB * CH_NB;
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int i = tx + 32 * p, c = ty + 32 * q;
      const bool live = (i >= c && i < nb);
      D[c + i * CH_NB] = live ? mm[p][q] / root[i] : 0.0;
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
  for (int e = threadIdx.x; e < CH_NB * CH_NB; e += blockDim.x) {  // zero the ragged edge
    int i = e % CH_NB, c = e / CH_NB;
    if (i >= nb || c >= nc) P[i + c * CH_LD] = 0.0;
  }
  __syncthreads();
  // out = D' P with 4 x 4 register tiles (D is upper with zeros below the diagonal)
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int l = 0; l < nb; ++l) {
    double x[4], y[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) x[a] = D[l + (tx + 16 * a) * CH_LD];
#pragma unroll
    for (int b = 0; b < 4; ++b) y[b] = P[l + (ty + 16 * b) * CH_LD];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      int i = tx + 16 * a, c = ty + 16 * b;
      if (i < nb && c < nc) H[(k0 + i) + (long)(c0 + c) * m] = acc[a][b];
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
// Inverse of the factor.  Diagonal tiles: X_ii = Dinv_i (stored in Uinv and, transposed, UinvT).
extern "C" __global__ void k_trtri_diag(int m, const double* __restrict__ Dinv,
                                        double* __restrict__ Uinv, double* __restrict__ UinvT) {
  const int ib = blockIdx.x;
  const int i0 = ib * CH_NB, ni = min(CH_NB, m - i0);
  const double* D = Dinv + (long)ib * CH_NB * CH_NB;
  for (int e = threadIdx.x; e < ni * ni; e += blockDim.x) {
    int r = e % ni, c = e / ni;
    double v = D[r + c * CH_NB];  // zero below the diagonal
    Uinv[(i0 + r) + (long)(i0 + c) * m] = v;
    UinvT[(i0 + c) + (long)(i0 + r) * m] = v;
  }
}

// 8-byte asynchronous global -> shared copy; src_bytes 0 writes zero (masked element).
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool in) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
               "r"(in ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Level `level` >= 1 of the recursive inverse: groups of 2^level tiles, left half L (2^(level-1)
// full tiles), right half R (possibly ragged).  phase 0: T = U[L,R] X[R,R] into Tmp[L,R];
// phase 1: X[L,R] = -X[L,L] T.  X's strictly lower part is never stored: loads mask it to zero.
// grid = (row tiles of L, column tiles of R, groups).  The K loop is a two-stage pipeline: the
// next 64-wide chunk of both operands streams into shared memory (cp.async, zero-filled where
// masked or out of range) while the tensor cores work on the current one.
// Dynamic shared memory: two stages of two tiles.
extern "C" __global__ void __launch_bounds__(SDPXG_THREADS)
k_trinv_level(const double* __restrict__ F, double* __restrict__ Uinv, double* __restrict__ UinvT,
              double* __restrict__ Tmp, int n, int level, int phase) {
  extern __shared__ double tl_sm[];
  const int g = 1 << level, h = g >> 1;
  const int L0 = blockIdx.z * g * CH_NB;
  const int R0 = L0 + h * CH_NB;
  if (R0 >= n) return;
  const int Ln = h * CH_NB;
  const int Rn = min(R0 + h * CH_NB, n) - R0;
  const int tm = blockIdx.x, tn = blockIdx.y;
  if (tm * CH_NB >= Ln || tn * CH_NB >= Rn) return;
  const double* A;
  const double* B;
  int ar, ac, br, bc, K;
  if (phase == 0) {
    A = F; ar = L0; ac = R0; B = Uinv; br = R0; bc = R0; K = Rn;
  } else {
    A = Uinv; ar = L0; ac = L0; B = Tmp; br = L0; bc = R0; K = Ln;
  }
  // triangular operands: skip the K chunks that are structurally zero
  int kbeg = 0, kend = K;
  if (phase == 0) kend = min(K, (tn + 1) * CH_NB);
  else kbeg = tm * CH_NB;
  // stage s: As = tl_sm + s * 2 * CH_NB * TI_LD ([r + k * TI_LD]), Bs = As + CH_NB * TI_LD
  auto load = [&](int k0, int s) {
    double* As = tl_sm + s * 2 * CH_NB * TI_LD;
    double* Bs = As + CH_NB * TI_LD;
    for (int e = threadIdx.x; e < CH_NB * CH_NB; e += blockDim.x) {
      const int r = e % CH_NB, k = e / CH_NB;
      const int gr = ar + tm * CH_NB + r, gc = ac + k0 + k;
      const bool in = (tm * CH_NB + r < Ln) && (k0 + k < K) && !(phase == 1 && gr > gc);
      cp_async8(As + r + k * TI_LD, in ? A + gr + (long)gc * n : A, in);
      const int hr = br + k0 + r, hc = bc + tn * CH_NB + k;
      const bool inb = (k0 + r < K) && (tn * CH_NB + k < Rn) && !(phase == 0 && hr > hc);
      cp_async8(Bs + r + k * TI_LD, inb ? B + hr + (long)hc * n : B, inb);
    }
    cp_async_commit();
  };
  // FP64 tensor cores: warp w owns the 8-column block w of the 64 x 64 output tile, eight
  // 8 x 8 accumulators; shared tiles with leading dimension TI_LD (4 mod 16: conflict-free
  // fragment reads).  Fragments: lane l holds A[l/4][l%4], B[l%4][l/4], C[l/4][2(l%4)+{0,1}].
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, q = lane & 3, rr = lane >> 2;
  double acc[8][2];
#pragma unroll
  for (int R = 0; R < 8; ++R) acc[R][0] = acc[R][1] = 0.0;
  int s = 0;
  if (kbeg < kend) load(kbeg, 0);
  for (int k0 = kbeg; k0 < kend; k0 += CH_NB, s ^= 1) {
    if (k0 + CH_NB < kend) {
      load(k0 + CH_NB, s ^ 1);  // its buffer was released by the barrier that ended step k0-64
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();  // chunk k0 is in shared memory for every thread
    const double* As = tl_sm + s * 2 * CH_NB * TI_LD;
    const double* Bs = As + CH_NB * TI_LD;
#pragma unroll 4
    for (int ks = 0; ks < CH_NB / 4; ++ks) {
      const int kk = ks * 4 + q;
      const double b = Bs[kk + (8 * w + rr) * TI_LD];
#pragma unroll
      for (int R = 0; R < 8; ++R) dmma_m8n8k4(acc[R][0], acc[R][1], As[(8 * R + rr) + kk * TI_LD], b);
    }
    __syncthreads();  // every warp is done with stage s before it is refilled
  }
#pragma unroll
  for (int R = 0; R < 8; ++R)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      int r = tm * CH_NB + 8 * R + rr, c = tn * CH_NB + 8 * w + 2 * q + e;
      if (r >= Ln || c >= Rn) continue;
      long gr = L0 + r, gc = R0 + c;
      if (phase == 0) {
        Tmp[gr + gc * n] = acc[R][e];
      } else {
        Uinv[gr + gc * n] = -acc[R][e];
        UinvT[gc + gr * n] = -acc[R][e];
      }
    }
}

// out[c] = sum over the stored triangle of column c of A (n x n): rows 0..c (upper) or c..n-1
// (lower), times v.  One warp per column: coalesced column reads.
extern "C" __global__ void k_tri_colgemv(const double* __restrict__ A, int n, int lower,
                                         const double* __restrict__ v, double* __restrict__ out) {
  // one warp per column, eight independent partial sums per lane so that each lane keeps eight
  // loads in flight (the matrix streams from HBM/L2 once per solve)
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= n) return;
  const int r0 = lower ? c : 0, r1 = lower ? n : c + 1;
  const double* col = A + (long)c * n;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int r = r0 + lane;
  for (; r + 7 * 32 < r1; r += 8 * 32) {
#pragma unroll
    for (int u = 0; u < 8; ++u) acc[u] = fma(__ldg(col + r + 32 * u), __ldg(v + r + 32 * u), acc[u]);
  }
  for (; r < r1; r += 32) acc[0] = fma(col[r], v[r], acc[0]);
  double t = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  t = warp_sum(t);
  if (lane == 0) out[c] = t;
}

// out[c] = rbase[c] + alpha * (column c of A) . v for a dense column-major n x n A restricted to
// a triangle (tri 0: all rows, 1: rows <= c, 2: rows >= c; other entries are never read).  One
// warp per (column, 256-row segment), eight loads in flight per lane, so every warp finishes in
// one memory round trip whatever the column length; the segment sums go to partial[seg][c] and
// the warp that finishes a column last (a ticket per column, reset for the next use) adds them
// in increasing segment order -- the result does not depend on the order the warps ran in.
#define CD_SEG 256
__device__ __forceinline__ void cd_seg_range(int tri, int c, int n, int& s0, int& s1) {
  const int nseg = (n + CD_SEG - 1) / CD_SEG;
  s0 = 0;
  s1 = nseg;
  if (tri == 1) s1 = c / CD_SEG + 1;  // rows 0..c
  if (tri == 2) s0 = c / CD_SEG;      // rows c..n-1
}

extern "C" __global__ void __launch_bounds__(256)
k_coldot_seg(const double* __restrict__ A, int n, int tri, const double* __restrict__ v,
             const double* __restrict__ rbase, double alpha, double* __restrict__ out,
             double* __restrict__ partial, unsigned* __restrict__ counters) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31, sg = blockIdx.y;
  if (c >= n) return;
  int s0, s1;
  cd_seg_range(tri, c, n, s0, s1);
  if (sg < s0 || sg >= s1) return;
  int r0 = sg * CD_SEG, r1 = min(n, r0 + CD_SEG);
  if (tri == 1) r1 = min(r1, c + 1);
  if (tri == 2) r0 = max(r0, c);
  const double* col = A + (long)c * n;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int r = r0 + lane + 32 * u;
    if (r < r1) acc[u] = __ldg(col + r) * __ldg(v + r);
  }
  double t = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  t = warp_sum(t);
  unsigned ticket = 0;
  if (lane == 0) {
    partial[(long)sg * n + c] = t;
    __threadfence();
    ticket = atomicAdd(counters + c, 1u);
  }
  ticket = __shfl_sync(0xffffffffu, ticket, 0);
  if (ticket != (unsigned)(s1 - s0 - 1)) return;
  if (lane == 0) {
    __threadfence();
    double sum = 0.0;
    for (int k = s0; k < s1; ++k) sum += __ldcg(partial + (long)k * n + c);
    out[c] = (rbase ? rbase[c] : 0.0) + alpha * sum;
    counters[c] = 0u;
  }
}

// e = r - H x for the symmetric H (both triangles stored): e_i = r_i - (column i of H) . x, one
// warp per column, coalesced, eight partial sums per lane (one launch, no partial buffer).
extern "C" __global__ void k_symv_cols(const double* __restrict__ H, int m,
                                       const double* __restrict__ x, const double* __restrict__ r,
                                       double* __restrict__ e) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= m) return;
  const double* col = H + (long)c * m;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int k = lane;
  for (; k + 7 * 32 < m; k += 8 * 32) {
#pragma unroll
    for (int u = 0; u < 8; ++u) acc[u] = fma(__ldg(col + k + 32 * u), __ldg(x + k + 32 * u), acc[u]);
  }
  for (; k < m; k += 32) acc[0] = fma(col[k], x[k], acc[0]);
  double t = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  t = warp_sum(t);
  if (lane == 0) e[c] = r[c] - t;
}
