// Condensed Schur complement of the PSD rows and the constraint-operator products.
//
// Data layout (uploaded once per problem):
//   For PSD block j the columns of A that touch it are stored densely, column-major,
//   as Acol[acol_off[j] + t * tri(n_j) + r], t < k_j, with their global indices
//   col_idx[col_ptr[j] + t].  The transpose map lists, per constraint i, its (block, t)
//   pairs in cone order: c2b_ptr[i] .. c2b_ptr[i+1] into c2b_blk / c2b_loc.
//
// Schur entry (kkt/condensed/psd.rs:1120-1570, scaling.rs:7-81):
//   H_ab = sum_j < A_aj , Ginv_j A_bj Ginv_j >  (+ P_ab)
// computed as T = svec(Ginv A Ginv) per column (k_schur_transform), one grouped GEMM
// S_j = Acol_j' T_j per block (k_schur_block_gemm), and a deterministic cone-order gather
// into the dense m x m matrix (k_schur_gather).
#include "common.cuh"

namespace {
constexpr int kMat = SDPXG_LD * SDPXG_NMAX;
}

// One CTA per (block, column) work item: item w -> block wblk[w], local column wloc[w].
extern "C" __global__ void __launch_bounds__(SDPXG_CONE_THREADS)
k_schur_transform(const BlockDesc* __restrict__ blocks, const int* __restrict__ wblk,
                  const int* __restrict__ wloc, const long* __restrict__ acol_off,
                  const double* __restrict__ Ginv, const double* __restrict__ Acol,
                  double* __restrict__ Tcol) {
  extern __shared__ double smem[];
  const int j = wblk[blockIdx.x], t = wloc[blockIdx.x];
  const BlockDesc bd = blocks[j];
  const int n = bd.n;
  const int tn = n * (n + 1) / 2;
  double* G = smem;
  double* X = G + kMat;
  double* Y = X + kMat;
  cta_load_mat(G, Ginv + bd.mat_off, n);
  const long off = acol_off[j] + (long)t * tn;
  cta_load_smat(X, Acol + off, n);
  __syncthreads();
  cta_gemm(Y, G, false, X, false, n);  // Y = Ginv A
  __syncthreads();
  cta_gemm(X, Y, false, G, false, n);  // X = Ginv A Ginv
  __syncthreads();
  cta_store_svec(Tcol + off, X, n);
}

// Grouped GEMM S_j = Acol_j' * Tcol_j (k_j x k_j, inner tri(n_j)) on the FP64 tensor cores.
// Tile list entries (block, tile row, tile col) of 32 x 32 output tiles; a 32-row K chunk of both
// operands is staged in shared memory, and each of the 8 warps owns two 8 x 8 output subtiles
// accumulated by mma.sync m8n8k4 (lane (r, q): A fragment A'(row r, k q), B fragment T(k q,
// column r); results C(r, 2q) and C(r, 2q + 1)).
#define SCHUR_TILE 32
#define SCHUR_KC 32
extern "C" __global__ void __launch_bounds__(SDPXG_THREADS)
k_schur_block_gemm(const BlockDesc* __restrict__ blocks, const int* __restrict__ tiles,
                   const int* __restrict__ kcount, const long* __restrict__ acol_off,
                   const long* __restrict__ s_off, const double* __restrict__ Acol,
                   const double* __restrict__ Tcol, double* __restrict__ S) {
  __shared__ double As[SCHUR_KC][SCHUR_TILE + 1];
  __shared__ double Ts[SCHUR_KC][SCHUR_TILE + 1];
  const int j = tiles[3 * blockIdx.x], ti = tiles[3 * blockIdx.x + 1],
            tj = tiles[3 * blockIdx.x + 2];
  const int n = blocks[j].n;
  const int tn = n * (n + 1) / 2;
  const int k = kcount[j];
  const double* A = Acol + acol_off[j];
  const double* T = Tcol + acol_off[j];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, r = lane >> 2, q = lane & 3;
  // subtiles w and w + 8 of the 4 x 4 grid of 8 x 8 subtiles
  const int I0 = w >> 2, J0 = w & 3, I1 = (w + 8) >> 2, J1 = (w + 8) & 3;
  double c00 = 0, c01 = 0, c10 = 0, c11 = 0;
  for (int r0 = 0; r0 < tn; r0 += SCHUR_KC) {
    for (int e = threadIdx.x; e < SCHUR_KC * SCHUR_TILE; e += blockDim.x) {
      int rr = e % SCHUR_KC, cc = e / SCHUR_KC;
      int rw = r0 + rr;
      int ca = ti * SCHUR_TILE + cc, cb = tj * SCHUR_TILE + cc;
      As[rr][cc] = (rw < tn && ca < k) ? A[(long)ca * tn + rw] : 0.0;
      Ts[rr][cc] = (rw < tn && cb < k) ? T[(long)cb * tn + rw] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < SCHUR_KC / 4; ++ks) {
      const int kk = 4 * ks + q;
      dmma_m8n8k4(c00, c01, As[kk][8 * I0 + r], Ts[kk][8 * J0 + r]);
      dmma_m8n8k4(c10, c11, As[kk][8 * I1 + r], Ts[kk][8 * J1 + r]);
    }
    __syncthreads();
  }
  double* out = S + s_off[j];
  const int a0 = ti * SCHUR_TILE + 8 * I0 + r, b0 = tj * SCHUR_TILE + 8 * J0 + 2 * q;
  const int a1 = ti * SCHUR_TILE + 8 * I1 + r, b1 = tj * SCHUR_TILE + 8 * J1 + 2 * q;
  if (a0 < k && b0 < k) out[a0 + (long)b0 * k] = c00;
  if (a0 < k && b0 + 1 < k) out[a0 + (long)(b0 + 1) * k] = c01;
  if (a1 < k && b1 < k) out[a1 + (long)b1 * k] = c10;
  if (a1 < k && b1 + 1 < k) out[a1 + (long)(b1 + 1) * k] = c11;
}

// H (m x m, full, column-major) = sum over shared blocks of S_j[la, lb], in cone order.
// One thread per (a, b) with a <= b; both triangles written (symmetrised by construction).
extern "C" __global__ void k_schur_gather(int m, const int* __restrict__ c2b_ptr,
                                          const int* __restrict__ c2b_blk,
                                          const int* __restrict__ c2b_loc,
                                          const int* __restrict__ kcount,
                                          const long* __restrict__ s_off,
                                          const double* __restrict__ S, double* __restrict__ H) {
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long total = (long)m * m;
  if (idx >= total) return;
  int a = (int)(idx % m), b = (int)(idx / m);
  if (a > b) return;
  int pa = c2b_ptr[a], ea = c2b_ptr[a + 1], pb = c2b_ptr[b], eb = c2b_ptr[b + 1];
  double acc = 0.0;
  while (pa < ea && pb < eb) {
    int ja = c2b_blk[pa], jb = c2b_blk[pb];
    if (ja < jb) {
      ++pa;
    } else if (jb < ja) {
      ++pb;
    } else {
      const int k = kcount[ja];
      const double* Sj = S + s_off[ja];
      int la = c2b_loc[pa], lb = c2b_loc[pb];
      // symmetric in exact arithmetic: average the two computed halves
      acc += 0.5 * (Sj[la + (long)lb * k] + Sj[lb + (long)la * k]);
      ++pa;
      ++pb;
    }
  }
  H[a + (long)b * m] = acc;
  H[b + (long)a * m] = acc;
}

// H += sym(P) for P given as an upper-triangular CSC (n x n).
extern "C" __global__ void k_add_upper_csc(int n, const int* __restrict__ colptr,
                                           const int* __restrict__ rowval,
                                           const double* __restrict__ val, double* __restrict__ H) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  for (int p = colptr[j]; p < colptr[j + 1]; ++p) {
    int i = rowval[p];
    if (i > j) continue;
    H[i + (long)j * n] += val[p];
    if (i != j) H[j + (long)i * n] += val[p];
  }
}

// y[rows of block j] = alpha * Acol_j x[cols_j] + beta * y   (one CTA per block, thread/row)
// One CTA per 64-row tile of a block (tile list ftile_blk / ftile_r0): 64 rows x 4 column
// groups; the four partial sums are combined in a fixed order (deterministic).
extern "C" __global__ void __launch_bounds__(256)
k_op_forward(const BlockDesc* __restrict__ blocks, const int* __restrict__ kcount,
             const int* __restrict__ col_ptr, const int* __restrict__ col_idx,
             const long* __restrict__ acol_off, const double* __restrict__ Acol,
             const int* __restrict__ ftile_blk, const int* __restrict__ ftile_r0,
             const double* __restrict__ x, long ldx, double alpha, double beta,
             double* __restrict__ y, long ldy) {
  __shared__ double part[4][64];
  const int j = ftile_blk[blockIdx.x], r0 = ftile_r0[blockIdx.x];
  const BlockDesc bd = blocks[j];
  const int tn = bd.n * (bd.n + 1) / 2;
  const int k = kcount[j];
  const double* A = Acol + acol_off[j];
  const int* cols = col_idx + col_ptr[j];
  const double* xc = x + (long)blockIdx.y * ldx;
  double* yc = y + (long)blockIdx.y * ldy;
  const int rr = threadIdx.x & 63, g = threadIdx.x >> 6;
  const int r = r0 + rr;
  double acc = 0.0;
  if (r < tn)
    for (int t = g; t < k; t += 4) acc = fma(A[(long)t * tn + r], xc[cols[t]], acc);
  part[g][rr] = acc;
  __syncthreads();
  if (g == 0 && r < tn) {
    double s = ((part[0][rr] + part[1][rr]) + part[2][rr]) + part[3][rr];
    double prev = (beta == 0.0) ? 0.0 : beta * yc[bd.svec_off + r];
    yc[bd.svec_off + r] = alpha * s + prev;
  }
}

// Per-block partial adjoint p[acol column] = Acol_j[:, t] . z_j  (one warp per column)
extern "C" __global__ void k_op_adjoint_partial(const BlockDesc* __restrict__ blocks,
                                                const int* __restrict__ wblk,
                                                const int* __restrict__ wloc,
                                                const int* __restrict__ col_ptr,
                                                const long* __restrict__ acol_off,
                                                const double* __restrict__ Acol,
                                                const double* __restrict__ z, long ldz,
                                                double* __restrict__ p, long ldp, int nwork) {
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= nwork) return;
  const int j = wblk[w], t = wloc[w];
  const BlockDesc bd = blocks[j];
  const int tn = bd.n * (bd.n + 1) / 2;
  const double* A = Acol + acol_off[j] + (long)t * tn;
  const double* zc = z + (long)blockIdx.y * ldz + bd.svec_off;
  double acc = 0.0;
  for (int r = lane; r < tn; r += 32) acc = fma(A[r], zc[r], acc);
  acc = warp_sum(acc);
  if (lane == 0) p[(long)blockIdx.y * ldp + col_ptr[j] + t] = acc;
}

// y[i] = alpha * sum over (block, t) of constraint i of p[...] + beta * y[i]  (cone order)
extern "C" __global__ void k_op_adjoint_gather(int n, const int* __restrict__ c2b_ptr,
                                               const int* __restrict__ c2b_blk,
                                               const int* __restrict__ c2b_loc,
                                               const int* __restrict__ col_ptr,
                                               const double* __restrict__ p, long ldp,
                                               double alpha, double beta, double* __restrict__ y,
                                               long ldy) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* pc = p + (long)blockIdx.y * ldp;
  double acc = 0.0;
  for (int q = c2b_ptr[i]; q < c2b_ptr[i + 1]; ++q) acc += pc[col_ptr[c2b_blk[q]] + c2b_loc[q]];
  double* yc = y + (long)blockIdx.y * ldy;
  double prev = (beta == 0.0) ? 0.0 : beta * yc[i];
  yc[i] = alpha * acc + prev;
}
