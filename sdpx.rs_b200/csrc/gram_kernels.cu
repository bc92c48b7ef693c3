// Rank-one (Gram) form of the PSD constraint operator.
//
// When every column of A restricted to PSD block j is rank one, svec(sigma_t u_t u_t') with
// sigma_t = +-1 (the sampled bootstrap SDPs: A_ij = w v v' with v a basis column), the block
// is stored as its factor U_j = [u_1 .. u_k] (n_j x k_j, column-major) and signs sigma.  Then
// with V_j = Rinv_j U_j (Ginv_j = Rinv_j' Rinv_j from the NT scaling):
//   Schur block   S_j[a][b] = < A_a, Ginv A_b Ginv > = sigma_a sigma_b (V_j' V_j)[a][b]^2
//   forward       (A x)_j   = svec(U_j diag(sigma x) U_j')
//   adjoint       (A' z)_t += sigma_t u_t' smat(z_j) u_t
// -- the same entries as the ordinary condensed path (kkt/condensed/psd.rs:1299-1534,
// scaling.rs:74-81) and as the reference's sampled Gram update for rank-one terms
// (sampled/mod.rs:1973-2025: H_pq = w_p w_q K_pq^2 with K = V'V, V = Rinv Q), at
// O(n^2 k + n k^2) work per block instead of O(k n^3 + k^2 n^2), and reading n k instead
// of k n(n+1)/2 doubles of operator data.
#include "common.cuh"

#define GR_LD SDPXG_LD  // the layout of cta_load_mat / cta_load_smat

// C (64 x nc, padded) = A (64 x 64, padded) B (64 x nc, padded) on the FP64 tensor cores,
// one 8 x 8 output tile per warp at a time; K = 64 (zero padding makes the tail exact).
__device__ __forceinline__ void gr_gemm_nn(double* C, const double* A, const double* B, int nr,
                                           int nc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int rt = (nr + 7) >> 3, ct = (nc + 7) >> 3;
  const int r = lane >> 2, q = lane & 3;
  for (int t = warp; t < rt * ct; t += nwarps) {
    const int ti = (t % rt) << 3, tj = (t / rt) << 3;
    double d0 = 0.0, d1 = 0.0;
#pragma unroll
    for (int kg = 0; kg < 4; ++kg) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int k = (kg << 4) + (u << 2) + q;
        a[u] = A[(ti + r) + k * GR_LD];
        b[u] = B[k + (tj + r) * GR_LD];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) dmma_m8n8k4(d0, d1, a[u], b[u]);
    }
    C[(ti + r) + (tj + 2 * q) * GR_LD] = d0;
    C[(ti + r) + (tj + 2 * q + 1) * GR_LD] = d1;
  }
}

// U chunk: rows < n, columns c0 .. c0 + 63 (< k) of a block's factor into padded shared memory.
__device__ __forceinline__ void gr_load_chunk(double* S, const double* __restrict__ U, int n, int k,
                                              int c0) {
  for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
    const int r = e & 63, c = e >> 6;
    S[r + c * GR_LD] = (r < n && c0 + c < k) ? U[(long)(c0 + c) * n + r] : 0.0;
  }
}

// V_j[:, c0 .. c0+63] = Rinv_j U_j[:, c0 .. c0+63]; item (block, column chunk).
extern "C" __global__ void __launch_bounds__(256)
k_gram_basis(const BlockDesc* __restrict__ blocks, const int* __restrict__ item_blk,
             const int* __restrict__ item_c0, const int* __restrict__ kcount,
             const long* __restrict__ gu_off, const double* __restrict__ Rinv,
             const double* __restrict__ U, double* __restrict__ V) {
  extern __shared__ double gsm[];
  double* Rs = gsm;
  double* Us = Rs + 64 * GR_LD;
  double* Cs = Us + 64 * GR_LD;
  const int j = item_blk[blockIdx.x], c0 = item_c0[blockIdx.x];
  const BlockDesc bd = blocks[j];
  const int n = bd.n, k = kcount[j];
  const int nc = min(64, k - c0);
  cta_load_mat(Rs, Rinv + bd.mat_off, n);
  gr_load_chunk(Us, U + gu_off[j], n, k, c0);
  __syncthreads();
  gr_gemm_nn(Cs, Rs, Us, n, nc);
  __syncthreads();
  double* out = V + gu_off[j] + (long)c0 * n;
  for (int e = threadIdx.x; e < n * nc; e += blockDim.x) out[e] = Cs[(e % n) + (e / n) * GR_LD];
}

// S_j tile (32 x 32): S[a][b] = sigma_a sigma_b (sum_r V[r][a] V[r][b])^2.  Both triangles are
// computed with the same products in the same order, so S_j is exactly symmetric.
extern "C" __global__ void __launch_bounds__(256)
k_gram_schur(const BlockDesc* __restrict__ blocks, const int* __restrict__ tiles,
             const int* __restrict__ kcount, const int* __restrict__ col_ptr,
             const long* __restrict__ gu_off, const long* __restrict__ s_off,
             const double* __restrict__ gsig, const double* __restrict__ V,
             double* __restrict__ S) {
  __shared__ double Va[64][33];
  __shared__ double Vb[64][33];
  const int j = tiles[3 * blockIdx.x], ti = tiles[3 * blockIdx.x + 1], tj = tiles[3 * blockIdx.x + 2];
  const int n = blocks[j].n, k = kcount[j];
  const double* Vj = V + gu_off[j];
  for (int e = threadIdx.x; e < 64 * 32; e += blockDim.x) {
    const int r = e & 63, c = e >> 6;
    const int ca = ti * 32 + c, cb = tj * 32 + c;
    Va[r][c] = (r < n && ca < k) ? Vj[(long)ca * n + r] : 0.0;
    Vb[r][c] = (r < n && cb < k) ? Vj[(long)cb * n + r] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
  for (int r = 0; r < n; ++r) {
    const double x0 = Va[r][2 * tx], x1 = Va[r][2 * tx + 1];
    const double y0 = Vb[r][2 * ty], y1 = Vb[r][2 * ty + 1];
    c00 = fma(x0, y0, c00);
    c01 = fma(x0, y1, c01);
    c10 = fma(x1, y0, c10);
    c11 = fma(x1, y1, c11);
  }
  const int a0 = ti * 32 + 2 * tx, b0 = tj * 32 + 2 * ty;
  const double* sg = gsig + col_ptr[j];
  double* out = S + s_off[j];
  const double cv[2][2] = {{c00, c01}, {c10, c11}};
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const int a = a0 + u, b = b0 + v;
      if (a < k && b < k) out[a + (long)b * k] = (sg[a] * sg[b]) * (cv[u][v] * cv[u][v]);
    }
}

// y_j = alpha svec(U_j diag(sigma x_cols) U_j') + beta y_j, K = k_j split in 64-column chunks.
// One CTA per (Gram block, chunk) item (the items of a block are consecutive, chunk order):
// it stages its 64 columns of U (coalesced, column t at Us[t * GR_LD + row], zero padded) and
// their weights d_t = sigma_t x[col_t], forms the upper 8 x 8 tiles of U_c diag(d) U_c' on the
// FP64 tensor cores (one warp per tile) into part[item] (64 x 64, column-major), and takes a
// ticket on cnt[j].  The block's last CTA (the ticket is reset for the next launch) sums the
// chunk partials in chunk order -- the same result for every arrival order -- and writes y.
#define GR_KCH 64
extern "C" __global__ void __launch_bounds__(256)
k_gram_forward(const BlockDesc* __restrict__ blocks, const int* __restrict__ item_blk,
               const int* __restrict__ item_c0, const int* __restrict__ kcount,
               const int* __restrict__ col_ptr, const int* __restrict__ col_idx,
               const long* __restrict__ gu_off, const double* __restrict__ gsig,
               const double* __restrict__ U, const double* __restrict__ x, double alpha,
               double beta, double* __restrict__ y, double* __restrict__ part,
               unsigned* __restrict__ cnt) {
  __shared__ __align__(16) double Us[GR_KCH * GR_LD];
  __shared__ double d[GR_KCH];
  __shared__ bool last;
  const int it = blockIdx.x, j = item_blk[it], c0 = item_c0[it];
  const BlockDesc bd = blocks[j];
  const int n = bd.n, k = kcount[j], kc = min(GR_KCH, k - c0);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, r = lane >> 2, q = lane & 3;
  const double* Uj = U + gu_off[j];
  for (int e = threadIdx.x; e < GR_KCH * GR_LD; e += blockDim.x) {
    const int t = e / GR_LD, row = e - t * GR_LD;
    Us[e] = (t < kc && row < n) ? Uj[(long)(c0 + t) * n + row] : 0.0;
  }
  for (int t = threadIdx.x; t < GR_KCH; t += blockDim.x)
    d[t] = (t < kc) ? gsig[col_ptr[j] + c0 + t] * x[col_idx[col_ptr[j] + c0 + t]] : 0.0;
  __syncthreads();
  double* P = part + (size_t)it * (SDPXG_NMAX * SDPXG_NMAX);
  const int T = (n + 7) >> 3, ntile = T * (T + 1) / 2;
  for (int tile = w; tile < ntile; tile += (int)(blockDim.x >> 5)) {
    int J = 0, I = tile;  // upper tiles column by column: (0,0), (0,1), (1,1), (0,2), ...
    while (I > J) {
      I -= J + 1;
      ++J;
    }
    double d0 = 0.0, d1 = 0.0;
#pragma unroll 4
    for (int ks = 0; ks < GR_KCH / 4; ++ks) {
      const int t = 4 * ks + q;
      const double a = d[t] * Us[t * GR_LD + 8 * I + r];  // (U diag(d))[row][t]
      const double b = Us[t * GR_LD + 8 * J + r];          // U'[t][col]
      dmma_m8n8k4(d0, d1, a, b);
    }
    P[(8 * J + 2 * q) * SDPXG_NMAX + 8 * I + r] = d0;
    P[(8 * J + 2 * q + 1) * SDPXG_NMAX + 8 * I + r] = d1;
  }
  __threadfence();
  __syncthreads();
  const int nch = (k + GR_KCH - 1) / GR_KCH;
  if (threadIdx.x == 0) {
    const unsigned tk = atomicAdd(&cnt[j], 1u);
    last = (tk == (unsigned)(nch - 1));
    if (last) cnt[j] = 0u;  // ready for the next launch (stream order)
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double* P0 = part + (size_t)(it - c0 / GR_KCH) * (SDPXG_NMAX * SDPXG_NMAX);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int row = e % n, col = e / n;
    if (row > col) continue;
    double v = 0.0;
    for (int c = 0; c < nch; ++c)
      v += __ldcg(P0 + (size_t)c * (SDPXG_NMAX * SDPXG_NMAX) + col * SDPXG_NMAX + row);
    const long idx = bd.svec_off + (long)col * (col + 1) / 2 + row;
    const double s2 = (row == col) ? v : v * SDPXG_SQRT2;
    y[idx] = alpha * s2 + ((beta == 0.0) ? 0.0 : beta * y[idx]);
  }
}

// p[col_ptr[j] + t] = sigma_t u_t' smat(z_j) u_t for the columns of one 64-column chunk.
extern "C" __global__ void __launch_bounds__(256)
k_gram_adjoint(const BlockDesc* __restrict__ blocks, const int* __restrict__ item_blk,
               const int* __restrict__ item_c0, const int* __restrict__ kcount,
               const int* __restrict__ col_ptr, const long* __restrict__ gu_off,
               const double* __restrict__ gsig, const double* __restrict__ U,
               const double* __restrict__ z, double* __restrict__ p) {
  extern __shared__ double gsm[];
  double* Zs = gsm;
  double* Us = Zs + 64 * GR_LD;
  double* Ws = Us + 64 * GR_LD;
  const int j = item_blk[blockIdx.x], c0 = item_c0[blockIdx.x];
  const BlockDesc bd = blocks[j];
  const int n = bd.n, k = kcount[j];
  const int nc = min(64, k - c0);
  cta_load_smat(Zs, z + bd.svec_off, n);
  gr_load_chunk(Us, U + gu_off[j], n, k, c0);
  __syncthreads();
  gr_gemm_nn(Ws, Zs, Us, n, nc);  // W = Z U_chunk
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = warp; c < nc; c += blockDim.x >> 5) {
    double acc = 0.0;
    for (int r = lane; r < n; r += 32) acc = fma(Us[r + c * GR_LD], Ws[r + c * GR_LD], acc);
    acc = warp_sum(acc);
    if (lane == 0) p[col_ptr[j] + c0 + c] = gsig[col_ptr[j] + c0 + c] * acc;
  }
}
