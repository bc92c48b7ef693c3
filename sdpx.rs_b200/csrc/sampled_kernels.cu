// Matrix-valued sampled PSD blocks (the reference's SampledBlock with dim D > 1,
// crates/solver/src/solver/sampled/mod.rs:9-29, Schur entry 1973-1987, basis product 2065-2143).
//
// A block of order n = D h with basis Q (h x c) and weights w holds the primitive columns
// p = (s, r, k), r <= s < D, k < c (k fastest), each w_p svec(sym(e_r e_s') (x) q_k q_k').  With
// the expanded vectors u_a = e_i (x) q_k, a = i c + k, the column is w_p sym(u_a u_b') for the
// pair (a, b) = (r c + k, s c + k).  Then, with V = R^-1 U (n x Dc) and K = V'V:
//   Schur      S_pq = w_p w_q 1/2 (K_ad K_be + K_ae K_bd),   (a, b) of p, (d, e) of q
//   forward    (A x)_block = svec of the matrix whose (r, s) block of h x h entries is
//              f sum_k w_(s,r,k) x_(s,r,k) q_k q_k', f = 1 on the diagonal blocks, 1/2 off it
//   adjoint    (A' z)_p = w_p q_k' Z_rs q_k, Z_rs the (r, s) block of smat(z)
// Per-block metadata: MsDesc (common.cuh).
#include "common.cuh"

// V[:, a] = R^-1[:, i h .. (i+1) h) Q[:, k], a = i c + k.  grid (blocks, ceil(Dc / 8)), 256 threads:
// eight columns a per CTA, one thread per (row, a).
extern "C" __global__ void k_ms_basis(const BlockDesc* __restrict__ blocks, const MsDesc* __restrict__ ms,
                                      const double* __restrict__ Rinv, const double* __restrict__ Q,
                                      double* __restrict__ V) {
  const MsDesc d = ms[blockIdx.x];
  const BlockDesc bd = blocks[d.j];
  const int n = bd.n, r = d.D * d.c;
  const double* Ri = Rinv + bd.mat_off;
  for (int e = threadIdx.x; e < n * 8; e += blockDim.x) {
    const int row = e % n, a = blockIdx.y * 8 + e / n;
    if (a >= r) continue;
    const int i = a / d.c, k = a % d.c;
    const double* q = Q + d.q_off + (long)k * d.h;
    double acc = 0.0;
    for (int t = 0; t < d.h; ++t) acc = fma(Ri[row + (long)(i * d.h + t) * n], q[t], acc);
    V[d.v_off + row + (long)a * n] = acc;
  }
}

// K = V'V (Dc x Dc, both triangles from the same products: exactly symmetric).
extern "C" __global__ void k_ms_gram(const BlockDesc* __restrict__ blocks, const MsDesc* __restrict__ ms,
                                     const double* __restrict__ V, double* __restrict__ K) {
  const MsDesc d = ms[blockIdx.x];
  const int n = blocks[d.j].n, r = d.D * d.c;
  const long e = (long)blockIdx.y * blockDim.x + threadIdx.x;
  if (e >= (long)r * r) return;
  const int a = (int)(e % r), b = (int)(e / r);
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  const double* va = V + d.v_off + (long)lo * n;
  const double* vb = V + d.v_off + (long)hi * n;
  double acc = 0.0;
  for (int t = 0; t < n; ++t) acc = fma(va[t], vb[t], acc);
  K[d.k_off + e] = acc;
}

// S_j[p][q] = w_p w_q 1/2 (K_ad K_be + K_ae K_bd) (sampled/mod.rs:1973-1987), column-major k_j x k_j
// at s_off[j]; pairs[2 t], pairs[2 t + 1] = (a, b) of the block's t-th primitive.
extern "C" __global__ void k_ms_schur(const MsDesc* __restrict__ ms, const int* __restrict__ kcount,
                                      const int* __restrict__ col_ptr, const long* __restrict__ s_off,
                                      const double* __restrict__ w, const int* __restrict__ pairs,
                                      const double* __restrict__ K, double* __restrict__ S) {
  const MsDesc d = ms[blockIdx.x];
  const int kj = kcount[d.j], r = d.D * d.c, c0 = col_ptr[d.j];
  const long e = (long)blockIdx.y * blockDim.x + threadIdx.x;
  if (e >= (long)kj * kj) return;
  const int p = (int)(e % kj), q = (int)(e / kj);
  const int a = pairs[2 * (c0 + p)], b = pairs[2 * (c0 + p) + 1];
  const int dd = pairs[2 * (c0 + q)], ee = pairs[2 * (c0 + q) + 1];
  const double* Kj = K + d.k_off;
  const double v = Kj[a + (long)dd * r] * Kj[b + (long)ee * r] + Kj[a + (long)ee * r] * Kj[b + (long)dd * r];
  S[s_off[d.j] + e] = w[c0 + p] * w[c0 + q] * 0.5 * v;
}

// y_block = alpha svec(sum_p w_p x_p sym(u_a u_b')) + beta y_block: one thread per svec entry.
extern "C" __global__ void k_ms_forward(const BlockDesc* __restrict__ blocks, const MsDesc* __restrict__ ms,
                                        const int* __restrict__ col_ptr, const int* __restrict__ col_idx,
                                        const double* __restrict__ w, const double* __restrict__ Q,
                                        const double* __restrict__ x, double alpha, double beta,
                                        double* __restrict__ y) {
  const MsDesc d = ms[blockIdx.x];
  const BlockDesc bd = blocks[d.j];
  const int n = bd.n, tn = n * (n + 1) / 2, c0 = col_ptr[d.j];
  const int e = blockIdx.y * blockDim.x + threadIdx.x;
  if (e >= tn) return;
  int col = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);  // svec entry e = col (col + 1) / 2 + row
  while (col * (col + 1) / 2 > e) --col;
  while ((col + 1) * (col + 2) / 2 <= e) ++col;
  const int row = e - col * (col + 1) / 2;
  const int bi = row / d.h, ti = row % d.h, bj = col / d.h, tj = col % d.h;
  const int s = bi > bj ? bi : bj, r = bi > bj ? bj : bi;
  const int pbase = (s * (s + 1) / 2 + r) * d.c;  // primitives (s, r, k) in order
  double acc = 0.0;
  for (int k = 0; k < d.c; ++k) {
    const double* q = Q + d.q_off + (long)k * d.h;
    const int t = pbase + k;
    acc = fma(w[c0 + t] * x[col_idx[c0 + t]], q[ti] * q[tj], acc);
  }
  double v = (bi == bj) ? acc : 0.5 * acc;
  if (row != col) v *= SDPXG_SQRT2;
  double* out = y + bd.svec_off + e;
  *out = beta == 0.0 ? alpha * v : fma(alpha, v, beta * *out);
}

// p[col_ptr[j] + t] = w_t q_k' Z_rs q_k for the block's primitive t = (s, r, k): one thread each.
extern "C" __global__ void k_ms_adjoint(const BlockDesc* __restrict__ blocks, const MsDesc* __restrict__ ms,
                                        const int* __restrict__ kcount, const int* __restrict__ col_ptr,
                                        const double* __restrict__ w, const int* __restrict__ pairs,
                                        const double* __restrict__ Q, const double* __restrict__ z,
                                        double* __restrict__ part) {
  const MsDesc d = ms[blockIdx.x];
  const BlockDesc bd = blocks[d.j];
  const int kj = kcount[d.j], c0 = col_ptr[d.j];
  const int t = blockIdx.y * blockDim.x + threadIdx.x;
  if (t >= kj) return;
  const int a = pairs[2 * (c0 + t)], b = pairs[2 * (c0 + t) + 1];
  const int r = a / d.c, s = b / d.c, k = a % d.c;
  const double* q = Q + d.q_off + (long)k * d.h;
  const double* zb = z + bd.svec_off;
  double acc = 0.0;
  for (int u = 0; u < d.h; ++u)
    for (int v = 0; v < d.h; ++v) {
      const int i = r * d.h + u, jj = s * d.h + v;  // Z(i, jj) from svec
      const int lo = i < jj ? i : jj, hi = i < jj ? jj : i;
      double zij = zb[hi * (hi + 1) / 2 + lo];
      if (lo != hi) zij *= SDPXG_RSQRT2;
      acc = fma(q[u] * q[v], zij, acc);
    }
  part[c0 + t] = w[c0 + t] * acc;
}
