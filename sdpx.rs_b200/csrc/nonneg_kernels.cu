// Nonnegative-orthant rows (the reference's NonnegativeCone, cones/nonnegativecone.rs): the NT
// scaling w = sqrt(s / z), lambda = sqrt(s z), the elementwise cone operators, Jordan products,
// unit shifts, step lengths, margins, and the rows' share of the constraint operator and of the
// condensed Schur complement, H += A_nn' diag(1 / w^2) A_nn.
//
// The orthant rows of all nonnegative cones form one index list idx[0 .. cnt) into the stacked
// cone vector (cone order), and their rows of A are stored densely, Ann[i + j * cnt].
#include "common.cuh"

extern "C" __global__ void k_nn_scale(int cnt, const int* __restrict__ idx,
                                      const double* __restrict__ s, const double* __restrict__ z,
                                      double* __restrict__ w, double* __restrict__ lam,
                                      uint32_t* __restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const int r = idx[i];
  const double si = s[r], zi = z[r];
  if (!(si > 0.0) || !(zi > 0.0) || !isfinite(si) || !isfinite(zi)) {
    atomicOr(status, SDPXG_ST_CHOL_FAIL);  // not interior
    return;
  }
  w[i] = sqrt(si / zi);
  lam[i] = sqrt(si * zi);
}

extern "C" __global__ void k_nn_identity(int cnt, double* __restrict__ w, double* __restrict__ lam) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) w[i] = lam[i] = 1.0;
}

// y = op(x) on the orthant rows; modes as k_congruence: 0 W, 1 W', 2 W^-1, 3 W^-T, 4 Hs, 5 Hs^-1.
extern "C" __global__ void k_nn_cone(int cnt, const int* __restrict__ idx, int mode,
                                     const double* __restrict__ w, const double* __restrict__ x,
                                     double* __restrict__ y, long ld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const long r = idx[i] + (long)blockIdx.y * ld;
  const double wi = w[i], xi = x[r];
  double v;
  switch (mode) {
    case 0: case 1: v = wi * xi; break;
    case 2: case 3: v = xi / wi; break;
    case 4: v = (wi * wi) * xi; break;
    default: v = xi / (wi * wi); break;
  }
  y[r] = v;
}

// x = y o z (elementwise Jordan product of the orthant)
extern "C" __global__ void k_nn_circ(int cnt, const int* __restrict__ idx, const double* __restrict__ y,
                                     const double* __restrict__ z, double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) x[idx[i]] = y[idx[i]] * z[idx[i]];
}

// x = lambda \ z
extern "C" __global__ void k_nn_lam_inv(int cnt, const int* __restrict__ idx,
                                        const double* __restrict__ lam, const double* __restrict__ z,
                                        double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) x[idx[i]] = z[idx[i]] / lam[i];
}

// ds = lambda o lambda
extern "C" __global__ void k_nn_affine_ds(int cnt, const int* __restrict__ idx,
                                          const double* __restrict__ lam, double* __restrict__ ds) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) ds[idx[i]] = lam[i] * lam[i];
}

// v += a * e (the orthant's unit element is the all-ones vector)
extern "C" __global__ void k_nn_shift(int cnt, const int* __restrict__ idx, double* __restrict__ v,
                                      double a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) v[idx[i]] += a;
}

// One CTA, in the NT-scaled form at the current iterate (z = lambda / w, s = lambda w):
// z + a dz >= 0  <=>  lambda + a w dz >= 0,  s + a ds >= 0  <=>  lambda + a ds / w >= 0.
// mode 0: out = {min(amax, min over w dz < 0 of -lambda / (w dz)), the same for ds / w};
// mode 1 (admission at amax): out = amax where lambda + amax (.) >= 0 holds on every row, else 0.
extern "C" __global__ void k_nn_step(int cnt, const int* __restrict__ idx,
                                     const double* __restrict__ w, const double* __restrict__ lam,
                                     const double* __restrict__ dz, const double* __restrict__ ds,
                                     double amax, int mode, double* __restrict__ out) {
  __shared__ double red[2][32];
  double az = amax, as = amax;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const int r = idx[i];
    const double gz = w[i] * dz[r], gs = ds[r] / w[i], l = lam[i];
    if (mode == 0) {
      if (gz < 0.0) az = fmin(az, -l / gz);
      if (gs < 0.0) as = fmin(as, -l / gs);
    } else {
      if (!(l + amax * gz >= 0.0)) az = 0.0;
      if (!(l + amax * gs >= 0.0)) as = 0.0;
    }
  }
  az = warp_min(az);
  as = warp_min(as);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
    red[0][wid] = az;
    red[1][wid] = as;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = red[0][0], b = red[1][0];
    for (int k = 1; k < nw; ++k) {
      a = fmin(a, red[0][k]);
      b = fmin(b, red[1][k]);
    }
    out[0] = a;
    out[1] = b;
  }
}

// One CTA: out = {min v, sum max(v, 0)} over the orthant rows (interior shifts of the start).
extern "C" __global__ void k_nn_margins(int cnt, const int* __restrict__ idx,
                                        const double* __restrict__ v, double* __restrict__ out) {
  __shared__ double red[2][32];
  double mn = INFINITY, pos = 0.0;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const double x = v[idx[i]];
    mn = fmin(mn, x);
    pos += fmax(x, 0.0);
  }
  mn = warp_min(mn);
  pos = warp_sum(pos);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
    red[0][wid] = mn;
    red[1][wid] = pos;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = red[0][0], b = red[1][0];
    for (int k = 1; k < nw; ++k) {
      a = fmin(a, red[0][k]);
      b += red[1][k];
    }
    out[0] = a;
    out[1] = b;
  }
}

// y[idx[i]] = alpha (A_nn x)_i + beta y[idx[i]]: one thread per orthant row (coalesced over i).
extern "C" __global__ void k_nn_forward(int cnt, int n, const int* __restrict__ idx,
                                        const double* __restrict__ Ann, const double* __restrict__ x,
                                        double alpha, double beta, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  double acc = 0.0;
  for (int j = 0; j < n; ++j) acc = fma(Ann[i + (long)j * cnt], x[j], acc);
  const int r = idx[i];
  y[r] = alpha * acc + ((beta == 0.0) ? 0.0 : beta * y[r]);
}

// y[j] += alpha (A_nn' z)_j: one warp per column j (contiguous), fixed-order warp reduction.
extern "C" __global__ void k_nn_adjoint(int cnt, int n, const int* __restrict__ idx,
                                        const double* __restrict__ Ann, const double* __restrict__ z,
                                        double alpha, double* __restrict__ y) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= n) return;
  const double* col = Ann + (long)j * cnt;
  double acc = 0.0;
  for (int i = lane; i < cnt; i += 32) acc = fma(col[i], z[idx[i]], acc);
  acc = warp_sum(acc);
  if (lane == 0) y[j] += alpha * acc;
}

// H (n x n, both triangles) += A_nn' diag(1 / w^2) A_nn, 32 x 32 output tiles, 2 x 2 per thread.
// Entry (a, b) and (b, a) use the same products in the same order: H stays exactly symmetric.
extern "C" __global__ void __launch_bounds__(256)
k_nn_schur(int cnt, int n, const double* __restrict__ Ann, const double* __restrict__ w,
           double* __restrict__ H) {
  __shared__ double As[32][33];
  __shared__ double Bs[32][33];
  const int ti = blockIdx.x, tj = blockIdx.y;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double c00 = 0, c01 = 0, c10 = 0, c11 = 0;
  for (int r0 = 0; r0 < cnt; r0 += 32) {
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
      const int rr = e % 32, cc = e / 32, r = r0 + rr;
      const int ca = ti * 32 + cc, cb = tj * 32 + cc;
      const double h = (r < cnt) ? 1.0 / w[r] : 0.0;
      As[rr][cc] = (r < cnt && ca < n) ? Ann[r + (long)ca * cnt] * h : 0.0;
      Bs[rr][cc] = (r < cnt && cb < n) ? Ann[r + (long)cb * cnt] * h : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int rr = 0; rr < 32; ++rr) {
      const double x0 = As[rr][2 * tx], x1 = As[rr][2 * tx + 1];
      const double y0 = Bs[rr][2 * ty], y1 = Bs[rr][2 * ty + 1];
      c00 = fma(x0, y0, c00);
      c01 = fma(x0, y1, c01);
      c10 = fma(x1, y0, c10);
      c11 = fma(x1, y1, c11);
    }
    __syncthreads();
  }
  const int a0 = ti * 32 + 2 * tx, b0 = tj * 32 + 2 * ty;
  const double cv[2][2] = {{c00, c01}, {c10, c11}};
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const int a = a0 + u, b = b0 + v;
      if (a < n && b < n) H[a + (long)b * n] += cv[u][v];
    }
}
