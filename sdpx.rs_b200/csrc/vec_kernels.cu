// Vector kernels of the interior-point iteration: linear combinations and deterministic
// reductions (fixed grid, fixed order: repeated runs give bitwise identical scalars).
#include "common.cuh"

#define RED_BLOCKS 148
#define RED_THREADS 256

// out = a*x + b*y + c*w  (null pointers contribute zero; out may alias any input)
extern "C" __global__ void k_lincomb(long n, double a, const double* x, double b, const double* y,
                                     double c, const double* w, double* out) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (x) v = a * x[i];
    if (y) v = fma(b, y[i], v);
    if (w) v = fma(c, w[i], v);
    out[i] = v;
  }
}

// Several independent updates in one launch: grid row r applies request r (the arithmetic of
// k_lincomb, so the same bits as the single launches).
extern "C" __global__ void k_lincomb_batch(LinBatch bt) {
  const LinReq q = bt.r[blockIdx.y];
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < q.n;
       i += (long)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (q.x) v = q.a * q.x[i];
    if (q.y) v = fma(q.b, q.y[i], v);
    if (q.w) v = fma(q.c, q.w[i], v);
    q.out[i] = v;
  }
}

// op 0: sum x*y;  op 1: sum (x*y)^2 (scaled 2-norm squared, y = scales or null);
// op 2: max |x*y|;  op 3: all finite (1.0 / 0.0) of x;  op 4: max(0, max -x*y) (y >= 0: a
// nonnegative scale, or a mask that selects rows)
__device__ __forceinline__ double red_elem(int op, const double* x, const double* y, long i) {
  double xv = x[i];
  double yv = y ? y[i] : 1.0;
  switch (op) {
    case 0: return xv * yv;
    case 1: { double t = xv * yv; return t * t; }
    case 2: return fabs(xv * yv);
    case 4: return fmax(0.0, -(xv * yv));
    default: return isfinite(xv) ? 1.0 : 0.0;
  }
}

__device__ __forceinline__ double red_combine(int op, double a, double b) {
  if (op == 2 || op == 4) return fmax(a, b);
  if (op == 3) return fmin(a, b);
  return a + b;
}

__device__ __forceinline__ double red_identity(int op) { return op == 3 ? 1.0 : 0.0; }

extern "C" __global__ void __launch_bounds__(RED_THREADS)
k_reduce_partial(int op, long n, const double* __restrict__ x, const double* __restrict__ y,
                 double* __restrict__ partial) {
  __shared__ double red[RED_THREADS / 32];
  double acc = red_identity(op);
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    acc = red_combine(op, acc, red_elem(op, x, y, i));
  for (int o = 16; o > 0; o >>= 1) acc = red_combine(op, acc, __shfl_xor_sync(0xffffffffu, acc, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = red_identity(op);
    for (int w = 0; w < RED_THREADS / 32; ++w) v = red_combine(op, v, red[w]);
    partial[blockIdx.x] = v;
  }
}

// One reduction per grid row: every block writes its partial, and the block that arrives last
// (a ticket on counter, reset to 0 for the next use) folds the partials in the fixed order of
// k_reduce_final and writes out -- the same value as the two-launch form, bit for bit.  An
// empty input (n = 0, x unread) gives the operation's identity.
__device__ __forceinline__ void reduce_fused_row(int op, long n, const double* __restrict__ x,
                                                 const double* __restrict__ y, double* __restrict__ partial,
                                                 unsigned* __restrict__ counter, double* __restrict__ out) {
  __shared__ double red[RED_THREADS / 32];
  __shared__ bool last;
  double acc = red_identity(op);
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    acc = red_combine(op, acc, red_elem(op, x, y, i));
  for (int o = 16; o > 0; o >>= 1) acc = red_combine(op, acc, __shfl_xor_sync(0xffffffffu, acc, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = red_identity(op);
    for (int w = 0; w < RED_THREADS / 32; ++w) v = red_combine(op, v, red[w]);
    partial[blockIdx.x] = v;
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x >= 32) return;
  __threadfence();
  double v = red_identity(op);
  for (int p = threadIdx.x; p < (int)gridDim.x; p += 32) v = red_combine(op, v, __ldcg(partial + p));
  for (int o = 16; o > 0; o >>= 1) v = red_combine(op, v, __shfl_xor_sync(0xffffffffu, v, o));
  if (threadIdx.x == 0) {
    *out = v;
    *counter = 0u;
  }
}

extern "C" __global__ void __launch_bounds__(RED_THREADS)
k_reduce_fused(int op, long n, const double* __restrict__ x, const double* __restrict__ y,
               double* __restrict__ partial, unsigned* __restrict__ counter,
               double* __restrict__ out) {
  reduce_fused_row(op, n, x, y, partial, counter, out);
}

// Several independent reductions in one launch: grid row r computes request r into slot
// first + r exactly as k_reduce_fused would (the same blocks per reduction, the same folding).
extern "C" __global__ void __launch_bounds__(RED_THREADS)
k_reduce_batch(RedBatch b, double* __restrict__ partial, unsigned* __restrict__ counters,
               double* __restrict__ slots, int first) {
  const RedReq q = b.r[blockIdx.y];
  const int s = first + blockIdx.y;
  reduce_fused_row(q.op, q.n, q.x, q.y, partial + (size_t)s * gridDim.x, counters + s, slots + s);
}

// One warp: lane l folds partials l, l+32, ... in order, then a fixed shuffle tree.
extern "C" __global__ void k_reduce_final(int op, int nparts, const double* __restrict__ partial,
                                          double* __restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  double v = red_identity(op);
  for (int p = threadIdx.x; p < nparts; p += 32) v = red_combine(op, v, partial[p]);
  for (int o = 16; o > 0; o >>= 1) v = red_combine(op, v, __shfl_xor_sync(0xffffffffu, v, o));
  if (threadIdx.x == 0) *out = v;
}

// Diagonal max |H_ii| of a dense m x m matrix (for the proportional static shift).
extern "C" __global__ void k_diag_absmax(const double* __restrict__ H, int m,
                                         double* __restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) acc = fmax(acc, fabs(H[i + (long)i * m]));
  acc = warp_max(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmax(v, red[w]);
    *out = v;
  }
}

// y = alpha * P x + beta * y for P in CSR (both triangles), one thread per row.
extern "C" __global__ void k_csr_spmv(int n, const int* __restrict__ rowptr,
                                      const int* __restrict__ colidx,
                                      const double* __restrict__ val, const double* __restrict__ x,
                                      double alpha, double beta, double* __restrict__ y) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double acc = 0.0;
  for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) acc = fma(val[p], x[colidx[p]], acc);
  y[r] = alpha * acc + (beta == 0.0 ? 0.0 : beta * y[r]);
}
