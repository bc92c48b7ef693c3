// MPFR dense LDL' kernels on MpFloat<N> arrays (see mp_ldl.cuh and mp.cuh).
#include <stdexcept>

#include "device.cuh"
#include "mp.cuh"
#include "mp_ldl.cuh"

namespace sdpxg {
namespace {

using mpd::Val;

__device__ __forceinline__ unsigned char* el(unsigned char* A, long i, long j, long ld, int N) {
  return A + (i + j * ld) * (8L * N + 8);
}
__device__ __forceinline__ const unsigned char* el(const unsigned char* A, long i, long j, long ld, int N) {
  return A + (i + j * ld) * (8L * N + 8);
}

// arrow.rs:156-242 ldl_dots on one block: columns in order; the pivot
// d_j = a_jj - dot(r_j, w_j) (the exact difference rounded once when that rounds to zero), the
// pivot rule, D^-1; then every later row i: r_ij = (a_ij - dot(r_i, w_j)) * d_j^-1,
// w_ij = r_ij d_j.  Dots are exact and rounded once; the other operations round once each.
// The block's lower triangle is copied into a row-major scratch R (and W is kept row-major) so
// that every dot reads two contiguous rows; each dot runs on one warp (mp_dot_sub_warp), warp 0
// for the pivot, the CTA's 32 warps over the later rows; R is written back at the end.
// Scratch: 2 size^2 elements (W, then R).
constexpr int kLeafThreads = 1024;
__global__ void __launch_bounds__(kLeafThreads) k_mp_ldl_dots(unsigned char* A, long lda, int off, int size, int N,
                                                              unsigned char* Wsc, unsigned char* dinv,
                                                              const unsigned char* reg, uint32_t* status) {
  __shared__ __align__(8) unsigned char sd[8 * mpd::kMaxN + 8];  // d_j
  __shared__ int s_fail;
  const long esz = 8L * N + 8;
  unsigned char* B = A + ((long)off + (long)off * lda) * esz;
  unsigned char* W = Wsc;                            // row-major: (i, c) at i * size + c
  unsigned char* R = Wsc + (long)size * size * esz;  // row-major copy of the lower triangle
  auto rm = [&](unsigned char* M, int i, int c) { return M + ((long)i * size + c) * esz; };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  if (threadIdx.x == 0) s_fail = 0;
  for (long wd = threadIdx.x; wd < (long)size * size * esz / 8; wd += blockDim.x) {  // R(i, c) = B(i, c)
    const long e = wd * 8 / esz, o = wd * 8 % esz;
    const int i = (int)(e / size), c = (int)(e % size);
    if (c <= i)
      *reinterpret_cast<unsigned long long*>(rm(R, i, c) + o) =
          *reinterpret_cast<const unsigned long long*>(el(B, i, c, lda, N) + o);
  }
  __syncthreads();
  for (int j = 0; j < size; ++j) {
    if (warp == 0) {  // the pivot: the dot over the lanes, the rest on lane 0
      bool ok = true;
      const Val a = mpd::mp_load(rm(R, j, j), N);
      const Val dot = mpd::mp_dot_sub_warp(nullptr, rm(R, j, 0), 1, rm(W, j, 0), 1, j, N, &ok);
      Val d = mpd::mp_addsub(a, dot, -1, N);
      if (d.zero && j > 0) d = mpd::mp_dot_sub_warp(&a, rm(R, j, 0), 1, rm(W, j, 0), 1, j, N, &ok);
      if (lane == 0) {
        if (reg) {  // DenseLeaf::pivot (arrow.rs:618-632), sign +1
          const Val eps = mpd::mp_load(reg, N), delta = mpd::mp_load(reg + 8 * N + 8, N);
          if (mpd::mp_cmp(d, eps, N) < 0) d = delta;
        }
        if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
        if (d.zero) {
          atomicOr(status, SDPXG_ST_PIVOT_FAIL);
          s_fail = 1;
        } else {
          mpd::mp_store(sd, N, d, status);
          mpd::mp_store(dinv + (long)j * esz, N, mpd::mp_recip(d, N), status);
        }
      }
    }
    __syncthreads();
    if (s_fail) return;
    const Val d = mpd::mp_load(sd, N);
    const Val di = mpd::mp_load(dinv + (long)j * esz, N);
    for (int i = j + 1 + warp; i < size; i += nwarps) {  // warp-uniform
      bool ok = true;
      const Val dot = mpd::mp_dot_sub_warp(nullptr, rm(R, i, 0), 1, rm(W, j, 0), 1, j, N, &ok);
      if (lane == 0) {
        if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
        const Val v = mpd::mp_mul(mpd::mp_addsub(mpd::mp_load(rm(R, i, j), N), dot, -1, N), di, N);
        mpd::mp_store(rm(R, i, j), N, v, status);
        mpd::mp_store(rm(W, i, j), N, mpd::mp_mul(v, d, N), status);
      }
    }
    __syncthreads();
  }
  for (long wd = threadIdx.x; wd < (long)size * size * esz / 8; wd += blockDim.x) {  // B(i, c) = R(i, c), c < i
    const long e = wd * 8 / esz, o = wd * 8 % esz;
    const int i = (int)(e / size), c = (int)(e % size);
    if (c < i)
      *reinterpret_cast<unsigned long long*>(el(B, i, c, lda, N) + o) =
          *reinterpret_cast<const unsigned long long*>(rm(R, i, c) + o);
  }
  for (int j = threadIdx.x; j < size; j += blockDim.x) {  // unit diagonal
    Val one = mpd::mp_zero();
    one.zero = false;
    one.m[N - 1] = 1ull << 63;
    one.s = 1 - 64LL * N;
    mpd::mp_store(el(B, j, j, lda, N), N, one, status);
  }
}

// arrow.rs:437-447: each row of B solves x L' = b by exact dots, x_j = b_j - dot(x_<j, L(j, <j)).
// One warp per row (the dots split over the lanes, mp_dot_sub_warp), four rows per CTA.
__global__ void __launch_bounds__(128) k_mp_solve_lt(const unsigned char* L, long ldl, int k, unsigned char* B,
                                                     long ldb, int m, int N, uint32_t* status) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= m) return;  // warp-uniform
  for (int j = 0; j < k; ++j) {
    bool ok = true;
    const Val x = mpd::mp_load(el(B, i, j, ldb, N), N);
    const Val dot = mpd::mp_dot_sub_warp(nullptr, el(B, i, 0, ldb, N), ldb, el(L, j, 0, ldl, N), ldl, j, N, &ok);
    if (lane == 0) {
      if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
      mpd::mp_store(el(B, i, j, ldb, N), N, mpd::mp_addsub(x, dot, -1, N), status);
    }
    __syncwarp();  // x_j visible to the lanes' next dot
  }
}

__global__ void k_mp_sub_block(unsigned char* B, long ldb, const unsigned char* P, long ldp, int m, int n, int N,
                               uint32_t* status) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)m * n) return;
  const int i = (int)(idx % m), j = (int)(idx / m);
  const Val b = mpd::mp_load(el(B, i, j, ldb, N), N), p = mpd::mp_load(el(P, i, j, ldp, N), N);
  mpd::mp_store(el(B, i, j, ldb, N), N, mpd::mp_addsub(b, p, -1, N), status);
}

__global__ void k_mp_copy_scale_cols(unsigned char* A, long lda, unsigned char* W, const unsigned char* d, int m,
                                     int n, int N, uint32_t* status) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)m * n) return;
  const int i = (int)(idx % m), j = (int)(idx / m);
  const long esz = 8L * N + 8;
  const Val a = mpd::mp_load(el(A, i, j, lda, N), N);
  unsigned char* w = el(W, i, j, m, N);
  const unsigned char* src = el(A, i, j, lda, N);
  for (long b = 0; b < esz; ++b) w[b] = src[b];
  mpd::mp_store(el(A, i, j, lda, N), N, mpd::mp_mul(a, mpd::mp_load(d + (long)j * esz, N), N), status);
}

__global__ void k_mp_sub_upper_t(unsigned char* A, long lda, const unsigned char* C, long ldc, int n, int N,
                                 uint32_t* status) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)n * n) return;
  const int b = (int)(idx % n), a = (int)(idx / n);  // entry (b, a) of the lower triangle
  if (b < a) return;
  const Val x = mpd::mp_load(el(A, b, a, lda, N), N), c = mpd::mp_load(el(C, a, b, ldc, N), N);
  mpd::mp_store(el(A, b, a, lda, N), N, mpd::mp_addsub(x, c, -1, N), status);
}

// XpotrfScalar::xpotrf for MpFloat (algebra/dense/blas/mpfr.rs:726-789): left-looking Cholesky
// of the stored triangle, entry (i, k), i >= k, at i * si + k * sk (lower: si = 1, sk = ld;
// upper: si = ld, sk = 1).  Per column j: d = a_jj - dot(l_j, l_j) (the dot exact and rounded
// once, the difference rounded), failure when d <= 0 (info = j + 1), l_jj = sqrt(d) rounded; then
// every later row i: l_ij = (a_ij - dot(l_i, l_j)) / l_jj, each operation rounded once.
__global__ void __launch_bounds__(128) k_mp_potrf(unsigned char* A, long si, long sk, int n, int N, int* info,
                                                  uint32_t* status) {
  __shared__ __align__(8) unsigned char sd[8 * mpd::kMaxN + 8];
  __shared__ int s_fail;
  const long esz = 8L * N + 8;
  auto at = [&](long i, long k) { return A + (i * si + k * sk) * esz; };
  if (threadIdx.x == 0) {
    s_fail = 0;
    *info = 0;
  }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    if (threadIdx.x < 32) {  // warp 0 forms the pivot's dot, its lane 0 the rest
      bool ok = true;
      const Val dot = mpd::mp_dot_sub_warp(nullptr, at(j, 0), sk, at(j, 0), sk, j, N, &ok);
      if (threadIdx.x == 0) {
        const Val a = mpd::mp_load(at(j, j), N);
        const Val d = mpd::mp_addsub(a, dot, -1, N);
        if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
        if (d.zero || d.neg) {
          mpd::mp_store(at(j, j), N, d, status);
          *info = j + 1;
          s_fail = 1;
        } else {
          const Val r = mpd::mp_sqrt(d, N);
          mpd::mp_store(at(j, j), N, r, status);
          mpd::mp_store(sd, N, r, status);
        }
      }
    }
    __syncthreads();
    if (s_fail) return;
    const Val r = mpd::mp_load(sd, N);
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      bool ok = true;
      const Val a = mpd::mp_load(at(i, j), N);
      const Val dot = mpd::mp_dot_sub(nullptr, at(i, 0), sk, at(j, 0), sk, j, N, &ok);
      if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
      mpd::mp_store(at(i, j), N, mpd::mp_div(mpd::mp_addsub(a, dot, -1, N), r, N), status);
    }
    __syncthreads();
  }
}

void check_limbs(int N) {
  if (N < 1 || N > mpd::kMaxN) throw std::invalid_argument("MPFR LDL: limbs must be in 1..8");
}

}  // namespace

void mp_launch_ldl_dots(unsigned char* A, long lda, int off, int size, int N, unsigned char* W, unsigned char* dinv,
                        const unsigned char* reg, uint32_t* status, cudaStream_t st) {
  check_limbs(N);
  if (size <= 0) return;
  if (size > kMpRecBase) throw std::invalid_argument("MPFR LDL: leaf above the recursion base");
  ++g_launches, k_mp_ldl_dots<<<1, kLeafThreads, 0, st>>>(A, lda, off, size, N, W, dinv, reg, status);
  check(cudaGetLastError(), "k_mp_ldl_dots");
}

// The stacked operands of the block product sum (rns_blas.rs:2656-2923 gemm_blocks_upper): block
// b's w_b x q_b factor y_b (column-major) fills rows [r0_b, r0_b + w_b) of the W x m matrices Y
// and Z at its global columns cols, Y = y_b and Z = d_b[r] * y_b (each product rounded once); every
// other entry is zero.  One thread per stacked entry (W x m): the block of a row by binary search
// over the row offsets, the column by a search of the block's sorted column list.
__global__ void k_mp_stack_blocks(int nb, const long* __restrict__ r0, const long* __restrict__ yoff,
                                  const long* __restrict__ coff, const int* __restrict__ qn,
                                  const unsigned char* __restrict__ y, const unsigned char* __restrict__ d,
                                  const unsigned long long* __restrict__ cols, long W, int m, int N,
                                  unsigned char* __restrict__ Z, unsigned char* __restrict__ Y,
                                  uint32_t* __restrict__ status) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= W * m) return;
  const long row = e % W;
  const int col = (int)(e / W);
  const size_t esz = 8 * (size_t)N + 8;
  int lo = 0, hi = nb - 1;  // last block with r0 <= row
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (r0[mid] <= row) lo = mid; else hi = mid - 1;
  }
  const int b = lo;
  const long r = row - r0[b], w = r0[b + 1] - r0[b];
  const unsigned long long* cb = cols + coff[b];
  int a = 0, z = qn[b] - 1, c = -1;
  while (a <= z) {
    const int mid = (a + z) / 2;
    if (cb[mid] == (unsigned long long)col) { c = mid; break; }
    if (cb[mid] < (unsigned long long)col) a = mid + 1; else z = mid - 1;
  }
  mpd::Val vy = mpd::mp_zero(), vz = mpd::mp_zero();
  if (c >= 0) {
    vy = mpd::mp_load(y + (size_t)(yoff[b] + r + (long)c * w) * esz, N);
    vz = mpd::mp_mul(mpd::mp_load(d + (size_t)(r0[b] + r) * esz, N), vy, N);
  }
  mpd::mp_store(Y + (size_t)e * esz, N, vy, status);
  mpd::mp_store(Z + (size_t)e * esz, N, vz, status);
}

void mp_launch_potrf(unsigned char* A, long lda, int n, bool lower, int N, int* info, uint32_t* status,
                     cudaStream_t st) {
  check_limbs(N);
  if (n <= 0) return;
  ++g_launches, k_mp_potrf<<<1, 128, 0, st>>>(A, lower ? 1 : lda, lower ? lda : 1, n, N, info, status);
  check(cudaGetLastError(), "k_mp_potrf");
}

void mp_launch_solve_lt(const unsigned char* L, long ldl, int k, unsigned char* B, long ldb, int m, int N,
                        uint32_t* status, cudaStream_t st) {
  check_limbs(N);
  if (m <= 0 || k <= 0) return;
  ++g_launches, k_mp_solve_lt<<<(m + 3) / 4, 128, 0, st>>>(L, ldl, k, B, ldb, m, N, status);
  check(cudaGetLastError(), "k_mp_solve_lt");
}

void mp_launch_sub_block(unsigned char* B, long ldb, const unsigned char* P, long ldp, int m, int n, int N,
                         uint32_t* status, cudaStream_t st) {
  if (m <= 0 || n <= 0) return;
  ++g_launches, k_mp_sub_block<<<(unsigned)(((long)m * n + 127) / 128), 128, 0, st>>>(B, ldb, P, ldp, m, n, N,
                                                                                      status);
  check(cudaGetLastError(), "k_mp_sub_block");
}

void mp_launch_copy_scale_cols(unsigned char* A, long lda, unsigned char* W, const unsigned char* d, int m, int n,
                               int N, uint32_t* status, cudaStream_t st) {
  if (m <= 0 || n <= 0) return;
  ++g_launches, k_mp_copy_scale_cols<<<(unsigned)(((long)m * n + 127) / 128), 128, 0, st>>>(A, lda, W, d, m, n, N,
                                                                                            status);
  check(cudaGetLastError(), "k_mp_copy_scale_cols");
}

void mp_launch_sub_upper_t(unsigned char* A, long lda, const unsigned char* C, long ldc, int n, int N,
                           uint32_t* status, cudaStream_t st) {
  if (n <= 0) return;
  ++g_launches, k_mp_sub_upper_t<<<(unsigned)(((long)n * n + 127) / 128), 128, 0, st>>>(A, lda, C, ldc, n, N,
                                                                                        status);
  check(cudaGetLastError(), "k_mp_sub_upper_t");
}

void mp_launch_stack_blocks(int nb, const long* r0, const long* yoff, const long* coff, const int* qn,
                            const unsigned char* y, const unsigned char* d, const unsigned long long* cols, long W,
                            int m, int N, unsigned char* Z, unsigned char* Y, uint32_t* status, cudaStream_t st) {
  check_limbs(N);
  if (W <= 0 || m <= 0) return;
  ++g_launches, k_mp_stack_blocks<<<(unsigned)((W * m + 127) / 128), 128, 0, st>>>(nb, r0, yoff, coff, qn, y, d,
                                                                                   cols, W, m, N, Z, Y, status);
  check(cudaGetLastError(), "k_mp_stack_blocks");
}

}  // namespace sdpxg
