// NT scaling of PSD blocks at MPFR width on the GPU: the reference's
// PSDTriangleCone::update_scaling (crates/solver/src/solver/cones/psdtrianglecone.rs:311-439) for
// MpFloat<N> (N <= 8), one CTA per block of order n <= 64:
//   S = mat(s), Z = mat(z) (off-diagonals times the working-precision 1/sqrt 2, matrix_math.rs:156-180)
//   L1 = chol(S), L2 = chol(Z)         exact-dot left-looking Cholesky (the reference's xpotrf,
//                                      algebra/dense/blas/mpfr.rs:726-789), the two factored
//                                      concurrently by the two halves of the CTA
//   M = L2' L1                          every entry an exact dot rounded once
//   M V = U Sigma                       right singular vectors by one-sided (Hestenes) Jacobi in
//                                      MpFloat arithmetic: the reference's MPFR right SVD
//                                      (mpfr_svd.rs, Golub-Kahan + dqds + inverse iteration) is
//                                      replaced by a method whose rotations of disjoint column
//                                      pairs run in parallel, one warp per pair (its column sums
//                                      exact dots over the lanes); singular values
//                                      are the final column norms, sorted descending
//   lambda = sigma, Lambda^-1/2 = 1 / sqrt(sigma)
//   R = L1 V Lambda^-1/2,  Rinv = Lambda^1/2 (L1^-T V)',  G = R R' (upper)
// V is unique up to the signs of its columns (and rotations within clusters of equal singular
// values); R, Rinv change with it as the reference's do, G, lambda and the congruences they define
// do not.  Per-block status: 0, or SDPXG_ST_CHOL_FAIL (s or z not interior), or
// SDPXG_ST_SVD_UNCONVERGED, and then the block's outputs are zeros; SDPXG_ST_EXACT_SPREAD in the shared status word when an exact dot
// exceeds the accumulator.
#include <stdexcept>

#include "device.cuh"
#include "mp.cuh"
#include "mp_ldl.cuh"

namespace sdpxg {
namespace {

using mpd::Val;

constexpr int kNtThreads = 512;  // 16 warps: up to 16 rotations of a round at once
constexpr int kNtWarps = kNtThreads / 32;
constexpr int kNtMaxSweeps = 80;

__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// a + b and a * b, rounded once
__device__ __forceinline__ Val add(const Val& a, const Val& b, int N) { return mpd::mp_addsub(a, b, 1, N); }
__device__ __forceinline__ Val sub(const Val& a, const Val& b, int N) { return mpd::mp_addsub(a, b, -1, N); }
__device__ __forceinline__ Val mul(const Val& a, const Val& b, int N) { return mpd::mp_mul(a, b, N); }

// Exact-dot Cholesky (lower, in place, column-major ld n) by a group of `nt` threads that
// synchronise on named barrier `bar`: the group's first warp forms each pivot (its dot split over
// the lanes), the group the column below it.
__device__ void chol_group(unsigned char* L, int n, int N, int t, int nt, int bar, unsigned char* sd,
                           volatile int* fail, uint32_t* status) {
  const long esz = 8L * N + 8;
  auto at = [&](int i, int k) { return L + ((long)i + (long)k * n) * esz; };
  for (int j = 0; j < n; ++j) {
    if (t < 32) {  // the group's first warp forms the pivot's dot, its lane 0 the rest
      bool ok = true;
      const Val dot = mpd::mp_dot_sub_warp(nullptr, at(j, 0), n, at(j, 0), n, j, N, &ok);
      if (t == 0) {
        const Val d = sub(mpd::mp_load(at(j, j), N), dot, N);
        if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
        if (d.zero || d.neg) {
          *fail = 1;
        } else {
          const Val r = mpd::mp_sqrt(d, N);
          mpd::mp_store(at(j, j), N, r, status);
          mpd::mp_store(sd, N, r, status);
        }
      }
    }
    named_sync(bar, nt);
    if (*fail) return;
    const Val r = mpd::mp_load(sd, N);
    for (int i = j + 1 + t; i < n; i += nt) {
      bool ok = true;
      const Val dot = mpd::mp_dot_sub(nullptr, at(i, 0), n, at(j, 0), n, j, N, &ok);
      if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
      mpd::mp_store(at(i, j), N, mpd::mp_div(sub(mpd::mp_load(at(i, j), N), dot, N), r, N), status);
    }
    named_sync(bar, nt);
  }
}

// One CTA per block (see the file comment).  Work: five n x n matrices per block at element
// 5 * mat (L1, L2, the Jacobi matrix A, V, X), two n-vectors at element 2 * vec (sigma, sqrt sigma).
__global__ void __launch_bounds__(kNtThreads) k_mp_nt_scale(const MpNtBlock* __restrict__ blocks, int N,
                                                            const unsigned char* __restrict__ s,
                                                            const unsigned char* __restrict__ z,
                                                            const unsigned char* __restrict__ frac,
                                                            unsigned char* __restrict__ work,
                                                            unsigned char* __restrict__ wvec,
                                                            unsigned char* __restrict__ lam,
                                                            unsigned char* __restrict__ lisqrt,
                                                            unsigned char* __restrict__ R,
                                                            unsigned char* __restrict__ Rinv,
                                                            unsigned char* __restrict__ G, int* __restrict__ bstatus,
                                                            uint32_t* __restrict__ status) {
  __shared__ __align__(8) unsigned char sd[2][8 * mpd::kMaxN + 8];
  __shared__ volatile int fail[2];
  __shared__ int rotated;
  __shared__ int perm[64];
  const MpNtBlock B = blocks[blockIdx.x];
  const int n = B.n, nn = n * n, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long esz = 8L * N + 8;
  auto el = [&](unsigned char* base, long e) { return base + e * esz; };
  unsigned char* L1 = work + 5 * B.mat * esz;
  unsigned char* L2 = L1 + nn * esz;
  unsigned char* A = L2 + nn * esz;
  unsigned char* V = A + nn * esz;
  unsigned char* X = V + nn * esz;
  unsigned char* sig = wvec + 2 * B.vec * esz;
  unsigned char* root = sig + n * esz;
  if (tid == 0) {
    fail[0] = fail[1] = 0;
    bstatus[blockIdx.x] = 0;
  }
  // S and Z, lower triangles (svec upper column order: (i, j), j <= i, at i (i + 1) / 2 + j)
  const Val fv = mpd::mp_load(frac, N);
  for (int e = tid; e < nn; e += kNtThreads) {
    const int i = e % n, j = e / n;
    Val sv = mpd::mp_zero(), zv = mpd::mp_zero();
    if (i >= j) {
      const long t = (long)i * (i + 1) / 2 + j;
      sv = mpd::mp_load(s + (B.svec + t) * esz, N);
      zv = mpd::mp_load(z + (B.svec + t) * esz, N);
      if (i != j) {
        sv = mul(sv, fv, N);
        zv = mul(zv, fv, N);
      }
    }
    mpd::mp_store(el(L1, e), N, sv, status);
    mpd::mp_store(el(L2, e), N, zv, status);
  }
  __syncthreads();
  if (tid < kNtThreads / 2)
    chol_group(L1, n, N, tid, kNtThreads / 2, 1, sd[0], &fail[0], status);
  else
    chol_group(L2, n, N, tid - kNtThreads / 2, kNtThreads / 2, 2, sd[1], &fail[1], status);
  __syncthreads();
  // a failed block's outputs are zeros
  auto zero_outputs = [&]() {
    for (int e = tid; e < nn; e += kNtThreads) {
      mpd::mp_store(el(R, B.mat + e), N, mpd::mp_zero(), status);
      mpd::mp_store(el(Rinv, B.mat + e), N, mpd::mp_zero(), status);
      mpd::mp_store(el(G, B.mat + e), N, mpd::mp_zero(), status);
    }
    for (int r = tid; r < n; r += kNtThreads) {
      mpd::mp_store(el(lam, B.vec + r), N, mpd::mp_zero(), status);
      mpd::mp_store(el(lisqrt, B.vec + r), N, mpd::mp_zero(), status);
    }
  };
  if (fail[0] || fail[1]) {
    if (tid == 0) bstatus[blockIdx.x] = SDPXG_ST_CHOL_FAIL;
    zero_outputs();
    return;
  }
  // A = M = L2' L1 (entry (i, j): rows k >= max(i, j)), V = I
  Val one = mpd::mp_zero();
  one.zero = false;
  one.m[N - 1] = 1ull << 63;
  one.s = 1 - 64LL * N;
  for (int e = tid; e < nn; e += kNtThreads) {
    const int i = e % n, j = e / n, k0 = i > j ? i : j;
    bool ok = true;
    const Val m = mpd::mp_dot_sub(nullptr, el(L2, k0 + (long)i * n), 1, el(L1, k0 + (long)j * n), 1, n - k0, N, &ok);
    if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
    mpd::mp_store(el(A, e), N, m, status);
    mpd::mp_store(el(V, e), N, i == j ? one : mpd::mp_zero(), status);
  }
  // One-sided Jacobi: sweeps of round-robin rounds (position 0 fixed, the others rotating), the
  // disjoint pairs of a round one per warp.  A pair rotates while |gamma| > 2^-(64N-8) sqrt(ab).
  const int mm = n + (n & 1);
  bool converged = n <= 1;
  for (int sweep = 0; sweep < kNtMaxSweeps && !converged; ++sweep) {
    __syncthreads();
    if (tid == 0) rotated = 0;
    for (int r = 0; r < mm - 1; ++r) {
      __syncthreads();
      for (int k = warp; k < mm / 2; k += kNtWarps) {
        const int pa = k, pb = mm - 1 - k;
        const int p = pa == 0 ? 0 : 1 + (pa - 1 + r) % (mm - 1);
        const int q = pb == 0 ? 0 : 1 + (pb - 1 + r) % (mm - 1);
        if (p >= n || q >= n) continue;
        // the three column sums as exact dots over the warp (every lane gets the same bits)
        bool okd = true;
        const Val aa = mpd::mp_dot_sub_warp(nullptr, el(A, (long)p * n), 1, el(A, (long)p * n), 1, n, N, &okd);
        const Val bb = mpd::mp_dot_sub_warp(nullptr, el(A, (long)q * n), 1, el(A, (long)q * n), 1, n, N, &okd);
        const Val gg = mpd::mp_dot_sub_warp(nullptr, el(A, (long)p * n), 1, el(A, (long)q * n), 1, n, N, &okd);
        if (!okd && lane == 0) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
        bool rot = !gg.zero && !aa.zero && !bb.zero;
        if (rot) {
          Val ab = mul(aa, bb, N);
          ab.s -= 2LL * (64 * N - 8);
          rot = mpd::mp_cmp(mul(gg, gg, N), ab, N) > 0;
        }
        if (!rot) continue;  // warp-uniform: every lane holds the same sums
        // zeta = (b - a) / (2 g), t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), c = 1/sqrt(1+t^2)
        Val g2 = gg;
        g2.s += 1;
        Val zeta = mul(sub(bb, aa, N), mpd::mp_recip_approx(g2, N), N);
        Val t;
        if (zeta.zero) {
          t = one;
        } else if (zeta.s + 64LL * N > 32LL * N + 8) {  // |zeta| > 2^(32N+8): t = 1 / (2 zeta)
          Val z2 = zeta;
          z2.s += 1;
          t = mpd::mp_recip_approx(z2, N);
        } else {
          Val az = zeta;
          az.neg = false;
          const Val w = add(one, mul(zeta, zeta, N), N);
          const Val sq = mul(w, mpd::mp_rsqrt_approx(w, N), N);
          t = mpd::mp_recip_approx(add(az, sq, N), N);
          t.neg = zeta.neg;
        }
        const Val c = mpd::mp_rsqrt_approx(add(one, mul(t, t, N), N), N);
        const Val sn = mul(c, t, N);
        for (int i = lane; i < n; i += 32) {
          unsigned char* M2[2] = {A, V};
          for (int w = 0; w < 2; ++w) {
            unsigned char* xp = el(M2[w], i + (long)p * n);
            unsigned char* xq = el(M2[w], i + (long)q * n);
            const Val vp = mpd::mp_load(xp, N), vq = mpd::mp_load(xq, N);
            mpd::mp_store(xp, N, sub(mul(c, vp, N), mul(sn, vq, N), N), status);
            mpd::mp_store(xq, N, add(mul(sn, vp, N), mul(c, vq, N), N), status);
          }
        }
        if (lane == 0) atomicAdd(&rotated, 1);
      }
    }
    __syncthreads();
    converged = rotated == 0;
  }
  if (!converged) {
    if (tid == 0) bstatus[blockIdx.x] = SDPXG_ST_SVD_UNCONVERGED;
    zero_outputs();
    return;
  }
  // singular values: column norms (exact sums of squares, correctly rounded roots), descending
  for (int j = tid; j < n; j += kNtThreads) {
    bool ok = true;
    const Val ss = mpd::mp_dot_sub(nullptr, el(A, (long)j * n), 1, el(A, (long)j * n), 1, n, N, &ok);
    if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
    mpd::mp_store(el(sig, j), N, mpd::mp_sqrt(ss, N), status);
  }
  __syncthreads();
  for (int j = tid; j < n; j += kNtThreads) {
    const Val sj = mpd::mp_load(el(sig, j), N);
    int rank = 0;
    for (int k = 0; k < n; ++k) {
      if (k == j) continue;
      const int c = mpd::mp_cmp(mpd::mp_load(el(sig, k), N), sj, N);
      rank += (c > 0 || (c == 0 && k < j)) ? 1 : 0;
    }
    perm[rank] = j;
  }
  __syncthreads();
  for (int r = tid; r < n; r += kNtThreads) {
    const Val sg = mpd::mp_load(el(sig, perm[r]), N);
    const Val rt = mpd::mp_sqrt(sg, N);
    mpd::mp_store(el(lam, B.vec + r), N, sg, status);
    mpd::mp_store(el(root, r), N, rt, status);
    mpd::mp_store(el(lisqrt, B.vec + r), N, mpd::mp_recip(rt, N), status);
  }
  __syncthreads();
  // R = L1 V Lambda^-1/2 (row i of L1 has entries k <= i); X = L1^-T V (back substitution)
  for (int e = tid; e < nn; e += kNtThreads) {
    const int i = e % n, r = e / n;
    bool ok = true;
    const Val d = mpd::mp_dot_sub(nullptr, el(L1, i), n, el(V, (long)perm[r] * n), 1, i + 1, N, &ok);
    if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
    mpd::mp_store(el(R, B.mat + e), N, mul(d, mpd::mp_load(el(lisqrt, B.vec + r), N), N), status);
  }
  for (int r = tid; r < n; r += kNtThreads) {
    for (int i = n - 1; i >= 0; --i) {
      bool ok = true;
      const Val b = mpd::mp_load(el(V, i + (long)perm[r] * n), N);
      const Val d = mpd::mp_dot_sub(&b, el(L1, i + 1 + (long)i * n), 1, el(X, i + 1 + (long)r * n), 1, n - 1 - i, N,
                                    &ok);
      if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
      mpd::mp_store(el(X, i + (long)r * n), N, mpd::mp_div(d, mpd::mp_load(el(L1, i + (long)i * n), N), N), status);
    }
  }
  __syncthreads();
  // Rinv(r, j) = sqrt(sigma_r) X(j, r); G = R R' (upper: exact dots of rows of R)
  for (int e = tid; e < nn; e += kNtThreads) {
    const int r = e % n, j = e / n;
    mpd::mp_store(el(Rinv, B.mat + e), N,
                  mul(mpd::mp_load(el(X, j + (long)r * n), N), mpd::mp_load(el(root, r), N), N), status);
    Val g = mpd::mp_zero();
    if (r <= j) {
      bool ok = true;
      g = mpd::mp_dot_sub(nullptr, el(R, B.mat + r), n, el(R, B.mat + j), n, n, N, &ok);
      if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
    }
    mpd::mp_store(el(G, B.mat + e), N, g, status);
  }
}

// The working-precision 1/sqrt 2 (FloatConst::FRAC_1_SQRT_2): sqrt(1/2) rounded once.
__global__ void k_mp_frac_sqrt2(int N, unsigned char* out, uint32_t* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Val h = mpd::mp_zero();
  h.zero = false;
  h.m[N - 1] = 1ull << 63;
  h.s = -64LL * N;  // 2^63 2^(64(N-1)) 2^-64N = 1/2
  mpd::mp_store(out, N, mpd::mp_sqrt(h, N), status);
}

}  // namespace

void mp_launch_nt_scale(const MpNtBlock* blocks, int nblk, int N, const unsigned char* s, const unsigned char* z,
                        unsigned char* frac, unsigned char* work, unsigned char* wvec, unsigned char* lam,
                        unsigned char* lisqrt, unsigned char* R, unsigned char* Rinv, unsigned char* G, int* bstatus,
                        uint32_t* status, cudaStream_t st) {
  if (N < 1 || N > mpd::kMaxN) throw std::invalid_argument("MPFR NT scaling: limbs must be in 1..8");
  if (nblk <= 0) return;
  ++g_launches, k_mp_frac_sqrt2<<<1, 32, 0, st>>>(N, frac, status);
  ++g_launches, k_mp_nt_scale<<<nblk, kNtThreads, 0, st>>>(blocks, N, s, z, frac, work, wvec, lam, lisqrt, R, Rinv,
                                                           G, bstatus, status);
  check(cudaGetLastError(), "k_mp_nt_scale");
}

}  // namespace sdpxg
