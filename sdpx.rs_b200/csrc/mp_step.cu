// Step-length bound of a PSD block at MPFR width on the GPU: the reference's
// step_length_psd_component for precisions above 64 bits (crates/solver/src/solver/cones/
// psdtrianglecone.rs:1180-1231, with eigval_min_f64 1233-1285, min_eigenvalue_f64 1287-1390,
// admits 1168-1178, lrscale_symmetric 1391-1406).  Per block, from the exact congruence
// Y = W-congruence of the direction (computed beforehand by the exact RNS congruence):
//   wv = svec(Y); Delta = mat(wv) scaled on both sides by Lambda^-1/2 (each product rounded)
//   n > 3: gamma = lambda_min of Delta's binary64 copy (Householder tridiagonalisation and Sturm
//          bisection, the reference's operation order, every FP64 operation rounded separately:
//          no contraction into FMA), accepted when its a priori bound 2 (n+1)^2 eps |Delta|_F is
//          within 1e-10 of max(|gamma|, 1/alpha_max), else certified by an exact-dot Cholesky of
//          I + alpha_c Delta at alpha_c = (1 - 1e-10) min(-1/gamma, alpha_max)
//   otherwise (n <= 3, a non-finite copy, a failed certificate): lambda_min of Delta in MpFloat
//          arithmetic by cyclic two-sided Jacobi (the reference's MPFR eigensolver,
//          algebra/dense/blas/mpfr_eigen.rs, is replaced by it; it agrees to working precision)
//   alpha = min(-1/gamma, alpha_max) when gamma < 0, else alpha_max.
// path[b]: 0 a priori bound, 1 certified, 2 MpFloat eigensolver, 3 the eigensolver did not converge
// (alpha = 0, the reference's zero step for a failed eigensolve).
#include <cfloat>
#include <stdexcept>

#include "device.cuh"
#include "mp.cuh"
#include "mp_ldl.cuh"

namespace sdpxg {
namespace {

using mpd::Val;

constexpr int kStThreads = 128;

__device__ __forceinline__ Val add(const Val& a, const Val& b, int N) { return mpd::mp_addsub(a, b, 1, N); }
__device__ __forceinline__ Val sub(const Val& a, const Val& b, int N) { return mpd::mp_addsub(a, b, -1, N); }
__device__ __forceinline__ Val mul(const Val& a, const Val& b, int N) { return mpd::mp_mul(a, b, N); }

// v rounded to binary64, to nearest with ties to even (values beyond the normal range become
// infinities or are rounded once more by ldexp into the subnormals).
__device__ inline double to_double(const Val& v, int N) {
  if (v.zero) return v.neg ? -0.0 : 0.0;
  const unsigned long long top = v.m[N - 1];  // top bit set
  unsigned long long mant = top >> 11;         // 53 bits
  const unsigned long long rest = top & 0x7FFull;
  bool sticky = (rest & 0x3FFull) != 0;
  for (int q = 0; q < N - 1 && !sticky; ++q) sticky = v.m[q] != 0;
  const bool half = (rest >> 10) & 1ull;
  if (half && (sticky || (mant & 1ull))) ++mant;  // may carry to 2^53: still exact in FP64
  // value = mant 2^(s + 64N - 53) (before the carry, mant < 2^53)
  const long long e = v.s + 64LL * N - 53;
  double r;
  if (e > 1100)
    r = HUGE_VAL;
  else if (e < -1200)
    r = 0.0;
  else
    r = ldexp((double)mant, (int)e);
  return v.neg ? -r : r;
}

// The reference's min_eigenvalue_f64 on a (n x n column-major, both triangles; overwritten), in
// its operation order with every operation rounded on its own.  d, e: n-entry scratch.  Returns
// false for a non-finite Gershgorin interval.
__device__ bool min_eigenvalue_f64(double* a, int n, double* d, double* e, double* out) {
  auto at = [&](int i, int j) -> double& { return a[i + j * n]; };
  for (int i = 0; i < n; ++i) d[i] = e[i] = 0.0;
  for (int i = n - 1; i >= 1; --i) {
    const int l = i - 1;
    double h = 0.0;
    if (l > 0) {
      double scale = -0.0;
      for (int k = 0; k <= l; ++k) scale = __dadd_rn(scale, fabs(at(i, k)));
      if (scale == 0.0) {
        e[i] = at(i, l);
      } else {
        for (int k = 0; k <= l; ++k) {
          at(i, k) = __ddiv_rn(at(i, k), scale);
          h = __dadd_rn(h, __dmul_rn(at(i, k), at(i, k)));
        }
        double f = at(i, l);
        const double g = f >= 0.0 ? -__dsqrt_rn(h) : __dsqrt_rn(h);
        e[i] = __dmul_rn(scale, g);
        h = __dsub_rn(h, __dmul_rn(f, g));
        at(i, l) = __dsub_rn(f, g);
        f = 0.0;
        for (int j = 0; j <= l; ++j) {
          double gg = 0.0;
          for (int k = 0; k <= j; ++k) gg = __dadd_rn(gg, __dmul_rn(at(j, k), at(i, k)));
          for (int k = j + 1; k <= l; ++k) gg = __dadd_rn(gg, __dmul_rn(at(k, j), at(i, k)));
          e[j] = __ddiv_rn(gg, h);
          f = __dadd_rn(f, __dmul_rn(e[j], at(i, j)));
        }
        const double hh = __ddiv_rn(f, __dadd_rn(h, h));
        for (int j = 0; j <= l; ++j) {
          const double ff = at(i, j);
          const double gg = __dsub_rn(e[j], __dmul_rn(hh, ff));
          e[j] = gg;
          for (int k = 0; k <= j; ++k)
            at(j, k) = __dsub_rn(at(j, k), __dadd_rn(__dmul_rn(ff, e[k]), __dmul_rn(gg, at(i, k))));
        }
      }
    } else {
      e[i] = at(i, l);
    }
    d[i] = h;
  }
  e[0] = 0.0;
  for (int i = 0; i < n; ++i) d[i] = at(i, i);
  const double tiny = __ddiv_rn(DBL_MIN, DBL_EPSILON);
  auto below = [&](double x) {
    int count = 0;
    double q = __dsub_rn(d[0], x);
    for (int i = 0; i < n; ++i) {
      if (i > 0) q = __dsub_rn(__dsub_rn(d[i], x), __ddiv_rn(__dmul_rn(e[i], e[i]), q));
      if (q == 0.0) q = -tiny;
      if (q < 0.0) ++count;
    }
    return count;
  };
  double lo = HUGE_VAL, hi = -HUGE_VAL;
  for (int i = 0; i < n; ++i) {
    const double r = __dadd_rn(fabs(e[i]), i + 1 < n ? fabs(e[i + 1]) : 0.0);
    lo = fmin(lo, __dsub_rn(d[i], r));
    hi = fmax(hi, __dadd_rn(d[i], r));
  }
  if (!isfinite(lo) || !isfinite(hi)) return false;
  const double width = fmax(__dsub_rn(hi, lo), __dmul_rn(fmax(fabs(hi), fabs(lo)), DBL_EPSILON));
  lo = __dsub_rn(lo, __dmul_rn(width, DBL_EPSILON));
  hi = __dadd_rn(hi, __dmul_rn(width, DBL_EPSILON));
  for (int it = 0; it < 128; ++it) {
    const double mid = __dmul_rn(0.5, __dadd_rn(lo, hi));
    if (mid <= lo || mid >= hi) break;
    if (below(mid) >= 1)
      hi = mid;
    else
      lo = mid;
  }
  *out = __dmul_rn(0.5, __dadd_rn(lo, hi));
  return true;
}


// lambda_min of the symmetric n x n A (column-major, full; overwritten) by cyclic two-sided Jacobi
// in MpFloat arithmetic, one warp (lanes over rows and columns).  false when 60 sweeps leave an
// off-diagonal entry above 2^-(64N-8) sqrt|a_pp a_qq|.
__device__ bool jacobi_min_eig(unsigned char* A, int n, int N, Val* out, uint32_t* status) {
  const long esz = 8L * N + 8;
  const int lane = threadIdx.x & 31;
  auto el = [&](int i, int j) { return A + ((long)i + (long)j * n) * esz; };
  Val one = mpd::mp_zero();
  one.zero = false;
  one.m[N - 1] = 1ull << 63;
  one.s = 1 - 64LL * N;
  bool converged = n <= 1;
  for (int sweep = 0; sweep < 60 && !converged; ++sweep) {
    int rotations = 0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const Val apq = mpd::mp_load(el(p, q), N);
        if (apq.zero) continue;
        const Val app = mpd::mp_load(el(p, p), N), aqq = mpd::mp_load(el(q, q), N);
        Val pp = mul(app, aqq, N);
        pp.neg = false;
        pp.s -= 2LL * (64 * N - 8);
        if (!pp.zero && mpd::mp_cmp(mul(apq, apq, N), pp, N) <= 0) continue;
        ++rotations;
        Val a2 = apq;
        a2.s += 1;
        const Val th = mul(sub(aqq, app, N), mpd::mp_recip_approx(a2, N), N);
        Val t;
        if (th.zero) {
          t = one;
        } else if (th.s + 64LL * N > 32LL * N + 8) {
          Val t2 = th;
          t2.s += 1;
          t = mpd::mp_recip_approx(t2, N);
        } else {
          Val ath = th;
          ath.neg = false;
          const Val w = add(mul(th, th, N), one, N);
          t = mpd::mp_recip_approx(add(ath, mul(w, mpd::mp_rsqrt_approx(w, N), N), N), N);
          t.neg = th.neg;
        }
        const Val c = mpd::mp_rsqrt_approx(add(one, mul(t, t, N), N), N);
        const Val sn = mul(c, t, N);
        for (int k = lane; k < n; k += 32) {  // columns p, q
          const Val kp = mpd::mp_load(el(k, p), N), kq = mpd::mp_load(el(k, q), N);
          mpd::mp_store(el(k, p), N, sub(mul(c, kp, N), mul(sn, kq, N), N), status);
          mpd::mp_store(el(k, q), N, add(mul(sn, kp, N), mul(c, kq, N), N), status);
        }
        __syncwarp();
        for (int k = lane; k < n; k += 32) {  // rows p, q
          const Val pk = mpd::mp_load(el(p, k), N), qk = mpd::mp_load(el(q, k), N);
          mpd::mp_store(el(p, k), N, sub(mul(c, pk, N), mul(sn, qk, N), N), status);
          mpd::mp_store(el(q, k), N, add(mul(sn, pk, N), mul(c, qk, N), N), status);
        }
        __syncwarp();
      }
    converged = rotations == 0;
  }
  Val mn = mpd::mp_load(el(0, 0), N);
  for (int i = 1; i < n; ++i) {
    const Val v = mpd::mp_load(el(i, i), N);
    if (mpd::mp_cmp(v, mn, N) < 0) mn = v;
  }
  *out = mn;
  return converged;
}

// One CTA per block: Delta from the congruence Y (n x n at element `mat`), then the bound.
// consts: the working-precision 1/sqrt 2 and alpha_max.
// work: 2 n^2 elements per block at 2 * mat (Delta, then I + alpha_c Delta or the Jacobi copy);
// fwork: n^2 + 2n doubles per block at mat + 2 vec.
__global__ void __launch_bounds__(kStThreads) k_mp_step_bound(const MpStepBlock* __restrict__ blocks, int N,
                                                              const unsigned char* __restrict__ Y,
                                                              const unsigned char* __restrict__ lisqrt,
                                                              const unsigned char* __restrict__ consts,
                                                              unsigned char* __restrict__ work, double* __restrict__ fwork,
                                                              unsigned char* __restrict__ alpha, int* __restrict__ path,
                                                              uint32_t* __restrict__ status) {
  __shared__ __align__(8) unsigned char s_alc[8 * mpd::kMaxN + 8], s_piv[8 * mpd::kMaxN + 8];
  __shared__ int s_mode, s_fail;  // mode: 0 accepted, 1 to certify, 2 eigensolver, 4 certified
  __shared__ double s_gamma;
  const MpStepBlock B = blocks[blockIdx.x];
  const int n = B.n, nn = n * n, tid = threadIdx.x;
  const long esz = 8L * N + 8;
  auto el = [&](unsigned char* base, long e) { return base + e * esz; };
  auto cel = [&](const unsigned char* base, long e) { return base + e * esz; };
  unsigned char* D = work + 2 * B.mat * esz;
  unsigned char* C = D + nn * esz;
  double* a = fwork + B.mat + 2 * B.vec;
  const Val frac = mpd::mp_load(cel(consts, 0), N), amax = mpd::mp_load(cel(consts, 1), N);
  // Delta(r, c) = mat(svec(Y))(r, c) * (d_r d_c), the upper entry (r <= c) mirrored: svec's
  // off-diagonal is (Y_rc + Y_cr) / sqrt 2 (Y exactly symmetric: 2 Y_rc exactly), mat's is that
  // times 1/sqrt 2, each product rounded once (matrix_math.rs:156-180, 231-260)
  for (int e = tid; e < nn; e += kStThreads) {
    const int r = e % n, c = e / n;
    if (r > c) continue;
    Val v = mpd::mp_load(cel(Y, B.mat + r + (long)c * n), N);
    if (r != c) {
      if (!v.zero) v.s += 1;
      v = mul(mul(v, frac, N), frac, N);
    }
    const Val dd = mul(mpd::mp_load(cel(lisqrt, B.vec + r), N), mpd::mp_load(cel(lisqrt, B.vec + c), N), N);
    v = mul(v, dd, N);
    mpd::mp_store(el(D, e), N, v, status);
    if (r != c) mpd::mp_store(el(D, c + (long)r * n), N, v, status);
  }
  __syncthreads();
  if (tid == 0) {
    s_mode = 2;
    s_fail = 0;
    if (n > 3) {
      const double amx = to_double(amax, N);
      bool ok = isfinite(amx);
      double sumsq = 0.0;
      for (int e = 0; e < nn && ok; ++e) {
        const double v = to_double(mpd::mp_load(el(D, e), N), N);
        if (!isfinite(v) || fabs(v) > 1e150) ok = false;
        sumsq = __dadd_rn(sumsq, __dmul_rn(v, v));
        a[e] = v;
      }
      double gamma = 0.0;
      if (ok) ok = min_eigenvalue_f64(a, n, a + nn, a + nn + n, &gamma);
      if (ok) {
        const double bound = __dmul_rn(__dmul_rn(__dmul_rn(2.0, (double)(n + 1) * (double)(n + 1)), DBL_EPSILON),
                                       __dsqrt_rn(sumsq));
        const double floor = (amx > 0.0 && isfinite(amx)) ? __ddiv_rn(1.0, amx) : 0.0;
        s_gamma = gamma;
        if (bound <= __dmul_rn(1e-10, fmax(fabs(gamma), floor))) {
          s_mode = 0;
        } else {
          s_mode = 1;
          Val alc = amax;
          if (gamma < 0.0 && __ddiv_rn(-1.0, gamma) < amx)
            alc = mpd::from_double(__ddiv_rn(-__dsub_rn(1.0, 1e-10), gamma), 0, N);
          mpd::mp_store(s_alc, N, alc, status);
        }
      }
    }
  }
  __syncthreads();
  if (s_mode == 1) {  // admits: exact-dot Cholesky of alpha_c Delta + I (symmetric: the lower factor)
    const Val alc = mpd::mp_load(s_alc, N);
    Val one = mpd::mp_zero();
    one.zero = false;
    one.m[N - 1] = 1ull << 63;
    one.s = 1 - 64LL * N;
    for (int e = tid; e < nn; e += kStThreads) {
      Val v = mul(mpd::mp_load(el(D, e), N), alc, N);
      if (e % n == e / n) v = add(v, one, N);
      mpd::mp_store(el(C, e), N, v, status);
    }
    __syncthreads();
    for (int j = 0; j < n; ++j) {
      if (tid < 32) {  // warp 0 forms the pivot's dot, its lane 0 the rest
        bool ok = true;
        const Val dot = mpd::mp_dot_sub_warp(nullptr, el(C, j), n, el(C, j), n, j, N, &ok);
        if (tid == 0) {
          const Val d = sub(mpd::mp_load(el(C, j + (long)j * n), N), dot, N);
          if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
          if (d.zero || d.neg) {
            s_fail = 1;
          } else {
            const Val r = mpd::mp_sqrt(d, N);
            mpd::mp_store(el(C, j + (long)j * n), N, r, status);
            mpd::mp_store(s_piv, N, r, status);
          }
        }
      }
      __syncthreads();
      if (s_fail) break;
      const Val r = mpd::mp_load(s_piv, N);
      for (int i = j + 1 + tid; i < n; i += kStThreads) {
        bool ok = true;
        const Val dot = mpd::mp_dot_sub(nullptr, el(C, i), n, el(C, j), n, j, N, &ok);
        if (!ok) atomicOr(status, SDPXG_ST_EXACT_SPREAD);
        mpd::mp_store(el(C, i + (long)j * n), N,
                      mpd::mp_div(sub(mpd::mp_load(el(C, i + (long)j * n), N), dot, N), r, N), status);
      }
      __syncthreads();
    }
    __syncthreads();
    if (tid == 0) s_mode = s_fail ? 2 : 4;
    __syncthreads();
  }
  Val gamma = mpd::mp_zero();
  int pth = s_mode == 0 ? 0 : (s_mode == 4 ? 1 : 2);
  bool eig_ok = true;
  if (s_mode == 2) {  // the MpFloat eigensolver on a copy of Delta
    for (int e = tid; e < nn; e += kStThreads) mpd::mp_store(el(C, e), N, mpd::mp_load(el(D, e), N), status);
    __syncthreads();
    if (tid < 32) eig_ok = jacobi_min_eig(C, n, N, &gamma, status);
  }
  if (tid != 0) return;
  if (s_mode != 2) gamma = mpd::from_double(s_gamma, 0, N);
  Val al;
  if (!eig_ok) {
    al = mpd::mp_zero();
    pth = 3;
  } else if (!gamma.zero && gamma.neg) {
    Val ng = mpd::mp_recip(gamma, N);
    ng.neg = !ng.neg;
    al = mpd::mp_cmp(ng, amax, N) < 0 ? ng : amax;
  } else {
    al = amax;
  }
  mpd::mp_store(el(alpha, blockIdx.x), N, al, status);
  path[blockIdx.x] = pth;
}
// X_b = mat(d_b): full symmetric, off-diagonals times the working-precision 1/sqrt 2 (rounded).
__global__ void k_mp_smat_blocks(const MpStepBlock* __restrict__ blocks, int N, const unsigned char* __restrict__ d,
                                 const unsigned char* __restrict__ consts, unsigned char* __restrict__ X,
                                 uint32_t* __restrict__ status) {
  const MpStepBlock B = blocks[blockIdx.x];
  const int n = B.n;
  const long esz = 8L * N + 8;
  const Val frac = mpd::mp_load(consts, N);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e % n, c = e / n, lo = r < c ? r : c, hi = r < c ? c : r;
    Val v = mpd::mp_load(d + (B.svec + (long)hi * (hi + 1) / 2 + lo) * esz, N);
    if (r != c) v = mul(v, frac, N);
    mpd::mp_store(X + (B.mat + e) * esz, N, v, status);
  }
}

// The working-precision 1/sqrt 2 into consts[0] (sqrt(1/2) rounded once).
__global__ void k_mp_step_consts(int N, unsigned char* consts, uint32_t* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Val h = mpd::mp_zero();
  h.zero = false;
  h.m[N - 1] = 1ull << 63;
  h.s = -64LL * N;
  mpd::mp_store(consts, N, mpd::mp_sqrt(h, N), status);
}

}  // namespace

void mp_launch_step_smat(const MpStepBlock* blocks, int nblk, int N, const unsigned char* d, unsigned char* consts,
                         unsigned char* X, uint32_t* status, cudaStream_t st) {
  if (N < 1 || N > mpd::kMaxN) throw std::invalid_argument("MPFR step length: limbs must be in 1..8");
  if (nblk <= 0) return;
  ++g_launches, k_mp_step_consts<<<1, 32, 0, st>>>(N, consts, status);
  ++g_launches, k_mp_smat_blocks<<<nblk, 128, 0, st>>>(blocks, N, d, consts, X, status);
  check(cudaGetLastError(), "k_mp_smat_blocks");
}

void mp_launch_step_bound(const MpStepBlock* blocks, int nblk, int N, const unsigned char* Y,
                          const unsigned char* lisqrt, unsigned char* consts, unsigned char* work, double* fwork,
                          unsigned char* alpha, int* path, uint32_t* status, cudaStream_t st) {
  if (N < 1 || N > mpd::kMaxN) throw std::invalid_argument("MPFR step length: limbs must be in 1..8");
  if (nblk <= 0) return;
  ++g_launches, k_mp_step_bound<<<nblk, kStThreads, 0, st>>>(blocks, N, Y, lisqrt, consts, work, fwork, alpha, path,
                                                             status);
  check(cudaGetLastError(), "k_mp_step_bound");
}

}  // namespace sdpxg
