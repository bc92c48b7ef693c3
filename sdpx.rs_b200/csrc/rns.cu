// Exact products of MpFloat<N> matrices through a residue number system (RNS), on the GPU.
//
// Restates the contract of the reference's RNS BLAS (crates/solver/src/algebra/dense/blas/
// rns_blas.rs:2134-2417 gemm): every entry of C = op(A) op(B) is the exact dot product rounded
// once to 64N bits, ties to even -- bit-identical to MpFloat::dot_fma (exactdot.rs:53-70).
//
// Two forms of the same product, bitwise equal (correct rounding has one answer):
//
// INT8 tensor-core form (the default, RNS_FORM_INT8):
//   k_rns_scan       per row of op(A) / column of op(B): lowest set-bit exponent lo and the
//                    width `bits` of the aligned integers (rns_blas.rs:2164-2183 alignment)
//   k_rns_pow2       2^s mod p for every prime and every bit position an entry can reach
//   k_rns8_residues  every entry as the integer M * 2^(e - 64N - lo) reduced to symmetric
//                    residues modulo L primes below 2^15, each split into two signed-byte
//                    digits r = lo + 256 hi, written as K-major byte planes
//                    (rns_blas.rs:929-986 panel residues)
//   k_i8_mod_gemm    per prime, the four digit products on tcgen05.mma kind::i8 with INT32
//                    accumulators in TMEM, recombined and reduced modulo the prime in the
//                    epilogue; K beyond 2^16 in chunks whose residues are added
//                    (rns_blas.rs:447-580 per-prime integer products)
//   k_rns_crt        Garner's mixed-radix CRT back to the signed integer, then one rounding to
//                    64N bits, ties to even (rns_blas.rs:1873-2125 CRT and pack,
//                    exactdot.rs:1316-1392 from_scaled_integer)
// FP64 form (RNS_FORM_FP64, the plain form on CUDA cores):
//   k_rns_residues   residues modulo primes below 2^21 as doubles
//   k_rns_gemm       one exact FP64 product per prime: symmetric residues keep |r| < 2^20, so
//                    8192 products sum exactly below 2^53; partial sums are reduced modulo the
//                    prime every 8192 terms
//   k_rns_crt        as above.
// The number of primes L follows the needed width 2*(64N) + spreads + log2(k) + 2 bits, the
// same bound as the reference's Plan (rns_blas.rs:2202-2208); the reference's own primes are
// 18-26 bits wide, the INT8 form uses 15-bit primes so that a residue is two signed bytes.
//
// Element layout (the reference's in-memory MpFloat<N>, arithmetic/src/lib.rs:333-340):
//   u64 limbs[N] (least significant first), i32 kind (sign * MPFR kind: 2 zero, 3 regular),
//   i32 exponent; a regular value is M * 2^(exponent - 64N) with the top bit of M set.
#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/sdpx_b200.h"
#include "engine.cuh"
#include "i8_gemm.cuh"
#include "mp_ldl.cuh"

using namespace sdpxg;

namespace sdpxg {
extern thread_local std::string g_last_error;
Engine* ctx_engine_any(sdpxg_ctx* c);
std::shared_ptr<void>* ctx_rns_slot(sdpxg_ctx* c);
}  // namespace sdpxg

#define RNS_MAXN 16    // limbs: up to 1024-bit values
#define RNS_MAXL 256   // primes (products of four 768-bit factors need about 220 of 15 bits)
#define RNS_MAXW 64    // 64-bit words of the reconstructed integer
#define RNS_KC 8192    // exact FP64 terms between two reductions modulo the prime
#define MP_ZERO 2
#define MP_REGULAR 3
#define MP_EXP_MAX ((1 << 30) - 1)

namespace {

__device__ __forceinline__ int elem_kind(const unsigned char* p, int N) {
  return *reinterpret_cast<const int*>(p + 8 * N);
}
__device__ __forceinline__ int elem_exp(const unsigned char* p, int N) {
  return *reinterpret_cast<const int*>(p + 8 * N + 4);
}

// x mod p by Barrett reduction, mu = floor((2^64 - 1) / p): the quotient estimate umulhi(x, mu)
// is at most two below floor(x / p), so two conditional subtractions finish; integer operations
// only (no conversions to and from FP64).
__device__ __forceinline__ uint32_t modb(unsigned long long x, uint32_t p, unsigned long long mu) {
  unsigned long long r = x - __umul64hi(x, mu) * p;
  if (r >= p) r -= p;
  if (r >= p) r -= p;
  return (uint32_t)r;
}

__device__ __forceinline__ uint32_t pow2mod(long long s, uint32_t p) {
  unsigned long long r = 1, b = 2 % p;
  while (s > 0) {
    if (s & 1) r = r * b % p;
    b = b * b % p;
    s >>= 1;
  }
  return (uint32_t)r;
}

}  // namespace

// Scan lines of a matrix view: element (x, y) at index x * sx + y * sy.
// lo[x] = min over regular entries of (exponent - 64N), bits[x] = max exponent - lo[x].
extern "C" __global__ void k_rns_scan(const unsigned char* __restrict__ X, int N, int nlines,
                                      int len, long sx, long sy, int* __restrict__ lo,
                                      int* __restrict__ bits, int* __restrict__ maxbits,
                                      uint32_t* __restrict__ status) {
  const int x = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (x >= nlines) return;
  const long esz = 8L * N + 8;
  const int p = 64 * N;
  int mn = INT_MAX, mx = INT_MIN;
  bool bad = false;
  for (int y = lane; y < len; y += 32) {
    const unsigned char* e = X + (x * sx + y * sy) * esz;
    int kind = abs(elem_kind(e, N));
    if (kind == MP_REGULAR) {
      int ex = elem_exp(e, N);
      mn = min(mn, ex - p);
      mx = max(mx, ex);
    } else if (kind != MP_ZERO) {
      bad = true;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0) {
    if (bad) atomicOr(status, SDPXG_ST_NONFINITE);
    if (mx == INT_MIN) {
      lo[x] = 0;
      bits[x] = 0;
    } else {
      lo[x] = mn;
      bits[x] = mx - mn;
      atomicMax(maxbits, mx - mn);
    }
  }
}

// Symmetric residues of every entry of a view for L primes: out[t * plane + x + y * ldx] when
// xmajor, else out[t * plane + y + x * ldy].
extern "C" __global__ void k_rns_residues(const unsigned char* __restrict__ X, int N, int nlines,
                                          int len, long sx, long sy, const int* __restrict__ lo,
                                          int L, const uint32_t* __restrict__ primes,
                                          const uint32_t* __restrict__ W, double* __restrict__ out,
                                          long plane, int xmajor) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)nlines * len) return;
  const int x = (int)(idx % nlines), y = (int)(idx / nlines);
  const long esz = 8L * N + 8;
  const unsigned char* e = X + (x * sx + y * sy) * esz;
  const long o = xmajor ? (x + (long)y * nlines) : (y + (long)x * len);
  const int kind = elem_kind(e, N);
  if (abs(kind) != MP_REGULAR) {
    for (int t = 0; t < L; ++t) out[t * plane + o] = 0.0;
    return;
  }
  const bool neg = kind < 0;
  const long long shift = (long long)elem_exp(e, N) - 64LL * N - lo[x];
  const unsigned long long* limbs = reinterpret_cast<const unsigned long long*>(e);
  for (int t = 0; t < L; ++t) {
    const uint32_t p = primes[t];
    unsigned long long r = 0;
    for (int q = 0; q < N; ++q) r = (r + (limbs[q] % p) * W[t * RNS_MAXN + q]) % p;
    r = r * pow2mod(shift, p) % p;
    long long s = (long long)r;
    if (s > (long long)(p / 2)) s -= p;
    if (neg) s = -s;
    out[t * plane + o] = (double)s;
  }
}

// Per-prime exact products: C_t = A_t B_t (m x n, inner k) with symmetric residues in FP64,
// reduced modulo p_t every RNS_KC terms.  grid (m/64, n/64, L), 256 threads, 4 x 4 per thread.
extern "C" __global__ void __launch_bounds__(256)
k_rns_gemm(const double* __restrict__ RA, const double* __restrict__ RB, double* __restrict__ RC,
           int m, int n, int k, const uint32_t* __restrict__ primes, long planeA, long planeB,
           long planeC, int upper_only) {
  __shared__ double As[32][65];  // [k][row]
  __shared__ double Bs[32][65];  // [k][col]
  const int t = blockIdx.z;
  const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
  if (upper_only && i0 > j0 + 63) return;
  const double p = (double)primes[t];
  const double* A = RA + t * planeA;
  const double* B = RB + t * planeB;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  int since = 0;
  for (int k0 = 0; k0 < k; k0 += 32) {
    __syncthreads();
    for (int e = threadIdx.x; e < 64 * 32; e += 256) {
      int r = e % 64, c = e / 64;  // A: row r of the tile, k offset c
      As[c][r] = (i0 + r < m && k0 + c < k) ? A[(i0 + r) + (long)(k0 + c) * m] : 0.0;
      int kr = e % 32, cc = e / 32;  // B: k offset kr, column cc of the tile
      Bs[kr][cc] = (k0 + kr < k && j0 + cc < n) ? B[(k0 + kr) + (long)(j0 + cc) * k] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < 32; ++kk) {
      double x[4], y[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) x[a] = As[kk][tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) y[b] = Bs[kk][ty + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
    }
    since += 32;
    if (since >= RNS_KC) {  // keep every partial sum exact: reduce modulo p
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] -= p * rint(acc[a][b] / p);
      since = 0;
    }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      int i = i0 + tx + 16 * a, j = j0 + ty + 16 * b;
      if (i < m && j < n) RC[t * planeC + i + (long)j * m] = acc[a][b] - p * rint(acc[a][b] / p);
    }
}

// 2^s mod p_t for s < S (row t of the table).
extern "C" __global__ void k_rns_pow2(int L, const int* __restrict__ primes, int S, uint32_t* __restrict__ out) {
  const int t = blockIdx.y, s = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L || s >= S) return;
  out[(size_t)t * S + s] = pow2mod(s, (uint32_t)primes[t]);
}

// (M 2^shift) mod p for the mantissa M = sum_q limbs[q] 2^(64q): Horner over the limbs with
// 2^32 and 2^64 mod p from the power table's row (row[s] = 2^s mod p, s < S, S > 64), each
// step one Barrett reduction, then one product with row[shift].
__device__ __forceinline__ uint32_t residue_of(const unsigned long long* limbs, int N, const uint32_t* row,
                                               int shift, uint32_t p, unsigned long long mu) {
  const unsigned long long c32 = row[32], c64 = row[64];
  unsigned long long r = 0;
#pragma unroll
  for (int q = RNS_MAXN - 1; q >= 0; --q) {
    if (q < N) {
      const unsigned long long v = limbs[q];
      const unsigned long long lm = modb((v >> 32) * c32 + (v & 0xFFFFFFFFull), p, mu);
      r = modb(r * c64 + lm, p, mu);
    }
  }
  return modb(r * row[shift], p, mu);
}

// INT8 form: symmetric residues modulo L primes below 2^15 of every entry of a view, each split
// into signed-byte digits r = lo + 256 hi (|hi| <= 64), written to K-major byte planes: digit d
// of prime t for line x (a row of op(A) or a column of op(B)) and inner index y at
// out[((2t + d) * Rpad + x) * Kld + y].  Lines >= nlines and y >= len (the padding) get zeros.
// One thread per (x, y), y fastest: the plane writes are coalesced.  The residue of
// M * 2^shift is (M mod p)(2^shift mod p) mod p, M mod p by Horner over the 64-bit limbs
// (residue_of: three power-table reads per prime).
extern "C" __global__ void k_rns8_residues(const unsigned char* __restrict__ X, int N, int nlines, int len,
                                           long sx, long sy, const int* __restrict__ lo, int L,
                                           const int* __restrict__ primes, const unsigned long long* __restrict__ mu,
                                           const uint32_t* __restrict__ pow2, int S, int8_t* __restrict__ out,
                                           int Rpad, int Kld) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)Rpad * Kld) return;
  const int y = (int)(idx % Kld), x = (int)(idx / Kld);
  const size_t plane = (size_t)Rpad * Kld;
  int8_t* o = out + (size_t)x * Kld + y;
  bool live = x < nlines && y < len;
  bool neg = false;
  int shift = 0;
  unsigned long long limbs[RNS_MAXN];
  if (live) {
    const unsigned char* e = X + ((long)x * sx + (long)y * sy) * (8L * N + 8);
    const int kind = elem_kind(e, N);
    live = abs(kind) == MP_REGULAR;
    if (live) {
      neg = kind < 0;
      shift = elem_exp(e, N) - 64 * N - lo[x];
      const unsigned long long* lp = reinterpret_cast<const unsigned long long*>(e);
#pragma unroll
      for (int q = 0; q < RNS_MAXN; ++q) limbs[q] = q < N ? lp[q] : 0ull;
    }
  }
  for (int t = 0; t < L; ++t) {
    int dlo = 0, dhi = 0;
    if (live) {
      const int p = primes[t];
      int r = (int)residue_of(limbs, N, pow2 + (size_t)t * S, shift, (uint32_t)p, mu[t]);
      if (r > p / 2) r -= p;
      if (neg) r = -r;
      dlo = ((r + 128) & 255) - 128;
      dhi = (r - dlo) >> 8;
    }
    o[(size_t)(2 * t) * plane] = (int8_t)dlo;
    o[(size_t)(2 * t + 1) * plane] = (int8_t)dhi;
  }
}

// Residues of an intermediate product (INT8 form, values in [0, p) as written by the modular
// GEMM: RC[t * plane + j * inner + r]) re-split into signed-byte digit planes for the next
// product: line j, inner index r at out[((2t + d) * Rpad + j) * Kld + r]; padding zeros.
extern "C" __global__ void k_rns8_replane(const int* __restrict__ RC, long plane, int lines, int inner, int L,
                                          const int* __restrict__ primes, int8_t* __restrict__ out, int Rpad,
                                          int Kld) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)Rpad * Kld) return;
  const int r = (int)(idx % Kld), j = (int)(idx / Kld);
  const size_t pl = (size_t)Rpad * Kld;
  int8_t* o = out + (size_t)j * Kld + r;
  const bool live = j < lines && r < inner;
  for (int t = 0; t < L; ++t) {
    int dlo = 0, dhi = 0;
    if (live) {
      const int p = primes[t];
      int v = RC[t * plane + (long)j * inner + r];
      if (v > p / 2) v -= p;
      dlo = ((v + 128) & 255) - 128;
      dhi = (v - dlo) >> 8;
    }
    o[(size_t)(2 * t) * pl] = (int8_t)dlo;
    o[(size_t)(2 * t + 1) * pl] = (int8_t)dhi;
  }
}

// out[i] = a[i] + c (exponent offsets of the congruence's second factor).
extern "C" __global__ void k_add_const_int(const int* __restrict__ a, int n, int c, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + c;
}
extern "C" __global__ void k_fill_int(int* __restrict__ a, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// Word w of S (WM words kept in registers: an unrolled select instead of a dynamic index).
template <int WM>
__device__ __forceinline__ unsigned long long word_at(const unsigned long long (&S)[WM], int w) {
  unsigned long long v = 0ull;
#pragma unroll
  for (int k = 0; k < WM; ++k) v = (k == w) ? S[k] : v;
  return v;
}

// CRT of the L residues of every output, then one rounding to 64N bits (ties to even).
// Residues are read as R (double: the FP64 form's exact integers, possibly negative; int: the
// INT8 form's residues in [0, p)).  With M = prod p_t, M_t = M / p_t and w_t = M_t^-1 mod p_t:
// c_t = r_t w_t mod p_t, S = sum_t c_t M_t (exact, WW words), f = sum_t c_t / p_t in FP64, and
// the signed integer is X = S - rint(f) M.  The prime set covers more than twice the largest |X|
// plus a margin (|X| < M / 4), so S / M = f sits within 1/4 of an integer and FP64's error
// (below L^2 2^-53) cannot move rint(f); X is then exact.  L products of a table row with one
// small factor per output, instead of Garner's L^2 / 2 modular steps.  S lives in registers: the
// kernel is instantiated for the smallest word count WM >= WW (launch_crt).
template <typename R, int WM>
__global__ void __launch_bounds__(128) k_rns_crt(const R* __restrict__ RC, long planeC, int m, int n, int L, int WW,
                                                 const uint32_t* __restrict__ primes,
                                                 const uint32_t* __restrict__ wt, const double* __restrict__ pinv,
                                                 const unsigned long long* __restrict__ mu,
                                                 const unsigned long long* __restrict__ MT,
                                                 const unsigned long long* __restrict__ Mbig,
                                                 const int* __restrict__ loA, const int* __restrict__ loB, int N,
                                                 int upper_only, unsigned char* __restrict__ C,
                                                 uint32_t* __restrict__ status) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)m * n) return;
  const int i = (int)(idx % m), j = (int)(idx / m);
  unsigned char* out = C + idx * (8L * N + 8);
  unsigned long long* ol = reinterpret_cast<unsigned long long*>(out);
  int* okind = reinterpret_cast<int*>(out + 8 * N);
  int* oexp = okind + 1;
  auto write_zero = [&]() {
    for (int q = 0; q < N; ++q) ol[q] = 0;
    *okind = MP_ZERO;
    *oexp = 0;
  };
  if (upper_only && i > j) {
    write_zero();
    return;
  }
  // S accumulates in 32-bit digits, one 64-bit accumulator each (c < 2^21 times a 32-bit digit
  // is below 2^53, so up to 2^11 primes sum without overflow), carried once after the loop
  unsigned long long acc[2 * WM];
#pragma unroll
  for (int w = 0; w < 2 * WM; ++w) acc[w] = 0ull;
  double f = 0.0;
  for (int t = 0; t < L; ++t) {
    const uint32_t p = primes[t];
    const double pi = pinv[t];
    long long r = (long long)RC[t * planeC + idx];
    if (!std::is_same<R, int>::value) {  // the FP64 form's exact integers (|r| < 2^53, any sign)
      r -= (long long)floor((double)r * pi) * (long long)p;  // within one multiple of p
      if (r < 0) r += p;
      if (r >= (long long)p) r -= p;
    }  // the INT8 form's residues are in [0, p) already
    const unsigned long long c = modb((unsigned long long)r * wt[t], p, mu[t]);
    f += (double)c * pi;
    const uint32_t* row = reinterpret_cast<const uint32_t*>(MT + (size_t)t * WW);  // 32-bit digits of M_t
#pragma unroll
    for (int w = 0; w < 2 * WM; ++w)  // S += c * M_t
      if (w < 2 * WW) acc[w] += c * (unsigned long long)row[w];
  }
  unsigned long long S[WM];
  {
    unsigned long long carry = 0;
#pragma unroll
    for (int w = 0; w < WM; ++w) {
      S[w] = 0ull;
      if (w < WW) {
        const unsigned long long lo = acc[2 * w] + carry;
        const unsigned long long hi = acc[2 * w + 1] + (lo >> 32);
        carry = hi >> 32;
        S[w] = (hi << 32) | (lo & 0xFFFFFFFFull);
      }
    }
  }
  // S -= k M (two's complement over WW words; |X| < M / 4 fits with room for the sign)
  const unsigned long long k = (unsigned long long)rint(f);
  {
    unsigned long long carry = 0, borrow = 0;
#pragma unroll
    for (int w = 0; w < WM; ++w) {
      if (w < WW) {
        const unsigned long long lo = Mbig[w] * k, hi = __umul64hi(Mbig[w], k);
        const unsigned long long km = lo + carry;
        carry = hi + (km < lo);
        const unsigned long long d1 = S[w] - km;
        const unsigned long long b1 = S[w] < km;
        const unsigned long long d2 = d1 - borrow;
        const unsigned long long b2 = d1 < borrow;
        S[w] = d2;
        borrow = b1 + b2;
      }
    }
  }
  const bool neg = (word_at(S, WW - 1) >> 63) != 0;
  if (neg) {  // magnitude
    unsigned long long cy = 1;
#pragma unroll
    for (int w = 0; w < WM; ++w) {
      if (w < WW) {
        S[w] = ~S[w] + cy;
        cy = (cy && S[w] == 0) ? 1ull : 0ull;
      }
    }
  }
  int top = -1;
#pragma unroll
  for (int w = WM - 1; w >= 0; --w)
    if (top < 0 && w < WW && S[w]) top = w;
  if (top < 0) {
    write_zero();
    return;
  }
  const int bitlen = top * 64 + 64 - __clzll(word_at(S, top));
  const int pbits = 64 * N;
  int shift = bitlen - pbits;
  auto window = [&](int start) -> unsigned long long {  // bits [start, start + 64) of S
    const int word = (start >= 0) ? start / 64 : -((-start + 63) / 64);
    const int off = start - 64 * word;
    const unsigned long long lo = word_at(S, word), hi = word_at(S, word + 1);
    return (lo >> off) | (off ? (hi << (64 - off)) : 0ull);
  };
  unsigned long long res[RNS_MAXN];
#pragma unroll
  for (int q = 0; q < RNS_MAXN; ++q) res[q] = q < N ? window(shift + 64 * q) : 0ull;
  if (shift > 0) {
    const int rb = shift - 1;
    const bool round_bit = (word_at(S, rb / 64) >> (rb % 64)) & 1ull;
    bool sticky = false;
#pragma unroll
    for (int w = 0; w < WM; ++w) sticky = sticky || (w < rb / 64 && S[w] != 0);
    if (rb % 64) sticky = sticky || ((word_at(S, rb / 64) & ((1ull << (rb % 64)) - 1)) != 0);
    if (round_bit && (sticky || (res[0] & 1ull))) {
      bool carry = true;
#pragma unroll
      for (int q = 0; q < RNS_MAXN; ++q) {
        if (q < N && carry) {
          res[q] += 1;
          carry = (res[q] == 0);
        }
      }
      if (carry) {
#pragma unroll
        for (int q = 0; q < RNS_MAXN; ++q)
          if (q == N - 1) res[q] = 1ull << 63;
        shift += 1;
      }
    }
  }
  const long long exponent = (long long)loA[i] + loB[j] + shift + pbits;
  if (exponent > MP_EXP_MAX || exponent < -MP_EXP_MAX) {
    atomicOr(status, SDPXG_ST_NONFINITE);
    write_zero();
    return;
  }
#pragma unroll
  for (int q = 0; q < RNS_MAXN; ++q)
    if (q < N) ol[q] = res[q];
  *okind = neg ? -MP_REGULAR : MP_REGULAR;
  *oexp = (int)exponent;
}

// The CRT kernel for WW words, instantiated with the smallest register width that holds them.
template <typename R>
void launch_crt(unsigned blocks, cudaStream_t st, const R* RC, long planeC, int m, int n, int L, int WW,
                const uint32_t* primes, const uint32_t* wt, const double* pinv, const unsigned long long* mu,
                const unsigned long long* MT,
                const unsigned long long* Mbig, const int* loA, const int* loB, int N, int upper_only,
                unsigned char* C, uint32_t* status) {
  if (WW <= 8)
    k_rns_crt<R, 8><<<blocks, 128, 0, st>>>(RC, planeC, m, n, L, WW, primes, wt, pinv, mu, MT, Mbig, loA, loB, N,
                                            upper_only, C, status);
  else if (WW <= 16)
    k_rns_crt<R, 16><<<blocks, 128, 0, st>>>(RC, planeC, m, n, L, WW, primes, wt, pinv, mu, MT, Mbig, loA, loB, N,
                                             upper_only, C, status);
  else if (WW <= 32)
    k_rns_crt<R, 32><<<blocks, 128, 0, st>>>(RC, planeC, m, n, L, WW, primes, wt, pinv, mu, MT, Mbig, loA, loB, N,
                                             upper_only, C, status);
  else
    k_rns_crt<R, RNS_MAXW><<<blocks, 128, 0, st>>>(RC, planeC, m, n, L, WW, primes, wt, pinv, mu, MT, Mbig, loA, loB,
                                                   N, upper_only, C, status);
}

// ---- exact forms of small factors (rns_blas.rs:2990-3194 diag_congruence, 4025-4174
// svec_quadratic, 4175-4277 symmetric_bilinear) ----
// Residues in [0, p_t) of a flat array of MpFloat<N> aligned at one exponent lo (the class's
// lowest set bit): entry e is (-1)^s M_e 2^(exp_e - 64N - lo); out[t * count + e].  absval drops
// the signs.  The residue is computed as in k_rns8_residues (residue_of).
extern "C" __global__ void k_rns_class_residues(const unsigned char* __restrict__ X, int N, int count, int lo,
                                                int absval, int L, const int* __restrict__ primes,
                                                const unsigned long long* __restrict__ mu,
                                                const uint32_t* __restrict__ pow2, int S, int* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const unsigned char* x = X + (size_t)e * (8 * N + 8);
  const int kind = elem_kind(x, N);
  if (abs(kind) != MP_REGULAR) {
    for (int t = 0; t < L; ++t) out[(size_t)t * count + e] = 0;
    return;
  }
  const bool neg = kind < 0 && !absval;
  const int shift = elem_exp(x, N) - 64 * N - lo;
  const unsigned long long* lp = reinterpret_cast<const unsigned long long*>(x);
  unsigned long long limbs[RNS_MAXN];
#pragma unroll
  for (int q = 0; q < RNS_MAXN; ++q) limbs[q] = q < N ? lp[q] : 0ull;
  for (int t = 0; t < L; ++t) {
    const int p = primes[t];
    int r = (int)residue_of(limbs, N, pow2 + (size_t)t * S, shift, (uint32_t)p, mu[t]);
    if (neg && r) r = p - r;
    out[(size_t)t * count + e] = r;
  }
}

// Right operand of the diagonal congruence: digit planes of (r_t(line j, inner r) * d_t(r)) mod
// p_t, symmetric, from the left operand's digit planes (the same layout as k_rns8_residues) and
// the residues of d (k entries per prime, in [0, p)).  Padding stays zero.
extern "C" __global__ void k_rns8_scale_planes(const int8_t* __restrict__ in, const int* __restrict__ dres, int k,
                                               int L, const int* __restrict__ primes, int8_t* __restrict__ out,
                                               int Rpad, int Kld) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)Rpad * Kld) return;
  const int r = (int)(idx % Kld);
  const size_t pl = (size_t)Rpad * Kld;
  for (int t = 0; t < L; ++t) {
    int dlo = 0, dhi = 0;
    if (r < k) {
      const int p = primes[t];
      const long long v = (long long)in[(size_t)(2 * t) * pl + idx] + 256LL * in[(size_t)(2 * t + 1) * pl + idx];
      long long w = v * dres[(size_t)t * k + r] % p;
      if (w < 0) w += p;
      int sv = (int)w;
      if (sv > p / 2) sv -= p;
      dlo = ((sv + 128) & 255) - 128;
      dhi = (sv - dlo) >> 8;
    }
    out[(size_t)(2 * t) * pl + idx] = (int8_t)dlo;
    out[(size_t)(2 * t + 1) * pl + idx] = (int8_t)dhi;
  }
}

// svec_quadratic residues: out[t * kmax + k] = sum_{i <= j} c_ij x_tri(j)+i q_ik q_jk mod p_t,
// c_ii = c[0] (the value 1), c_ij = c[1] (the working-precision sqrt 2).  One thread per (k, t).
extern "C" __global__ void k_rns_svec_quadratic(int h, int kmax, const int* __restrict__ xr, const int* __restrict__ qr,
                                                const int* __restrict__ cr, int L, const int* __restrict__ primes,
                                                int* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x, t = blockIdx.y;
  if (k >= kmax || t >= L) return;
  const unsigned long long p = (unsigned)primes[t];
  const int tri = h * (h + 1) / 2;
  const int* x = xr + (size_t)t * tri;
  const int* q = qr + (size_t)t * h * kmax + (size_t)k * h;
  const unsigned long long c0 = (unsigned)cr[2 * t], c1 = (unsigned)cr[2 * t + 1];
  unsigned long long acc = 0;  // terms below 2^15 each
  for (int j = 0; j < h; ++j) {
    const unsigned long long qj = (unsigned)q[j];
    unsigned long long row = 0;  // sum_{i < j} x_ij q_i, terms below 2^30
    for (int i = 0; i < j; ++i) row += (unsigned long long)(unsigned)x[j * (j + 1) / 2 + i] * (unsigned)q[i];
    row %= p;
    acc += (row * c1 % p) * qj % p;
    acc += ((unsigned long long)(unsigned)x[j * (j + 1) / 2 + j] * qj % p) * qj % p * c0 % p;
  }
  out[(size_t)t * kmax + k] = (int)(acc % p);
}

// symmetric_bilinear residues: out[t * np + s] = q_a' X q_b mod p_t for pair s = (a, b), X
// symmetric from its packed upper triangle (entry (i, j), i <= j, at tri(j) + i).
extern "C" __global__ void k_rns_bilinear(int h, int cols, const int* __restrict__ xr, const int* __restrict__ qr,
                                          const unsigned long long* __restrict__ pairs, int np, int L,
                                          const int* __restrict__ primes, int* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x, t = blockIdx.y;
  if (s >= np || t >= L) return;
  const unsigned long long p = (unsigned)primes[t];
  const int tri = h * (h + 1) / 2;
  const int* x = xr + (size_t)t * tri;
  const int* qa = qr + (size_t)t * h * cols + (size_t)pairs[2 * s] * h;
  const int* qb = qr + (size_t)t * h * cols + (size_t)pairs[2 * s + 1] * h;
  unsigned long long acc = 0;
  for (int j = 0; j < h; ++j) {
    unsigned long long u = 0;  // (X q_a)_j, terms below 2^30
    for (int i = 0; i < h; ++i) {
      const int lo = i < j ? i : j, hi = i < j ? j : i;
      u += (unsigned long long)(unsigned)x[hi * (hi + 1) / 2 + lo] * (unsigned)qa[i];
    }
    acc += (u % p) * (unsigned)qb[j] % p;
  }
  out[(size_t)t * np + s] = (int)(acc % p);
}

namespace {

// Host tables of one prime set (descending primes below 2^bits).
struct PrimeTables {
  int L = 0, WW = 0;
  std::vector<uint32_t> primes, W, wt;
  std::vector<double> pinv;
  std::vector<unsigned long long> mu;  // floor((2^64 - 1) / p_t), the Barrett constants
  std::vector<unsigned long long> M, MT;  // M = prod p_t; MT row t = M / p_t (WW words each)
};

// The largest RNS_MAXL primes below 2^bits, descending.
const std::vector<uint32_t>& prime_list(int bits) {
  static std::vector<uint32_t> ps21, ps15;
  static std::once_flag once21, once15;
  auto make = [](std::vector<uint32_t>& ps, int b) {
    const uint32_t top = 1u << b;
    std::vector<bool> comp(top, false);
    for (uint32_t i = 2; (uint64_t)i * i < top; ++i)
      if (!comp[i])
        for (uint32_t j = i * i; j < top; j += i) comp[j] = true;
    for (uint32_t q = top - 1; q > 2 && ps.size() < RNS_MAXL; --q)
      if (!comp[q]) ps.push_back(q);
  };
  if (bits == 15) {
    std::call_once(once15, [&] { make(ps15, 15); });
    return ps15;
  }
  std::call_once(once21, [&] { make(ps21, 21); });
  return ps21;
}

uint64_t powmod64(uint64_t b, uint64_t e, uint64_t p) {
  uint64_t r = 1 % p;
  b %= p;
  while (e) {
    if (e & 1) r = (unsigned __int128)r * b % p;
    b = (unsigned __int128)b * b % p;
    e >>= 1;
  }
  return r;
}

PrimeTables make_tables(const std::vector<uint32_t>& ps, int L) {
  PrimeTables T;
  T.L = L;
  T.primes.assign(ps.begin(), ps.begin() + L);
  T.W.assign((size_t)L * RNS_MAXN, 0);
  for (int t = 0; t < L; ++t)
    for (int q = 0; q < RNS_MAXN; ++q) T.W[t * RNS_MAXN + q] = (uint32_t)powmod64(2, 64ull * q, T.primes[t]);
  // M = prod p_t (WW words with room above it), M_t = M / p_t, w_t = M_t^-1 mod p_t
  double log2m = 0;
  for (uint32_t p : T.primes) log2m += std::log2((double)p);
  T.WW = std::min(RNS_MAXW, (int)(log2m / 64) + 2);
  auto mul_small = [&](std::vector<unsigned long long>& x, uint64_t p) {
    unsigned __int128 carry = 0;
    for (int w = 0; w < T.WW; ++w) {
      unsigned __int128 v = (unsigned __int128)x[w] * p + carry;
      x[w] = (unsigned long long)v;
      carry = v >> 64;
    }
  };
  T.M.assign(T.WW, 0);
  T.M[0] = 1;
  for (uint32_t p : T.primes) mul_small(T.M, p);
  T.MT.assign((size_t)L * T.WW, 0);
  T.wt.assign(L, 0);
  T.pinv.assign(L, 0.0);
  T.mu.assign(L, 0ull);
  for (int t = 0; t < L; ++t) {
    std::vector<unsigned long long> x(T.WW, 0);
    x[0] = 1;
    uint64_t rem = 1;  // M_t mod p_t
    const uint64_t p = T.primes[t];
    for (int s2 = 0; s2 < L; ++s2)
      if (s2 != t) {
        mul_small(x, T.primes[s2]);
        rem = rem * (T.primes[s2] % p) % p;
      }
    for (int w = 0; w < T.WW; ++w) T.MT[(size_t)t * T.WW + w] = x[w];
    T.wt[t] = (uint32_t)powmod64(rem, p - 2, p);
    T.pinv[t] = 1.0 / (double)p;
    T.mu[t] = ~0ull / p;
  }
  return T;
}

template <typename T>
void grow(DevBuf<T>& b, size_t n) {
  if (b.n < std::max<size_t>(n, 1)) b.alloc(std::max<size_t>(n, 1));
}

// Device copies of one prime set's tables (re-uploaded when L changes).
struct DevTables {
  DevBuf<uint32_t> primes, W, wt;
  DevBuf<double> pinv;
  DevBuf<unsigned long long> mu;
  DevBuf<int> iprimes;
  DevBuf<unsigned long long> M, MT;
  int L = -1;
  std::map<int, PrimeTables> host;
  const PrimeTables& get(int bits, int L_, cudaStream_t st) {
    auto it = host.find(L_);
    if (it == host.end()) it = host.emplace(L_, make_tables(prime_list(bits), L_)).first;
    const PrimeTables& T = it->second;
    if (L != L_) {
      grow(primes, L_); grow(W, T.W.size()); grow(wt, L_); grow(pinv, L_); grow(mu, L_);
      grow(iprimes, L_); grow(M, T.WW); grow(MT, T.MT.size());
      primes.upload(T.primes.data(), L_, st);
      W.upload(T.W.data(), T.W.size(), st);
      wt.upload(T.wt.data(), L_, st);
      pinv.upload(T.pinv.data(), L_, st);
      mu.upload(T.mu.data(), L_, st);
      std::vector<int> ip(T.primes.begin(), T.primes.end());
      iprimes.upload(ip.data(), L_, st);
      M.upload(T.M.data(), T.WW, st);
      MT.upload(T.MT.data(), T.MT.size(), st);
      L = L_;
    }
    return T;
  }
};

struct RnsWorkspace {
  DevBuf<unsigned char> a, b, c;  // staging of the host entry point
  DevBuf<int> loA, loB, bitsA, bitsB, maxbits, err;
  DevBuf<uint32_t> status, pow2;
  DevTables t21, t15;
  DevBuf<double> RA, RB, RC;  // FP64 form
  DevBuf<int8_t> PA, PB;      // INT8 form: digit planes
  DevBuf<int> RC8;            // INT8 form: residues of the product
  DevBuf<int> RT8, loX, bitsX, loB2;  // congruence: intermediate residues, X scan, column offsets
  DevBuf<int> cres, clo, cbits, cmax;   // exact forms: class residues, class scans
  DevBuf<unsigned char> zs, ys, fd;     // block products: stacked operands, staging
  DevBuf<long> boff;                    // block products: row, factor and column offsets
  DevBuf<int> bq;
  DevBuf<unsigned long long> bcols, bpairs;
  int form = 0;               // 0: INT8 tensor cores, 1: FP64
};

constexpr int kI8Chunk = 1 << 16;  // K per modular GEMM call (INT32 accumulators stay exact)

// The exact product on device buffers.  Returns 0, or 2 (non-finite operand, exponent spread
// too wide) with g_last_error set; *hs receives the device status word.
int32_t rns_product(RnsWorkspace& ws, cudaStream_t st, int form, int N, char ta, char tb, uint64_t m,
                    uint64_t n, uint64_t k, const unsigned char* dA, uint64_t lda, const unsigned char* dB,
                    uint64_t ldb, int upper_only, unsigned char* dC, uint32_t* hs_out) {
  grow(ws.loA, m); grow(ws.bitsA, m); grow(ws.loB, n); grow(ws.bitsB, n);
  grow(ws.maxbits, 2); grow(ws.status, 1); grow(ws.err, 1);
  check(cudaMemsetAsync(ws.maxbits.p, 0, 2 * sizeof(int), st), "memset");
  check(cudaMemsetAsync(ws.status.p, 0, sizeof(uint32_t), st), "memset");
  // op(A) rows: (i, l) -> i*sx + l*sy ; op(B) columns: (j, l) -> j*sx + l*sy
  const long asx = (ta == 'N') ? 1 : (long)lda, asy = (ta == 'N') ? (long)lda : 1;
  const long bsx = (tb == 'N') ? (long)ldb : 1, bsy = (tb == 'N') ? 1 : (long)ldb;
  if (k) {
    ++g_launches, k_rns_scan<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(dA, N, (int)m, (int)k, asx, asy, ws.loA,
                                                                   ws.bitsA, ws.maxbits, ws.status);
    ++g_launches, k_rns_scan<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(dB, N, (int)n, (int)k, bsx, bsy, ws.loB,
                                                                   ws.bitsB, ws.maxbits.p + 1, ws.status);
  } else {
    check(cudaMemsetAsync(ws.loA.p, 0, m * sizeof(int), st), "memset");
    check(cudaMemsetAsync(ws.loB.p, 0, n * sizeof(int), st), "memset");
  }
  int hb[2] = {0, 0};
  uint32_t hs = 0;
  copy_d2h(hb, ws.maxbits.p, 2 * sizeof(int), st);
  copy_d2h(&hs, ws.status.p, sizeof(uint32_t), st);
  check(cudaStreamSynchronize(st), "sync");
  if (hs) {
    if (hs_out) *hs_out = hs;
    g_last_error = "sdpxg_rns_gemm: non-finite operands are not supported";
    return 2;
  }
  // width of |sum| < k 2^(bitsA + bitsB); the CRT range must exceed twice that
  int lg = 0;
  while ((1ull << lg) < std::max<uint64_t>(k, 1)) ++lg;
  const double needed = (double)hb[0] + hb[1] + lg + 2;
  const int bits = form == 0 ? 15 : 21;
  const auto& ps = prime_list(bits);
  int L = 0;
  double acc = 0;
  while (L < RNS_MAXL && acc <= needed) acc += std::log2((double)ps[L++]);
  if (acc <= needed || (int)(acc / 64) + 2 > RNS_MAXW) {
    g_last_error = "sdpxg_rns_gemm: exponent spread too wide for the prime set";
    return 2;
  }
  DevTables& DT = form == 0 ? ws.t15 : ws.t21;
  const PrimeTables& T = DT.get(bits, L, st);
  const long planeC = (long)(m * n);
  if (form == 0) {
    const int Mpad = (int)((m + 127) / 128 * 128), Npad = (int)((n + 127) / 128 * 128);
    const int Kld = (int)((std::max<uint64_t>(k, 1) + 127) / 128 * 128);
    grow(ws.RC8, (size_t)L * planeC);
    if (k) {
      const int S = 64 * N + std::max(hb[0], hb[1]) + 1;
      grow(ws.pow2, (size_t)L * S);
      ++g_launches, k_rns_pow2<<<dim3((S + 255) / 256, L), 256, 0, st>>>(L, DT.iprimes, S, ws.pow2);
      grow(ws.PA, (size_t)L * 2 * Mpad * Kld);
      grow(ws.PB, (size_t)L * 2 * Npad * Kld);
      ++g_launches, k_rns8_residues<<<(unsigned)(((long)Mpad * Kld + 255) / 256), 256, 0, st>>>(
          dA, N, (int)m, (int)k, asx, asy, ws.loA, L, DT.iprimes, DT.mu, ws.pow2, S, ws.PA, Mpad, Kld);
      ++g_launches, k_rns8_residues<<<(unsigned)(((long)Npad * Kld + 255) / 256), 256, 0, st>>>(
          dB, N, (int)n, (int)k, bsx, bsy, ws.loB, L, DT.iprimes, DT.mu, ws.pow2, S, ws.PB, Npad, Kld);
      check(cudaMemsetAsync(ws.err.p, 0, sizeof(int), st), "memset");
      for (int k0 = 0; k0 < Kld; k0 += kI8Chunk) {
        I8GemmArgs ga;
        ga.Mpad = Mpad; ga.Npad = Npad; ga.Kld = Kld;
        ga.k0 = k0; ga.Kpad = std::min(kI8Chunk, Kld - k0);
        ga.m = (int)m; ga.n = (int)n; ga.L = L; ga.moduli = DT.iprimes;
        ga.upper_only = upper_only; ga.accumulate = k0 > 0; ga.out = ws.RC8.p; ga.plane = planeC;
        ga.err = ws.err.p;
        launch_i8_gemm(2, ws.PA, ws.PB, ga, st);
      }
    } else {
      check(cudaMemsetAsync(ws.RC8.p, 0, (size_t)L * planeC * sizeof(int), st), "memset");
    }
    ++g_launches, launch_crt<int>((unsigned)((m * n + 127) / 128), st, 
        ws.RC8, planeC, (int)m, (int)n, L, T.WW, DT.primes, DT.wt, DT.pinv, DT.mu, DT.MT, DT.M, ws.loA, ws.loB, N,
        upper_only ? 1 : 0, dC, ws.status);
  } else {
    const long planeA = (long)(m * std::max<uint64_t>(k, 1)), planeB = (long)(std::max<uint64_t>(k, 1) * n);
    grow(ws.RA, (size_t)L * planeA);
    grow(ws.RB, (size_t)L * planeB);
    grow(ws.RC, (size_t)L * planeC);
    if (k) {
      ++g_launches, k_rns_residues<<<(unsigned)((m * k + 255) / 256), 256, 0, st>>>(
          dA, N, (int)m, (int)k, asx, asy, ws.loA, L, DT.primes, DT.W, ws.RA, planeA, 1);
      ++g_launches, k_rns_residues<<<(unsigned)((n * k + 255) / 256), 256, 0, st>>>(
          dB, N, (int)n, (int)k, bsx, bsy, ws.loB, L, DT.primes, DT.W, ws.RB, planeB, 0);
      dim3 grid((unsigned)((m + 63) / 64), (unsigned)((n + 63) / 64), (unsigned)L);
      ++g_launches, k_rns_gemm<<<grid, 256, 0, st>>>(ws.RA, ws.RB, ws.RC, (int)m, (int)n, (int)k, DT.primes,
                                                     planeA, planeB, planeC, upper_only ? 1 : 0);
    } else {
      check(cudaMemsetAsync(ws.RC.p, 0, (size_t)L * planeC * sizeof(double), st), "memset");
    }
    ++g_launches, launch_crt<double>((unsigned)((m * n + 127) / 128), st, 
        ws.RC, planeC, (int)m, (int)n, L, T.WW, DT.primes, DT.wt, DT.pinv, DT.mu, DT.MT, DT.M, ws.loA, ws.loB, N,
        upper_only ? 1 : 0, dC, ws.status);
  }
  check(cudaGetLastError(), "rns launch");
  int herr = 0;
  copy_d2h(&hs, ws.status.p, sizeof(uint32_t), st);
  if (form == 0 && k) copy_d2h(&herr, ws.err.p, sizeof(int), st);
  check(cudaStreamSynchronize(st), "sync");
  if (herr) throw CudaError("modular INT8 GEMM: a bounded wait gave up");
  if (hs_out) *hs_out = hs;
  return 0;
}

// The exact congruence C = op(A) X op(A)' (INT8 form) on device buffers: op(A) m x k aligned per
// row (lo_i), X k x k aligned as one block (lo_x, so that its scale factors out of the sums),
// then per prime T = X A~' and C = A~ T on the tensor cores, and the CRT with the exponents
// lo_i + lo_j + lo_x.  Width: |C| < k^2 2^(2 max bits(A) + bits(X)), so the primes cover
// 2 bits(A) + bits(X) + 2 log2 k + 2 bits.  Returns 0 or 2 (non-finite, too wide).
int32_t rns_congruence(RnsWorkspace& ws, cudaStream_t st, int N, char ta, uint64_t m, uint64_t k,
                       const unsigned char* dA, uint64_t lda, const unsigned char* dX, uint64_t ldx, int upper_only,
                       unsigned char* dC, uint32_t* hs_out) {
  grow(ws.loA, m); grow(ws.bitsA, m); grow(ws.loX, k); grow(ws.bitsX, k); grow(ws.loB2, m);
  grow(ws.maxbits, 2); grow(ws.status, 1); grow(ws.err, 1);
  check(cudaMemsetAsync(ws.maxbits.p, 0, 2 * sizeof(int), st), "memset");
  check(cudaMemsetAsync(ws.status.p, 0, sizeof(uint32_t), st), "memset");
  const long asx = (ta == 'N') ? 1 : (long)lda, asy = (ta == 'N') ? (long)lda : 1;
  ++g_launches, k_rns_scan<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(dA, N, (int)m, (int)k, asx, asy, ws.loA,
                                                                 ws.bitsA, ws.maxbits, ws.status);
  // X by columns (line c: entries (r, c), r < k), combined on the host into one alignment
  ++g_launches, k_rns_scan<<<(unsigned)((k + 7) / 8), 256, 0, st>>>(dX, N, (int)k, (int)k, (long)ldx, 1, ws.loX,
                                                                 ws.bitsX, ws.maxbits.p + 1, ws.status);
  int hb[2] = {0, 0};
  uint32_t hs = 0;
  std::vector<int> hlo(k), hbits(k);
  copy_d2h(hb, ws.maxbits.p, 2 * sizeof(int), st);
  copy_d2h(&hs, ws.status.p, sizeof(uint32_t), st);
  copy_d2h(hlo.data(), ws.loX.p, k * sizeof(int), st);
  copy_d2h(hbits.data(), ws.bitsX.p, k * sizeof(int), st);
  check(cudaStreamSynchronize(st), "sync");
  if (hs) {
    if (hs_out) *hs_out = hs;
    g_last_error = "sdpxg_rns_congruence: non-finite operands are not supported";
    return 2;
  }
  // one alignment for the whole of X: lowest bit over all regular entries, and its width
  long long lo_x = LLONG_MAX, top_x = LLONG_MIN;
  for (uint64_t c = 0; c < k; ++c)
    if (hbits[c] > 0 || hlo[c] != 0) {  // a column with a regular entry (an all-zero one reports 0, 0)
      lo_x = std::min<long long>(lo_x, hlo[c]);
      top_x = std::max<long long>(top_x, (long long)hlo[c] + hbits[c]);
    }
  if (lo_x == LLONG_MAX) lo_x = top_x = 0;
  if (top_x - lo_x > (1 << 20)) {
    g_last_error = "sdpxg_rns_congruence: exponent spread too wide";
    return 2;
  }
  const int bits_x = (int)(top_x - lo_x);
  int lg = 0;
  while ((1ull << lg) < std::max<uint64_t>(k, 1)) ++lg;
  const double needed = 2.0 * hb[0] + bits_x + 2.0 * lg + 2;
  const auto& ps = prime_list(15);
  int L = 0;
  double acc = 0;
  while (L < RNS_MAXL && acc <= needed) acc += std::log2((double)ps[L++]);
  if (acc <= needed || (int)(acc / 64) + 2 > RNS_MAXW) {
    g_last_error = "sdpxg_rns_congruence: exponent spread too wide for the prime set";
    return 2;
  }
  DevTables& DT = ws.t15;
  const PrimeTables& T = DT.get(15, L, st);
  const int Mpad = (int)((m + 127) / 128 * 128), Kpad = (int)((k + 127) / 128 * 128);
  const long planeT = (long)(k * m), planeC = (long)(m * m);
  grow(ws.RT8, (size_t)L * planeT);
  grow(ws.RC8, (size_t)L * planeC);
  const int S = 64 * N + std::max(hb[0], bits_x) + 1;
  grow(ws.pow2, (size_t)L * S);
  ++g_launches, k_rns_pow2<<<dim3((S + 255) / 256, L), 256, 0, st>>>(L, DT.iprimes, S, ws.pow2);
  grow(ws.PA, (size_t)L * 2 * Mpad * Kpad);  // A~ (rows of op(A)), used by both products
  grow(ws.PB, (size_t)L * 2 * (size_t)std::max(Kpad, Mpad) * Kpad);
  ++g_launches, k_rns8_residues<<<(unsigned)(((long)Mpad * Kpad + 255) / 256), 256, 0, st>>>(
      dA, N, (int)m, (int)k, asx, asy, ws.loA, L, DT.iprimes, DT.mu, ws.pow2, S, ws.PA, Mpad, Kpad);
  ++g_launches, k_fill_int<<<(unsigned)((k + 255) / 256), 256, 0, st>>>(ws.loX, (int)k, (int)lo_x);
  // X~ by rows (line r: entries (r, c)): the left operand of T = X~ A~'
  ++g_launches, k_rns8_residues<<<(unsigned)(((long)Kpad * Kpad + 255) / 256), 256, 0, st>>>(
      dX, N, (int)k, (int)k, 1, (long)ldx, ws.loX, L, DT.iprimes, DT.mu, ws.pow2, S, ws.PB, Kpad, Kpad);
  check(cudaMemsetAsync(ws.err.p, 0, sizeof(int), st), "memset");
  for (int k0 = 0; k0 < Kpad; k0 += kI8Chunk) {  // T (k x m) = X~ A~'
    I8GemmArgs ga;
    ga.Mpad = Kpad; ga.Npad = Mpad; ga.Kld = Kpad; ga.k0 = k0; ga.Kpad = std::min(kI8Chunk, Kpad - k0);
    ga.m = (int)k; ga.n = (int)m; ga.L = L; ga.moduli = DT.iprimes; ga.accumulate = k0 > 0;
    ga.out = ws.RT8.p; ga.plane = planeT; ga.err = ws.err.p;
    launch_i8_gemm(2, ws.PB, ws.PA, ga, st);
  }
  // columns of T as the right operand of C = A~ T (line j, inner r)
  ++g_launches, k_rns8_replane<<<(unsigned)(((long)Mpad * Kpad + 255) / 256), 256, 0, st>>>(
      ws.RT8, planeT, (int)m, (int)k, L, DT.iprimes, ws.PB, Mpad, Kpad);
  for (int k0 = 0; k0 < Kpad; k0 += kI8Chunk) {  // C (m x m) = A~ T
    I8GemmArgs ga;
    ga.Mpad = Mpad; ga.Npad = Mpad; ga.Kld = Kpad; ga.k0 = k0; ga.Kpad = std::min(kI8Chunk, Kpad - k0);
    ga.m = (int)m; ga.n = (int)m; ga.L = L; ga.moduli = DT.iprimes; ga.upper_only = upper_only;
    ga.accumulate = k0 > 0; ga.out = ws.RC8.p; ga.plane = planeC; ga.err = ws.err.p;
    launch_i8_gemm(2, ws.PA, ws.PB, ga, st);
  }
  ++g_launches, k_add_const_int<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(ws.loA, (int)m, (int)lo_x, ws.loB2);
  ++g_launches, launch_crt<int>((unsigned)((m * m + 127) / 128), st, 
      ws.RC8, planeC, (int)m, (int)m, L, T.WW, DT.primes, DT.wt, DT.pinv, DT.mu, DT.MT, DT.M, ws.loA, ws.loB2, N,
      upper_only ? 1 : 0, dC, ws.status);
  check(cudaGetLastError(), "congruence launch");
  int herr = 0;
  copy_d2h(&hs, ws.status.p, sizeof(uint32_t), st);
  copy_d2h(&herr, ws.err.p, sizeof(int), st);
  check(cudaStreamSynchronize(st), "sync");
  if (herr) throw CudaError("modular INT8 GEMM: a bounded wait gave up");
  if (hs_out) *hs_out = hs;
  return 0;
}


// ---- exact forms of small factors: every output is one exact sum of products of MpFloat
// factors, rounded once.  Each operand is one class aligned at its lowest set bit, so a term's
// integer is the product of its factors' integers and every term of an output carries the same
// power of two; per prime the sums run on CUDA cores (the shapes are per-block sized), and the
// CRT rounds once. ----

// Scans of `n` flat arrays (one line each) into (lo, bits) on the host; returns false (status
// bits in *hs) when an operand is not finite.
bool scan_classes(RnsWorkspace& ws, cudaStream_t st, int N, const unsigned char* const* arr, const int* count, int n,
                  int* lo, int* bits, uint32_t* hs) {
  grow(ws.clo, n); grow(ws.cbits, n); grow(ws.cmax, n); grow(ws.status, 1);
  check(cudaMemsetAsync(ws.status.p, 0, sizeof(uint32_t), st), "memset");
  check(cudaMemsetAsync(ws.cmax.p, 0, n * sizeof(int), st), "memset");
  for (int c = 0; c < n; ++c)
    ++g_launches, k_rns_scan<<<1, 32, 0, st>>>(arr[c], N, 1, count[c], 0, 1, ws.clo.p + c, ws.cbits.p + c,
                                               ws.cmax.p + c, ws.status);
  copy_d2h(lo, ws.clo.p, n * sizeof(int), st);
  copy_d2h(bits, ws.cbits.p, n * sizeof(int), st);
  copy_d2h(hs, ws.status.p, sizeof(uint32_t), st);
  check(cudaStreamSynchronize(st), "sync");
  return *hs == 0;
}

// Primes (15 bits) covering `needed` bits, or 0 when the set is too small.
int primes_for(double needed) {
  const auto& ps = prime_list(15);
  int L = 0;
  double acc = 0;
  while (L < RNS_MAXL && acc <= needed) acc += std::log2((double)ps[L++]);
  if (acc <= needed || (int)(acc / 64) + 2 > RNS_MAXW) return 0;
  return L;
}

int ceil_log2(uint64_t v) {
  int lg = 0;
  while ((1ull << lg) < std::max<uint64_t>(v, 1)) ++lg;
  return lg;
}

// CRT of `count` outputs (residues ws.RC8[t * count + o]) at exponent `lo` into dOut.
void crt_vector(RnsWorkspace& ws, cudaStream_t st, DevTables& DT, const PrimeTables& T, int N, int L, int count,
                int lo, unsigned char* dOut) {
  grow(ws.loA, count); grow(ws.loB, 1);
  ++g_launches, k_fill_int<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(ws.loA, count, lo);
  ++g_launches, k_fill_int<<<1, 32, 0, st>>>(ws.loB, 1, 0);
  ++g_launches, launch_crt<int>((unsigned)((count + 127) / 128), st, 
      ws.RC8, count, count, 1, L, T.WW, DT.primes, DT.wt, DT.pinv, DT.mu, DT.MT, DT.M, ws.loA, ws.loB, N, 0, dOut,
      ws.status);
}

// The residue tables of the classes: class c's residues at ws.cres + off[c] * L (count[c] per prime).
void class_residues(RnsWorkspace& ws, cudaStream_t st, DevTables& DT, int N, int L, const unsigned char* const* arr,
                    const int* count, const int* lo, const int* absval, int n, int maxbits, size_t* off) {
  size_t total = 0;
  for (int c = 0; c < n; ++c) {
    off[c] = total;
    total += (size_t)std::max(count[c], 1);
  }
  grow(ws.cres, total * L);
  const int S = 64 * N + maxbits + 1;
  grow(ws.pow2, (size_t)L * S);
  ++g_launches, k_rns_pow2<<<dim3((S + 255) / 256, L), 256, 0, st>>>(L, DT.iprimes, S, ws.pow2);
  for (int c = 0; c < n; ++c)
    if (count[c])
      ++g_launches, k_rns_class_residues<<<(unsigned)((count[c] + 127) / 128), 128, 0, st>>>(
          arr[c], N, count[c], lo[c], absval[c], L, DT.iprimes, DT.mu, ws.pow2, S, ws.cres.p + off[c] * L);
}

// v[k] = sum_{i <= j} c_ij x_tri(j)+i q_ik q_jk (c_ii = 1, c_ij = sqrt2), k < kmax, each rounded
// once (rns_blas.rs:4025-4174 svec_quadratic).  dC2 holds the two coefficients (1, sqrt2).
int32_t rns_svec_quadratic(RnsWorkspace& ws, cudaStream_t st, int N, int h, int kmax, const unsigned char* dQ,
                           int abs_q, const unsigned char* dX, const unsigned char* dC2, unsigned char* dOut,
                           uint32_t* hs_out) {
  const int tri = h * (h + 1) / 2;
  const unsigned char* arr[3] = {dQ, dX, dC2};
  const int count[3] = {h * kmax, tri, 2};
  int lo[3], bits[3];
  uint32_t hs = 0;
  if (!scan_classes(ws, st, N, arr, count, 3, lo, bits, &hs)) {
    if (hs_out) *hs_out = hs;
    g_last_error = "sdpxg_rns_svec_quadratic: non-finite operands are not supported";
    return 2;
  }
  const int L = primes_for(2.0 * bits[0] + bits[1] + bits[2] + ceil_log2((uint64_t)tri) + 2);
  if (!L) {
    g_last_error = "sdpxg_rns_svec_quadratic: exponent spread too wide for the prime set";
    return 2;
  }
  DevTables& DT = ws.t15;
  const PrimeTables& T = DT.get(15, L, st);
  size_t off[3];
  const int absv[3] = {abs_q, 0, 0};
  class_residues(ws, st, DT, N, L, arr, count, lo, absv, 3, std::max(bits[0], std::max(bits[1], bits[2])), off);
  grow(ws.RC8, (size_t)L * kmax);
  ++g_launches, k_rns_svec_quadratic<<<dim3((unsigned)((kmax + 63) / 64), (unsigned)L), 64, 0, st>>>(
      h, kmax, ws.cres.p + off[1] * L, ws.cres.p + off[0] * L, ws.cres.p + off[2] * L, L, DT.iprimes, ws.RC8);
  crt_vector(ws, st, DT, T, N, L, kmax, 2 * lo[0] + lo[1] + lo[2], dOut);
  check(cudaGetLastError(), "svec_quadratic launch");
  copy_d2h(&hs, ws.status.p, sizeof(uint32_t), st);
  check(cudaStreamSynchronize(st), "sync");
  if (hs_out) *hs_out = hs;
  return 0;
}

// out[s] = q_a' X q_b for the pairs s = (a, b), each the exact sum rounded once
// (rns_blas.rs:4175-4277 symmetric_bilinear); X packed upper without svec factors.
int32_t rns_bilinear(RnsWorkspace& ws, cudaStream_t st, int N, int h, int cols, const unsigned char* dQ,
                     const unsigned char* dX, const unsigned long long* dPairs, int np, unsigned char* dOut,
                     uint32_t* hs_out) {
  const unsigned char* arr[2] = {dQ, dX};
  const int count[2] = {h * cols, h * (h + 1) / 2};
  int lo[2], bits[2];
  uint32_t hs = 0;
  if (!scan_classes(ws, st, N, arr, count, 2, lo, bits, &hs)) {
    if (hs_out) *hs_out = hs;
    g_last_error = "sdpxg_rns_symmetric_bilinear: non-finite operands are not supported";
    return 2;
  }
  const int L = primes_for(2.0 * bits[0] + bits[1] + 2 * ceil_log2((uint64_t)h) + 2);
  if (!L) {
    g_last_error = "sdpxg_rns_symmetric_bilinear: exponent spread too wide for the prime set";
    return 2;
  }
  DevTables& DT = ws.t15;
  const PrimeTables& T = DT.get(15, L, st);
  size_t off[2];
  const int absv[2] = {0, 0};
  class_residues(ws, st, DT, N, L, arr, count, lo, absv, 2, std::max(bits[0], bits[1]), off);
  grow(ws.RC8, (size_t)L * np);
  ++g_launches, k_rns_bilinear<<<dim3((unsigned)((np + 63) / 64), (unsigned)L), 64, 0, st>>>(
      h, cols, ws.cres.p + off[1] * L, ws.cres.p + off[0] * L, dPairs, np, L, DT.iprimes, ws.RC8);
  crt_vector(ws, st, DT, T, N, L, np, 2 * lo[0] + lo[1], dOut);
  check(cudaGetLastError(), "symmetric_bilinear launch");
  copy_d2h(&hs, ws.status.p, sizeof(uint32_t), st);
  check(cudaStreamSynchronize(st), "sync");
  if (hs_out) *hs_out = hs;
  return 0;
}

// C = A' diag(d) A (m x m) for A k x m (ld lda), every entry the exact sum rounded once
// (rns_blas.rs:2990-3194 diag_congruence), on the INT8 tensor cores: the columns of A aligned
// per column (lo_j), d as one class (lo_d); the right operand's residues are the left operand's
// times d's, and the CRT exponent of (i, j) is lo_i + lo_j + lo_d.
int32_t rns_diag_congruence(RnsWorkspace& ws, cudaStream_t st, int N, uint64_t m, uint64_t k,
                            const unsigned char* dA, uint64_t lda, const unsigned char* dD, int upper_only,
                            unsigned char* dC, uint32_t* hs_out) {
  grow(ws.loA, m); grow(ws.bitsA, m); grow(ws.loB2, m);
  grow(ws.maxbits, 2); grow(ws.status, 1); grow(ws.err, 1);
  const unsigned char* arr[1] = {dD};
  const int count[1] = {(int)k};
  int lo_d = 0, bits_d = 0;
  uint32_t hs = 0;
  if (!scan_classes(ws, st, N, arr, count, 1, &lo_d, &bits_d, &hs)) {
    if (hs_out) *hs_out = hs;
    g_last_error = "sdpxg_rns_diag_congruence: non-finite operands are not supported";
    return 2;
  }
  check(cudaMemsetAsync(ws.maxbits.p, 0, 2 * sizeof(int), st), "memset");
  ++g_launches, k_rns_scan<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(dA, N, (int)m, (int)k, (long)lda, 1, ws.loA,
                                                                 ws.bitsA, ws.maxbits, ws.status);
  int hb[2] = {0, 0};
  copy_d2h(hb, ws.maxbits.p, 2 * sizeof(int), st);
  copy_d2h(&hs, ws.status.p, sizeof(uint32_t), st);
  check(cudaStreamSynchronize(st), "sync");
  if (hs) {
    if (hs_out) *hs_out = hs;
    g_last_error = "sdpxg_rns_diag_congruence: non-finite operands are not supported";
    return 2;
  }
  const int L = primes_for(2.0 * hb[0] + bits_d + ceil_log2(k) + 2);
  if (!L) {
    g_last_error = "sdpxg_rns_diag_congruence: exponent spread too wide for the prime set";
    return 2;
  }
  DevTables& DT = ws.t15;
  const PrimeTables& T = DT.get(15, L, st);
  const int Mpad = (int)((m + 127) / 128 * 128), Kpad = (int)((k + 127) / 128 * 128);
  const long planeC = (long)(m * m);
  grow(ws.RC8, (size_t)L * planeC);
  size_t off[1];
  const int absv[1] = {0};
  class_residues(ws, st, DT, N, L, arr, count, &lo_d, absv, 1, std::max(hb[0], bits_d), off);
  const int S = 64 * N + std::max(hb[0], bits_d) + 1;  // the table class_residues just built
  grow(ws.PA, (size_t)L * 2 * Mpad * Kpad);
  grow(ws.PB, (size_t)L * 2 * Mpad * Kpad);
  ++g_launches, k_rns8_residues<<<(unsigned)(((long)Mpad * Kpad + 255) / 256), 256, 0, st>>>(
      dA, N, (int)m, (int)k, (long)lda, 1, ws.loA, L, DT.iprimes, DT.mu, ws.pow2, S, ws.PA, Mpad, Kpad);
  ++g_launches, k_rns8_scale_planes<<<(unsigned)(((long)Mpad * Kpad + 255) / 256), 256, 0, st>>>(
      ws.PA, ws.cres.p + off[0] * L, (int)k, L, DT.iprimes, ws.PB, Mpad, Kpad);
  check(cudaMemsetAsync(ws.err.p, 0, sizeof(int), st), "memset");
  for (int k0 = 0; k0 < Kpad; k0 += kI8Chunk) {
    I8GemmArgs ga;
    ga.Mpad = Mpad; ga.Npad = Mpad; ga.Kld = Kpad; ga.k0 = k0; ga.Kpad = std::min(kI8Chunk, Kpad - k0);
    ga.m = (int)m; ga.n = (int)m; ga.L = L; ga.moduli = DT.iprimes; ga.upper_only = upper_only;
    ga.accumulate = k0 > 0; ga.out = ws.RC8.p; ga.plane = planeC; ga.err = ws.err.p;
    launch_i8_gemm(2, ws.PA, ws.PB, ga, st);
  }
  ++g_launches, k_add_const_int<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(ws.loA, (int)m, lo_d, ws.loB2);
  ++g_launches, launch_crt<int>((unsigned)((m * m + 127) / 128), st, 
      ws.RC8, planeC, (int)m, (int)m, L, T.WW, DT.primes, DT.wt, DT.pinv, DT.mu, DT.MT, DT.M, ws.loA, ws.loB2, N,
      upper_only ? 1 : 0, dC, ws.status);
  check(cudaGetLastError(), "diag_congruence launch");
  int herr = 0;
  copy_d2h(&hs, ws.status.p, sizeof(uint32_t), st);
  copy_d2h(&herr, ws.err.p, sizeof(int), st);
  check(cudaStreamSynchronize(st), "sync");
  if (herr) throw CudaError("modular INT8 GEMM: a bounded wait gave up");
  if (hs_out) *hs_out = hs;
  return 0;
}

// Upper triangle of sum_b Z_b' Y_b with Z_b = diag(d_b) Y_b rounded entrywise, the exact sum over
// every block and row rounded once (rns_blas.rs:2656-2923 gemm_blocks_upper): the blocks are
// stacked into W x m operands (zeros off their columns, Z rounded while stacking) and multiplied
// by the exact product (W = the blocks' total width).  hr0/hyoff/hcoff/hq: host offsets.
int32_t rns_blocks_upper(RnsWorkspace& ws, cudaStream_t st, int N, uint64_t m, int nb, const std::vector<long>& hr0,
                         const std::vector<long>& hyoff, const std::vector<long>& hcoff, const std::vector<int>& hq,
                         const unsigned char* dY, const unsigned char* dD, const unsigned long long* dCols,
                         unsigned char* dC, uint32_t* hs_out) {
  const size_t esz = 8 * (size_t)N + 8;
  const long W = hr0[nb];
  grow(ws.boff, 3 * (size_t)nb + 1);
  grow(ws.bq, nb);
  std::vector<long> offs(hr0.begin(), hr0.end());
  offs.insert(offs.end(), hyoff.begin(), hyoff.end());
  offs.insert(offs.end(), hcoff.begin(), hcoff.end());
  ws.boff.upload(offs.data(), offs.size(), st);
  ws.bq.upload(hq.data(), nb, st);
  grow(ws.zs, (size_t)W * m * esz);
  grow(ws.ys, (size_t)W * m * esz);
  grow(ws.status, 1);
  check(cudaMemsetAsync(ws.status.p, 0, sizeof(uint32_t), st), "memset");
  mp_launch_stack_blocks(nb, ws.boff.p, ws.boff.p + nb + 1, ws.boff.p + 2 * nb + 1, ws.bq.p, dY, dD, dCols, W,
                         (int)m, N, ws.zs, ws.ys, ws.status, st);
  return rns_product(ws, st, ws.form, N, 'T', 'N', m, m, (uint64_t)W, ws.zs, (uint64_t)W, ws.ys, (uint64_t)W, 1, dC,
                     hs_out);
}

// The reference's dense MPFR LDL' (ArrowLDLSolver::try_dense -> ldl_rec, arrow.rs:255-470) on
// device MpFloat<N> arrays: blocks up to 128 by the exact-dot kernel, larger blocks halved with
// W21 = A21 L11^-T (solve_lt), L21 = W21 D1^-1 and A22 -= W21 L21' as one exact product (INT8
// tensor-core RNS, every entry rounded once) then subtracted.  Status bits accumulate in *status.
struct MpLdl {
  RnsWorkspace& ws;
  cudaStream_t st;
  int N;
  const unsigned char* reg;  // device (eps, delta) or null
  uint32_t* status;          // device status word
  size_t esz() const { return 8 * (size_t)N + 8; }

  // the exact product C = op(A) op(B) (m x n, ld m) into C
  void product(char ta, char tb, int m, int n, int k, const unsigned char* A, long lda, const unsigned char* B,
               long ldb, int upper, DevBuf<unsigned char>& C) {
    C.alloc((size_t)m * n * esz());
    uint32_t hs = 0;
    if (rns_product(ws, st, 0, N, ta, tb, m, n, k, A, lda, B, ldb, upper, C, &hs) != 0)
      throw std::runtime_error(g_last_error);
    if (hs) throw std::runtime_error("MPFR LDL: exact product reported status " + std::to_string(hs));
  }
  // X L' = B, L unit lower k x k (ld ldl), B m x k (ld ldb), X over B (arrow.rs:430-470)
  void solve_lt(const unsigned char* L, long ldl, int k, unsigned char* B, long ldb, int m) {
    if (m <= 0 || k <= 0) return;
    if (k <= kMpRecBase) {
      mp_launch_solve_lt(L, ldl, k, B, ldb, m, N, status, st);
      return;
    }
    const int k1 = k / 2, k2 = k - k1;
    solve_lt(L, ldl, k1, B, ldb, m);
    DevBuf<unsigned char> P;
    product('N', 'T', m, k2, k1, B, ldb, L + (size_t)k1 * esz(), ldl, 0, P);  // B1 L21'
    mp_launch_sub_block(B + (size_t)k1 * ldb * esz(), ldb, P, m, m, k2, N, status, st);
    solve_lt(L + ((size_t)k1 + (size_t)k1 * ldl) * esz(), ldl, k2, B + (size_t)k1 * ldb * esz(), ldb, m);
  }
  // arrow.rs:255-420 on the diagonal block at (off, off), size `size`; D^-1 into dinv + off
  void ldl_rec(unsigned char* A, long lda, int off, int size, unsigned char* dinv, DevBuf<unsigned char>& Wleaf) {
    if (size <= kMpRecBase) {
      mp_launch_ldl_dots(A, lda, off, size, N, Wleaf, dinv + (size_t)off * esz(), reg, status, st);
      return;
    }
    const int n1 = size / 2, n2 = size - n1;
    ldl_rec(A, lda, off, n1, dinv, Wleaf);
    unsigned char* A11 = A + ((size_t)off + (size_t)off * lda) * esz();
    unsigned char* A21 = A + ((size_t)off + n1 + (size_t)off * lda) * esz();
    solve_lt(A11, lda, n1, A21, lda, n2);  // W21 = A21 L11^-T in place
    DevBuf<unsigned char> W, C;
    W.alloc((size_t)n2 * n1 * esz());
    mp_launch_copy_scale_cols(A21, lda, W, dinv + (size_t)off * esz(), n2, n1, N, status, st);  // L21 = W21 D1^-1
    // (W L21')(a, b) for a <= b, subtracted from A22(b, a)
    product('N', 'T', n2, n2, n1, W, n2, A21, lda, 1, C);
    unsigned char* A22 = A + ((size_t)off + n1 + ((size_t)off + n1) * lda) * esz();
    mp_launch_sub_upper_t(A22, lda, C, n2, n2, N, status, st);
    ldl_rec(A, lda, off + n1, n2, dinv, Wleaf);
  }
};

RnsWorkspace& workspace(sdpxg_ctx* ctx) {
  auto slot = ctx_rns_slot(ctx);
  if (!*slot) *slot = std::make_shared<RnsWorkspace>();
  return *static_cast<RnsWorkspace*>(slot->get());
}

// Shared argument checks of both entry points; returns the element counts of A and B.
void check_args(uint32_t limbs, char ta, char tb, uint64_t m, uint64_t n, uint64_t k, uint64_t lda, uint64_t ldb,
                size_t* na, size_t* nb) {
  if ((ta != 'N' && ta != 'T') || (tb != 'N' && tb != 'T')) throw std::invalid_argument("bad transpose flag");
  if (m > (1u << 30) || n > (1u << 30) || k > (1u << 30)) throw std::invalid_argument("size overflow");
  const uint64_t ar = (ta == 'N') ? m : k, ac = (ta == 'N') ? k : m;
  const uint64_t br = (tb == 'N') ? k : n, bc = (tb == 'N') ? n : k;
  if (lda < std::max<uint64_t>(ar, 1) || ldb < std::max<uint64_t>(br, 1))
    throw std::invalid_argument("leading dimension too small");
  *na = ac ? lda * (ac - 1) + ar : 0;
  *nb = bc ? ldb * (bc - 1) + br : 0;
  (void)limbs;
}

bool device_memory(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int32_t sdpxg_rns_set_form(sdpxg_ctx* ctx, uint32_t form) {
  try {
    if (!ctx_engine_any(ctx)) throw std::invalid_argument("null context");
    if (form > 1) throw std::invalid_argument("form must be 0 (INT8 tensor cores) or 1 (FP64)");
    workspace(ctx).form = (int)form;
    return 0;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    g_last_error = "internal error";
    return 5;
  }
}

extern "C" int32_t sdpxg_rns_gemm(sdpxg_ctx* ctx, uint32_t limbs, char ta, char tb, uint64_t m,
                                  uint64_t n, uint64_t k, const void* A, uint64_t lda,
                                  const void* B, uint64_t ldb, uint32_t upper_only, void* C,
                                  uint32_t* status) {
  try {
    Engine* E = ctx_engine_any(ctx);
    if (!E) throw std::invalid_argument("null context");
    const int N = (int)limbs;
    if (N < 1 || N > RNS_MAXN) {
      g_last_error = "sdpxg_rns_gemm: limbs must be in 1..16";
      return 2;
    }
    size_t na = 0, nb = 0;
    check_args(limbs, ta, tb, m, n, k, lda, ldb, &na, &nb);
    if (m == 0 || n == 0) return 0;
    if (!A || !B || !C) throw std::invalid_argument("null pointer");
    const size_t esz = 8 * (size_t)N + 8;
    RnsWorkspace& ws = workspace(ctx);
    cudaStream_t st = E->st;
    check(cudaSetDevice(E->device), "cudaSetDevice");
    grow(ws.a, na * esz);
    grow(ws.b, nb * esz);
    grow(ws.c, m * n * esz);
    if (na) ws.a.upload(static_cast<const unsigned char*>(A), na * esz, st);
    if (nb) ws.b.upload(static_cast<const unsigned char*>(B), nb * esz, st);
    uint32_t hs = 0;
    const int32_t rc = rns_product(ws, st, ws.form, N, ta, tb, m, n, k, ws.a, lda, ws.b, ldb, upper_only ? 1 : 0,
                                   ws.c, &hs);
    if (status) *status = hs;
    if (rc) return rc;
    copy_d2h(C, ws.c.p, m * n * esz, st);
    check(cudaStreamSynchronize(st), "sync");
    return 0;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    g_last_error = "internal error";
    return 5;
  }
}

extern "C" int32_t sdpxg_rns_gemm_device(sdpxg_ctx* ctx, uint32_t limbs, char ta, char tb, uint64_t m,
                                         uint64_t n, uint64_t k, const void* d_A, uint64_t lda,
                                         const void* d_B, uint64_t ldb, uint32_t upper_only, void* d_C,
                                         uint32_t* status) {
  try {
    Engine* E = ctx_engine_any(ctx);
    if (!E) throw std::invalid_argument("null context");
    const int N = (int)limbs;
    if (N < 1 || N > RNS_MAXN) {
      g_last_error = "sdpxg_rns_gemm_device: limbs must be in 1..16";
      return 2;
    }
    size_t na = 0, nb = 0;
    check_args(limbs, ta, tb, m, n, k, lda, ldb, &na, &nb);
    if (m == 0 || n == 0) return 0;
    if (!d_A || !d_B || !d_C) throw std::invalid_argument("null pointer");
    check(cudaSetDevice(E->device), "cudaSetDevice");
    if ((na && !device_memory(d_A)) || (nb && !device_memory(d_B)) || !device_memory(d_C))
      throw std::invalid_argument("sdpxg_rns_gemm_device: A, B and C must be device pointers");
    RnsWorkspace& ws = workspace(ctx);
    uint32_t hs = 0;
    const int32_t rc = rns_product(ws, E->st, ws.form, N, ta, tb, m, n, k, static_cast<const unsigned char*>(d_A),
                                   lda, static_cast<const unsigned char*>(d_B), ldb, upper_only ? 1 : 0,
                                   static_cast<unsigned char*>(d_C), &hs);
    if (status) *status = hs;
    return rc;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    g_last_error = "internal error";
    return 5;
  }
}

extern "C" int32_t sdpxg_rns_congruence(sdpxg_ctx* ctx, uint32_t limbs, char ta, uint64_t m, uint64_t k,
                                        const void* A, uint64_t lda, const void* X, uint64_t ldx,
                                        uint32_t upper_only, void* C, uint32_t* status) {
  try {
    Engine* E = ctx_engine_any(ctx);
    if (!E) throw std::invalid_argument("null context");
    const int N = (int)limbs;
    if (N < 1 || N > RNS_MAXN) {
      g_last_error = "sdpxg_rns_congruence: limbs must be in 1..16";
      return 2;
    }
    if (ta != 'N' && ta != 'T') throw std::invalid_argument("bad transpose flag");
    if (m > (1u << 20) || k > (1u << 20)) throw std::invalid_argument("size overflow");
    const uint64_t ar = ta == 'N' ? m : k, ac = ta == 'N' ? k : m;
    if (lda < std::max<uint64_t>(ar, 1) || ldx < std::max<uint64_t>(k, 1))
      throw std::invalid_argument("leading dimension too small");
    if (m == 0) return 0;
    if (!A || !X || !C) throw std::invalid_argument("null pointer");
    const size_t esz = 8 * (size_t)N + 8;
    const size_t na = ac ? lda * (ac - 1) + ar : 0, nx = k ? ldx * (k - 1) + k : 0;
    RnsWorkspace& ws = workspace(ctx);
    cudaStream_t st = E->st;
    check(cudaSetDevice(E->device), "cudaSetDevice");
    if (k == 0) {  // empty sums: zeros
      std::vector<unsigned char> z(m * m * esz, 0);
      for (size_t e = 0; e < m * m; ++e) *reinterpret_cast<int*>(&z[e * esz + 8 * N]) = MP_ZERO;
      std::memcpy(C, z.data(), z.size());
      if (status) *status = 0;
      return 0;
    }
    grow(ws.a, na * esz);
    grow(ws.b, nx * esz);
    grow(ws.c, m * m * esz);
    ws.a.upload(static_cast<const unsigned char*>(A), na * esz, st);
    ws.b.upload(static_cast<const unsigned char*>(X), nx * esz, st);
    uint32_t hs = 0;
    const int32_t rc = rns_congruence(ws, st, N, ta, m, k, ws.a, lda, ws.b, ldx, upper_only ? 1 : 0, ws.c, &hs);
    if (status) *status = hs;
    if (rc) return rc;
    copy_d2h(C, ws.c.p, m * m * esz, st);
    check(cudaStreamSynchronize(st), "sync");
    return 0;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    g_last_error = "internal error";
    return 5;
  }
}

extern "C" int32_t sdpxg_mp_ldl_device(sdpxg_ctx* ctx, uint32_t limbs, uint64_t n, void* d_A, uint64_t lda,
                                       const void* d_reg, void* d_dinv, uint32_t* status) {
  try {
    Engine* E = ctx_engine_any(ctx);
    if (!E) throw std::invalid_argument("null context");
    const int N = (int)limbs;
    if (N < 1 || N > kMpMaxLimbs) {
      g_last_error = "sdpxg_mp_ldl: limbs must be in 1..8";
      return 2;
    }
    if (n == 0) return 0;
    if (n > (1u << 20) || lda < n) throw std::invalid_argument("bad size or leading dimension");
    if (!d_A || !d_dinv) throw std::invalid_argument("null pointer");
    check(cudaSetDevice(E->device), "cudaSetDevice");
    if (!device_memory(d_A) || !device_memory(d_dinv) || (d_reg && !device_memory(d_reg)))
      throw std::invalid_argument("sdpxg_mp_ldl_device: A, reg and dinv must be device pointers");
    RnsWorkspace& ws = workspace(ctx);
    DevBuf<uint32_t> stw(1);
    check(cudaMemsetAsync(stw.p, 0, sizeof(uint32_t), E->st), "memset");
    MpLdl f{ws, E->st, N, static_cast<const unsigned char*>(d_reg), stw.p};
    DevBuf<unsigned char> Wleaf(2 * (size_t)kMpRecBase * kMpRecBase * f.esz());  // the leaves' W and R
    f.ldl_rec(static_cast<unsigned char*>(d_A), (long)lda, 0, (int)n, static_cast<unsigned char*>(d_dinv), Wleaf);
    uint32_t hs = 0;
    copy_d2h(&hs, stw.p, sizeof(uint32_t), E->st);
    check(cudaStreamSynchronize(E->st), "sync");
    if (status) *status = hs;
    if (hs & SDPXG_ST_EXACT_SPREAD) {
      g_last_error = "sdpxg_mp_ldl: an exact dot's exponent spread exceeds the device accumulator";
      return 2;
    }
    return 0;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    g_last_error = "internal error";
    return 5;
  }
}

extern "C" int32_t sdpxg_mp_ldl(sdpxg_ctx* ctx, uint32_t limbs, uint64_t n, const void* A, uint64_t lda,
                                const void* reg, void* L, void* dinv, uint32_t* status) {
  try {
    Engine* E = ctx_engine_any(ctx);
    if (!E) throw std::invalid_argument("null context");
    const int N = (int)limbs;
    if (N < 1 || N > kMpMaxLimbs) {
      g_last_error = "sdpxg_mp_ldl: limbs must be in 1..8";
      return 2;
    }
    if (n == 0) return 0;
    if (n > (1u << 20) || lda < n) throw std::invalid_argument("bad size or leading dimension");
    if (!A || !L || !dinv) throw std::invalid_argument("null pointer");
    const size_t esz = 8 * (size_t)N + 8;
    check(cudaSetDevice(E->device), "cudaSetDevice");
    DevBuf<unsigned char> dA(n * n * esz), dD(n * esz), dR(2 * esz);
    check(cudaMemcpy2DAsync(dA.p, n * esz, A, lda * esz, n * esz, n, cudaMemcpyHostToDevice, E->st), "H2D");
    g_h2d_bytes += n * n * esz;
    if (reg) dR.upload(static_cast<const unsigned char*>(reg), 2 * esz, E->st);
    const int32_t rc = sdpxg_mp_ldl_device(ctx, limbs, n, dA.p, n, reg ? dR.p : nullptr, dD.p, status);
    if (rc) return rc;
    copy_d2h(L, dA.p, n * n * esz, E->st);
    copy_d2h(dinv, dD.p, n * esz, E->st);
    check(cudaStreamSynchronize(E->st), "sync");
    return 0;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    g_last_error = "internal error";
    return 5;
  }
}

extern "C" int32_t sdpxg_mp_potrf(sdpxg_ctx* ctx, uint32_t limbs, char uplo, uint64_t n, void* A, uint64_t lda,
                                  int32_t* info, uint32_t* status) {
  try {
    Engine* E = ctx_engine_any(ctx);
    if (!E) throw std::invalid_argument("null context");
    const int N = (int)limbs;
    if (N < 1 || N > kMpMaxLimbs) {
      g_last_error = "sdpxg_mp_potrf: limbs must be in 1..8";
      return 2;
    }
    if (uplo != 'L' && uplo != 'U') throw std::invalid_argument("uplo must be 'L' or 'U'");
    if (n > (1u << 16) || lda < std::max<uint64_t>(n, 1)) throw std::invalid_argument("bad size or leading dimension");
    if (!info) throw std::invalid_argument("null pointer");
    *info = 0;
    if (n == 0) return 0;
    if (!A) throw std::invalid_argument("null pointer");
    const size_t esz = 8 * (size_t)N + 8;
    check(cudaSetDevice(E->device), "cudaSetDevice");
    DevBuf<unsigned char> dA(n * n * esz);
    DevBuf<int> dinfo(1);
    DevBuf<uint32_t> stw(1);
    check(cudaMemsetAsync(stw.p, 0, sizeof(uint32_t), E->st), "memset");
    check(cudaMemcpy2DAsync(dA.p, n * esz, A, lda * esz, n * esz, n, cudaMemcpyHostToDevice, E->st), "H2D");
    g_h2d_bytes += n * n * esz;
    mp_launch_potrf(dA.p, (long)n, (int)n, uplo == 'L', N, dinfo.p, stw.p, E->st);
    check(cudaMemcpy2DAsync(A, lda * esz, dA.p, n * esz, n * esz, n, cudaMemcpyDeviceToHost, E->st), "D2H");
    g_d2h_bytes += n * n * esz;
    uint32_t hs = 0;
    copy_d2h(&hs, stw.p, sizeof(uint32_t), E->st);
    copy_d2h(info, dinfo.p, sizeof(int), E->st);
    check(cudaStreamSynchronize(E->st), "sync");
    if (status) *status = hs;
    if (hs & SDPXG_ST_EXACT_SPREAD) {
      g_last_error = "sdpxg_mp_potrf: an exact dot's exponent spread exceeds the device accumulator";
      return 2;
    }
    return 0;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    g_last_error = "internal error";
    return 5;
  }
}

// ---- entry points of the exact forms (host arrays in the reference's MpFloat<N> layout) ----
namespace {
template <class F>
int32_t rns_entry(F&& f) {
  try {
    return f();
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    g_last_error = "internal error";
    return 5;
  }
}
Engine* entry_engine(sdpxg_ctx* ctx, uint32_t limbs, const char* name, uint32_t max_limbs) {
  Engine* E = ctx_engine_any(ctx);
  if (!E) throw std::invalid_argument("null context");
  if (limbs < 1 || limbs > max_limbs)
    throw std::invalid_argument(std::string(name) + ": limbs must be in 1.." + std::to_string(max_limbs));
  check(cudaSetDevice(E->device), "cudaSetDevice");
  return E;
}
void zero_outputs(void* out, size_t count, int N) {
  const size_t esz = 8 * (size_t)N + 8;
  unsigned char* o = static_cast<unsigned char*>(out);
  std::memset(o, 0, count * esz);
  for (size_t e = 0; e < count; ++e) *reinterpret_cast<int*>(o + e * esz + 8 * N) = MP_ZERO;
}
}  // namespace

extern "C" int32_t sdpxg_rns_diag_congruence(sdpxg_ctx* ctx, uint32_t limbs, uint64_t m, uint64_t k, const void* A,
                                             uint64_t lda, const void* d, uint32_t upper_only, void* C,
                                             uint32_t* status) {
  return rns_entry([&]() -> int32_t {
    Engine* E = entry_engine(ctx, limbs, "sdpxg_rns_diag_congruence", RNS_MAXN);
    const int N = (int)limbs;
    if (m > (1u << 20) || k > (1u << 20)) throw std::invalid_argument("size overflow");
    if (lda < std::max<uint64_t>(k, 1)) throw std::invalid_argument("leading dimension too small");
    if (status) *status = 0;
    if (m == 0) return 0;
    if (!A || !d || !C) throw std::invalid_argument("null pointer");
    if (k == 0) {
      zero_outputs(C, m * m, N);
      return 0;
    }
    const size_t esz = 8 * (size_t)N + 8, na = lda * (m - 1) + k;
    RnsWorkspace& ws = workspace(ctx);
    cudaStream_t st = E->st;
    grow(ws.a, na * esz);
    grow(ws.b, k * esz);
    grow(ws.c, m * m * esz);
    ws.a.upload(static_cast<const unsigned char*>(A), na * esz, st);
    ws.b.upload(static_cast<const unsigned char*>(d), k * esz, st);
    uint32_t hs = 0;
    const int32_t rc = rns_diag_congruence(ws, st, N, m, k, ws.a, lda, ws.b, upper_only ? 1 : 0, ws.c, &hs);
    if (status) *status = hs;
    if (rc) return rc;
    copy_d2h(C, ws.c.p, m * m * esz, st);
    check(cudaStreamSynchronize(st), "sync");
    return 0;
  });
}

extern "C" int32_t sdpxg_rns_svec_quadratic(sdpxg_ctx* ctx, uint32_t limbs, uint64_t h, uint64_t kmax, const void* Q,
                                            uint32_t abs_q, const void* x, const void* sqrt2, void* out,
                                            uint32_t* status) {
  return rns_entry([&]() -> int32_t {
    Engine* E = entry_engine(ctx, limbs, "sdpxg_rns_svec_quadratic", RNS_MAXN);
    const int N = (int)limbs;
    if (h > 4096 || kmax > (1u << 20)) throw std::invalid_argument("size overflow");
    if (status) *status = 0;
    if (kmax == 0) return 0;
    if (!Q || !x || !sqrt2 || !out) throw std::invalid_argument("null pointer");
    if (h == 0) {
      zero_outputs(out, kmax, N);
      return 0;
    }
    const size_t esz = 8 * (size_t)N + 8, tri = h * (h + 1) / 2;
    RnsWorkspace& ws = workspace(ctx);
    cudaStream_t st = E->st;
    grow(ws.a, h * kmax * esz);
    grow(ws.b, tri * esz);
    grow(ws.fd, 2 * esz);
    grow(ws.c, kmax * esz);
    std::vector<unsigned char> c2(2 * esz, 0);  // (1, sqrt2): 1 = 2^63 in the top limb, exponent 1
    reinterpret_cast<unsigned long long*>(c2.data())[N - 1] = 1ull << 63;
    *reinterpret_cast<int*>(&c2[8 * N]) = MP_REGULAR;
    *reinterpret_cast<int*>(&c2[8 * N + 4]) = 1;
    std::memcpy(&c2[esz], sqrt2, esz);
    ws.a.upload(static_cast<const unsigned char*>(Q), h * kmax * esz, st);
    ws.b.upload(static_cast<const unsigned char*>(x), tri * esz, st);
    ws.fd.upload(c2.data(), 2 * esz, st);
    uint32_t hs = 0;
    const int32_t rc = rns_svec_quadratic(ws, st, N, (int)h, (int)kmax, ws.a, abs_q ? 1 : 0, ws.b, ws.fd, ws.c, &hs);
    if (status) *status = hs;
    if (rc) return rc;
    copy_d2h(out, ws.c.p, kmax * esz, st);
    check(cudaStreamSynchronize(st), "sync");
    return 0;
  });
}

extern "C" int32_t sdpxg_rns_symmetric_bilinear(sdpxg_ctx* ctx, uint32_t limbs, uint64_t h, uint64_t columns,
                                                const void* Q, const void* X, uint64_t npairs, const uint64_t* pairs,
                                                void* out, uint32_t* status) {
  return rns_entry([&]() -> int32_t {
    Engine* E = entry_engine(ctx, limbs, "sdpxg_rns_symmetric_bilinear", RNS_MAXN);
    const int N = (int)limbs;
    if (h > 4096 || columns > (1u << 20) || npairs > (1u << 24)) throw std::invalid_argument("size overflow");
    if (status) *status = 0;
    if (npairs == 0) return 0;
    if (!Q || !X || !pairs || !out) throw std::invalid_argument("null pointer");
    for (uint64_t s = 0; s < 2 * npairs; ++s)
      if (pairs[s] >= columns) throw std::invalid_argument("pair column out of range");
    if (h == 0) {
      zero_outputs(out, npairs, N);
      return 0;
    }
    const size_t esz = 8 * (size_t)N + 8, tri = h * (h + 1) / 2;
    RnsWorkspace& ws = workspace(ctx);
    cudaStream_t st = E->st;
    grow(ws.a, h * columns * esz);
    grow(ws.b, tri * esz);
    grow(ws.c, npairs * esz);
    grow(ws.bpairs, 2 * npairs);
    ws.a.upload(static_cast<const unsigned char*>(Q), h * columns * esz, st);
    ws.b.upload(static_cast<const unsigned char*>(X), tri * esz, st);
    ws.bpairs.upload(reinterpret_cast<const unsigned long long*>(pairs), 2 * npairs, st);
    uint32_t hs = 0;
    const int32_t rc = rns_bilinear(ws, st, N, (int)h, (int)columns, ws.a, ws.b, ws.bpairs, (int)npairs, ws.c, &hs);
    if (status) *status = hs;
    if (rc) return rc;
    copy_d2h(out, ws.c.p, npairs * esz, st);
    check(cudaStreamSynchronize(st), "sync");
    return 0;
  });
}

extern "C" int32_t sdpxg_rns_gemm_blocks_upper(sdpxg_ctx* ctx, uint32_t limbs, uint64_t m, uint64_t nblocks,
                                               const uint64_t* widths, const uint64_t* counts, const void* y,
                                               const void* d, const uint64_t* columns, void* C, uint32_t* status) {
  return rns_entry([&]() -> int32_t {
    Engine* E = entry_engine(ctx, limbs, "sdpxg_rns_gemm_blocks_upper", kMpMaxLimbs);
    const int N = (int)limbs;
    if (m > (1u << 16) || nblocks > (1u << 20)) throw std::invalid_argument("size overflow");
    if (status) *status = 0;
    if (m == 0) return 0;
    if (!C || (nblocks && (!widths || !counts))) throw std::invalid_argument("null pointer");
    std::vector<long> r0(1, 0), yoff, coff;
    std::vector<int> q;
    long ytot = 0, ctot = 0;
    for (uint64_t b = 0; b < nblocks; ++b) {
      if (widths[b] > (1u << 20) || counts[b] > m) throw std::invalid_argument("block extent out of range");
      if (widths[b] == 0 || counts[b] == 0) continue;  // an empty block adds nothing
      yoff.push_back(ytot);
      coff.push_back(ctot);
      q.push_back((int)counts[b]);
      r0.push_back(r0.back() + (long)widths[b]);
      ytot += (long)(widths[b] * counts[b]);
      ctot += (long)counts[b];
    }
    // columns of every (nonempty or not) block, in order: validate sorted and in range
    uint64_t cpos = 0;
    std::vector<unsigned long long> cols;
    for (uint64_t b = 0; b < nblocks; ++b) {
      for (uint64_t c = 0; c < counts[b]; ++c) {
        const uint64_t v = columns[cpos + c];
        if (v >= m || (c && v <= columns[cpos + c - 1]))
          throw std::invalid_argument("block columns must be increasing and below m");
        if (widths[b]) cols.push_back(v);
      }
      cpos += counts[b];
    }
    const int nb = (int)q.size();
    if (nb == 0 || r0.back() * (long)m > (1L << 28)) {
      if (nb == 0) {
        zero_outputs(C, m * m, N);
        return 0;
      }
      throw std::invalid_argument("stacked block operands too large");
    }
    if (!y || !d || !columns) throw std::invalid_argument("null pointer");
    // the inputs of the nonempty blocks, packed in order
    const size_t esz = 8 * (size_t)N + 8;
    std::vector<unsigned char> hy((size_t)ytot * esz), hd((size_t)r0.back() * esz);
    {
      const unsigned char* ys = static_cast<const unsigned char*>(y);
      const unsigned char* ds = static_cast<const unsigned char*>(d);
      size_t yi = 0, di = 0, yo = 0, dO = 0;
      for (uint64_t b = 0; b < nblocks; ++b) {
        const size_t ny = widths[b] * counts[b], nd = widths[b];
        if (widths[b] && counts[b]) {
          std::memcpy(&hy[yo * esz], ys + yi * esz, ny * esz);
          std::memcpy(&hd[dO * esz], ds + di * esz, nd * esz);
          yo += ny;
          dO += nd;
        }
        yi += ny;
        di += nd;
      }
    }
    RnsWorkspace& ws = workspace(ctx);
    cudaStream_t st = E->st;
    grow(ws.a, hy.size());
    grow(ws.b, hd.size());
    grow(ws.c, m * m * esz);
    grow(ws.bcols, cols.size());
    ws.a.upload(hy.data(), hy.size(), st);
    ws.b.upload(hd.data(), hd.size(), st);
    ws.bcols.upload(cols.data(), cols.size(), st);
    uint32_t hs = 0;
    const int32_t rc = rns_blocks_upper(ws, st, N, m, nb, r0, yoff, coff, q, ws.a, ws.b, ws.bcols, ws.c, &hs);
    if (status) *status = hs;
    if (rc) return rc;
    copy_d2h(C, ws.c.p, m * m * esz, st);
    check(cudaStreamSynchronize(st), "sync");
    return 0;
  });
}

extern "C" int32_t sdpxg_mp_nt_scale(sdpxg_ctx* ctx, uint32_t limbs, uint64_t nblocks, const uint64_t* orders,
                                     const void* s, const void* z, void* lambda, void* lisqrt, void* R, void* Rinv,
                                     void* G, int32_t* block_status, uint32_t* status) {
  return rns_entry([&]() -> int32_t {
    Engine* E = entry_engine(ctx, limbs, "sdpxg_mp_nt_scale", kMpMaxLimbs);
    const int N = (int)limbs;
    if (status) *status = 0;
    if (nblocks == 0) return 0;
    if (nblocks > (1u << 20)) throw std::invalid_argument("size overflow");
    if (!orders || !s || !z || !lambda || !lisqrt || !R || !Rinv || !G || !block_status)
      throw std::invalid_argument("null pointer");
    std::vector<MpNtBlock> desc;
    std::vector<int> slot;  // block index of each nonempty descriptor
    long tri = 0, sq = 0, lin = 0;
    for (uint64_t b = 0; b < nblocks; ++b) {
      if (orders[b] > 64) throw std::invalid_argument("sdpxg_mp_nt_scale: block orders must be at most 64");
      block_status[b] = 0;
      const long n = (long)orders[b];
      if (n) {
        desc.push_back({(int)n, tri, sq, lin});
        slot.push_back((int)b);
      }
      tri += n * (n + 1) / 2;
      sq += n * n;
      lin += n;
    }
    const size_t esz = 8 * (size_t)N + 8;
    cudaStream_t st = E->st;
    DevBuf<MpNtBlock> dd(std::max<size_t>(desc.size(), 1));
    DevBuf<unsigned char> ds(tri * esz + esz), dz(tri * esz + esz), dwork(5 * sq * esz + esz), dwv(2 * lin * esz + esz);
    DevBuf<unsigned char> dlam(lin * esz + esz), dlis(lin * esz + esz), dR(sq * esz + esz), dRi(sq * esz + esz),
        dG(sq * esz + esz), dfrac(esz);
    DevBuf<int> dbs(std::max<size_t>(desc.size(), 1));
    DevBuf<uint32_t> stw(1);
    check(cudaMemsetAsync(stw.p, 0, sizeof(uint32_t), st), "memset");
    if (!desc.empty()) dd.upload(desc.data(), desc.size(), st);
    ds.upload(static_cast<const unsigned char*>(s), tri * esz, st);
    dz.upload(static_cast<const unsigned char*>(z), tri * esz, st);
    // blocks of order 0 keep zero-filled outputs
    check(cudaMemsetAsync(dR.p, 0, sq * esz + esz, st), "memset");
    mp_launch_nt_scale(dd, (int)desc.size(), N, ds, dz, dfrac, dwork, dwv, dlam, dlis, dR, dRi, dG, dbs, stw, st);
    std::vector<int> hbs(desc.size());
    uint32_t hs = 0;
    copy_d2h(lambda, dlam.p, lin * esz, st);
    copy_d2h(lisqrt, dlis.p, lin * esz, st);
    copy_d2h(R, dR.p, sq * esz, st);
    copy_d2h(Rinv, dRi.p, sq * esz, st);
    copy_d2h(G, dG.p, sq * esz, st);
    if (!desc.empty()) copy_d2h(hbs.data(), dbs.p, desc.size() * sizeof(int), st);
    copy_d2h(&hs, stw.p, sizeof(uint32_t), st);
    check(cudaStreamSynchronize(st), "sync");
    for (size_t i = 0; i < desc.size(); ++i) block_status[slot[i]] = hbs[i];
    if (status) *status = hs;
    if (hs & SDPXG_ST_EXACT_SPREAD) {
      g_last_error = "sdpxg_mp_nt_scale: an exact dot's exponent spread exceeds the device accumulator";
      return 2;
    }
    return 0;
  });
}

extern "C" int32_t sdpxg_mp_step_length(sdpxg_ctx* ctx, uint32_t limbs, uint64_t nblocks, const uint64_t* orders,
                                        uint32_t primal, const void* d, const void* Rx, const void* lisqrt,
                                        const void* alpha_max, void* alpha, int32_t* path, uint32_t* status) {
  return rns_entry([&]() -> int32_t {
    Engine* E = entry_engine(ctx, limbs, "sdpxg_mp_step_length", kMpMaxLimbs);
    const int N = (int)limbs;
    if (status) *status = 0;
    if (nblocks == 0) return 0;
    if (nblocks > (1u << 20)) throw std::invalid_argument("size overflow");
    if (!orders || !d || !Rx || !lisqrt || !alpha_max || !alpha || !path) throw std::invalid_argument("null pointer");
    std::vector<MpStepBlock> desc;
    std::vector<int> slot;
    long tri = 0, sq = 0, lin = 0, fw = 0;
    for (uint64_t b = 0; b < nblocks; ++b) {
      if (orders[b] > 64) throw std::invalid_argument("sdpxg_mp_step_length: block orders must be at most 64");
      const long n = (long)orders[b];
      if (n) {
        desc.push_back({(int)n, tri, sq, lin});
        slot.push_back((int)b);
      }
      tri += n * (n + 1) / 2;
      sq += n * n;
      lin += n;
      fw += n * n + 2 * n;
    }
    const size_t esz = 8 * (size_t)N + 8;
    cudaStream_t st = E->st;
    RnsWorkspace& ws = workspace(ctx);
    DevBuf<MpStepBlock> dd(std::max<size_t>(desc.size(), 1));
    DevBuf<unsigned char> dD(tri * esz + esz), dR(sq * esz + esz), dL(lin * esz + esz), dX(sq * esz + esz),
        dY(sq * esz + esz), dwork(2 * sq * esz + esz), dconst(2 * esz), dal(std::max<size_t>(desc.size(), 1) * esz);
    DevBuf<double> dfw(fw + 1);
    DevBuf<int> dpath(std::max<size_t>(desc.size(), 1));
    DevBuf<uint32_t> stw(1);
    check(cudaMemsetAsync(stw.p, 0, sizeof(uint32_t), st), "memset");
    if (!desc.empty()) dd.upload(desc.data(), desc.size(), st);
    dD.upload(static_cast<const unsigned char*>(d), tri * esz, st);
    dR.upload(static_cast<const unsigned char*>(Rx), sq * esz, st);
    dL.upload(static_cast<const unsigned char*>(lisqrt), lin * esz, st);
    check(cudaMemcpyAsync(dconst.p + esz, alpha_max, esz, cudaMemcpyHostToDevice, st), "H2D");
    g_h2d_bytes += esz;
    mp_launch_step_smat(dd, (int)desc.size(), N, dD, dconst, dX, stw, st);
    // Y_b: the exact W-congruence of the direction (mul_Wx_scratch, psdtrianglecone.rs:860-917):
    // primal (ds) Rinv X Rinv', dual (dz) R' X R
    for (const MpStepBlock& b : desc) {
      uint32_t hs = 0;
      const int32_t rc = rns_congruence(ws, st, N, primal ? 'N' : 'T', (uint64_t)b.n, (uint64_t)b.n,
                                        dR.p + b.mat * esz, (uint64_t)b.n, dX.p + b.mat * esz, (uint64_t)b.n, 0,
                                        dY.p + b.mat * esz, &hs);
      if (rc) return rc;
    }
    mp_launch_step_bound(dd, (int)desc.size(), N, dY, dL, dconst, dwork, dfw, dal, dpath, stw, st);
    std::vector<unsigned char> hal(desc.size() * esz);
    std::vector<int> hpath(desc.size());
    uint32_t hs = 0;
    if (!desc.empty()) {
      copy_d2h(hal.data(), dal.p, desc.size() * esz, st);
      copy_d2h(hpath.data(), dpath.p, desc.size() * sizeof(int), st);
    }
    copy_d2h(&hs, stw.p, sizeof(uint32_t), st);
    check(cudaStreamSynchronize(st), "sync");
    unsigned char* out = static_cast<unsigned char*>(alpha);
    for (uint64_t b = 0; b < nblocks; ++b) {  // an empty block bounds nothing: alpha_max
      std::memcpy(out + b * esz, alpha_max, esz);
      path[b] = 0;
    }
    for (size_t i = 0; i < desc.size(); ++i) {
      std::memcpy(out + (size_t)slot[i] * esz, &hal[i * esz], esz);
      path[slot[i]] = hpath[i];
    }
    if (status) *status = hs;
    if (hs & SDPXG_ST_EXACT_SPREAD) {
      g_last_error = "sdpxg_mp_step_length: an exact dot's exponent spread exceeds the device accumulator";
      return 2;
    }
    return 0;
  });
}
