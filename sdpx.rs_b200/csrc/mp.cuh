// Correctly rounded MpFloat<N> arithmetic on the GPU (N 64-bit limbs, round to nearest, ties to
// even: the MPFR contract of crates/arithmetic/src/lib.rs that the reference's MpFloat follows).
//
// Element layout (the reference's in-memory MpFloat<N>, lib.rs:333-340): u64 limbs[N], least
// significant first, i32 kind = sign * MPFR kind (2 zero, 3 regular), i32 exponent; a regular
// value is M * 2^(exponent - 64N) with the top bit of M set.
//
// Every operation forms its exact result as a wide integer times a power of two and rounds it
// once (mp_round):
//   mp_addsub           aligned exact sum (operands more than 64N + 64 bits apart: the smaller
//                       one lies below a 2^-64 fraction of an ulp and leaves the larger unchanged)
//   mp_mul              2N-limb product
//   mp_recip, mp_div,   the integer quotient floor(2^(128N + 2) / M), floor(M_a 2^(64N + 2) / M_b)
//   mp_sqrt             or root floor(sqrt(M 2^e)) with its remainder folded into a sticky bit;
//                       the quotient or root from a Newton estimate corrected exactly by its
//                       multiword remainder (the same integers a long division would give)
//   mp_dot_sub          a - sum x_c y_c (or sum x_c y_c) exact in a two's-complement fixed-point
//                       accumulator of up to kAccWords words, rounded once -- the exact dot of
//                       exactdot.rs:53-70; terms spread beyond the accumulator report failure.
#pragma once
#include <climits>
#include <cstdint>

namespace mpd {

constexpr int kMaxN = 8;        // limbs: up to 512-bit values
constexpr int kAccWords = 40;   // exact-dot accumulator: 2560 bits of spread + width
constexpr int kWideWords = 2 * kMaxN + 3;
constexpr int kKindZero = 2, kKindRegular = 3;
constexpr int kExpMax = (1 << 30) - 1;

struct Val {
  unsigned long long m[kMaxN];  // mantissa, top bit of limb N-1 set (unless zero)
  long long s;                  // scale: value = (-1)^neg M 2^s
  bool neg, zero;
};

__device__ __forceinline__ Val mp_load(const unsigned char* p, int N) {
  Val v;
  const unsigned long long* l = reinterpret_cast<const unsigned long long*>(p);
  const int kind = *reinterpret_cast<const int*>(p + 8 * N);
  const int ex = *reinterpret_cast<const int*>(p + 8 * N + 4);
  v.zero = (kind == kKindZero || kind == -kKindZero);
  v.neg = kind < 0;
#pragma unroll
  for (int q = 0; q < kMaxN; ++q) v.m[q] = (q < N && !v.zero) ? l[q] : 0ull;
  v.s = (long long)ex - 64LL * N;
  return v;
}

// Store v (zeros as +0); an exponent outside the MPFR range sets bit 4 (non-finite) of *status.
__device__ __forceinline__ void mp_store(unsigned char* p, int N, const Val& v, uint32_t* status) {
  unsigned long long* l = reinterpret_cast<unsigned long long*>(p);
  int* kind = reinterpret_cast<int*>(p + 8 * N);
  const long long ex = v.s + 64LL * N;
  if (v.zero || ex > kExpMax || ex < -kExpMax) {
    if (!v.zero && status) atomicOr(status, 4u);
    for (int q = 0; q < N; ++q) l[q] = 0ull;
    kind[0] = kKindZero;
    kind[1] = 0;
    return;
  }
  for (int q = 0; q < N; ++q) l[q] = v.m[q];
  kind[0] = v.neg ? -kKindRegular : kKindRegular;
  kind[1] = (int)ex;
}

__device__ __forceinline__ Val mp_zero() {
  Val v;
#pragma unroll
  for (int q = 0; q < kMaxN; ++q) v.m[q] = 0ull;
  v.s = 0;
  v.neg = false;
  v.zero = true;
  return v;
}

// Round S (W little-endian words, magnitude) * 2^scale to N limbs, ties to even.
__device__ inline Val mp_round(const unsigned long long* S, int W, bool neg, long long scale, int N) {
  int top = -1;
  for (int w = W - 1; w >= 0; --w)
    if (S[w]) {
      top = w;
      break;
    }
  if (top < 0) return mp_zero();
  const int bitlen = top * 64 + 64 - __clzll(S[top]);
  int shift = bitlen - 64 * N;
  auto window = [&](int start) -> unsigned long long {  // bits [start, start + 64) of S
    const int word = (start >= 0) ? start / 64 : -((-start + 63) / 64);
    const int off = start - 64 * word;
    const unsigned long long lo = (word >= 0 && word < W) ? S[word] : 0ull;
    const unsigned long long hi = (word + 1 >= 0 && word + 1 < W) ? S[word + 1] : 0ull;
    return (lo >> off) | (off ? (hi << (64 - off)) : 0ull);
  };
  Val v;
  v.zero = false;
  v.neg = neg;
#pragma unroll
  for (int q = 0; q < kMaxN; ++q) v.m[q] = q < N ? window(shift + 64 * q) : 0ull;
  if (shift > 0) {
    const int rb = shift - 1;
    const bool round_bit = (S[rb / 64] >> (rb % 64)) & 1ull;
    bool sticky = false;
    for (int w = 0; w < rb / 64; ++w) sticky = sticky || (S[w] != 0);
    if (rb % 64) sticky = sticky || ((S[rb / 64] & ((1ull << (rb % 64)) - 1)) != 0);
    if (round_bit && (sticky || (v.m[0] & 1ull))) {
      bool carry = true;
      for (int q = 0; q < N && carry; ++q) {
        v.m[q] += 1;
        carry = (v.m[q] == 0);
      }
      if (carry) {
        v.m[N - 1] = 1ull << 63;
        shift += 1;
      }
    }
  }
  v.s = scale + shift;
  return v;
}

// dst += src << sh (bits) over W words (two's complement); src has n words.
__device__ __forceinline__ void add_shifted(unsigned long long* dst, int W, const unsigned long long* src, int n,
                                            long long sh) {
  const int q = (int)(sh >> 6), r = (int)(sh & 63);
  unsigned long long carry = 0;
  for (int i = 0; i <= n && q + i < W; ++i) {
    const unsigned long long lo = i < n ? src[i] : 0ull;
    const unsigned long long prev = (i > 0 && i - 1 < n) ? src[i - 1] : 0ull;
    const unsigned long long part = r ? ((lo << r) | (prev >> (64 - r))) : lo;
    const unsigned long long a = dst[q + i];
    const unsigned long long t = a + part;
    const unsigned long long c1 = t < a;
    const unsigned long long t2 = t + carry;
    const unsigned long long c2 = t2 < t;
    dst[q + i] = t2;
    carry = c1 + c2;
  }
  for (int i = q + n + 1; i < W && carry; ++i) {
    dst[i] += carry;
    carry = dst[i] == 0;
  }
}
// dst -= src << sh (two's complement over W words)
__device__ __forceinline__ void sub_shifted(unsigned long long* dst, int W, const unsigned long long* src, int n,
                                            long long sh) {
  const int q = (int)(sh >> 6), r = (int)(sh & 63);
  unsigned long long borrow = 0;
  for (int i = 0; i <= n && q + i < W; ++i) {
    const unsigned long long lo = i < n ? src[i] : 0ull;
    const unsigned long long prev = (i > 0 && i - 1 < n) ? src[i - 1] : 0ull;
    const unsigned long long part = r ? ((lo << r) | (prev >> (64 - r))) : lo;
    const unsigned long long a = dst[q + i];
    const unsigned long long t = a - part;
    const unsigned long long b1 = a < part;
    const unsigned long long t2 = t - borrow;
    const unsigned long long b2 = t < borrow;
    dst[q + i] = t2;
    borrow = b1 + b2;
  }
  for (int i = q + n + 1; i < W && borrow; ++i) {
    const unsigned long long a = dst[i];
    dst[i] = a - borrow;
    borrow = a < borrow;
  }
}

// a + sign * b, exact then rounded (sign = -1: subtraction).
__device__ inline Val mp_addsub(const Val& a, const Val& b, int sign, int N) {
  Val bb = b;
  if (sign < 0) bb.neg = !bb.neg;
  if (bb.zero) {
    if (a.zero) {  // (+0) + (-0) = +0 under round to nearest
      Val z = mp_zero();
      z.neg = a.neg && bb.neg;
      return z;
    }
    return a;
  }
  if (a.zero) return bb;
  const long long gap = 64LL * N + 64;
  const long long d = a.s - bb.s;
  if (d > gap) return a;
  if (d < -gap) return bb;
  const long long lo = a.s < bb.s ? a.s : bb.s;
  const int W = 2 * N + 3;
  unsigned long long A[kWideWords] = {}, B[kWideWords] = {};
  add_shifted(A, W, a.m, N, a.s - lo);
  add_shifted(B, W, bb.m, N, bb.s - lo);
  bool neg;
  if (a.neg == bb.neg) {
    add_shifted(A, W, B, W, 0);
    neg = a.neg;
  } else {
    int cmp = 0;
    for (int w = W - 1; w >= 0 && !cmp; --w) cmp = A[w] > B[w] ? 1 : (A[w] < B[w] ? -1 : 0);
    if (cmp == 0) return mp_zero();
    if (cmp > 0) {
      sub_shifted(A, W, B, W, 0);
      neg = a.neg;
    } else {
      sub_shifted(B, W, A, W, 0);
      for (int w = 0; w < W; ++w) A[w] = B[w];
      neg = bb.neg;
    }
  }
  return mp_round(A, W, neg, lo, N);
}

__device__ inline Val mp_mul(const Val& a, const Val& b, int N) {
  if (a.zero || b.zero) {
    Val z = mp_zero();
    z.neg = a.neg != b.neg;
    return z;
  }
  unsigned long long P[2 * kMaxN + 1] = {};
  for (int i = 0; i < N; ++i) {
    unsigned long long carry = 0;
    for (int j = 0; j < N; ++j) {
      const unsigned long long lo = a.m[i] * b.m[j], hi = __umul64hi(a.m[i], b.m[j]);
      const unsigned long long t = P[i + j] + lo;
      const unsigned long long c1 = t < lo;
      const unsigned long long t2 = t + carry;
      const unsigned long long c2 = t2 < t;
      P[i + j] = t2;
      carry = hi + c1 + c2;
    }
    P[i + N] += carry;
  }
  return mp_round(P, 2 * N, a.neg != b.neg, a.s + b.s, N);
}

// sign of a - b: -1, 0, 1.
__device__ inline int mp_cmp(const Val& a, const Val& b, int N) {
  if (a.zero && b.zero) return 0;
  const Val d = mp_addsub(a, b, -1, N);
  return d.zero ? 0 : (d.neg ? -1 : 1);
}

// a - sum_c x[c] y[c] (a given) or sum_c x[c] y[c] (a null), the exact value rounded once.
// x_c at x + c * xs, y_c at y + c * ys (element strides).  *ok = false when the terms do not
// fit the accumulator.
__device__ inline Val mp_dot_sub(const Val* a, const unsigned char* x, long xs, const unsigned char* y, long ys,
                                 int count, int N, bool* ok) {
  const long esz = 8L * N + 8;
  long long lo = LLONG_MAX, hi = LLONG_MIN;
  for (int c = 0; c < count; ++c) {
    const Val xv = mp_load(x + c * xs * esz, N), yv = mp_load(y + c * ys * esz, N);
    if (xv.zero || yv.zero) continue;
    const long long s = xv.s + yv.s;
    lo = s < lo ? s : lo;
    hi = s > hi ? s : hi;
  }
  if (a && !a->zero) {  // the addend's top bit sits where a product term's would at scale s - 64N
    lo = a->s < lo ? a->s : lo;
    hi = (a->s - 64LL * N) > hi ? (a->s - 64LL * N) : hi;
  }
  if (lo == LLONG_MAX) return mp_zero();
  const long long span = hi - lo + 128LL * N + 72;  // largest term's width + log2(count) + sign
  const int W = (int)((span + 63) / 64) + 1;
  if (W > kAccWords) {
    *ok = false;
    return mp_zero();
  }
  unsigned long long acc[kAccWords];
  for (int w = 0; w < W; ++w) acc[w] = 0ull;
  if (a && !a->zero) {
    if (a->neg)
      sub_shifted(acc, W, a->m, N, a->s - lo);
    else
      add_shifted(acc, W, a->m, N, a->s - lo);
  }
  for (int c = 0; c < count; ++c) {
    const Val xv = mp_load(x + c * xs * esz, N), yv = mp_load(y + c * ys * esz, N);
    if (xv.zero || yv.zero) continue;
    unsigned long long P[2 * kMaxN] = {};
    for (int i = 0; i < N; ++i) {
      unsigned long long carry = 0;
      for (int j = 0; j < N; ++j) {
        const unsigned long long plo = xv.m[i] * yv.m[j], phi = __umul64hi(xv.m[i], yv.m[j]);
        const unsigned long long t = P[i + j] + plo;
        const unsigned long long c1 = t < plo;
        const unsigned long long t2 = t + carry;
        const unsigned long long c2 = t2 < t;
        P[i + j] = t2;
        carry = phi + c1 + c2;
      }
      P[i + N] += carry;
    }
    const bool term_neg = (xv.neg != yv.neg) != (a != nullptr);  // a - sum: products subtract
    if (term_neg)
      sub_shifted(acc, W, P, 2 * N, xv.s + yv.s - lo);
    else
      add_shifted(acc, W, P, 2 * N, xv.s + yv.s - lo);
  }
  const bool neg = (acc[W - 1] >> 63) != 0;
  if (neg) {  // magnitude of a two's-complement value
    unsigned long long carry = 1;
    for (int w = 0; w < W; ++w) {
      acc[w] = ~acc[w] + carry;
      carry = (carry && acc[w] == 0) ? 1ull : 0ull;
    }
  }
  return mp_round(acc, W, neg, lo, N);
}

// A value as (double in [0.5, 1), binary exponent): v = f 2^e.
__device__ __forceinline__ double frac_exp(const Val& v, int N, long long* e) {
  const double top = (double)(v.m[N - 1] >> 11) * 0x1p-53;  // the top 53 bits, in [0.5, 1)
  *e = v.s + 64LL * N;
  return v.neg ? -top : top;
}

// f 2^e as a Val (f a finite nonzero double).
__device__ inline Val from_double(double f, long long e, int N) {
  Val v = mp_zero();
  if (f == 0.0) return v;
  int fe = 0;
  const double m = frexp(fabs(f), &fe);  // m in [0.5, 1)
  v.zero = false;
  v.neg = f < 0;
  v.m[N - 1] = (unsigned long long)(m * 0x1p64);  // exact: 53 significant bits
  v.s = e + fe - 64LL * N;
  return v;
}

// mp_dot_sub computed by a whole warp (every lane calls it with the same arguments; every lane
// gets the result): the lanes take the terms c = lane, lane + 32, ..., each accumulates its
// terms exactly in the same fixed-point frame (the warp-wide lowest scale), the partial
// accumulators are added exactly by a shuffle tree, and lane 0 rounds once -- the bits of
// mp_dot_sub, about thirty times faster for long dots.
__device__ inline Val mp_dot_sub_warp(const Val* a, const unsigned char* x, long xs, const unsigned char* y, long ys,
                                      int count, int N, bool* ok) {
  const long esz = 8L * N + 8;
  const int lane = threadIdx.x & 31;
  long long lo = LLONG_MAX, hi = LLONG_MIN;
  for (int c = lane; c < count; c += 32) {
    const Val xv = mp_load(x + c * xs * esz, N), yv = mp_load(y + c * ys * esz, N);
    if (xv.zero || yv.zero) continue;
    const long long s = xv.s + yv.s;
    lo = s < lo ? s : lo;
    hi = s > hi ? s : hi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const long long l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = l2 < lo ? l2 : lo;
    hi = h2 > hi ? h2 : hi;
  }
  if (a && !a->zero) {
    lo = a->s < lo ? a->s : lo;
    hi = (a->s - 64LL * N) > hi ? (a->s - 64LL * N) : hi;
  }
  if (lo == LLONG_MAX) return mp_zero();
  const long long span = hi - lo + 128LL * N + 72;
  const int W = (int)((span + 63) / 64) + 1;
  if (W > kAccWords) {
    *ok = false;
    return mp_zero();
  }
  unsigned long long acc[kAccWords];
  for (int w = 0; w < W; ++w) acc[w] = 0ull;
  if (lane == 0 && a && !a->zero) {
    if (a->neg)
      sub_shifted(acc, W, a->m, N, a->s - lo);
    else
      add_shifted(acc, W, a->m, N, a->s - lo);
  }
  for (int c = lane; c < count; c += 32) {
    const Val xv = mp_load(x + c * xs * esz, N), yv = mp_load(y + c * ys * esz, N);
    if (xv.zero || yv.zero) continue;
    unsigned long long P[2 * kMaxN] = {};
    for (int i = 0; i < N; ++i) {
      unsigned long long carry = 0;
      for (int j = 0; j < N; ++j) {
        const unsigned long long plo = xv.m[i] * yv.m[j], phi = __umul64hi(xv.m[i], yv.m[j]);
        const unsigned long long t = P[i + j] + plo;
        const unsigned long long c1 = t < plo;
        const unsigned long long t2 = t + carry;
        const unsigned long long c2 = t2 < t;
        P[i + j] = t2;
        carry = phi + c1 + c2;
      }
      P[i + N] += carry;
    }
    const bool term_neg = (xv.neg != yv.neg) != (a != nullptr);
    if (term_neg)
      sub_shifted(acc, W, P, 2 * N, xv.s + yv.s - lo);
    else
      add_shifted(acc, W, P, 2 * N, xv.s + yv.s - lo);
  }
  for (int o = 16; o > 0; o >>= 1) {  // exact two's-complement sum of the partial accumulators
    unsigned long long carry = 0;
    for (int w = 0; w < W; ++w) {
      const unsigned long long b = __shfl_down_sync(0xffffffffu, acc[w], o);
      const unsigned long long t = acc[w] + b;
      const unsigned long long c1 = t < b;
      const unsigned long long t2 = t + carry;
      const unsigned long long c2 = t2 < t;
      acc[w] = t2;
      carry = c1 + c2;
    }
  }
  Val r = mp_zero();
  if (lane == 0) {
    const bool neg = (acc[W - 1] >> 63) != 0;
    if (neg) {
      unsigned long long carry = 1;
      for (int w = 0; w < W; ++w) {
        acc[w] = ~acc[w] + carry;
        carry = (carry && acc[w] == 0) ? 1ull : 0ull;
      }
    }
    r = mp_round(acc, W, neg, lo, N);
  }
#pragma unroll
  for (int q = 0; q < kMaxN; ++q) r.m[q] = __shfl_sync(0xffffffffu, r.m[q], 0);
  r.s = __shfl_sync(0xffffffffu, r.s, 0);
  r.neg = __shfl_sync(0xffffffffu, (int)r.neg, 0) != 0;
  r.zero = __shfl_sync(0xffffffffu, (int)r.zero, 0) != 0;
  return r;
}

// 1 / x and 1 / sqrt(x) by Newton's iteration from an FP64 seed (quadratic convergence: four
// steps carry 53 bits past 512): accurate to a few units in the last place, not correctly
// rounded -- used only for the Jacobi rotation parameters, whose orthogonality they bound.
__device__ inline Val mp_recip_approx(const Val& x, int N) {
  long long e;
  const double f = frac_exp(x, N, &e);
  Val y = from_double(1.0 / f, -e, N);
  const Val two = from_double(0.5, 2, N);
  const int steps = N <= 2 ? 2 : (N <= 4 ? 3 : 4);
  for (int k = 0; k < steps; ++k) y = mp_mul(y, mp_addsub(two, mp_mul(x, y, N), -1, N), N);
  return y;
}
__device__ inline Val mp_rsqrt_approx(const Val& x, int N) {  // x > 0
  long long e;
  const double f = frac_exp(x, N, &e);
  // x = f 2^e: 1/sqrt(x) = (1/sqrt(f 2^(e mod 2))) 2^(-(e - e mod 2) / 2)
  const long long odd = e & 1;
  Val y = from_double(1.0 / sqrt(f * (odd ? 2.0 : 1.0)), -((e - odd) / 2), N);
  const Val three = from_double(0.75, 2, N);
  const int steps = N <= 2 ? 2 : (N <= 4 ? 3 : 4);
  for (int k = 0; k < steps; ++k) {
    Val t = mp_addsub(three, mp_mul(x, mp_mul(y, y, N), N), -1, N);
    t.s -= 1;  // / 2
    y = mp_mul(y, t, N);
  }
  return y;
}


// ---- correctly rounded reciprocal, quotient and square root ----
// Each forms the exact integer quotient (or root) and remainder that a binary long division (or
// digit-by-digit root) would give, from a Newton estimate in MpFloat arithmetic corrected exactly:
// the remainder of the estimate is computed in multiword integers and the estimate stepped by
// one until 0 <= remainder < divisor (a few steps: the estimate is within a few units); the
// remainder then becomes the sticky bit of one rounding to 64N bits, ties to even.
constexpr int kQW = kMaxN + 2;      // quotient / root words (N + 1 used)
constexpr int kRW = 2 * kMaxN + 4;  // remainder words, two's complement

// P = A (na words) * B (nb words), na + nb words.
__device__ inline void mul_words(const unsigned long long* A, int na, const unsigned long long* B, int nb,
                                 unsigned long long* P) {
  for (int i = 0; i < na + nb; ++i) P[i] = 0ull;
  for (int i = 0; i < na; ++i) {
    unsigned long long carry = 0;
    for (int j = 0; j < nb; ++j) {
      const unsigned long long lo = A[i] * B[j], hi = __umul64hi(A[i], B[j]);
      const unsigned long long t = P[i + j] + lo;
      const unsigned long long c1 = t < lo;
      const unsigned long long t2 = t + carry;
      const unsigned long long c2 = t2 < t;
      P[i + j] = t2;
      carry = hi + c1 + c2;
    }
    P[i + nb] = carry;
  }
}
// R += M (M n words, zero-extended; R W words, two's complement); R -= M.
__device__ inline void addw(unsigned long long* R, int W, const unsigned long long* M, int n) {
  unsigned long long carry = 0;
  for (int w = 0; w < W; ++w) {
    const unsigned long long m = w < n ? M[w] : 0ull;
    const unsigned long long t = R[w] + m;
    const unsigned long long c1 = t < m;
    const unsigned long long t2 = t + carry;
    carry = c1 + (t2 < t);
    R[w] = t2;
  }
}
__device__ inline void subw(unsigned long long* R, int W, const unsigned long long* M, int n) {
  unsigned long long borrow = 0;
  for (int w = 0; w < W; ++w) {
    const unsigned long long m = w < n ? M[w] : 0ull;
    const unsigned long long t = R[w] - m;
    const unsigned long long b1 = R[w] < m;
    const unsigned long long t2 = t - borrow;
    borrow = b1 + (t < borrow);
    R[w] = t2;
  }
}
// Non-negative R (W words) against M (n words): -1, 0, 1.
__device__ inline int cmpw(const unsigned long long* R, int W, const unsigned long long* M, int n) {
  for (int w = W - 1; w >= 0; --w) {
    const unsigned long long m = w < n ? M[w] : 0ull;
    if (R[w] != m) return R[w] > m ? 1 : -1;
  }
  return 0;
}
__device__ inline void incw(unsigned long long* Q, int W) {
  for (int w = 0; w < W; ++w)
    if (++Q[w] != 0ull) break;
}
__device__ inline void decw(unsigned long long* Q, int W) {
  for (int w = 0; w < W; ++w)
    if (Q[w]-- != 0ull) break;
}
// floor(mantissa(v) 2^(s_v + sh)) into Q (QW words); v > 0.
__device__ inline void to_int_words(const Val& v, int N, long long sh, unsigned long long* Q, int QW) {
  for (int w = 0; w < QW; ++w) Q[w] = 0ull;
  const long long t = v.s + sh;  // Q = M_v 2^t
  if (t >= 0) {
    const int q = (int)(t >> 6), r = (int)(t & 63);
    for (int i = 0; i <= N; ++i) {
      const unsigned long long lo = i < N ? v.m[i] : 0ull, prev = i > 0 ? v.m[i - 1] : 0ull;
      if (q + i < QW) Q[q + i] = r ? ((lo << r) | (prev >> (64 - r))) : lo;
    }
  } else {
    const long long u = -t;
    const int q = (int)(u >> 6), r = (int)(u & 63);
    for (int w = 0; w < QW; ++w) {
      const int i = w + q;
      const unsigned long long lo = i < N ? v.m[i] : 0ull, hi = (i + 1) < N ? v.m[i + 1] : 0ull;
      Q[w] = r ? ((lo >> r) | (hi << (64 - r))) : lo;
    }
  }
}
// Step Q until R = X - Q D lies in [0, D) (D n words; R kRW words, two's complement).
__device__ inline void fix_quotient(unsigned long long* Q, int QW, unsigned long long* R, const unsigned long long* D,
                                    int n) {
  for (int it = 0; it < 4096 && (R[kRW - 1] >> 63); ++it) {
    decw(Q, QW);
    addw(R, kRW, D, n);
  }
  for (int it = 0; it < 4096 && cmpw(R, kRW, D, n) >= 0; ++it) {
    incw(Q, QW);
    subw(R, kRW, D, n);
  }
}
__device__ inline Val round_with_sticky(const unsigned long long* Q, int QW, const unsigned long long* R, bool neg,
                                        long long scale, int N) {
  bool sticky = false;
  for (int w = 0; w < kRW; ++w) sticky = sticky || R[w];
  unsigned long long S[kQW + 1];
  unsigned long long carry = sticky ? 1ull : 0ull;
  for (int w = 0; w <= QW; ++w) {  // S = 2 Q + sticky
    const unsigned long long q = w < QW ? Q[w] : 0ull;
    S[w] = (q << 1) | carry;
    carry = q >> 63;
  }
  return mp_round(S, QW + 1, neg, scale, N);
}

// 1 / d: Q = floor(2^K / M_d), K = 128N + 2, remainder sticky.
__device__ inline Val mp_recip(const Val& d, int N) {
  const int K = 128 * N + 2, QW = N + 1;
  Val m = d;  // M_d 2^-64N in [1/2, 1)
  m.neg = false;
  m.s = -64LL * N;
  const Val y = mp_recip_approx(m, N);  // ~ 2^64N / M_d
  unsigned long long Q[kQW], R[kRW], P[kRW];
  to_int_words(y, N, K - 64LL * N, Q, QW);  // ~ 2^K / M_d
  mul_words(Q, QW, d.m, N, P);               // QW + N words
  for (int w = 0; w < kRW; ++w) R[w] = 0ull;
  R[K >> 6] = 1ull << (K & 63);
  subw(R, kRW, P, QW + N);
  fix_quotient(Q, QW, R, d.m, N);
  return round_with_sticky(Q, QW, R, d.neg, -(long long)K - d.s - 1, N);
}

// a / b: Q = floor(M_a 2^K / M_b), K = 64N + 2, remainder sticky.  b must be nonzero.
__device__ inline Val mp_div(const Val& a, const Val& b, int N) {
  if (a.zero) {
    Val z = mp_zero();
    z.neg = a.neg != b.neg;
    return z;
  }
  const int K = 64 * N + 2, QW = N + 1;
  Val an = a, bn = b;
  an.neg = bn.neg = false;
  an.s = bn.s = -64LL * N;
  const Val q = mp_mul(an, mp_recip_approx(bn, N), N);  // ~ M_a / M_b
  unsigned long long Q[kQW], R[kRW], P[kRW];
  to_int_words(q, N, K, Q, QW);
  mul_words(Q, QW, b.m, N, P);
  for (int w = 0; w < kRW; ++w) R[w] = 0ull;
  for (int w = 0; w < N; ++w) {  // M_a 2^K: K = 64 N + 2
    R[w + N] |= a.m[w] << 2;
    R[w + N + 1] |= a.m[w] >> 62;
  }
  subw(R, kRW, P, QW + N);
  fix_quotient(Q, QW, R, b.m, N);
  return round_with_sticky(Q, QW, R, a.neg != b.neg, a.s - b.s - K - 1, N);
}

// sqrt(a), a >= 0: Y = floor(sqrt(M 2^e)), the radicand 2 (64N + 2) bits wide (e even with s - e),
// remainder sticky.
__device__ inline Val mp_sqrt(const Val& a, int N) {
  if (a.zero) return a;
  const int RB = 64 * N + 2, QW = N + 1;
  long long e = 2LL * RB - 64LL * N;
  if ((a.s - e) & 1) e += 1;
  Val x = a;  // M 2^e
  x.neg = false;
  x.s = e;
  const Val y = mp_mul(x, mp_rsqrt_approx(x, N), N);  // ~ sqrt(M 2^e)
  unsigned long long Y[kQW], R[kRW], P[kRW], T[kQW + 1];
  to_int_words(y, N, 0, Y, QW);
  mul_words(Y, QW, Y, QW, P);  // Y^2, 2 QW words
  for (int w = 0; w < kRW; ++w) R[w] = 0ull;
  {
    const int q = (int)(e >> 6), r = (int)(e & 63);  // X = M 2^e
    for (int i = 0; i <= N; ++i) {
      const unsigned long long lo = i < N ? a.m[i] : 0ull, prev = i > 0 ? a.m[i - 1] : 0ull;
      R[q + i] |= r ? ((lo << r) | (prev >> (64 - r))) : lo;
    }
  }
  subw(R, kRW, P, 2 * QW);
  // 0 <= R = X - Y^2 <= 2Y: while negative Y -= 1, R += 2Y + 1 (new Y); while R > 2Y, R -= 2Y + 1, Y += 1
  for (int it = 0; it < 4096 && (R[kRW - 1] >> 63); ++it) {
    decw(Y, QW);
    unsigned long long c = 1;
    for (int w = 0; w <= QW; ++w) {  // T = 2Y + 1
      const unsigned long long v = w < QW ? Y[w] : 0ull, pv = w > 0 ? Y[w - 1] : 0ull;
      T[w] = (v << 1) | (pv >> 63) | c;
      c = 0;
    }
    addw(R, kRW, T, QW + 1);
  }
  for (int it = 0; it < 4096; ++it) {
    unsigned long long c = 1;
    for (int w = 0; w <= QW; ++w) {  // T = 2Y + 1
      const unsigned long long v = w < QW ? Y[w] : 0ull, pv = w > 0 ? Y[w - 1] : 0ull;
      T[w] = (v << 1) | (pv >> 63) | c;
      c = 0;
    }
    if (cmpw(R, kRW, T, QW + 1) < 0) break;
    subw(R, kRW, T, QW + 1);
    incw(Y, QW);
  }
  return round_with_sticky(Y, QW, R, false, (a.s - e) / 2 - 1, N);
}

}  // namespace mpd
