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
//   mp_recip            binary long division of 2^(128N + 2) by the mantissa, the remainder
//                       folded into a sticky bit
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

// 1 / d: the quotient of 2^K (K = 128N + 2) by the mantissa by binary long division, the
// remainder folded into a sticky low bit.
__device__ inline Val mp_recip(const Val& d, int N) {
  const int K = 128 * N + 2;
  const int QW = 2 * N + 2;
  unsigned long long Q[2 * kMaxN + 2] = {}, R[kMaxN + 1] = {};
  for (int bit = K; bit >= 0; --bit) {
    unsigned long long carry = (bit == K) ? 1ull : 0ull;  // R = 2 R + (bit == K)
    for (int w = 0; w <= N; ++w) {
      const unsigned long long nc = R[w] >> 63;
      R[w] = (R[w] << 1) | carry;
      carry = nc;
    }
    int cmp = R[N] ? 1 : 0;
    for (int w = N - 1; w >= 0 && !cmp; --w) cmp = R[w] > d.m[w] ? 1 : (R[w] < d.m[w] ? -1 : 0);
    if (cmp >= 0) {
      unsigned long long borrow = 0;
      for (int w = 0; w <= N; ++w) {
        const unsigned long long dm = w < N ? d.m[w] : 0ull;
        const unsigned long long t = R[w] - dm;
        const unsigned long long b1 = R[w] < dm;
        const unsigned long long t2 = t - borrow;
        const unsigned long long b2 = t < borrow;
        R[w] = t2;
        borrow = b1 + b2;
      }
      Q[bit >> 6] |= 1ull << (bit & 63);
    }
  }
  bool sticky = false;
  for (int w = 0; w <= N; ++w) sticky = sticky || R[w];
  unsigned long long S[2 * kMaxN + 3] = {};  // S = 2 Q + sticky at scale -(K + s) - 1
  unsigned long long carry = sticky ? 1ull : 0ull;
  for (int w = 0; w < QW + 1; ++w) {
    const unsigned long long q = w < QW ? Q[w] : 0ull;
    S[w] = (q << 1) | carry;
    carry = q >> 63;
  }
  return mp_round(S, QW + 1, d.neg, -(long long)K - d.s - 1, N);
}

// a / b: the quotient of M_a 2^K (K = 64N + 2) by M_b by binary long division, remainder folded
// into a sticky bit.  b must be nonzero.
__device__ inline Val mp_div(const Val& a, const Val& b, int N) {
  if (a.zero) {
    Val z = mp_zero();
    z.neg = a.neg != b.neg;
    return z;
  }
  const int K = 64 * N + 2;
  const int DB = 64 * N + K;  // dividend bits
  unsigned long long Q[2 * kMaxN + 2] = {}, R[kMaxN + 1] = {};
  for (int bit = DB - 1; bit >= 0; --bit) {
    // next dividend bit: bit (bit - K) of M_a, zero below K
    const int src = bit - K;
    unsigned long long carry = (src >= 0) ? ((a.m[src >> 6] >> (src & 63)) & 1ull) : 0ull;
    for (int w = 0; w <= N; ++w) {
      const unsigned long long nc = R[w] >> 63;
      R[w] = (R[w] << 1) | carry;
      carry = nc;
    }
    int cmp = R[N] ? 1 : 0;
    for (int w = N - 1; w >= 0 && !cmp; --w) cmp = R[w] > b.m[w] ? 1 : (R[w] < b.m[w] ? -1 : 0);
    if (cmp >= 0) {
      unsigned long long borrow = 0;
      for (int w = 0; w <= N; ++w) {
        const unsigned long long dm = w < N ? b.m[w] : 0ull;
        const unsigned long long t = R[w] - dm;
        const unsigned long long b1 = R[w] < dm;
        const unsigned long long t2 = t - borrow;
        const unsigned long long b2 = t < borrow;
        R[w] = t2;
        borrow = b1 + b2;
      }
      Q[bit >> 6] |= 1ull << (bit & 63);
    }
  }
  bool sticky = false;
  for (int w = 0; w <= N; ++w) sticky = sticky || R[w];
  const int QW = (DB + 63) / 64;
  unsigned long long S[2 * kMaxN + 3] = {};
  unsigned long long carry = sticky ? 1ull : 0ull;
  for (int w = 0; w < QW + 1; ++w) {
    const unsigned long long q = w < QW ? Q[w] : 0ull;
    S[w] = (q << 1) | carry;
    carry = q >> 63;
  }
  // a / b = (Q + R/M_b) 2^(s_a - s_b - K)
  return mp_round(S, QW + 1, a.neg != b.neg, a.s - b.s - K - 1, N);
}

// sqrt(a), a >= 0: the integer square root of M 2^e (e making the exponent even and the radicand
// 2(64N + 2) bits wide) by the bit-pair restoring method, remainder folded into a sticky bit.
__device__ inline Val mp_sqrt(const Val& a, int N) {
  if (a.zero) return a;
  const int RB = 64 * N + 2;              // root bits
  long long e = 2LL * RB - 64LL * N;      // radicand = M 2^e has 2 RB bits (M has 64N)
  if ((a.s - e) & 1) e += 1;              // a = M 2^s = (M 2^e) 2^(s - e), s - e even
  const int XB = 64 * N + (int)e;         // radicand bit length bound
  unsigned long long Y[kMaxN + 2] = {}, R[kMaxN + 3] = {};
  const int W = N + 2;
  for (int pair = (XB + 1) / 2 - 1; pair >= 0; --pair) {
    // R = 4 R + next two radicand bits (bits 2 pair + 1, 2 pair of M 2^e)
    unsigned long long two = 0;
    for (int t = 1; t >= 0; --t) {
      const long long bit = 2LL * pair + t - e;
      const unsigned long long b = (bit >= 0 && bit < 64LL * N) ? ((a.m[bit >> 6] >> (bit & 63)) & 1ull) : 0ull;
      two = (two << 1) | b;
    }
    unsigned long long carry = two;
    for (int w = 0; w <= W; ++w) {
      const unsigned long long nc = R[w] >> 62;
      R[w] = (R[w] << 2) | carry;
      carry = nc;
    }
    // T = 4 Y + 1; if R >= T: R -= T, Y = 2Y + 1 else Y = 2Y
    unsigned long long T[kMaxN + 3] = {};
    carry = 1;
    for (int w = 0; w <= W; ++w) {
      const unsigned long long y = w < W ? Y[w] : 0ull;
      const unsigned long long prev = (w > 0 && w - 1 < W) ? Y[w - 1] : 0ull;
      T[w] = (y << 2) | (prev >> 62) | carry;
      carry = 0;
    }
    int cmp = 0;
    for (int w = W; w >= 0 && !cmp; --w) cmp = R[w] > T[w] ? 1 : (R[w] < T[w] ? -1 : 0);
    const bool take = cmp >= 0;
    if (take) {
      unsigned long long borrow = 0;
      for (int w = 0; w <= W; ++w) {
        const unsigned long long t1 = R[w] - T[w];
        const unsigned long long b1 = R[w] < T[w];
        const unsigned long long t2 = t1 - borrow;
        const unsigned long long b2 = t1 < borrow;
        R[w] = t2;
        borrow = b1 + b2;
      }
    }
    carry = take ? 1ull : 0ull;
    for (int w = 0; w < W; ++w) {
      const unsigned long long nc = Y[w] >> 63;
      Y[w] = (Y[w] << 1) | carry;
      carry = nc;
    }
  }
  bool sticky = false;
  for (int w = 0; w <= W; ++w) sticky = sticky || R[w];
  unsigned long long S[kMaxN + 3] = {};
  unsigned long long c2 = sticky ? 1ull : 0ull;
  for (int w = 0; w < W + 1; ++w) {
    const unsigned long long y = w < W ? Y[w] : 0ull;
    S[w] = (y << 1) | c2;
    c2 = y >> 63;
  }
  // sqrt(M 2^e 2^(s - e)) = Y' 2^((s - e) / 2), Y' = Y + frac
  return mp_round(S, W + 1, false, (a.s - e) / 2 - 1, N);
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


}  // namespace mpd
