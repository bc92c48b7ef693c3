// Split-precision FP64 products (Ozaki scheme II) on the INT8 tensor cores; see ozaki.cuh.
#include <cmath>
#include <mutex>
#include <stdexcept>

#include "i8_gemm.cuh"
#include "ozaki.cuh"

namespace sdpxg {
namespace {

// Sixteen pairwise coprime moduli <= 256 (256 = 2^8, 255 = 3*5*17, 253 = 11*23, 247 = 13*19,
// 217 = 7*31, the rest prime): their product P is about 2^126.4.  A constant function of the
// index, so that in the kernels' unrolled loops every reduction is by a literal modulus.
__host__ __device__ constexpr int oz_mod(int t) {
  return t == 0 ? 256 : t == 1 ? 255 : t == 2 ? 253 : t == 3 ? 251 : t == 4 ? 247 : t == 5 ? 241 : t == 6 ? 239
       : t == 7 ? 233 : t == 8 ? 229 : t == 9 ? 227 : t == 10 ? 223 : t == 11 ? 217 : t == 12 ? 211
       : t == 13 ? 199 : t == 14 ? 197 : 193;
}
constexpr int kModuli[kOzMod] = {oz_mod(0),  oz_mod(1),  oz_mod(2),  oz_mod(3),  oz_mod(4),  oz_mod(5),
                                 oz_mod(6),  oz_mod(7),  oz_mod(8),  oz_mod(9),  oz_mod(10), oz_mod(11),
                                 oz_mod(12), oz_mod(13), oz_mod(14), oz_mod(15)};

// Garner tables, passed by value: inv[t] = (p_0 ... p_{t-1})^-1 mod p_t, pre[s][t] =
// (p_0 ... p_{s-1}) mod p_t.
struct OzTables {
  int p[kOzMod];
  int inv[kOzMod];
  short pre[kOzMod][kOzMod];
};

const OzTables& tables() {
  static OzTables T;
  static std::once_flag once;
  std::call_once(once, [] {
    for (int t = 0; t < kOzMod; ++t) {
      const int p = kModuli[t];
      T.p[t] = p;
      long prod = 1;
      for (int s = 0; s < kOzMod; ++s) {
        T.pre[s][t] = (short)(s <= t ? prod : 0);
        if (s < t) prod = prod * (kModuli[s] % p) % p;
      }
      // prod = (p_0 ... p_{t-1}) mod p; its inverse by search (p <= 256)
      int inv = 1;
      for (int x = 1; x < p; ++x)
        if ((long)x * prod % p == 1) {
          inv = x;
          break;
        }
      T.inv[t] = t == 0 ? 1 : inv;
    }
  });
  return T;
}

double log2_product() {
  double s = 0;
  for (int p : kModuli) s += std::log2((double)p);
  return s;
}

// Per-line maxima of |X| as FP64 bit patterns (non-negative doubles order like their bits), by
// atomicMax into a zeroed array; a non-finite entry sets SDPXG_ST_NONFINITE.
// ALONG_K (sk == 1): one warp per line reading along k.  Otherwise (consecutive lines
// consecutive in memory): CTAs of 32 lines x 8 warps over a 256-wide k range, lanes along lines.
template <bool ALONG_K>
__global__ void k_oz_amax(const double* __restrict__ X, int rows, int K, long sr, long sk,
                          unsigned long long* __restrict__ amax, uint32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double m = 0.0;
  bool bad = false;
  int row;
  if (ALONG_K) {
    row = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (row >= rows) return;
    for (int k = lane; k < K; k += 32) {
      const double v = X[row * sr + k];
      bad |= !isfinite(v);
      m = fmax(m, fabs(v));
    }
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    bad = __any_sync(0xffffffffu, bad);
    if (lane != 0) return;
  } else {
    __shared__ double part[8][32];
    row = blockIdx.x * 32 + lane;
    const int k0 = blockIdx.y * 256, k1 = min(K, k0 + 256);
    if (row < rows)
      for (int k = k0 + warp; k < k1; k += 8) {
        const double v = X[row + (long)k * sk];
        bad |= !isfinite(v);
        m = fmax(m, fabs(v));
      }
    part[warp][lane] = bad ? __longlong_as_double(0x7ff8000000000000LL) : m;
    __syncthreads();
    if (warp != 0 || row >= rows) return;
    m = 0.0;
    for (int w = 0; w < 8; ++w) {
      const double v = part[w][lane];
      bad |= isnan(v);
      m = isnan(v) ? m : fmax(m, v);
    }
  }
  if (bad) {
    atomicOr(status, SDPXG_ST_NONFINITE);
    m = __longlong_as_double(0x7ff0000000000000LL);
  }
  atomicMax(amax + row, (unsigned long long)__double_as_longlong(m));
}

// Shift of a line with maximum `bits`: b - 1 - floor(log2 max) puts the line below 2^b; 0 for a
// zero or non-finite line.
__device__ __forceinline__ int oz_shift(unsigned long long bits, int b) {
  const double m = __longlong_as_double((long long)bits);
  return (m > 0.0 && isfinite(m)) ? b - 1 - ilogb(m) : 0;
}

// Symmetric residue in [-(p-1)/2, p/2] of the integer (neg ? -1 : 1) (hi 2^32 + lo), hi < 2^30:
// 32-bit reductions by the literal modulus p (the caller's loop is unrolled).
__device__ __forceinline__ int oz_sym_residue(uint32_t hi, uint32_t lo, bool neg, const int p) {
  const uint32_t c = (uint32_t)((1ull << 32) % (unsigned)p);
  int r = (int)(((hi % (unsigned)p) * c + lo % (unsigned)p) % (unsigned)p);
  if (neg && r) r = p - r;
  if (r > p / 2) r -= p;
  return r;
}

// Residues of the quantised lines as signed-byte planes: out[(l * Rpad + x) * Kld + k] =
// rint(X(x, k) 2^shift[x]) mod p_l (symmetric), zeros in the padding.  One CTA per tile of
// 32 lines x 128 k, staged in shared memory so that both the reads (along whichever index is
// contiguous) and the 16-byte plane writes are coalesced.
constexpr int kResPitch = 144;  // bytes per staged line (128 + 16: 16-byte aligned rows)
__global__ void __launch_bounds__(256) k_oz_residues(const double* __restrict__ X, int rows, int K, long sr, long sk,
                                                     const unsigned long long* __restrict__ amax, int b,
                                                     int8_t* __restrict__ out, int Rpad, int Kld) {
  extern __shared__ int8_t tile[];  // [kOzMod][32][kResPitch]
  const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 128;
  const bool along_k = (sk == 1);
  for (int e = threadIdx.x; e < 32 * 128; e += 256) {
    const int rr = along_k ? e / 128 : e % 32;
    const int kk = along_k ? e % 128 : e / 32;
    const int x = r0 + rr, k = k0 + kk;
    long long q = 0;
    if (x < rows && k < K) {
      const double v = X[(long)x * sr + (long)k * sk];
      if (isfinite(v)) q = llrint(ldexp(v, oz_shift(amax[x], b)));
    }
    const unsigned long long u = (unsigned long long)(q < 0 ? -q : q);
    const uint32_t hi = (uint32_t)(u >> 32), lo = (uint32_t)u;
#pragma unroll
    for (int l = 0; l < kOzMod; ++l)
      tile[(l * 32 + rr) * kResPitch + kk] = (int8_t)oz_sym_residue(hi, lo, q < 0, oz_mod(l));
  }
  __syncthreads();
  const int rr = threadIdx.x >> 3, c = threadIdx.x & 7;
#pragma unroll 4
  for (int l = 0; l < kOzMod; ++l) {
    const uint4 v = *reinterpret_cast<const uint4*>(tile + (l * 32 + rr) * kResPitch + 16 * c);
    *reinterpret_cast<uint4*>(out + ((size_t)l * Rpad + r0 + rr) * Kld + k0 + 16 * c) = v;
  }
}

// C(i, j) = alpha * 2^-(sL_i + sR_j) * X_ij + beta * C(i, j), X_ij the integer product rebuilt
// from its residues by Garner's algorithm with symmetric digits v_t in [-p_t/2, p_t/2]
// (X = v_0 + p_0 (v_1 + p_1 (v_2 + ...)), exact for |X| < P/2) and evaluated by Horner's rule
// in double-double arithmetic (error-free FMA product and two-sum per step: about 2^-100
// relative), so the FP64 value of X is its correct rounding except within 2^-100 of a tie.
__global__ void k_oz_garner(const int8_t* __restrict__ PC, long plane, int M, int N,
                            const unsigned long long* __restrict__ aL, const unsigned long long* __restrict__ aR,
                            int b, OzTables T, double alpha, double beta, double* __restrict__ C, long ldc,
                            int upper_only) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)M * N) return;
  const int i = (int)(idx % M), j = (int)(idx / M);
  if (upper_only && i > j) return;
  int v[kOzMod];
#pragma unroll
  for (int t = 0; t < kOzMod; ++t) {
    const int p = oz_mod(t);
    int r = (int)PC[t * plane + idx] % p;
    if (r < 0) r += p;
    int u = 0;
#pragma unroll
    for (int s = 0; s < t; ++s) u += v[s] * (int)T.pre[s][t];
    int d = (r - u) % p;
    if (d < 0) d += p;
    d = d * T.inv[t] % p;
    if (d > p / 2) d -= p;
    v[t] = d;
  }
  double h = (double)v[kOzMod - 1], lo = 0.0;
#pragma unroll
  for (int t = kOzMod - 2; t >= 0; --t) {
    const double p = (double)oz_mod(t), vt = (double)v[t];
    const double ph = h * p, pe = fma(h, p, -ph);  // h p = ph + pe exactly
    const double s = ph + vt, bb = s - ph;
    const double se = (ph - (s - bb)) + (vt - bb);  // ph + vt = s + se exactly
    const double tt = se + pe + lo * p;
    h = s + tt;
    lo = tt - (h - s);
  }
  double x = ldexp(h + lo, -(oz_shift(aL[i], b) + oz_shift(aR[j], b)));
  double* c = C + i + (long)j * ldc;
  *c = beta == 0.0 ? alpha * x : fma(alpha, x, beta * *c);
}

template <typename T>
void grow(DevBuf<T>& b, size_t n) {
  if (b.n < std::max<size_t>(n, 1)) b.alloc(std::max<size_t>(n, 1));
}

void line_maxima(const double* X, int rows, int K, long sr, long sk, unsigned long long* amax, uint32_t* status,
                 cudaStream_t st) {
  check(cudaMemsetAsync(amax, 0, (size_t)rows * sizeof(unsigned long long), st), "memset");
  if (sk == 1) {
    ++g_launches, k_oz_amax<true><<<(unsigned)(((long)rows * 32 + 255) / 256), 256, 0, st>>>(X, rows, K, sr, sk,
                                                                                              amax, status);
  } else {
    if (sr != 1) throw std::invalid_argument("split GEMM: one operand index must be contiguous");
    ++g_launches, k_oz_amax<false><<<dim3((unsigned)((rows + 31) / 32), (unsigned)((K + 255) / 256)), 256, 0, st>>>(
        X, rows, K, sr, sk, amax, status);
  }
}

}  // namespace

int ozaki_bits(int K) {
  int lg = 0;
  while ((1L << lg) < std::max(K, 1)) ++lg;
  const int b = (int)std::floor((log2_product() - 2.0 - lg) / 2.0);
  return std::min(b, 62);
}

void ozaki_gemm(OzakiWorkspace& ws, cudaStream_t st, int M, int N, int K, const double* L, long l_sr, long l_sk,
                const double* R, long r_sr, long r_sk, double alpha, double beta, double* C, long ldc,
                int upper_only) {
  if (M <= 0 || N <= 0) return;
  if (K <= 0 || K > (1 << 16)) throw std::invalid_argument("split GEMM: K must be in 1..65536");
  if (!L || !R || !C) throw std::invalid_argument("split GEMM: null operand");
  const OzTables& T = tables();
  if (!ws.init) {
    grow(ws.moduli, kOzMod);
    ws.moduli.upload(kModuli, kOzMod, st);
    grow(ws.status, 1);
    grow(ws.err, 1);
    check(cudaMemsetAsync(ws.status.p, 0, sizeof(uint32_t), st), "memset");
    check(cudaMemsetAsync(ws.err.p, 0, sizeof(int), st), "memset");
    static std::once_flag attr;
    std::call_once(attr, [] {
      check(cudaFuncSetAttribute(k_oz_residues, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzMod * 32 * kResPitch),
            "oz residues smem");
    });
    ws.init = true;
  }
  const int b = ozaki_bits(K);
  const int Mpad = (M + 127) / 128 * 128, Npad = (N + 255) / 256 * 256, Kld = (K + 127) / 128 * 128;
  grow(ws.amaxL, M);
  grow(ws.amaxR, N);
  grow(ws.PL, (size_t)kOzMod * Mpad * Kld);
  grow(ws.PR, (size_t)kOzMod * Npad * Kld);
  grow(ws.PC, (size_t)kOzMod * M * N);
  line_maxima(L, M, K, l_sr, l_sk, ws.amaxL, ws.status, st);
  line_maxima(R, N, K, r_sr, r_sk, ws.amaxR, ws.status, st);
  const size_t rsm = (size_t)kOzMod * 32 * kResPitch;
  ++g_launches, k_oz_residues<<<dim3(Kld / 128, Mpad / 32), 256, rsm, st>>>(L, M, K, l_sr, l_sk, ws.amaxL, b, ws.PL,
                                                                            Mpad, Kld);
  ++g_launches, k_oz_residues<<<dim3(Kld / 128, Npad / 32), 256, rsm, st>>>(R, N, K, r_sr, r_sk, ws.amaxR, b, ws.PR,
                                                                            Npad, Kld);
  I8GemmArgs ga;
  ga.Mpad = Mpad; ga.Npad = Npad; ga.Kld = Kld; ga.k0 = 0; ga.Kpad = Kld;
  ga.m = M; ga.n = N; ga.L = kOzMod; ga.moduli = ws.moduli; ga.upper_only = upper_only;
  ga.out = ws.PC.p; ga.plane = (long)M * N; ga.err = ws.err.p;
  launch_i8_gemm(1, ws.PL, ws.PR, ga, st);
  ++g_launches, k_oz_garner<<<(unsigned)(((long)M * N + 255) / 256), 256, 0, st>>>(
      ws.PC, (long)M * N, M, N, ws.amaxL, ws.amaxR, b, T, alpha, beta, C, ldc, upper_only);
  check(cudaGetLastError(), "split GEMM launch");
}

}  // namespace sdpxg
