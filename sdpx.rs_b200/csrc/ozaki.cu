// Split-precision FP64 products (Ozaki scheme II) on the INT8 tensor cores; see ozaki.cuh.
#include <cmath>
#include <mutex>
#include <stdexcept>

#include "i8_gemm.cuh"
#include "ozaki.cuh"

namespace sdpxg {
namespace {

// Sixteen pairwise coprime moduli <= 256 (256 = 2^8, 255 = 3*5*17, 253 = 11*23, 247 = 13*19,
// 217 = 7*31, the rest prime): their product P is about 2^126.4.
constexpr int kModuli[kOzMod] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193};

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

// Per-line power-of-two shifts: shift[x] = b - 1 - floor(log2 max_k |X(x, k)|) (0 for a zero
// line), so every entry of the line scaled by 2^shift lies below 2^b in magnitude.
// ALONG_K: one warp per line reading along k (sk == 1); otherwise one thread per line
// (consecutive lines are consecutive in memory, sr == 1).
template <bool ALONG_K>
__global__ void k_oz_shift(const double* __restrict__ X, int rows, int K, long sr, long sk, int b,
                           int* __restrict__ shift, uint32_t* __restrict__ status) {
  const long gt = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int row = ALONG_K ? (int)(gt >> 5) : (int)gt;
  const int lane = threadIdx.x & 31;
  if (row >= rows) return;
  double amax = 0.0;
  bool bad = false;
  if (ALONG_K) {
    for (int k = lane; k < K; k += 32) {
      const double v = X[row * sr + (long)k * sk];
      bad |= !isfinite(v);
      amax = fmax(amax, fabs(v));
    }
    for (int o = 16; o; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    bad = __any_sync(0xffffffffu, bad);
  } else {
    for (int k = 0; k < K; ++k) {
      const double v = X[row * sr + (long)k * sk];
      bad |= !isfinite(v);
      amax = fmax(amax, fabs(v));
    }
  }
  if (!ALONG_K || lane == 0) {
    shift[row] = (amax > 0.0 && isfinite(amax)) ? (b - 1 - ilogb(amax)) : 0;
    if (bad) atomicOr(status, SDPXG_ST_NONFINITE);
  }
}

// Residues of the quantised lines as signed-byte planes: out[(l * Rpad + x) * Kld + k] =
// rint(X(x, k) 2^shift[x]) mod p_l (symmetric), zeros in the padding.  One CTA per tile of
// 32 lines x 128 k, staged in shared memory so that both the reads (along whichever index is
// contiguous) and the 16-byte plane writes are coalesced.
constexpr int kResPitch = 144;  // bytes per staged line (128 + 16: 16-byte aligned rows)
__global__ void __launch_bounds__(256) k_oz_residues(const double* __restrict__ X, int rows, int K, long sr, long sk,
                                                     const int* __restrict__ shift, OzTables T,
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
      if (isfinite(v)) q = llrint(ldexp(v, shift[x]));
    }
#pragma unroll
    for (int l = 0; l < kOzMod; ++l) {
      const int p = T.p[l];
      int r = (int)(q % p);
      if (r > p / 2) r -= p;
      if (r < -(p / 2)) r += p;
      tile[(l * 32 + rr) * kResPitch + kk] = (int8_t)r;
    }
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
__global__ void k_oz_garner(const int8_t* __restrict__ PC, long plane, int M, int N, const int* __restrict__ sL,
                            const int* __restrict__ sR, OzTables T, double alpha, double beta,
                            double* __restrict__ C, long ldc, int upper_only) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)M * N) return;
  const int i = (int)(idx % M), j = (int)(idx / M);
  if (upper_only && i > j) return;
  int v[kOzMod];
#pragma unroll
  for (int t = 0; t < kOzMod; ++t) {
    const int p = T.p[t];
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
    const double p = (double)T.p[t], vt = (double)v[t];
    const double ph = h * p, pe = fma(h, p, -ph);  // h p = ph + pe exactly
    const double s = ph + vt, bb = s - ph;
    const double se = (ph - (s - bb)) + (vt - bb);  // ph + vt = s + se exactly
    const double tt = se + pe + lo * p;
    h = s + tt;
    lo = tt - (h - s);
  }
  double x = ldexp(h + lo, -(sL[i] + sR[j]));
  double* c = C + i + (long)j * ldc;
  *c = beta == 0.0 ? alpha * x : fma(alpha, x, beta * *c);
}

template <typename T>
void grow(DevBuf<T>& b, size_t n) {
  if (b.n < std::max<size_t>(n, 1)) b.alloc(std::max<size_t>(n, 1));
}

void line_shifts(const double* X, int rows, int K, long sr, long sk, int b, int* shift, uint32_t* status,
                 cudaStream_t st) {
  if (sk == 1) {
    ++g_launches, k_oz_shift<true><<<(unsigned)(((long)rows * 32 + 255) / 256), 256, 0, st>>>(X, rows, K, sr, sk, b,
                                                                                               shift, status);
  } else {
    ++g_launches, k_oz_shift<false><<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(X, rows, K, sr, sk, b, shift,
                                                                                    status);
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
  grow(ws.shiftL, M);
  grow(ws.shiftR, N);
  grow(ws.PL, (size_t)kOzMod * Mpad * Kld);
  grow(ws.PR, (size_t)kOzMod * Npad * Kld);
  grow(ws.PC, (size_t)kOzMod * M * N);
  line_shifts(L, M, K, l_sr, l_sk, b, ws.shiftL, ws.status, st);
  line_shifts(R, N, K, r_sr, r_sk, b, ws.shiftR, ws.status, st);
  const size_t rsm = (size_t)kOzMod * 32 * kResPitch;
  ++g_launches, k_oz_residues<<<dim3(Kld / 128, Mpad / 32), 256, rsm, st>>>(L, M, K, l_sr, l_sk, ws.shiftL, T, ws.PL,
                                                                            Mpad, Kld);
  ++g_launches, k_oz_residues<<<dim3(Kld / 128, Npad / 32), 256, rsm, st>>>(R, N, K, r_sr, r_sk, ws.shiftR, T, ws.PR,
                                                                            Npad, Kld);
  I8GemmArgs ga;
  ga.Mpad = Mpad; ga.Npad = Npad; ga.Kld = Kld; ga.k0 = 0; ga.Kpad = Kld;
  ga.m = M; ga.n = N; ga.L = kOzMod; ga.moduli = ws.moduli; ga.upper_only = upper_only;
  ga.out = ws.PC.p; ga.plane = (long)M * N; ga.err = ws.err.p;
  launch_i8_gemm(1, ws.PL, ws.PR, ga, st);
  ++g_launches, k_oz_garner<<<(unsigned)(((long)M * N + 255) / 256), 256, 0, st>>>(
      ws.PC, (long)M * N, M, N, ws.shiftL, ws.shiftR, T, alpha, beta, C, ldc, upper_only);
  check(cudaGetLastError(), "split GEMM launch");
}

}  // namespace sdpxg
