// Modular INT8 tensor-core GEMM on sm_100a: one CTA per (128-row tile, tile_n-column tile,
// modulus).  Warp-specialised, non-persistent:
//   warp 4 (one lane)  TMA producer: K-blocks of 128 bytes of every digit plane of A and B into a
//                      ring of shared-memory stages (128-byte swizzle), completion counted in
//                      bytes on the stage's `full` mbarrier;
//   warp 5 (one lane)  MMA issuer: 4 x tcgen05.mma.kind::i8 (K = 32 bytes each) per digit pair and
//                      stage into TMEM accumulators (one per digit sum), tcgen05.commit frees the
//                      stage; a last commit signals the epilogue;
//   warps 0-3          epilogue: tcgen05.ld of the accumulators (warp w reads TMEM lanes
//                      32w..32w+31 = output rows), reduction modulo the tile's modulus, coalesced
//                      stores (consecutive lanes = consecutive rows of a column-major plane).
// Every wait is bounded; a wait that gives up sets bit 0 of args.err, the other roles stop at
// their next wait, outstanding TMA copies are drained (bounded) and TMEM is released before exit.
#include <cuda.h>

#include <array>
#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <stdexcept>
#include <cstdio>
#include <string>

#include "device.cuh"
#include "i8_gemm.cuh"
#include "tc05.cuh"

namespace sdpxg {
namespace {

constexpr int kBM = 128;     // rows per tile (MMA M)
constexpr int kKB = 128;     // K bytes per stage (one 128-byte swizzle row)
constexpr int kThreads = 192;

// Tile configurations: variant 0 (the default), variant 1 (half the tile width, deeper stage
// ring) and variant 2 (two CTAs per SM: a two-stage ring each, so that one CTA's epilogue overlaps
// the other's main loop); the autotuner picks per shape class.  Every variant gives the same bits.
constexpr int kVariants = 3;
template <int DIGITS, int VAR>
struct Cfg;
template <>
struct Cfg<1, 0> {
  static constexpr int BN = 256, STAGES = 4, NACC = 1, TMEM_COLS = 256, CTAS = 1;
};
template <>
struct Cfg<1, 1> {
  static constexpr int BN = 128, STAGES = 6, NACC = 1, TMEM_COLS = 128, CTAS = 1;
};
template <>
struct Cfg<1, 2> {
  static constexpr int BN = 256, STAGES = 2, NACC = 1, TMEM_COLS = 256, CTAS = 2;
};
template <>
struct Cfg<2, 0> {
  static constexpr int BN = 128, STAGES = 3, NACC = 3, TMEM_COLS = 512, CTAS = 1;
};
template <>
struct Cfg<2, 1> {
  static constexpr int BN = 64, STAGES = 4, NACC = 3, TMEM_COLS = 256, CTAS = 1;
};
template <>
struct Cfg<2, 2> {
  static constexpr int BN = 64, STAGES = 2, NACC = 3, TMEM_COLS = 256, CTAS = 2;
};

template <int DIGITS, int VAR>
constexpr int stage_bytes() {
  return DIGITS * (kBM * kKB + Cfg<DIGITS, VAR>::BN * kKB);
}
template <int DIGITS, int VAR>
constexpr size_t smem_bytes() {
  // stages, then 2 * STAGES + 1 mbarriers, the TMEM address, the abort flag and the consumed
  // count, plus 1024 bytes to align the stage ring to the swizzle atom
  return (size_t)Cfg<DIGITS, VAR>::STAGES * stage_bytes<DIGITS, VAR>() + (2 * Cfg<DIGITS, VAR>::STAGES + 1) * 8 + 16 +
         1024;
}

__device__ __forceinline__ void give_up(volatile int* abort, int* err) {
  *abort = 1;
  if (err) atomicOr(err, 1);
}

// Symmetric residue of v modulo p (|v| < 2^31, 2 <= p <= 256) in [-(p-1)/2, p/2]: the quotient
// rounded from an FP64 product (v and v/p are exact to far below 1/2 in FP64, so it is the
// nearest integer to v/p up to a tie), the remainder in 32-bit integers (exact modulo 2^32, and
// the true remainder is small), then at most one correction each way.
__device__ __forceinline__ int sym_mod_small(int v, int p, double pinv) {
  const int q = __double2int_rn((double)v * pinv);
  int r = v - q * p;
  if (r > p / 2) r -= p;
  if (r < -((p - 1) / 2)) r += p;
  return r;
}
// Residue of v modulo p in [0, p) for |v| < 2^50, p < 2^15: FP64 quotient as above (v exact in
// FP64), remainder in 64-bit integers, one correction.
__device__ __forceinline__ int mod_wide(long long v, int p, double pinv) {
  const long long q = __double2ll_rn((double)v * pinv);
  long long r = v - q * p;
  if (r < 0) r += p;
  if (r >= p) r -= p;
  return (int)r;
}

template <int DIGITS, int VAR>
__global__ void __launch_bounds__(kThreads, Cfg<DIGITS, VAR>::CTAS)
    k_i8_mod_gemm(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, I8GemmArgs a) {
  constexpr int BN = Cfg<DIGITS, VAR>::BN, STAGES = Cfg<DIGITS, VAR>::STAGES, NACC = Cfg<DIGITS, VAR>::NACC;
  constexpr int TCOLS = Cfg<DIGITS, VAR>::TMEM_COLS;
  constexpr int SB = stage_bytes<DIGITS, VAR>();
  constexpr int A_TILE = kBM * kKB, B_TILE = BN * kKB;
  const int tm = blockIdx.x, tn = blockIdx.y, l = blockIdx.z;
  if (a.upper_only && tm * kBM > tn * BN + BN - 1) return;  // every entry of the tile has i > j

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)STAGES * SB);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* consumed = reinterpret_cast<int*>(tmem_slot + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc05::mbar_init(&full[s], 1);
      tc05::mbar_init(&empty[s], 1);
    }
    tc05::mbar_init(done, 1);
    *abort = 0;
    *consumed = 0;
    tc05::fence_barrier_init();
  }
  if (warp == 0) {
    __syncwarp();  // the .sync.aligned allocation needs the whole warp converged
    tc05::tmem_alloc(tmem_slot, TCOLS);
    tc05::tmem_relinquish();
  }
  tc05::tc_fence_before();
  __syncthreads();
  tc05::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nk = a.Kpad / kKB;
  int issued = 0;

  if (warp == 4 && lane == 0) {  // ---- TMA producer ----
    tc05::tma_prefetch_map(&tA);
    tc05::tma_prefetch_map(&tB);
    for (int it = 0; it < nk; ++it) {
      const int s = it % STAGES, r = it / STAGES;
      if (r > 0 && !tc05::mbar_wait(&empty[s], (r - 1) & 1, abort)) {
        give_up(abort, a.err);
        break;
      }
      tc05::mbar_arrive_expect_tx(&full[s], SB);
      uint8_t* st = smem + (size_t)s * SB;
      const int x = a.k0 + it * kKB;
#pragma unroll
      for (int d = 0; d < DIGITS; ++d) {
        tc05::tma_load_2d(st + d * A_TILE, &tA, &full[s], x, (l * DIGITS + d) * a.Mpad + tm * kBM);
        tc05::tma_load_2d(st + DIGITS * A_TILE + d * B_TILE, &tB, &full[s], x,
                          (l * DIGITS + d) * a.Npad + tn * BN);
      }
      issued = it + 1;
    }
  } else if (warp == 5 && lane == 0) {  // ---- MMA issuer ----
    constexpr uint32_t idesc = tc05::idesc_i8(kBM, BN);
    int it = 0;
    for (; it < nk; ++it) {
      const int s = it % STAGES, r = it / STAGES;
      if (!tc05::mbar_wait(&full[s], r & 1, abort)) {
        give_up(abort, a.err);
        break;
      }
      tc05::tc_fence_after();
      const uint32_t st = tc05::smem_u32(smem + (size_t)s * SB);
#pragma unroll
      for (int kk = 0; kk < kKB / 32; ++kk) {
        const uint32_t first = (it == 0 && kk == 0) ? 0u : 1u;
        if (DIGITS == 1) {
          const uint64_t ad = tc05::sdesc_k_sw128(st) + 2 * kk;
          const uint64_t bd = tc05::sdesc_k_sw128(st + A_TILE) + 2 * kk;
          tc05::mma_i8(tmem, ad, bd, idesc, first);
        } else {
          const uint64_t a0 = tc05::sdesc_k_sw128(st) + 2 * kk;
          const uint64_t a1 = tc05::sdesc_k_sw128(st + A_TILE) + 2 * kk;
          const uint64_t b0 = tc05::sdesc_k_sw128(st + 2 * A_TILE) + 2 * kk;
          const uint64_t b1 = tc05::sdesc_k_sw128(st + 2 * A_TILE + B_TILE) + 2 * kk;
          tc05::mma_i8(tmem, a0, b0, idesc, first);               // D0 += lo lo
          tc05::mma_i8(tmem + BN, a0, b1, idesc, first);          // D1 += lo hi
          tc05::mma_i8(tmem + BN, a1, b0, idesc, 1u);             // D1 += hi lo
          tc05::mma_i8(tmem + 2 * BN, a1, b1, idesc, first);      // D2 += hi hi
        }
      }
      tc05::mma_commit(&empty[s]);
    }
    *consumed = it;
    tc05::mma_commit(done);  // completes once every MMA issued above has
  } else if (warp < 4) {  // ---- epilogue ----
    const bool waited = tc05::mbar_wait(done, 0, abort);
    if (!waited) give_up(abort, a.err);
    // warp-uniform decision: tcgen05.ld is .sync.aligned
    const bool go = __all_sync(0xffffffffu, waited && !*abort);
    tc05::tc_fence_after();
    if (go) {
      const int row = warp * 32 + lane;
      const int i = tm * kBM + row;
      const int p = a.moduli[l];
      const double pinv = 1.0 / (double)p;
      const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t acc[NACC][32];
#pragma unroll
        for (int q = 0; q < NACC; ++q) tc05::tmem_ld32(lane_base + q * BN + c0, acc[q]);
        tc05::tmem_ld_wait();
        const int j0 = tn * BN + c0;
        if (i < a.m) {
          if (DIGITS == 1) {
            int8_t* out = static_cast<int8_t*>(a.out) + (long)l * a.plane;
#pragma unroll
            for (int q = 0; q < 32; ++q) {
              const int j = j0 + q;
              if (j < a.n) {
                out[(long)j * a.m + i] = (int8_t)sym_mod_small((int)acc[0][q], p, pinv);
              }
            }
          } else {
            int* out = static_cast<int*>(a.out) + (long)l * a.plane;
#pragma unroll
            for (int q = 0; q < 32; ++q) {
              const int j = j0 + q;
              if (j < a.n) {
                long long v = (long long)(int)acc[0][q] + ((long long)(int)acc[NACC > 1 ? 1 : 0][q] << 8) +
                              ((long long)(int)acc[NACC > 2 ? 2 : 0][q] << 16);
                long long r = mod_wide(v, p, pinv);
                if (a.accumulate) {
                  r += out[(long)j * a.m + i];
                  if (r >= p) r -= p;
                }
                out[(long)j * a.m + i] = (int)r;
              }
            }
          }
        }
      }
    }
  }
  __syncthreads();
  if (warp == 4 && lane == 0) {  // copies the MMA issuer never consumed must land before exit
    for (int it = *consumed; it < issued; ++it) tc05::mbar_wait(&full[it % STAGES], (it / STAGES) & 1, nullptr);
  }
  tc05::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc05::tc_fence_after();
    tc05::tmem_dealloc(tmem, TCOLS);
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  if (!fn) throw CudaError("cuTensorMapEncodeTiled is not available");
  return fn;
}

// Byte matrix of `rows` rows of `kpad` bytes (row stride kpad), boxes of box_rows x 128 bytes,
// 128-byte swizzle.
CUtensorMap byte_map(const int8_t* base, long rows, int kpad, int box_rows) {
  if (reinterpret_cast<uintptr_t>(base) % 16) throw std::invalid_argument("TMA base not 16-byte aligned");
  if (kpad % kKB) throw std::invalid_argument("K padding must be a multiple of 128");
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)kpad};
  const cuuint32_t box[2] = {(cuuint32_t)kKB, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

// Optional CUDA-event timing of every launch (sdpx_b200_set_i8_timing): events on the launch
// stream around the kernel, host-synchronised, so only for measurement runs.
std::atomic<int> g_i8_timing{0};
std::mutex g_i8_mu;
double g_i8_ms = 0.0, g_i8_ops = 0.0, g_i8_alg_ops = 0.0;
uint64_t g_i8_count = 0;

// One launch of variant VAR (returns after queueing; with timing on, after the event).
template <int DIGITS, int VAR>
void launch_variant(const int8_t* A, const int8_t* B, const I8GemmArgs& a, cudaStream_t st, float* ms_out) {
  constexpr int BN = Cfg<DIGITS, VAR>::BN;
  static std::once_flag attr;
  std::call_once(attr, [] {
    check(cudaFuncSetAttribute(k_i8_mod_gemm<DIGITS, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem_bytes<DIGITS, VAR>()),
          "i8 gemm smem attribute");
  });
  const CUtensorMap ta = byte_map(A, (long)a.L * DIGITS * a.Mpad, a.Kld, kBM);
  const CUtensorMap tb = byte_map(B, (long)a.L * DIGITS * a.Npad, a.Kld, BN);
  const dim3 grid(a.Mpad / kBM, a.Npad / BN, a.L);
  const bool timed = ms_out != nullptr || g_i8_timing.load() != 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (timed) {
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    check(cudaEventRecord(e0, st), "event");
  }
  ++g_launches;
  k_i8_mod_gemm<DIGITS, VAR><<<grid, kThreads, smem_bytes<DIGITS, VAR>(), st>>>(ta, tb, a);
  check(cudaGetLastError(), "k_i8_mod_gemm launch");
  if (timed) {
    check(cudaEventRecord(e1, st), "event");
    check(cudaEventSynchronize(e1), "event sync");
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, e0, e1), "event time");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms_out) *ms_out = ms;
    if (g_i8_timing.load()) {
      double tiles = 0;  // tiles actually computed (upper_only skips those below the diagonal)
      for (int tm = 0; tm < a.Mpad / kBM; ++tm)
        for (int tn = 0; tn < a.Npad / BN; ++tn)
          if (!(a.upper_only && tm * kBM > tn * BN + BN - 1)) tiles += 1;
      std::lock_guard<std::mutex> lk(g_i8_mu);
      g_i8_ms += ms;
      g_i8_ops += 2.0 * DIGITS * DIGITS * tiles * kBM * BN * (double)a.Kpad * a.L;
      g_i8_alg_ops += 2.0 * DIGITS * DIGITS * (double)a.m * a.n * (double)a.Kpad * a.L;
      ++g_i8_count;
    }
  }
}

// Autotuner of the tile configuration.  A shape class is (digits, ceil log2 of Mpad, Npad and
// the K range, moduli); the first launch of a class (outside stream capture, not accumulating
// into an earlier chunk's residues) runs every variant on the real operands, times each with
// CUDA events on the launch stream and keeps the fastest for the rest of the process.  All
// variants compute the same exact integers, so the choice never changes a result.
// SDPX_B200_AUTOTUNE=0 keeps variant 0; SDPX_B200_I8_CONFIG=v or sdpx_b200_i8_config forces one.
struct Tuner {
  std::mutex mu;
  std::map<std::array<int, 5>, std::pair<int, std::array<float, kVariants>>> table;
  int forced = -1;
  bool enabled = true;
  Tuner() {
    const char* e = std::getenv("SDPX_B200_AUTOTUNE");
    enabled = !(e && e[0] == '0');
    const char* f = std::getenv("SDPX_B200_I8_CONFIG");  // a fixed configuration, e.g. for a profile
    if (f && f[0] >= '0' && f[0] < '0' + kVariants && f[1] == 0) forced = f[0] - '0';
  }
};
Tuner& tuner() {
  static Tuner t;
  return t;
}
int lg2(long v) {
  int l = 0;
  while ((1L << l) < v) ++l;
  return l;
}

template <int DIGITS>
void launch(const int8_t* A, const int8_t* B, const I8GemmArgs& a, cudaStream_t st) {
  constexpr int BN = Cfg<DIGITS, 0>::BN;  // the padding rule: a multiple of every variant's width
  static_assert(Cfg<DIGITS, 0>::BN % Cfg<DIGITS, 1>::BN == 0 && Cfg<DIGITS, 0>::BN % Cfg<DIGITS, 2>::BN == 0,
                "variant widths must divide the padding");
  if (a.Mpad <= 0 || a.Npad <= 0 || a.Kpad <= 0 || a.Mpad % kBM || a.Npad % BN || a.Kpad % kKB ||
      a.Kld % kKB || a.k0 % kKB || a.k0 < 0 || a.k0 + a.Kpad > a.Kld)
    throw std::invalid_argument("i8 GEMM: padded extents must be multiples of the tile");
  if (a.m > a.Mpad || a.n > a.Npad || a.L <= 0 || a.L > 65535 || !a.moduli || !a.out)
    throw std::invalid_argument("i8 GEMM: bad arguments");
  if (a.Kpad > (1 << 17)) throw std::invalid_argument("i8 GEMM: K above 2^17 per call is not exact");
  Tuner& T = tuner();
  const std::array<int, 5> key = {DIGITS, lg2(a.Mpad), lg2(a.Npad), lg2(a.Kpad), lg2(a.L)};
  int var = 0;
  bool tune = false;
  {
    std::lock_guard<std::mutex> lk(T.mu);
    if (T.forced >= 0) {
      var = T.forced;
    } else if (T.enabled) {
      auto it = T.table.find(key);
      if (it != T.table.end()) {
        var = it->second.first;
      } else {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        check(cudaStreamIsCapturing(st, &cs), "capture status");
        tune = cs == cudaStreamCaptureStatusNone && !a.accumulate;
      }
    }
  }
  auto run = [&](int v, float* ms) {
    if (v == 0)
      launch_variant<DIGITS, 0>(A, B, a, st, ms);
    else if (v == 1)
      launch_variant<DIGITS, 1>(A, B, a, st, ms);
    else
      launch_variant<DIGITS, 2>(A, B, a, st, ms);
  };
  if (!tune) {
    run(var, nullptr);
    return;
  }
  // warm every variant, then time each; variant 0 runs last and leaves its (identical) output
  std::array<float, kVariants> ms{};
  for (int pass = 0; pass < 2; ++pass)
    for (int v = kVariants - 1; v >= 0; --v) run(v, &ms[v]);
  int best = 0;
  for (int v = 1; v < kVariants; ++v)
    if (ms[v] < ms[best]) best = v;
  std::lock_guard<std::mutex> lk(T.mu);
  T.table[key] = {best, ms};
}

}  // namespace

void i8_timing(int on) {
  std::lock_guard<std::mutex> lk(g_i8_mu);
  g_i8_timing = on;
  g_i8_ms = g_i8_ops = g_i8_alg_ops = 0.0;
  g_i8_count = 0;
}
void i8_times(double* ms, double* ops, double* alg_ops, uint64_t* count) {
  std::lock_guard<std::mutex> lk(g_i8_mu);
  *ms = g_i8_ms;
  *ops = g_i8_ops;
  *alg_ops = g_i8_alg_ops;
  *count = g_i8_count;
}

void i8_set_config(int variant) {
  std::lock_guard<std::mutex> lk(tuner().mu);
  tuner().forced = variant;
}
std::string i8_tuning_table() {
  std::lock_guard<std::mutex> lk(tuner().mu);
  std::string out;
  for (const auto& kv : tuner().table) {
    char line[192];
    std::snprintf(line, sizeof line,
                  "digits %d Mpad<=2^%d Npad<=2^%d K<=2^%d L<=2^%d -> variant %d (%.4f ms, %.4f ms, %.4f ms)\n",
                  kv.first[0], kv.first[1], kv.first[2], kv.first[3], kv.first[4], kv.second.first,
                  (double)kv.second.second[0], (double)kv.second.second[1], (double)kv.second.second[2]);
    out += line;
  }
  return out;
}

void launch_i8_gemm(int digits, const int8_t* A, const int8_t* B, const I8GemmArgs& args, cudaStream_t st) {
  if (digits == 1)
    launch<1>(A, B, args, st);
  else if (digits == 2)
    launch<2>(A, B, args, st);
  else
    throw std::invalid_argument("i8 GEMM: digits must be 1 or 2");
}

}  // namespace sdpxg
