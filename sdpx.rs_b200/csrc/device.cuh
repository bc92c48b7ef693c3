// Host-side helpers: device buffers, kernel launch wrappers and the batched scalar reducer.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <initializer_list>
#include <cstdint>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"

namespace sdpxg {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

inline void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// Bytes this library copied between host and device in this process (all handles): the
// end-to-end traffic of a solve, read through sdpx_b200_transfer_bytes.
inline std::atomic<uint64_t> g_h2d_bytes{0}, g_d2h_bytes{0};

inline void copy_h2d(void* d, const void* h, size_t bytes, cudaStream_t st) {
  if (!bytes) return;
  check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st), "H2D");
  g_h2d_bytes += bytes;
}

inline void copy_d2h(void* h, const void* d, size_t bytes, cudaStream_t st) {
  if (!bytes) return;
  check(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st), "D2H");
  g_d2h_bytes += bytes;
}

// Device blocks this library has obtained in this process (from the cache below or from
// cudaMalloc), read through sdpx_b200_device_allocations: a call that must not allocate leaves
// it unchanged.
inline std::atomic<uint64_t> g_dev_allocs{0};

// Device allocations are recycled through a process-wide cache instead of going back to the
// driver: the next handle (an e2e loop, a new problem) takes the blocks the last one released,
// without cudaMalloc's mapping cost and cudaFree's unmapping.  A block is released the way
// cudaFree releases it -- after a device synchronisation, so no queued work can still touch it
// when it is handed out again.  Best fit among cached blocks of at most twice the request; at
// most kCacheBytes are kept per device (the largest blocks go back to the driver first).
class DeviceCache {
 public:
  static constexpr size_t kCacheBytes = size_t(8) << 30;
  static DeviceCache& get() {
    static DeviceCache c;
    return c;
  }
  // A cached block of at least `bytes` (its true size in *got), or nullptr.
  void* take(size_t bytes, int dev, size_t* got) {
    std::lock_guard<std::mutex> lk(mu_);
    auto& f = free_[dev & 15];
    auto it = f.lower_bound(bytes);
    if (it == f.end() || it->first > 2 * bytes + (size_t(1) << 20)) return nullptr;
    void* p = it->second;
    *got = it->first;
    held_[dev & 15] -= it->first;
    f.erase(it);
    return p;
  }
  // bytes: the size the block was allocated with; dev: the device it lives on (made current for
  // the synchronisation and any eviction, the caller's current device restored after)
  void give(void* p, size_t bytes, int dev) {
    int cur = dev;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaDeviceSynchronize();  // what cudaFree would wait for
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto& f = free_[dev & 15];
      f.emplace(bytes, p);
      held_[dev & 15] += bytes;
      while (held_[dev & 15] > kCacheBytes && !f.empty()) {
        auto last = std::prev(f.end());
        cudaFree(last->second);
        held_[dev & 15] -= last->first;
        f.erase(last);
      }
    }
    if (cur != dev) cudaSetDevice(cur);
  }

 private:
  std::mutex mu_;
  std::multimap<size_t, void*> free_[16];
  size_t held_[16] = {};
};

// Device buffer with grow-only storage: alloc() reuses the allocation when it is large enough,
// so a handle that is re-prepared with a new problem (batches of instances) allocates only when
// a buffer grows, and never frees in between (cudaFree synchronises the whole device, which
// would stall every other instance running on it).  n is the requested element count.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  size_t cap = 0;    // elements the block holds
  size_t bytes = 0;  // true size of the block (a cached block may be larger than asked for)
  int dev = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), cap(o.cap), bytes(o.bytes), dev(o.dev) {
    o.p = nullptr;
    o.n = o.cap = o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; cap = o.cap; bytes = o.bytes; dev = o.dev;
      o.p = nullptr; o.n = o.cap = o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    if (count <= cap && p) {
      n = count;
      return;
    }
    release();
    n = count;
    if (count) {
      check(cudaGetDevice(&dev), "cudaGetDevice");
      const size_t want = count * sizeof(T);
      size_t got = want;
      void* q = DeviceCache::get().take(want, dev, &got);
      if (!q) check(cudaMalloc(&q, want), "cudaMalloc");
      ++g_dev_allocs;
      p = static_cast<T*>(q);
      bytes = got;
      cap = got / sizeof(T);
    }
  }
  void release() {
    if (p) DeviceCache::get().give(p, bytes, dev);
    p = nullptr;
    n = cap = bytes = 0;
  }
  void upload(const T* h, size_t count, cudaStream_t st) {
    copy_h2d(p, h, count * sizeof(T), st);
  }
  void upload(const std::vector<T>& h, cudaStream_t st) {
    if (h.size() > n) alloc(h.size());
    upload(h.data(), h.size(), st);
  }
  operator T*() const { return p; }
};

// Page-locked host buffer: scalar device-to-host reads skip the pageable staging copy.
template <typename T>
struct PinnedBuf {
  T* p = nullptr;
  size_t n = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() { release(); }
  size_t cap = 0;
  void alloc(size_t count) {  // grow-only, like DevBuf
    if (count <= cap && p) {
      n = count;
      return;
    }
    release();
    n = count;
    if (count) {
      check(cudaMallocHost(&p, count * sizeof(T)), "cudaMallocHost");
      cap = count;
    }
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = cap = 0;
  }
  T& operator[](size_t i) { return p[i]; }
  const T& operator[](size_t i) const { return p[i]; }
};

// Kernel declarations (defined in the *_kernels.cu translation units of this library).
extern "C" {
__global__ void k_nt_factor(const BlockDesc*, const double*, const double*, double*, double*,
                            uint32_t*);
__global__ void k_nt_svd(const BlockDesc*, double*, double*, double*, double*, double*, uint32_t*);
__global__ void k_identity_scaling(const BlockDesc*, double*, double*, double*, double*, double*);
__global__ void k_ginv_from_rinv(const BlockDesc*, const double*, double*);
__global__ void k_congruence(const BlockDesc*, int, const double*, const double*, const double*,
                             double*, long);
__global__ void k_circ_op(const BlockDesc*, const double*, const double*, double*);
__global__ void k_lam_inv_circ(const BlockDesc*, const double*, const double*, double*);
__global__ void k_affine_ds(const BlockDesc*, const double*, double*);
__global__ void k_shift_unit(const BlockDesc*, double*, double);
__global__ void k_step_length(const BlockDesc*, const double*, const double*, const double*,
                              const double*, const double*, double, int, double*, uint32_t*);
__global__ void k_margins(const BlockDesc*, const double*, long, double*, uint32_t*, int);
__global__ void k_schur_transform(const BlockDesc*, const int*, const int*, const long*,
                                  const double*, const double*, double*);
__global__ void k_schur_block_gemm(const BlockDesc*, const int*, const int*, const long*,
                                   const long*, const double*, const double*, double*);
__global__ void k_schur_gather(int, const int*, const int*, const int*, const int*, const long*,
                               const double*, double*);
__global__ void k_add_upper_csc(int, const int*, const int*, const double*, double*);
__global__ void k_op_forward(const BlockDesc*, const int*, const int*, const int*, const long*,
                             const double*, const int*, const int*, const double*, long, double,
                             double, double*, long);
__global__ void k_op_adjoint_partial(const BlockDesc*, const int*, const int*, const int*,
                                     const long*, const double*, const double*, long, double*,
                                     long, int);
__global__ void k_op_adjoint_gather(int, const int*, const int*, const int*, const int*,
                                    const double*, long, double, double, double*, long);
__global__ void k_potrf_diag(double*, int, int, double, double, int, const double*, double*,
                             uint32_t*);
__global__ void k_trsm_panel(double*, int, int, const double*);
__global__ void k_gram_basis(const BlockDesc*, const int*, const int*, const int*, const long*,
                             const double*, const double*, double*);
__global__ void k_gram_schur(const BlockDesc*, const int*, const int*, const int*, const long*,
                             const long*, const double*, const double*, double*);
__global__ void k_gram_forward(const BlockDesc*, const int*, const int*, const int*, const int*,
                               const int*, const long*, const double*, const double*,
                               const double*, double, double, double*, double*, unsigned*);
__global__ void k_gram_adjoint(const BlockDesc*, const int*, const int*, const int*, const int*,
                               const long*, const double*, const double*, const double*, double*);
__global__ void k_chol_dataflow(double*, int, int, const unsigned*, int, int*, double, double, int,
                                const double*, double*, uint32_t*);
__global__ void k_syrk_update(double*, int, int);
__global__ void k_trtri_diag(int, const double*, double*, double*);
__global__ void k_trinv_level(const double*, double*, double*, double*, int, int, int);
__global__ void k_tri_colgemv(const double*, int, int, const double*, double*);
__global__ void k_shifted_copy(const double*, double*, int, double, double*);
__global__ void k_strided_diag(const double*, long, int, double, double*);
__global__ void k_transpose_block(const double*, long, int, int, double*, long);
__global__ void k_symv_cols(const double*, int, const double*, const double*, double*);
__global__ void k_coldot_seg(const double*, int, int, const double*, const double*, double, double*,
                             double*, unsigned*);
__global__ void k_lincomb(long, double, const double*, double, const double*, double,
                          const double*, double*);
__global__ void k_reduce_partial(int, long, const double*, const double*, double*);
__global__ void k_reduce_final(int, int, const double*, double*);
__global__ void k_reduce_fused(int, long, const double*, const double*, double*, unsigned*, double*);
__global__ void k_reduce_batch(RedBatch, double*, unsigned*, double*, int);
__global__ void k_lincomb_batch(LinBatch);
__global__ void k_refine_head(const double*, const double*, const double*, const double*,
                              const double*, int, RefineCtl*, RefineParams, cudaGraphConditionalHandle);
__global__ void k_refine_step(const double*, RefineCtl*, RefineParams, cudaGraphConditionalHandle);
__global__ void k_refine_outer_init(const double*, const double*, const double*, const double*,
                                    RefineCtl*, RefineParams, cudaGraphConditionalHandle);
__global__ void k_refine_outer_step(const double*, const double*, RefineCtl*, RefineParams,
                                    cudaGraphConditionalHandle);
__global__ void k_refine_copy(const int*, long, double*, const double*, const int*, long, double*,
                              const double*);
__global__ void k_diag_absmax(const double*, int, double*);
__global__ void k_nn_scale(int, const int*, const double*, const double*, double*, double*, uint32_t*);
__global__ void k_nn_identity(int, double*, double*);
__global__ void k_nn_cone(int, const int*, int, const double*, const double*, double*, long);
__global__ void k_nn_circ(int, const int*, const double*, const double*, double*);
__global__ void k_nn_lam_inv(int, const int*, const double*, const double*, double*);
__global__ void k_nn_affine_ds(int, const int*, const double*, double*);
__global__ void k_nn_shift(int, const int*, double*, double);
__global__ void k_nn_step(int, const int*, const double*, const double*, const double*, const double*,
                          double, int, double*);
__global__ void k_nn_margins(int, const int*, const double*, double*);
__global__ void k_nn_forward(int, int, const int*, const double*, const double*, double, double, double*);
__global__ void k_nn_adjoint(int, int, const int*, const double*, const double*, double, double*);
__global__ void k_nn_schur(int, int, const double*, const double*, double*);
__global__ void k_ms_basis(const BlockDesc*, const MsDesc*, const double*, const double*, double*);
__global__ void k_ms_gram(const BlockDesc*, const MsDesc*, const double*, double*);
__global__ void k_ms_schur(const MsDesc*, const int*, const int*, const long*, const double*, const int*,
                           const double*, double*);
__global__ void k_ms_forward(const BlockDesc*, const MsDesc*, const int*, const int*, const double*,
                             const double*, const double*, double, double, double*);
__global__ void k_ms_adjoint(const BlockDesc*, const MsDesc*, const int*, const int*, const double*, const int*,
                             const double*, const double*, double*);
__global__ void k_csr_spmv(int, const int*, const int*, const double*, const double*, double,
                           double, double*);
}

// Kernel launches issued by this library in this process (every launch site increments it).
inline std::atomic<uint64_t> g_launches{0};  // atomic: handles may run on many host threads

enum RedOp { RED_DOT = 0, RED_SUMSQ = 1, RED_MAXABS = 2, RED_FINITE = 3, RED_NEGMAX = 4 };

// Queues reductions into device scalar slots; fetch() copies them back in one transfer.
class Reducer {
 public:
  static constexpr int kBlocks = 148;
  static constexpr int kSlots = 64;
  void init() {
    partial_.alloc((size_t)kBlocks * kSlots);
    slots_.alloc(kSlots);
    counters_.alloc(kSlots);
    check(cudaMemset(counters_.p, 0, kSlots * sizeof(unsigned)), "reducer counters");
    host_.alloc(kSlots);
  }
  int add(cudaStream_t st, int op, long n, const double* x, const double* y) {
    if (count_ >= kSlots) throw CudaError("reducer slots exhausted");
    if (n > 0 && !x) throw std::invalid_argument("null device buffer: reduction input");
    int s = count_++;
    if (n > 0) {
      ++g_launches, k_reduce_fused<<<kBlocks, 256, 0, st>>>(op, n, x, y, partial_.p + (size_t)s * kBlocks,
                                                          counters_.p + s, slots_.p + s);
    } else {  // an empty input: the operation's identity (1 for the finite test, 0 otherwise)
      copy_h2d(slots_.p + s, &id_[op], sizeof(double), st);
    }
    return s;
  }
  // Consecutive reductions in one launch (slots first, first + 1, ...; the same values as the
  // same adds one by one).  Returns the first slot.
  int add_batch(cudaStream_t st, std::initializer_list<RedReq> reqs) {
    const int k = (int)reqs.size();
    if (k == 0 || k > kRedBatchMax) throw std::invalid_argument("reduction batch size");
    if (count_ + k > kSlots) throw CudaError("reducer slots exhausted");
    RedBatch b{};
    int i = 0;
    for (const RedReq& q : reqs) {
      if (q.n > 0 && !q.x) throw std::invalid_argument("null device buffer: reduction input");
      b.r[i++] = q;
    }
    const int first = count_;
    count_ += k;
    ++g_launches, k_reduce_batch<<<dim3(kBlocks, k), 256, 0, st>>>(b, partial_.p, counters_.p, slots_.p, first);
    return first;
  }
  int count() const { return count_; }
  // Device address of a slot (read by the control kernels of the device-driven solves).
  const double* slot(int s) const { return slots_.p + s; }
  // Slots queued by a replayed captured segment (its reductions ran inside the graph).
  void set_count(int c) { count_ = c; }
  const PinnedBuf<double>& fetch(cudaStream_t st) {
    if (count_) {
      copy_d2h(host_.p, slots_.p, count_ * sizeof(double), st);
    }
    check(cudaStreamSynchronize(st), "reducer sync");
    count_ = 0;
    return host_;
  }

 private:
  DevBuf<double> partial_, slots_;
  DevBuf<unsigned> counters_;  // arrival tickets of k_reduce_fused, one per slot (self-resetting)
  PinnedBuf<double> host_;
  int count_ = 0;
  const double id_[5] = {0.0, 0.0, 0.0, 1.0, 0.0};
};

}  // namespace sdpxg
