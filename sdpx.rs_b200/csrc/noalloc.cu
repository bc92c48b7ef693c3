// sdpxg_solve_noalloc: the refined reduced solve of sdpxg_solve_many for callers that cannot
// allocate device memory when they call it.
//
// Some hosts own all of their device memory: an application that reserves the GPU's memory up
// front for its own pool, or a real-time loop in which a cudaMalloc (which may synchronise the
// whole device) is not allowed.  They can still create a context and factor once at set-up,
// but every later solve must run without allocating.  This entry point takes device pointers
// for the right-hand sides and the solutions and keeps all of its per-call scratch (the solve
// intermediate, the refinement vectors and the reduction slots) in
// one file-scope device array, g_noalloc_scratch, of fixed size.  It calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// Limits and sharing:
//  * n (the Schur dimension of the uploaded problem) must be at most SDPXG_NOALLOC_MAXN;
//    larger problems are rejected with return code 2 and a message.
//  * The array lives in every GPU that loads this library until the process exits
//    (SDPXG_NOALLOC_DOUBLES doubles, about 0.17 MB).
//  * Every call shares the array and it keeps the last call's contents.  Nothing in it has to
//    start at zero: each kernel writes every scratch element before another reads it.  Calls
//    whose work overlaps on the GPU (two host threads, or contexts on different streams of the
//    same device) race on the array; callers must serialise them.
//  * Host code cannot use the array's name as a device address, so the first call on each
//    device (with that device current) looks its address up with cudaGetSymbolAddress and
//    caches it.  Make that first call before any stream capture.
//  * The solve runs on the context's stream, which is not ordered after the caller's streams:
//    the caller finishes writing d_rhs (e.g. synchronises its stream) before the call; d_out is
//    complete when the call returns.  The caller's current device is restored on every exit.
#include <mutex>
#include <string>

#include "../../include/sdpx_b200.h"
#include "hsd.cuh"

using namespace sdpxg;

namespace sdpxg {
extern thread_local std::string g_last_error;
}

struct sdpxg_ctx;  // defined in kernel_api.cu
namespace sdpxg {
Engine* ctx_engine(sdpxg_ctx* ctx);
}

#define SDPXG_NOALLOC_MAXN 4096
#define SDPXG_NOALLOC_RED_BLOCKS 148
// tri (n) + e (n) + dx (n) + cand (n) + e2 (n) + 3 reduction slots
#define SDPXG_NOALLOC_DOUBLES (5 * SDPXG_NOALLOC_MAXN + 3 * (SDPXG_NOALLOC_RED_BLOCKS + 1))

static __device__ __align__(256) double g_noalloc_scratch[SDPXG_NOALLOC_DOUBLES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Once per device, with that device current: the device address of the static array.
double* scratch_for_current_device() {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (rc != cudaSuccess)
      throw std::runtime_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(rc));
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  return g_scratch_ptr[dev];
}

// Restores the caller's current device when the entry point returns or throws.
struct DeviceRestore {
  int saved = -1;
  DeviceRestore() {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
  }
  ~DeviceRestore() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};

// True when p is memory the GPU addresses as device (or managed) memory.
bool is_device_pointer(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // reset the error the failed query recorded
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// One reduction into slot `slot` of the scratch reduction area, no host transfer.
void reduce_into(cudaStream_t st, int op, long n, const double* x, double* partial, double* slot) {
  ++g_launches, k_reduce_partial<<<SDPXG_NOALLOC_RED_BLOCKS, 256, 0, st>>>(op, n, x, nullptr, partial);
  ++g_launches, k_reduce_final<<<1, 32, 0, st>>>(op, SDPXG_NOALLOC_RED_BLOCKS, partial, slot);
}

}  // namespace

extern "C" int32_t sdpxg_solve_noalloc(sdpxg_ctx* ctx, const double* d_rhs, double* d_out,
                                       uint32_t ncols) {
  try {
    if (!ctx) throw std::invalid_argument("null context");
    Engine* Ep = ctx_engine(ctx);
    if (!Ep) throw std::invalid_argument("no problem uploaded");
    Engine& E = *Ep;
    const int n = E.n;
    if (n > SDPXG_NOALLOC_MAXN) {
      sdpxg::g_last_error = "sdpxg_solve_noalloc: Schur dimension " + std::to_string(n) +
                            " exceeds the compiled maximum " + std::to_string(SDPXG_NOALLOC_MAXN);
      return 2;
    }
    if (ncols && (!d_rhs || !d_out)) throw std::invalid_argument("null pointer");
    if (!E.factored()) throw std::invalid_argument("no factorization: call sdpxg_factor first");
    DeviceRestore restore;
    check(cudaSetDevice(E.device), "cudaSetDevice");
    if (ncols && (!is_device_pointer(d_rhs) || !is_device_pointer(d_out)))
      throw std::invalid_argument("d_rhs and d_out must be device pointers");
    double* base = scratch_for_current_device();
    double* tri = base;
    double* en = tri + SDPXG_NOALLOC_MAXN;
    double* dx = en + SDPXG_NOALLOC_MAXN;
    double* cand = dx + SDPXG_NOALLOC_MAXN;
    double* e2 = cand + SDPXG_NOALLOC_MAXN;
    double* red = e2 + SDPXG_NOALLOC_MAXN;
    double* slots = red + 3 * SDPXG_NOALLOC_RED_BLOCKS;
    cudaStream_t st = E.st;
    const Settings cfg;  // binary64 refinement defaults, as in sdpxg_solve_many
    const int grid = (n + 7) / 8;
    auto trisolve = [&](const double* r, double* x) {
      ++g_launches, k_tri_colgemv<<<grid, 256, 0, st>>>(E.uinv(), n, 0, r, tri);
      ++g_launches, k_tri_colgemv<<<grid, 256, 0, st>>>(E.uinvT(), n, 1, tri, x);
    };
    auto residual = [&](const double* r, const double* x, double* e) {
      ++g_launches, k_symv_cols<<<(n + 7) / 8, 256, 0, st>>>(E.Hsave(), n, x, r, e);
    };
    auto fetch = [&](int count, double* host) {
      check(cudaMemcpyAsync(host, slots, count * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
      check(cudaStreamSynchronize(st), "sync");
    };
    auto copy = [&](double* dst, const double* src) {
      check(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, st), "d2d");
    };
    for (uint32_t c = 0; c < ncols; ++c) {
      const double* r = d_rhs + (size_t)c * n;
      double* x = d_out + (size_t)c * n;
      trisolve(r, x);
      residual(r, x, en);
      reduce_into(st, RED_MAXABS, n, r, red, slots);
      reduce_into(st, RED_MAXABS, n, en, red + SDPXG_NOALLOC_RED_BLOCKS, slots + 1);
      reduce_into(st, RED_FINITE, n, x, red + 2 * SDPXG_NOALLOC_RED_BLOCKS, slots + 2);
      double h[3];
      fetch(3, h);
      double normb = h[0], norme = h[1];
      if (h[2] != 1.0 || !std::isfinite(norme)) throw std::runtime_error("reduced solve failed");
      const double tol = cfg.ir_abstol + cfg.ir_reltol * normb;
      bool converged = norme <= tol;
      for (int it = 0; it < cfg.ir_max_iter && !converged; ++it) {
        double previous = norme;
        trisolve(en, dx);
        ++g_launches, k_lincomb<<<std::min((n + 255) / 256, 1184), 256, 0, st>>>(
            n, 1.0, x, 1.0, dx, 0.0, nullptr, cand);
        residual(r, cand, e2);
        reduce_into(st, RED_MAXABS, n, e2, red, slots);
        fetch(1, h);
        norme = h[0];
        if (!std::isfinite(norme)) throw std::runtime_error("reduced solve failed");
        double ratio = previous / norme;
        if (ratio < cfg.ir_stop_ratio) {
          if (ratio > 1.0) copy(x, cand);
          break;
        }
        copy(x, cand);
        copy(en, e2);
        converged = norme <= tol;
      }
    }
    check(cudaGetLastError(), "launch");
    check(cudaStreamSynchronize(st), "sync");
    return 0;
  } catch (const std::invalid_argument& e) {
    sdpxg::g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    sdpxg::g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    sdpxg::g_last_error = "internal error";
    return 5;
  }
}
