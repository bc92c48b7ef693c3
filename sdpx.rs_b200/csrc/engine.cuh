// Device engine: problem upload and the per-iteration hot-path operations on one GPU.
//
// Everything an iteration touches stays resident in HBM; the host receives scalars only
// (reductions, status words, per-block step bounds).  The operations map onto the
// reference's KKTSolver / DirectLDLSolver / Cone seams:
//   nt_scale          Cone::update_scaling            (cones/psdtrianglecone.rs:311)
//   assemble          CondensedKKTSolver::assemble    (kkt/condensed/mod.rs:1962)
//   factor            DirectLDLKKTSolver::factor_with_shift + DenseBlockSolver
//                     (kkt/direct/solver.rs:758, kkt/ldl/dense_block.rs:95)
//   trisolve / symv   DenseBlockSolver::solve / residual (dense_block.rs:604-719)
//   apply_cone        PsdBlock::apply and the W products (kkt/condensed/psd.rs:1968)
//   step_bounds       Cone::step_length (cones/psdtrianglecone.rs:475)
#pragma once
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <utility>
#include <string>
#include <unordered_map>

#include "device.cuh"
#include "host_parallel.h"
#include "ozaki.cuh"

namespace sdpxg {

constexpr int kMatD = SDPXG_LD * SDPXG_NMAX;
constexpr size_t kSmemNtFactor = (3 * kMatD + 2 * SDPXG_CHOL_SCRATCH) * sizeof(double);
constexpr size_t kSmemNt = (5 * kMatD + 2 * SDPXG_NMAX) * sizeof(double) + (SDPXG_NMAX + 1) * sizeof(int);
constexpr size_t kSmemCong = 4 * kMatD * sizeof(double);
constexpr size_t kSmemCirc = 2 * kMatD * sizeof(double);
constexpr size_t kSmemStep = (4 * kMatD + SDPXG_CHOL_SCRATCH + 4 * SDPXG_NMAX + 32) * sizeof(double);
constexpr size_t kSmemMarg = (kMatD + 5 * SDPXG_NMAX + 32) * sizeof(double);
constexpr size_t kSmemTrans = 3 * kMatD * sizeof(double);
constexpr size_t kSmemTrsm = 2 * 64 * 65 * sizeof(double);
constexpr size_t kSmemSyrk = 2 * 64 * 66 * sizeof(double);
constexpr size_t kSmemTrtri = 2 * 64 * 65 * sizeof(double);
constexpr size_t kSmemTrinv = 4 * 64 * 68 * sizeof(double);  // k_trinv_level: 2 stages x 2 tiles
constexpr size_t kSmemDf = (3 * 64 * 68 + 2 * 8 * 64) * sizeof(double);  // k_chol_dataflow
constexpr size_t kSmemGram = 3 * kMatD * sizeof(double);                 // k_gram_basis/adjoint
constexpr int kDfMaxTiles = 256;  // dataflow schedule up to m = 16384 (nt^3/6 items)

// Rank-one test of one PSD column block: svec v (upper, column order, off-diagonal x sqrt2) of
// an n x n matrix M.  On success M = sigma u u' entrywise to a few ulps (32 eps relative to
// each entry, exact zeros kept), with u scaled from the column of the largest diagonal.
inline bool rank_one_column(const double* v, int n, double* u, double* sigma) {
  int p = 0;
  double best = -1.0;
  for (int i = 0; i < n; ++i) {
    const double a = std::fabs(v[i * (i + 3) / 2]);  // diagonal (i, i) sits at i(i+1)/2 + i
    if (a > best) {
      best = a;
      p = i;
    }
  }
  if (!(best > 0.0)) {  // among rank-one matrices only the zero matrix has a zero diagonal
    for (int e = 0; e < n * (n + 1) / 2; ++e)
      if (v[e] != 0.0) return false;
    for (int i = 0; i < n; ++i) u[i] = 0.0;
    *sigma = 1.0;
    return true;
  }
  const double mpp = v[p * (p + 3) / 2], sg = mpp > 0.0 ? 1.0 : -1.0;
  const double r = std::sqrt(std::fabs(mpp));
  if (!std::isfinite(r)) return false;
  for (int i = 0; i < n; ++i) {
    const double mip = (i == p) ? mpp
                       : (i < p ? v[p * (p + 1) / 2 + i] : v[i * (i + 1) / 2 + p]) * SDPXG_RSQRT2;
    u[i] = sg * mip / r;
  }
  const double tol = 32.0 * 2.220446049250313e-16;
  const double* e = v;
  for (int j = 0; j < n; ++j) {
    const double uj = sg * u[j];
    for (int i = 0; i < j; ++i, ++e) {  // off-diagonal svec entry sqrt2 M_ij
      const double g = SDPXG_SQRT2 * (uj * u[i]);
      if (!(std::fabs(*e - g) <= tol * (std::fabs(*e) + std::fabs(g)))) return false;
    }
    const double g = uj * u[j];
    if (!(std::fabs(*e - g) <= tol * (std::fabs(*e) + std::fabs(g)))) return false;
    ++e;
  }
  *sigma = sg;
  return true;
}

// Work list of the dataflow Cholesky (k_chol_dataflow): POTRF(k), TRSM(k, j), GEMM(k, i, j) of
// the right-looking tiled algorithm in a topological order with one step of look-ahead: the
// update of tile row k + 1, POTRF(k + 1) and its TRSM row come before the rest of step k's
// trailing update.  Encoded type << 30 | k << 20 | i << 10 | j.
inline std::vector<unsigned> chol_schedule(int nt) {
  auto code = [](unsigned type, int k, int i, int j) {
    return (type << 30) | ((unsigned)k << 20) | ((unsigned)i << 10) | (unsigned)j;
  };
  std::vector<unsigned> it;
  if (nt <= 0) return it;
  // ticket 0: the critical-path chain (every POTRF(k), TRSM(k, k+1) and GEMM(k, k+1, k+1))
  it.push_back(code(3u, 0, 0, 0));
  // then step by step the rest of each step: the TRSM row beyond k + 1, and the trailing
  // updates row by row (rows k + 1 and k + 2 first feed the chain's next two steps)
  for (int k = 0; k + 1 < nt; ++k) {
    for (int j = k + 2; j < nt; ++j) it.push_back(code(1u, k, k, j));
    for (int i = k + 1; i < nt; ++i)
      for (int j = i; j < nt; ++j)
        if (!(i == k + 1 && j == k + 1)) it.push_back(code(2u, k, i, j));
  }
  return it;
}

// Replays a work list in ticket order and checks that every item's inputs come from earlier
// items or from chain steps whose own inputs come from earlier items -- the condition under
// which k_chol_dataflow cannot deadlock (the chain, ticket 0, only waits on items that precede
// every item waiting on it) -- and that every tile ends factored.  False on any violation.
inline bool chol_schedule_valid(const std::vector<unsigned>& it, int nt) {
  std::vector<int> upd((size_t)nt * nt, 0), fin((size_t)nt * nt, 0);
  auto U = [&](int i, int j) -> int& { return upd[(size_t)i * nt + j]; };
  auto Fn = [&](int i, int j) -> int& { return fin[(size_t)i * nt + j]; };
  bool chain = false;
  int step = 0;          // next chain step
  bool diag_done = false;  // the chain's POTRF of `step` is done, its TRSM is pending
  auto advance = [&]() {
    while (chain && step < nt) {
      const int s = step;
      if (!diag_done) {
        if (s > 0 && (U(s, s) != s - 1 || !Fn(s - 1, s))) return;  // GEMM(s-1, s, s) inputs
        U(s, s) = s;
        Fn(s, s) = 1;
        diag_done = true;
      }
      if (s + 1 < nt) {
        if (U(s, s + 1) != s) return;  // TRSM(s, s+1) input
        Fn(s, s + 1) = 1;
      }
      diag_done = false;
      ++step;
    }
  };
  for (size_t t = 0; t < it.size(); ++t) {
    const unsigned c = it[t];
    const int type = (int)(c >> 30), k = (int)((c >> 20) & 1023u);
    const int i = (int)((c >> 10) & 1023u), j = (int)(c & 1023u);
    if (k >= nt || i >= nt || j >= nt) return false;
    if (type == 3) {
      if (t != 0 || chain) return false;
      chain = true;
      advance();
      continue;
    }
    advance();
    if (type == 1) {
      if (i != k || j <= k + 1 || !Fn(k, k) || U(k, j) != k) return false;
      Fn(k, j) = 1;
    } else if (type == 2) {
      if (i <= k || j < i || (i == k + 1 && j == k + 1) || !Fn(k, i) || !Fn(k, j) || U(i, j) != k)
        return false;
      U(i, j) = k + 1;
    } else {
      return false;
    }
  }
  advance();
  if (!chain || step != nt) return false;
  for (int i = 0; i < nt; ++i)
    for (int j = i; j < nt; ++j)
      if (!Fn(i, j) || U(i, j) != i) return false;
  return true;
}
constexpr int kNB = 64;

// Factorisation forms of the Schur complement.
//   kFormPlain  one FP64 dataflow Cholesky of the whole matrix, then its explicit inverse;
//   kFormSplit  (m >= kSplitMin) H = [H11 H12; H12' H22] in two halves: FP64 dataflow Cholesky
//               and inverse of the diagonal blocks (pivots and the dynamic pivot rule stay FP64),
//               and the four large products -- U12 = X11' H12, S = H22 - U12' U12,
//               W = X11 U12, X12 = -W X22 -- as split-precision (Ozaki-II) INT8 tensor-core
//               GEMMs.  The refinement against the unshifted FP64 Schur complement is unchanged.
enum FactorForm { kFormPlain = 0, kFormSplit = 1 };
constexpr int kSplitMin = 1024;

// Equilibrated problem in host memory (CSC, int64 indices as in the reference ABI).
// std::vector storage whose resize() leaves new elements default-initialised (unset for
// arithmetic types): the large CSC arrays of a prepare are written right away by parallel loops,
// so zero-filling them first on one thread -- and taking every first-touch page fault there --
// is wasted time.
template <typename T>
struct UninitAlloc : std::allocator<T> {
  using value_type = T;
  template <class U>
  struct rebind {
    using other = UninitAlloc<U>;
  };
  UninitAlloc() = default;
  template <class U>
  UninitAlloc(const UninitAlloc<U>&) noexcept {}
  template <class U>
  void construct(U* ptr) noexcept {
    ::new (static_cast<void*>(ptr)) U;
  }
  template <class U, class... Args>
  void construct(U* ptr, Args&&... args) {
    ::new (static_cast<void*>(ptr)) U(std::forward<Args>(args)...);
  }
};
using I64Vec = std::vector<int64_t, UninitAlloc<int64_t>>;
using F64Vec = std::vector<double, UninitAlloc<double>>;

struct HostProblem {
  int n = 0, m = 0;
  std::vector<int64_t> Pcolptr, Prow;
  std::vector<double> Pval;
  I64Vec Acolptr, Arow;
  F64Vec Aval;
  std::vector<double> q, b;
  std::vector<int> psd;  // PSD block orders in cone order
  // all cones in order: (1, d) nonnegative orthant of dimension d, (3, d) PSD triangle of order d;
  // empty means every cone is PSD (the orders in psd)
  std::vector<std::pair<int, int>> cones;
  // Factor-authoritative sampled blocks (sdpx_prepare_sampled): the PSD block starting at row
  // `row_start` holds the columns col0 .. col0 + count - 1, column col0 + k being
  // weight[k] svec(q_k q_k') with q_k column k of `basis` (order x count, column-major).  The
  // engine uses these factors instead of testing the materialised columns.
  struct Sampled {
    int row_start = 0, col0 = 0, count = 0, order = 0;  // count: basis columns; order: dim * basis rows
    int dim = 1;                                        // matrix blocks per side
    std::vector<double> basis, weight;                  // basis (order / dim) x count; tri(dim) count weights
  };
  std::vector<Sampled> sampled;
};

// Cone operator modes of k_congruence.
enum ConeMode { CM_W = 0, CM_WT = 1, CM_WINV = 2, CM_WINVT = 3, CM_HS = 4, CM_HINV = 5 };

// Every wrapper checks its device pointers on the host before launching: a missing buffer is
// reported as an error instead of reaching a kernel.
inline void need(const void* p, const char* what) {
  if (!p) throw std::invalid_argument(std::string("null device buffer: ") + what);
}

// Kernel-phase timers: CUDA events recorded on the engine's stream around each phase.
enum KernelPhase { KT_SCALE = 0, KT_ASSEMBLE, KT_FACTOR, KT_TRISOLVE, KT_CONE, KT_STEP, KT_SYMV, KT_TRINV,
                   KT_SPLIT, KT_N };

class Engine {
 public:
  cudaStream_t st = nullptr;
  bool timing = false;
  double kt_ms[KT_N] = {0};
  uint64_t kt_count[KT_N] = {0};
  void reset_timers() {
    for (int k = 0; k < KT_N; ++k) { kt_ms[k] = 0; kt_count[k] = 0; }
  }
  int n = 0, m = 0, nblk = 0;
  int nchol = 0;  // Schur tiles per side
  int factor_form = kFormPlain;  // SDPX_B200_FORM=split or sdpx_b200_set_form
  OzakiWorkspace oz;             // split-precision GEMM scratch
  bool split_active() const { return factor_form == kFormSplit && n >= kSplitMin; }
  bool gram_enabled = true;  // rank-one blocks use the Gram form (SDPX_B200_GRAM=0 disables)
  int gram_blocks() const { return ngram_; }
  int sampled_matrix_blocks() const { return nms_; }
  int nn_count() const { return nnn_; }
  std::vector<int> nn_rows;  // orthant rows of the stacked cone vector (cone order)
  std::vector<BlockDesc> hblocks;
  std::vector<int> hk;  // columns per block
  Reducer red;

  Engine() = default;
  ~Engine() {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second.exec);
    for (auto& kv : programs_) cudaGraphExecDestroy(kv.second.exec);
    for (auto& e : ev_) if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  // ---- captured segments ----
  // A segment is a straight run of launches, copies and queued reductions between two host
  // reads whose shape depends only on the device pointers in its key (fixed scalars).  The
  // first run captures it into a CUDA graph (stream capture on this engine's stream); later
  // runs launch the instantiated graph.  The reducer's slot count is restored on replay.
  // Eager when graphs are off (SDPX_B200_GRAPHS=0) or while phase timing is on (its events
  // synchronize the host).
  bool graphs_enabled = true;
  // Captured graphs hold device pointers by value: drop them whenever buffers they may reference
  // are (re)allocated (a new upload, a new solver's work vectors).
  void clear_graphs() {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second.exec);
    graphs_.clear();
    for (auto& kv : programs_) cudaGraphExecDestroy(kv.second.exec);
    programs_.clear();
  }
  template <typename F>
  void segment(int id, std::initializer_list<const void*> ptrs, F&& body) {
    if (!graphs_enabled || timing || n == 0 || m == 0) {
      body();
      return;
    }
    if (red.count() != 0) throw CudaError("a captured segment must start with an empty reducer");
    std::string key(reinterpret_cast<const char*>(&id), sizeof id);
    for (const void* p : ptrs) key.append(reinterpret_cast<const char*>(&p), sizeof p);
    auto it = graphs_.find(key);
    if (it != graphs_.end()) {
      check(cudaGraphLaunch(it->second.exec, st), "cudaGraphLaunch");
      red.set_count(it->second.red_count);
      g_launches += it->second.launches;
      return;
    }
    if (graphs_.size() >= kMaxGraphs) clear_graphs();  // bound the cache
    uint64_t kernels = 0;
    cudaGraph_t g = capture(body, &kernels);
    cudaGraphExec_t ex = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    check(e, "cudaGraphInstantiate");
    graphs_[key] = {ex, red.count(), kernels};
    check(cudaGraphLaunch(ex, st), "cudaGraphLaunch");
  }
  // Capture a straight run of launches on this engine's stream into a graph (not instantiated)
  // and count its kernel nodes.
  template <typename F>
  cudaGraph_t capture(F&& body, uint64_t* kernels) {
    check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      body();
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cudaGraph_t g = nullptr;
    check(cudaStreamEndCapture(st, &g), "end capture");
    size_t nn = 0;
    uint64_t k = 0;
    check(cudaGraphGetNodes(g, nullptr, &nn), "graph nodes");
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) check(cudaGraphGetNodes(g, nodes.data(), &nn), "graph nodes");
    for (cudaGraphNode_t nd : nodes) {
      cudaGraphNodeType ty;
      check(cudaGraphNodeGetType(nd, &ty), "graph node type");
      k += (ty == cudaGraphNodeTypeKernel);
    }
    if (kernels) *kernels = k;
    return g;
  }
  // Instantiated graphs with device-side control flow (the refined KKT solve), keyed like the
  // segments and dropped with them.  Kernel counts: fixed per launch, per inner and per outer
  // refinement step.
  struct Program {
    cudaGraphExec_t exec = nullptr;
    uint64_t fixed = 0, per_inner = 0, per_outer = 0;
  };
  Program* find_program(const std::string& key) {
    auto it = programs_.find(key);
    return it == programs_.end() ? nullptr : &it->second;
  }
  Program* add_program(const std::string& key, const Program& pg) {
    if (programs_.size() >= kMaxGraphs) clear_graphs();
    return &(programs_[key] = pg);
  }
  void tbegin(int k) {
    if (timing) check(cudaEventRecord(ev_[2 * k], st), "event");
  }
  void tend(int k) {
    if (!timing) return;
    check(cudaEventRecord(ev_[2 * k + 1], st), "event");
    check(cudaEventSynchronize(ev_[2 * k + 1]), "event sync");
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, ev_[2 * k], ev_[2 * k + 1]), "event time");
    kt_ms[k] += ms;
    kt_count[k]++;
  }

  int device = 0;

  void init(int dev) {
    device = dev;
    check(cudaSetDevice(device), "cudaSetDevice");
    check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    set_smem(reinterpret_cast<const void*>(k_nt_factor), kSmemNtFactor);
    set_smem(reinterpret_cast<const void*>(k_nt_svd), kSmemNt);
    set_smem(reinterpret_cast<const void*>(k_congruence), kSmemCong);
    set_smem(reinterpret_cast<const void*>(k_circ_op), kSmemCirc);
    set_smem(reinterpret_cast<const void*>(k_step_length), kSmemStep);
    set_smem(reinterpret_cast<const void*>(k_margins), kSmemMarg);
    set_smem(reinterpret_cast<const void*>(k_schur_transform), kSmemTrans);
    set_smem(reinterpret_cast<const void*>(k_trsm_panel), kSmemTrsm);
    set_smem(reinterpret_cast<const void*>(k_syrk_update), kSmemSyrk);
    set_smem(reinterpret_cast<const void*>(k_trinv_level), kSmemTrinv);
    set_smem(reinterpret_cast<const void*>(k_potrf_diag), kSmemTrtri);
    set_smem(reinterpret_cast<const void*>(k_chol_dataflow), kSmemDf);
    set_smem(reinterpret_cast<const void*>(k_gram_basis), kSmemGram);
    set_smem(reinterpret_cast<const void*>(k_gram_adjoint), kSmemGram);
    {
      const char* g = std::getenv("SDPX_B200_GRAM");  // "0": ordinary Schur form for every block
      gram_enabled = !(g && g[0] == '0');
      const char* c = std::getenv("SDPX_B200_GRAPHS");  // "0": launch every segment eagerly
      graphs_enabled = !(c && c[0] == '0');
      const char* f = std::getenv("SDPX_B200_FORM");  // "split": split-precision factorisation
      factor_form = (f && std::string(f) == "split") ? kFormSplit : kFormPlain;
    }
    red.init();
    status_.alloc(1);
    hstat_.alloc(1);
    for (auto& e : ev_) check(cudaEventCreate(&e), "event create");
  }

  // host-side upload breakdown of the last upload (structure, rank-one test, device copies)
  std::string upload_report() const {
    char buf[160];
    std::snprintf(buf, sizeof buf, "structure %.3f s, rank-one test %.3f s, copies %.3f s",
                  up_t_[0], up_t_[1], up_t_[2]);
    return buf;
  }

  void upload(const HostProblem& p) {
    const auto u0 = std::chrono::steady_clock::now();
    clear_graphs();
    factor_ok_ = false;  // the factor (and its inverse) belong to the previous problem
    n = p.n;
    m = p.m;
    hblocks.clear();
    nn_rows.clear();
    {
      std::vector<std::pair<int, int>> cl = p.cones;
      if (cl.empty())
        for (int d : p.psd) cl.push_back({3, d});
      int row = 0, mat = 0, vec = 0;
      for (const auto& c : cl) {
        if (c.first == 3) {
          const int d = c.second;
          if (d > SDPXG_NMAX) throw std::invalid_argument("PSD block order above 64 is not supported");
          hblocks.push_back({d, row, mat, vec});
          row += d * (d + 1) / 2;
          mat += d * d;
          vec += d;
        } else if (c.first == 1) {
          for (int i = 0; i < c.second; ++i) nn_rows.push_back(row + i);
          row += c.second;
        } else {
          throw std::invalid_argument("cone kind not supported on the GPU path");
        }
      }
      if (row != m) throw std::invalid_argument("cone rows do not match A");
      matlen_ = mat;
      veclen_ = vec;
    }
    nblk = (int)hblocks.size();
    nnn_ = (int)nn_rows.size();
    // per-block dense column storage of A.  Columns of A are independent: the block memberships,
    // the dense columns and the rank-one tests run on the host threads (rows within a column are
    // sorted, so a block's entries are one contiguous range found by binary search).
    hk.assign(nblk, 0);
    std::vector<std::vector<std::pair<int, int>>> c2b(n);  // (block, local)
    parallel_for(n, col_grain(n, p.Aval.size()), [&](int64_t c0, int64_t c1, int) {
      for (int64_t c = c0; c < c1; ++c) {
        const int64_t p0 = p.Acolptr[c], p1 = p.Acolptr[c + 1];
        int64_t q0 = p0;
        for (int j = 0; j < nblk && q0 < p1; ++j) {
          const int r0 = hblocks[j].svec_off, r1 = r0 + hblocks[j].n * (hblocks[j].n + 1) / 2;
          q0 = std::lower_bound(p.Arow.begin() + q0, p.Arow.begin() + p1, (int64_t)r0) - p.Arow.begin();
          const int64_t q1 =
              std::lower_bound(p.Arow.begin() + q0, p.Arow.begin() + p1, (int64_t)r1) - p.Arow.begin();
          if (q1 > q0) c2b[c].push_back({j, 0});
          q0 = q1;
        }
      }
    });
    std::vector<std::vector<int>> bcols(nblk);
    for (int c = 0; c < n; ++c)
      for (auto& e : c2b[c]) {
        e.second = hk[e.first]++;
        bcols[e.first].push_back(c);
      }
    std::vector<long> acol_off(nblk), s_off(nblk);
    std::vector<int> col_ptr(nblk + 1, 0), col_idx;
    long aoff = 0, soff = 0;
    for (int j = 0; j < nblk; ++j) {
      int tn = hblocks[j].n * (hblocks[j].n + 1) / 2;
      acol_off[j] = aoff;
      aoff += (long)tn * hk[j];
      s_off[j] = soff;
      soff += (long)hk[j] * hk[j];
      col_ptr[j + 1] = col_ptr[j] + hk[j];
      col_idx.insert(col_idx.end(), bcols[j].begin(), bcols[j].end());
    }
    // (block, local column) items in block order: item i is column i - col_ptr[j] of block j
    const int nitems = col_ptr[nblk];
    std::vector<int> item_blk(nitems);
    for (int j = 0; j < nblk; ++j)
      for (int t = col_ptr[j]; t < col_ptr[j + 1]; ++t) item_blk[t] = j;
    F64Vec acol(aoff);
    const int64_t item_grain = std::max<int64_t>(1, nitems * 65536LL / std::max<int64_t>(aoff, 1));
    parallel_for(nitems, item_grain, [&](int64_t i0, int64_t i1, int) {
      for (int64_t it = i0; it < i1; ++it) {
        const int j = item_blk[it], t = (int)(it - col_ptr[j]), c = bcols[j][t];
        const int r0 = hblocks[j].svec_off, tn = hblocks[j].n * (hblocks[j].n + 1) / 2;
        double* dst = &acol[acol_off[j] + (long)t * tn];
        std::fill(dst, dst + tn, 0.0);
        const int64_t p1 = p.Acolptr[c + 1];
        int64_t q = std::lower_bound(p.Arow.begin() + p.Acolptr[c], p.Arow.begin() + p1, (int64_t)r0) -
                    p.Arow.begin();
        for (; q < p1 && p.Arow[q] < r0 + tn; ++q) dst[p.Arow[q] - r0] = p.Aval[q];
      }
    });
    const auto u1 = std::chrono::steady_clock::now();
    // rank-one (Gram) blocks keep only their factor; the others keep dense columns
    std::vector<char> gram(nblk, 0);
    std::vector<long> gu_off(nblk, 0);
    std::vector<double> gu, gsig(col_ptr[nblk], 1.0);
    ngram_ = 0;
    std::vector<const HostProblem::Sampled*> sampled_of(nblk, nullptr), ms_of(nblk, nullptr);
    for (const auto& sb : p.sampled) {
      int j = 0;
      while (j < nblk && hblocks[j].svec_off != sb.row_start) ++j;
      const int prims = sb.dim * (sb.dim + 1) / 2 * sb.count;
      if (j == nblk || hblocks[j].n != sb.order || hk[j] != prims)
        throw std::invalid_argument("sampled block does not match its PSD cone or columns");
      for (int t = 0; t < prims; ++t)
        if (bcols[j][t] != sb.col0 + t) throw std::invalid_argument("sampled block columns are not its own");
      (sb.dim == 1 ? sampled_of : ms_of)[j] = &sb;
    }
    if (gram_enabled || !p.sampled.empty()) {
      std::vector<long> u_off(nblk + 1, 0);
      for (int j = 0; j < nblk; ++j) u_off[j + 1] = u_off[j] + (long)hblocks[j].n * hk[j];
      std::vector<double> u_all(u_off[nblk]);
      std::vector<char> col_ok(nitems, 0);
      parallel_for(nitems, item_grain, [&](int64_t i0, int64_t i1, int) {
        for (int64_t it = i0; it < i1; ++it) {
          const int j = item_blk[it], t = (int)(it - col_ptr[j]);
          const int nj = hblocks[j].n, tn = nj * (nj + 1) / 2;
          if (const HostProblem::Sampled* sb = sampled_of[j]) {  // the given factor, exactly
            std::copy(sb->basis.begin() + (long)t * nj, sb->basis.begin() + (long)(t + 1) * nj,
                      u_all.begin() + u_off[j] + (long)t * nj);
            gsig[it] = sb->weight[t];
            col_ok[it] = 1;
          } else if (gram_enabled && !ms_of[j]) {
            col_ok[it] = rank_one_column(&acol[acol_off[j] + (long)t * tn], nj,
                                         &u_all[u_off[j] + (long)t * nj], &gsig[it]);
          }
        }
      });
      for (int j = 0; j < nblk; ++j) {
        if (hk[j] == 0) continue;
        bool ok = true;
        for (int t = col_ptr[j]; t < col_ptr[j + 1] && ok; ++t) ok = col_ok[t] != 0;
        if (!ok) {
          for (int t = col_ptr[j]; t < col_ptr[j + 1]; ++t) gsig[t] = 1.0;
          continue;
        }
        gram[j] = 1;
        ngram_++;
        gu_off[j] = (long)gu.size();
        gu.insert(gu.end(), u_all.begin() + u_off[j], u_all.begin() + u_off[j + 1]);
      }
    }
    // matrix-valued sampled blocks (dim > 1) keep their factors in a form of their own
    nms_ = 0;
    std::vector<MsDesc> msd;
    std::vector<double> msq, msw(col_ptr[nblk], 0.0);
    std::vector<int> mspairs(2 * (size_t)std::max(col_ptr[nblk], 1), 0);
    long msv = 0, msk = 0;
    int ms_rmax = 0, ms_kmax = 0, ms_tnmax = 0;
    for (int j = 0; j < nblk; ++j) {
      const HostProblem::Sampled* sb = ms_of[j];
      if (!sb) continue;
      gram[j] = 2;
      const int D = sb->dim, h = sb->order / D, c = sb->count, r = D * c;
      MsDesc d{j, D, h, c, (long)msq.size(), msv, msk};
      msd.push_back(d);
      msq.insert(msq.end(), sb->basis.begin(), sb->basis.end());
      msv += (long)hblocks[j].n * r;
      msk += (long)r * r;
      ms_rmax = std::max(ms_rmax, r);
      ms_kmax = std::max(ms_kmax, hk[j]);
      ms_tnmax = std::max(ms_tnmax, hblocks[j].n * (hblocks[j].n + 1) / 2);
      int t = 0;
      for (int ss = 0; ss < D; ++ss)
        for (int rr = 0; rr <= ss; ++rr)
          for (int k = 0; k < c; ++k, ++t) {  // primitive (s, r, k): the pair (r c + k, s c + k)
            msw[col_ptr[j] + t] = sb->weight[t];
            mspairs[2 * (col_ptr[j] + t)] = rr * c + k;
            mspairs[2 * (col_ptr[j] + t) + 1] = ss * c + k;
          }
      nms_++;
    }
    if (ngram_ > 0 || nms_ > 0) {  // repack the dense columns of the ordinary blocks only
      F64Vec packed;
      long off = 0;
      for (int j = 0; j < nblk; ++j) {
        const long len = (long)hblocks[j].n * (hblocks[j].n + 1) / 2 * hk[j];
        if (gram[j]) {
          acol_off[j] = 0;
          continue;
        }
        packed.insert(packed.end(), acol.begin() + acol_off[j], acol.begin() + acol_off[j] + len);
        acol_off[j] = off;
        off += len;
      }
      acol.swap(packed);
      aoff = off;
    }
    const auto u2 = std::chrono::steady_clock::now();
    std::vector<int> c2b_ptr(n + 1, 0), c2b_blk, c2b_loc;
    for (int c = 0; c < n; ++c) {
      for (auto& e : c2b[c]) {
        c2b_blk.push_back(e.first);
        c2b_loc.push_back(e.second);
      }
      c2b_ptr[c + 1] = (int)c2b_blk.size();
    }
    std::vector<int> wblk, wloc, tiles, gtiles, gitem_blk, gitem_c0, gblk;
    for (int j = 0; j < nblk; ++j) {
      if (gram[j] == 2) continue;  // matrix-valued sampled: kernels of their own
      if (gram[j]) {
        gblk.push_back(j);
        for (int c0 = 0; c0 < hk[j]; c0 += 64) {
          gitem_blk.push_back(j);
          gitem_c0.push_back(c0);
        }
      } else {
        for (int t = 0; t < hk[j]; ++t) {
          wblk.push_back(j);
          wloc.push_back(t);
        }
      }
      std::vector<int>& tl = gram[j] ? gtiles : tiles;
      int nt = (hk[j] + 31) / 32;
      for (int tj = 0; tj < nt; ++tj)
        for (int ti = 0; ti < nt; ++ti) {
          tl.push_back(j);
          tl.push_back(ti);
          tl.push_back(tj);
        }
    }
    ncol_ = col_ptr[nblk];
    ngtiles_ = (int)gtiles.size() / 3;
    ngitem_ = (int)gitem_blk.size();
    ngblk_ = (int)gblk.size();
    gU_.alloc(std::max<size_t>(gu.size(), 1)); gU_.upload(gu.data(), gu.size(), st);
    gV_.alloc(std::max<size_t>(gu.size(), 1));
    gsig_.alloc(std::max<size_t>(gsig.size(), 1)); gsig_.upload(gsig.data(), gsig.size(), st);
    gu_off_.alloc(std::max(nblk, 1)); gu_off_.upload(gu_off.data(), nblk, st);
    gtiles_.alloc(std::max<size_t>(gtiles.size(), 1)); gtiles_.upload(gtiles.data(), gtiles.size(), st);
    gitem_blk_.alloc(std::max(ngitem_, 1)); gitem_blk_.upload(gitem_blk.data(), gitem_blk.size(), st);
    gitem_c0_.alloc(std::max(ngitem_, 1)); gitem_c0_.upload(gitem_c0.data(), gitem_c0.size(), st);
    gblk_.alloc(std::max(ngblk_, 1)); gblk_.upload(gblk.data(), gblk.size(), st);
    ms_desc_.alloc(std::max(nms_, 1)); ms_desc_.upload(msd.data(), msd.size(), st);
    ms_q_.alloc(std::max<size_t>(msq.size(), 1)); ms_q_.upload(msq.data(), msq.size(), st);
    ms_w_.alloc(std::max<size_t>(msw.size(), 1)); ms_w_.upload(msw.data(), msw.size(), st);
    ms_pairs_.alloc(mspairs.size()); ms_pairs_.upload(mspairs.data(), mspairs.size(), st);
    ms_v_.alloc(std::max<long>(msv, 1));
    ms_k_.alloc(std::max<long>(msk, 1));
    ms_rmax_ = ms_rmax;
    ms_kmax_ = ms_kmax;
    ms_tnmax_ = ms_tnmax;
    gf_part_.alloc((size_t)std::max(ngitem_, 1) * SDPXG_NMAX * SDPXG_NMAX);
    gf_cnt_.alloc(std::max(nblk, 1));
    check(cudaMemsetAsync(gf_cnt_.p, 0, std::max(nblk, 1) * sizeof(unsigned), st), "gram tickets");
    nwork_ = (int)wblk.size();
    ntiles_ = (int)tiles.size() / 3;
    // symmetric P in CSR (both triangles) for the x-row products
    std::vector<std::vector<std::pair<int, double>>> prow(n);
    for (int c = 0; c < n; ++c)
      for (int64_t q = p.Pcolptr[c]; q < p.Pcolptr[c + 1]; ++q) {
        int r = (int)p.Prow[q];
        if (r > c) continue;
        prow[r].push_back({c, p.Pval[q]});
        if (r != c) prow[c].push_back({r, p.Pval[q]});
      }
    std::vector<int> prp(n + 1, 0), pci;
    std::vector<double> pv;
    for (int r = 0; r < n; ++r) {
      std::sort(prow[r].begin(), prow[r].end());
      for (auto& e : prow[r]) {
        pci.push_back(e.first);
        pv.push_back(e.second);
      }
      prp[r + 1] = (int)pci.size();
    }
    p_nnz_ = (int)pci.size();
    std::vector<int> pup_ptr(n + 1, 0), pup_row;
    std::vector<double> pup_val;
    for (int c = 0; c < n; ++c) {
      for (int64_t q = p.Pcolptr[c]; q < p.Pcolptr[c + 1]; ++q)
        if (p.Prow[q] <= c) {
          pup_row.push_back((int)p.Prow[q]);
          pup_val.push_back(p.Pval[q]);
        }
      pup_ptr[c + 1] = (int)pup_row.size();
    }

    blocks_.alloc(nblk);
    blocks_.upload(hblocks.data(), nblk, st);
    R_.alloc(matlen_); Rinv_.alloc(matlen_); Ginv_.alloc(matlen_);
    lam_.alloc(veclen_); lisqrt_.alloc(veclen_);
    acol_.alloc(aoff); acol_.upload(acol.data(), aoff, st);
    tcol_.alloc(aoff);
    S_.alloc(std::max<long>(soff, 1));
    acol_off_.alloc(nblk); acol_off_.upload(acol_off.data(), nblk, st);
    s_off_.alloc(nblk); s_off_.upload(s_off.data(), nblk, st);
    kcount_.alloc(nblk); kcount_.upload(hk.data(), nblk, st);
    col_ptr_.alloc(nblk + 1); col_ptr_.upload(col_ptr.data(), nblk + 1, st);
    col_idx_.alloc(std::max<size_t>(col_idx.size(), 1)); col_idx_.upload(col_idx.data(), col_idx.size(), st);
    c2b_ptr_.alloc(n + 1); c2b_ptr_.upload(c2b_ptr.data(), n + 1, st);
    c2b_blk_.alloc(std::max<size_t>(c2b_blk.size(), 1)); c2b_blk_.upload(c2b_blk.data(), c2b_blk.size(), st);
    c2b_loc_.alloc(std::max<size_t>(c2b_loc.size(), 1)); c2b_loc_.upload(c2b_loc.data(), c2b_loc.size(), st);
    wblk_.alloc(std::max(nwork_, 1)); wblk_.upload(wblk.data(), wblk.size(), st);
    wloc_.alloc(std::max(nwork_, 1)); wloc_.upload(wloc.data(), wloc.size(), st);
    {  // 64-row tiles of every block for the forward product
      std::vector<int> fb, fr;
      for (int j = 0; j < nblk; ++j) {
        if (gram[j]) continue;  // Gram and matrix-valued sampled blocks have their own operators
        int tn = hblocks[j].n * (hblocks[j].n + 1) / 2;
        for (int r0 = 0; r0 < tn; r0 += 64) {
          fb.push_back(j);
          fr.push_back(r0);
        }
      }
      nftile_ = (int)fb.size();
      ftile_blk_.alloc(std::max(nftile_, 1)); ftile_blk_.upload(fb.data(), fb.size(), st);
      ftile_r0_.alloc(std::max(nftile_, 1)); ftile_r0_.upload(fr.data(), fr.size(), st);
    }
    tiles_.alloc(std::max<size_t>(tiles.size(), 1)); tiles_.upload(tiles.data(), tiles.size(), st);
    prp_.alloc(n + 1); prp_.upload(prp.data(), n + 1, st);
    pci_.alloc(std::max(p_nnz_, 1)); pci_.upload(pci.data(), pci.size(), st);
    pv_.alloc(std::max(p_nnz_, 1)); pv_.upload(pv.data(), pv.size(), st);
    pup_ptr_.alloc(n + 1); pup_ptr_.upload(pup_ptr.data(), n + 1, st);
    pup_row_.alloc(std::max<size_t>(pup_row.size(), 1)); pup_row_.upload(pup_row.data(), pup_row.size(), st);
    pup_val_.alloc(std::max<size_t>(pup_val.size(), 1)); pup_val_.upload(pup_val.data(), pup_val.size(), st);
    pup_nnz_ = (int)pup_row.size();
    adj_part_.alloc(std::max<size_t>((size_t)ncol_ * 2, 1));
    nchol = (n + kNB - 1) / kNB;
    Hsave_.alloc((size_t)n * n);
    F_.alloc((size_t)n * n);
    Dinv_.alloc((size_t)std::max(nchol, 1) * kNB * kNB);
    diag0_.alloc(std::max(n, 1));
    tri_y_.alloc(std::max(n, 1));
    gv_part_.alloc((size_t)std::max(n, 1) * ((n + 255) / 256 + 1));
    gv_cnt_.alloc(std::max(n, 1));
    check(cudaMemsetAsync(gv_cnt_.p, 0, gv_cnt_.n * sizeof(unsigned), st), "gemv counters");
    Uinv_.alloc((size_t)n * n);
    UinvT_.alloc((size_t)n * n);
    Tmp_.alloc((size_t)n * n);
    make_schedule(nchol, df_list_, df_sync_, &df_items_, &df_grid_);
    if (split_active()) prepare_split();
    step_out_.alloc(2 * (nblk + 1));
    hblk_.alloc(2 * (nblk + 1));
    {  // nonnegative-orthant rows: index list and their rows of A, dense (nnn x n)
      nn_idx_.alloc(std::max(nnn_, 1));
      nn_idx_.upload(nn_rows.data(), nn_rows.size(), st);
      nnw_.alloc(std::max(nnn_, 1));
      nnlam_.alloc(std::max(nnn_, 1));
      std::vector<double> ann((size_t)nnn_ * n, 0.0);
      if (nnn_) {
        std::vector<int> pos(m, -1);
        for (int i = 0; i < nnn_; ++i) pos[nn_rows[i]] = i;
        for (int c = 0; c < n; ++c)
          for (int64_t q = p.Acolptr[c]; q < p.Acolptr[c + 1]; ++q) {
            const int r = (int)p.Arow[q];
            if (pos[r] >= 0) ann[(size_t)pos[r] + (size_t)c * nnn_] = p.Aval[q];
          }
      }
      Ann_.alloc(std::max<size_t>(ann.size(), 1));
      Ann_.upload(ann.data(), ann.size(), st);
    }
    marg_out_.alloc(2 * (nblk + 1));
    scal_.alloc(4);
    check(cudaStreamSynchronize(st), "upload sync");
    const auto u3 = std::chrono::steady_clock::now();
    auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    up_t_[0] = sec(u0, u1);
    up_t_[1] = sec(u1, u2);
    up_t_[2] = sec(u2, u3);
  }

  // ---- status word ----
  void clear_status() { check(cudaMemsetAsync(status_.p, 0, sizeof(uint32_t), st), "memset"); }
  uint32_t read_status() {
    copy_d2h(hstat_.p, status_.p, sizeof(uint32_t), st);
    check(cudaStreamSynchronize(st), "status sync");
    return hstat_[0];
  }

  // ---- cone scaling ----
  void identity_scaling() {
    if (nblk) ++g_launches, k_identity_scaling<<<nblk, 256, 0, st>>>(blocks_, R_, Rinv_, Ginv_, lam_, lisqrt_);
    if (nnn_) ++g_launches, k_nn_identity<<<(nnn_ + 255) / 256, 256, 0, st>>>(nnn_, nnw_, nnlam_);
  }
  bool nt_scale(const double* s, const double* z) {
    need(s, "nt_scale s");
    need(z, "nt_scale z");
    clear_status();
    tbegin(KT_SCALE);
    if (nblk) {
      ++g_launches, k_nt_factor<<<nblk, SDPXG_CONE_THREADS, kSmemNtFactor, st>>>(blocks_, s, z, R_, Rinv_,
                                                                                  status_);
      ++g_launches, k_nt_svd<<<nblk, SDPXG_NT_SVD_THREADS, kSmemNt, st>>>(blocks_, R_, Rinv_, Ginv_, lam_,
                                                                           lisqrt_, status_);
    }
    if (nnn_)
      ++g_launches, k_nn_scale<<<(nnn_ + 255) / 256, 256, 0, st>>>(nnn_, nn_idx_, s, z, nnw_, nnlam_, status_);
    launched("k_nt_factor, k_nt_svd");
    tend(KT_SCALE);
    return read_status() == 0;
  }

  // Scaling given by the caller (the condensed KKT's sync from the cones' R and R^-1): per PSD
  // block the n_j x n_j column-major R and R^-1 stacked in cone order (sum n_j^2 each); G^-1 =
  // R^-T R^-1 is formed on the device.  lambda is not set (only the Schur assembly and the
  // operators read this scaling).
  void set_scaling(const double* hR, const double* hRinv) {
    if (!nblk) return;
    if (!hR || !hRinv) throw std::invalid_argument("null pointer");
    R_.upload(hR, matlen_, st);
    Rinv_.upload(hRinv, matlen_, st);
    ++g_launches, k_ginv_from_rinv<<<nblk, 256, 0, st>>>(blocks_, Rinv_, Ginv_);
    launched("k_ginv_from_rinv");
    check(cudaStreamSynchronize(st), "scaling sync");
  }

  // y = op(x) for cone operator `mode`, ncols columns with stride ld.
  void cone_apply(int mode, const double* x, double* y, int ncols = 1, long ld = 0) {
    need(x, "cone_apply x");
    need(y, "cone_apply y");
    if (!nblk && !nnn_) return;
    tbegin(KT_CONE);
    if (nblk)
      ++g_launches, k_congruence<<<dim3(nblk, ncols), SDPXG_CONE_THREADS, kSmemCong, st>>>(
          blocks_, mode, R_, Rinv_, x, y, ld ? ld : m);
    if (nnn_)
      ++g_launches, k_nn_cone<<<dim3((nnn_ + 255) / 256, ncols), 256, 0, st>>>(nnn_, nn_idx_, mode, nnw_, x,
                                                                               y, ld ? ld : m);
    launched("k_congruence");
    tend(KT_CONE);
  }
  void circ_op(const double* y, const double* z, double* x) {
    need(y, "circ y");
    need(z, "circ z");
    need(x, "circ x");
    if (nblk) ++g_launches, k_circ_op<<<nblk, SDPXG_CONE_THREADS, kSmemCirc, st>>>(blocks_, y, z, x);
    if (nnn_) ++g_launches, k_nn_circ<<<(nnn_ + 255) / 256, 256, 0, st>>>(nnn_, nn_idx_, y, z, x);
    launched("k_circ_op");
  }
  void lam_inv_circ(const double* z, double* x) {
    need(z, "lam_inv z");
    need(x, "lam_inv x");
    if (nblk) ++g_launches, k_lam_inv_circ<<<nblk, 256, 0, st>>>(blocks_, lam_, z, x);
    if (nnn_) ++g_launches, k_nn_lam_inv<<<(nnn_ + 255) / 256, 256, 0, st>>>(nnn_, nn_idx_, nnlam_, z, x);
  }
  void affine_ds(double* ds) {
    need(ds, "affine_ds");
    if (nblk) ++g_launches, k_affine_ds<<<nblk, 256, 0, st>>>(blocks_, lam_, ds);
    if (nnn_) ++g_launches, k_nn_affine_ds<<<(nnn_ + 255) / 256, 256, 0, st>>>(nnn_, nn_idx_, nnlam_, ds);
  }
  void shift_unit(double* v, double a) {
    need(v, "shift_unit");
    if (nblk) ++g_launches, k_shift_unit<<<nblk, 64, 0, st>>>(blocks_, v, a);
    if (nnn_) ++g_launches, k_nn_shift<<<(nnn_ + 255) / 256, 256, 0, st>>>(nnn_, nn_idx_, v, a);
  }
  // per-block (dual, primal) bounds; returns false on an eigen failure
  bool step_bounds(const double* dz, const double* ds, double amax, int mode, double* az,
                   double* as) {
    need(dz, "step dz");
    need(ds, "step ds");
    *az = amax;
    *as = amax;
    if (!nblk && !nnn_) return true;
    clear_status();
    tbegin(KT_STEP);
    if (nblk)
      ++g_launches, k_step_length<<<dim3(nblk, 2), SDPXG_CONE_THREADS, kSmemStep, st>>>(
          blocks_, R_, Rinv_, lisqrt_, dz, ds, amax, mode, step_out_, status_);
    if (nnn_)
      ++g_launches, k_nn_step<<<1, 256, 0, st>>>(nnn_, nn_idx_, nnw_, nnlam_, dz, ds, amax, mode,
                                                 step_out_.p + 2 * nblk);
    launched("k_step_length");
    tend(KT_STEP);
    const PinnedBuf<double>& h = hblk_;
    const int parts = nblk + (nnn_ ? 1 : 0);
    copy_d2h(hblk_.p, step_out_.p, 2 * parts * sizeof(double), st);
    uint32_t s = read_status();
    for (int j = 0; j < parts; ++j) {
      *az = std::min(*az, h[2 * j]);
      *as = std::min(*as, h[2 * j + 1]);
    }
    return s == 0;
  }
  // (lambda_min, sum of positive eigenvalues) per PSD block of v, then (min, sum of positive
  // entries) over the orthant rows when there are any
  // min_only: per PSD block min(lambda_min, 0) and 0 (the original-coordinate acceptance
  // test); otherwise lambda_min and the sum of the positive eigenvalues.
  bool margins(const double* v, std::vector<double>& out, bool min_only = false) {
    need(v, "margins v");
    const int parts = nblk + (nnn_ ? 1 : 0);
    out.assign(2 * parts, 0.0);
    if (!parts) return true;
    clear_status();
    if (nblk)
      ++g_launches, k_margins<<<dim3(nblk, 1), SDPXG_CONE_THREADS, kSmemMarg, st>>>(blocks_, v, m, marg_out_,
                                                                                    status_, min_only ? 1 : 0);
    if (nnn_) ++g_launches, k_nn_margins<<<1, 256, 0, st>>>(nnn_, nn_idx_, v, marg_out_.p + 2 * nblk);
    launched("k_margins");
    copy_d2h(hblk_.p, marg_out_.p, 2 * parts * sizeof(double), st);
    const bool ok = read_status() == 0;
    for (int j = 0; j < 2 * parts; ++j) out[j] = hblk_[j];
    return ok;
  }

  // ---- constraint operator ----
  // y = alpha * A x + beta * y   (rows m)
  void A_forward(const double* x, double alpha, double beta, double* y) {
    need(x, "A_forward x");
    need(y, "A_forward y");
    if (nnn_) {
      ++g_launches, k_nn_forward<<<(nnn_ + 255) / 256, 256, 0, st>>>(nnn_, n, nn_idx_, Ann_, x, alpha, beta,
                                                                     y);
      launched("k_nn_forward");
    }
    if (!nblk) return;
    if (nftile_) {
      ++g_launches, k_op_forward<<<dim3(nftile_, 1), 256, 0, st>>>(
          blocks_, kcount_, col_ptr_, col_idx_, acol_off_, acol_, ftile_blk_, ftile_r0_, x, n, alpha,
          beta, y, m);
      launched("k_op_forward");
    }
    if (nms_) {
      ++g_launches, k_ms_forward<<<dim3(nms_, (ms_tnmax_ + 255) / 256), 256, 0, st>>>(
          blocks_, ms_desc_, col_ptr_, col_idx_, ms_w_, ms_q_, x, alpha, beta, y);
      launched("k_ms_forward");
    }
    if (ngblk_) {
      ++g_launches, k_gram_forward<<<ngitem_, 256, 0, st>>>(
          blocks_, gitem_blk_, gitem_c0_, kcount_, col_ptr_, col_idx_, gu_off_, gsig_, gU_, x,
          alpha, beta, y, gf_part_, gf_cnt_);
      launched("k_gram_forward");
    }
  }
  // y = alpha * A' z + beta * y   (length n)
  void A_adjoint(const double* z, double alpha, double beta, double* y) {
    need(z, "A_adjoint z");
    need(y, "A_adjoint y");
    if (nwork_) {
      int wpb = 8;
      ++g_launches, k_op_adjoint_partial<<<dim3((nwork_ + wpb - 1) / wpb, 1), 256, 0, st>>>(
          blocks_, wblk_, wloc_, col_ptr_, acol_off_, acol_, z, m, adj_part_, ncol_, nwork_);
      launched("k_op_adjoint_partial");
    }
    if (nms_) {
      ++g_launches, k_ms_adjoint<<<dim3(nms_, (ms_kmax_ + 127) / 128), 128, 0, st>>>(
          blocks_, ms_desc_, kcount_, col_ptr_, ms_w_, ms_pairs_, ms_q_, z, adj_part_);
      launched("k_ms_adjoint");
    }
    if (ngitem_) {
      ++g_launches, k_gram_adjoint<<<ngitem_, 256, kSmemGram, st>>>(
          blocks_, gitem_blk_, gitem_c0_, kcount_, col_ptr_, gu_off_, gsig_, gU_, z, adj_part_);
      launched("k_gram_adjoint");
    }
    if (n) {
      ++g_launches, k_op_adjoint_gather<<<dim3((n + 255) / 256, 1), 256, 0, st>>>(
          n, c2b_ptr_, c2b_blk_, c2b_loc_, col_ptr_, adj_part_, ncol_, alpha, beta, y, n);
      launched("k_op_adjoint_gather");
    }
    if (n && nnn_) {
      ++g_launches, k_nn_adjoint<<<(n + 7) / 8, 256, 0, st>>>(nnn_, n, nn_idx_, Ann_, z, alpha, y);
      launched("k_nn_adjoint");
    }
  }
  // y = alpha * P x + beta * y  (P symmetric)
  void P_mult(const double* x, double alpha, double beta, double* y) {
    need(x, "P_mult x");
    need(y, "P_mult y");
    if (!n) return;
    if (p_nnz_ == 0) {
      lincomb(n, 0.0, nullptr, beta, beta == 0.0 ? nullptr : y, 0.0, nullptr, y);
      return;
    }
    ++g_launches, k_csr_spmv<<<(n + 255) / 256, 256, 0, st>>>(n, prp_, pci_, pv_, x, alpha, beta, y);
    launched("k_csr_spmv");
  }
  bool has_P() const { return p_nnz_ > 0; }

  // ---- Schur complement ----
  bool assemble() {
    factor_ok_ = false;  // the factor no longer matches the Schur complement being rebuilt
    tbegin(KT_ASSEMBLE);
    if (nwork_) {
      ++g_launches, k_schur_transform<<<nwork_, SDPXG_CONE_THREADS, kSmemTrans, st>>>(blocks_, wblk_, wloc_, acol_off_,
                                                                   Ginv_, acol_, tcol_);
      launched("k_schur_transform");
      ++g_launches, k_schur_block_gemm<<<ntiles_, 256, 0, st>>>(blocks_, tiles_, kcount_, acol_off_, s_off_, acol_,
                                                  tcol_, S_);
      launched("k_schur_block_gemm");
    }
    if (ngitem_) {  // rank-one blocks: V = Rinv U, S = (sigma sigma') o (V'V)^2
      ++g_launches, k_gram_basis<<<ngitem_, 256, kSmemGram, st>>>(blocks_, gitem_blk_, gitem_c0_, kcount_,
                                                                 gu_off_, Rinv_, gU_, gV_);
      launched("k_gram_basis");
      ++g_launches, k_gram_schur<<<ngtiles_, 256, 0, st>>>(blocks_, gtiles_, kcount_, col_ptr_, gu_off_,
                                                          s_off_, gsig_, gV_, S_);
      launched("k_gram_schur");
    }
    if (nms_) {  // matrix-valued sampled blocks: V = Rinv U, K = V'V, S from K
      ++g_launches, k_ms_basis<<<dim3(nms_, (ms_rmax_ + 7) / 8), 256, 0, st>>>(blocks_, ms_desc_, Rinv_, ms_q_,
                                                                           ms_v_);
      ++g_launches, k_ms_gram<<<dim3(nms_, (unsigned)(((long)ms_rmax_ * ms_rmax_ + 255) / 256)), 256, 0, st>>>(
          blocks_, ms_desc_, ms_v_, ms_k_);
      ++g_launches, k_ms_schur<<<dim3(nms_, (unsigned)(((long)ms_kmax_ * ms_kmax_ + 255) / 256)), 256, 0, st>>>(
          ms_desc_, kcount_, col_ptr_, s_off_, ms_w_, ms_pairs_, ms_k_, S_);
      launched("k_ms_schur");
    }
    long tot = (long)n * n;
    if (tot) {
      ++g_launches, k_schur_gather<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, c2b_ptr_, c2b_blk_, c2b_loc_,
                                                                  kcount_, s_off_, S_, Hsave_);
      launched("k_schur_gather");
    }
    if (pup_nnz_) {
      ++g_launches, k_add_upper_csc<<<(n + 255) / 256, 256, 0, st>>>(n, pup_ptr_, pup_row_, pup_val_, Hsave_);
    }
    if (nnn_ && n) {  // orthant rows: H += A_nn' diag(1 / w^2) A_nn
      const unsigned t = (n + 31) / 32;
      ++g_launches, k_nn_schur<<<dim3(t, t), 256, 0, st>>>(nnn_, n, Ann_, nnw_, Hsave_);
      launched("k_nn_schur");
    }
    tend(KT_ASSEMBLE);
    int s = red.add(st, RED_FINITE, tot, Hsave_, nullptr);
    return red.fetch(st)[s] == 1.0;
  }
  double schur_diag_absmax() {
    if (!n) return 0.0;
    ++g_launches, k_diag_absmax<<<1, 1024, 0, st>>>(Hsave_, n, scal_);
    copy_d2h(hblk_.p, scal_.p, sizeof(double), st);
    check(cudaStreamSynchronize(st), "diag sync");
    return hblk_[0];
  }
  // Storage of one dense factorisation: source matrix H (contiguous n x n), its shifted copy
  // that becomes U, the diagonal-tile inverses, the original diagonal, the explicit inverse X
  // and its transpose, a GEMM scratch, and the dataflow work list.
  struct FactorBufs {
    int n = 0, nchol = 0, df_items = 0, df_grid = 0;
    const double* H = nullptr;
    double *F = nullptr, *Dinv = nullptr, *diag0 = nullptr, *Uinv = nullptr, *UinvT = nullptr, *Tmp = nullptr;
    const unsigned* df_list = nullptr;
    int* df_sync = nullptr;
  };
  // A diagonal block of the split form with storage of its own (contiguous, so every dense
  // kernel runs on it unchanged).
  struct SubFactor {
    DevBuf<double> H, F, Dinv, diag0, Uinv, UinvT, Tmp;
    DevBuf<unsigned> df_list;
    DevBuf<int> df_sync;
    FactorBufs b;
  };

  // The dataflow work list of an nt x nt tile grid (validated before upload) and its grid size.
  void make_schedule(int nt, DevBuf<unsigned>& list, DevBuf<int>& sync, int* items_out, int* grid_out) {
    *items_out = 0;
    *grid_out = 0;
    if (nt <= 0 || nt > kDfMaxTiles) return;
    std::vector<unsigned> items = chol_schedule(nt);
    if (!chol_schedule_valid(items, nt)) throw CudaError("invalid Cholesky work list");
    list.alloc(items.size());
    list.upload(items.data(), items.size(), st);
    sync.alloc(2 + 2 * (size_t)nt * nt);
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    // one CTA per SM: the chain CTA (the critical path) then has its SM to itself; the
    // trailing updates are far from saturating the others
    *items_out = (int)items.size();
    *grid_out = std::max(1, std::min(sms, *items_out));
  }

  FactorBufs full_bufs() {
    FactorBufs b;
    b.n = n; b.nchol = nchol; b.df_items = df_items_; b.df_grid = df_grid_;
    b.H = Hsave_; b.F = F_; b.Dinv = Dinv_; b.diag0 = diag0_; b.Uinv = Uinv_; b.UinvT = UinvT_; b.Tmp = Tmp_;
    b.df_list = df_list_; b.df_sync = df_sync_;
    return b;
  }

  void setup_sub(SubFactor& s, int ns) {
    const int nt = (ns + kNB - 1) / kNB;
    s.H.alloc((size_t)ns * ns);
    s.F.alloc((size_t)ns * ns);
    s.Dinv.alloc((size_t)nt * kNB * kNB);
    s.diag0.alloc(ns);
    s.Uinv.alloc((size_t)ns * ns);
    s.UinvT.alloc((size_t)ns * ns);
    s.Tmp.alloc((size_t)ns * ns);
    s.b = FactorBufs();
    s.b.n = ns;
    s.b.nchol = nt;
    make_schedule(nt, s.df_list, s.df_sync, &s.b.df_items, &s.b.df_grid);
    s.b.H = s.H; s.b.F = s.F; s.b.Dinv = s.Dinv; s.b.diag0 = s.diag0; s.b.Uinv = s.Uinv;
    s.b.UinvT = s.UinvT; s.b.Tmp = s.Tmp; s.b.df_list = s.df_list; s.b.df_sync = s.df_sync;
  }
  int split_n1() const { return ((n / 2 + kNB - 1) / kNB) * kNB; }
  void prepare_split() {
    const int n1 = split_n1(), n2 = n - n1;
    if (sub1_.b.n != n1) setup_sub(sub1_, n1);
    if (sub2_.b.n != n2) setup_sub(sub2_, n2);
  }

  // F = chol(H + eps I) of one factorisation's buffers (dynamic pivot rule); the status word
  // collects pivot failures.  diag_src (stride diag_stride): when given, the pivot rule's
  // original diagonal is taken from there (+ eps) instead of from H.
  void launch_chol(const FactorBufs& b, double eps, bool dynamic, double dyn_eps, double dyn_delta,
                   const double* diag_src = nullptr, long diag_stride = 0) {
    ++g_launches, k_shifted_copy<<<1184, 256, 0, st>>>(b.H, b.F, b.n, eps, b.diag0);
    if (diag_src)
      ++g_launches, k_strided_diag<<<(b.n + 255) / 256, 256, 0, st>>>(diag_src, diag_stride, b.n, eps, b.diag0);
    if (b.df_items > 0) {  // one persistent launch over the whole tile schedule
      check(cudaMemsetAsync(b.df_sync, 0, (2 + 2 * (size_t)b.nchol * b.nchol) * sizeof(int), st),
            "dataflow sync reset");
      ++g_launches, k_chol_dataflow<<<b.df_grid, 256, kSmemDf, st>>>(
          b.F, b.n, b.nchol, b.df_list, b.df_items, b.df_sync, dyn_eps, dyn_delta, dynamic ? 1 : 0, b.diag0,
          b.Dinv, status_);
    }
    for (int kb = 0; b.df_items == 0 && kb < b.nchol; ++kb) {
      ++g_launches, k_potrf_diag<<<1, 1024, kSmemTrtri, st>>>(b.F, b.n, kb, dyn_eps, dyn_delta, dynamic ? 1 : 0,
                                                              b.diag0, b.Dinv, status_);
      int rest = b.nchol - kb - 1;
      if (rest > 0) {
        ++g_launches, k_trsm_panel<<<rest, SDPXG_THREADS, kSmemTrsm, st>>>(b.F, b.n, kb, b.Dinv);
        ++g_launches, k_syrk_update<<<rest * (rest + 1) / 2, SDPXG_THREADS, kSmemSyrk, st>>>(b.F, b.n, kb);
      }
    }
    launched("factor");
  }
  // X = U^-1 of one factorisation: diagonal tiles, then one batched GEMM pair per level.
  void launch_trinv(const FactorBufs& b) {
    ++g_launches, k_trtri_diag<<<b.nchol, SDPXG_THREADS, 0, st>>>(b.n, b.Dinv, b.Uinv, b.UinvT);
    for (int level = 1; (1 << (level - 1)) < b.nchol; ++level) {
      const int g = 1 << level, h = g >> 1;
      dim3 grid(h, h, (b.nchol + g - 1) / g);
      for (int phase = 0; phase < 2; ++phase)
        ++g_launches, k_trinv_level<<<grid, SDPXG_THREADS, kSmemTrinv, st>>>(b.F, b.Uinv, b.UinvT, b.Tmp, b.n,
                                                                             level, phase);
    }
    launched("trinv");
  }
  void copy_block(double* dst, long ldd, const double* src, long lds, int rows, int cols) {
    if (rows <= 0 || cols <= 0) return;
    check(cudaMemcpy2DAsync(dst, ldd * sizeof(double), src, lds * sizeof(double), rows * sizeof(double), cols,
                            cudaMemcpyDeviceToDevice, st),
          "block copy");
  }

  // F = chol(Hsave + eps I) with the dynamic pivot rule, then X = F^-1 explicitly.
  bool factor(double eps, bool dynamic, double dyn_eps, double dyn_delta) {
    factor_ok_ = false;
    if (!n) return true;
    if (split_active()) return factor_split(eps, dynamic, dyn_eps, dyn_delta);
    clear_status();
    const FactorBufs b = full_bufs();
    tbegin(KT_FACTOR);
    launch_chol(b, eps, dynamic, dyn_eps, dyn_delta);
    tend(KT_FACTOR);
    uint32_t s = read_status();
    if (s & SDPXG_ST_SYNC_TIMEOUT) throw CudaError("factorization: a bounded inter-CTA wait gave up");
    factor_ok_ = (s == 0);
    if (factor_ok_) {
      tbegin(KT_TRINV);
      launch_trinv(b);
      tend(KT_TRINV);
    }
    return factor_ok_;
  }

  // The split form (kFormSplit).  With n1 = n/2 rounded up to the tile and n2 = n - n1:
  //   U11' U11 = H11 + eps I (FP64 dataflow), X11 = U11^-1 (FP64)
  //   U12 = X11' H12                       split-precision GEMM
  //   U22' U22 = H22 + eps I - U12' U12      split-precision GEMM, then FP64 dataflow, X22 (FP64)
  //   X12 = -(X11 U12) X22                  two split-precision GEMMs
  // so that U = [U11 U12; 0 U22] and X = U^-1 = [X11 X12; 0 X22], with the same pivot rule on
  // the same original diagonal as the plain form.  Only the upper triangles of X and U and the
  // lower triangle of X' are assembled (the solves read nothing else).
  bool factor_split(double eps, bool dynamic, double dyn_eps, double dyn_delta) {
    prepare_split();
    const int n1 = split_n1(), n2 = n - n1;
    const long ldn = n;
    clear_status();
    check(cudaMemsetAsync(oz_status_word(), 0, sizeof(uint32_t), st), "memset");
    // phase timers: the dataflow launches under KT_FACTOR, the diagonal-block inverses under
    // KT_TRINV, the split-precision products and the assembly under KT_SPLIT
    copy_block(sub1_.H, n1, Hsave_, ldn, n1, n1);
    copy_block(sub2_.H, n2, Hsave_ + (long)n1 * ldn + n1, ldn, n2, n2);
    tbegin(KT_FACTOR);
    launch_chol(sub1_.b, eps, dynamic, dyn_eps, dyn_delta);
    tend(KT_FACTOR);
    // the inverse kernels write the upper triangles only; the split-precision products read
    // X11 and X22 whole, so their lower triangles must be zeros, not a recycled block's contents
    check(cudaMemsetAsync(sub1_.Uinv.p, 0, (size_t)n1 * n1 * sizeof(double), st), "memset");
    check(cudaMemsetAsync(sub2_.Uinv.p, 0, (size_t)n2 * n2 * sizeof(double), st), "memset");
    tbegin(KT_TRINV);
    launch_trinv(sub1_.b);
    tend(KT_TRINV);
    double* U12 = F_.p + (long)n1 * ldn;  // F[0:n1, n1:n]
    tbegin(KT_SPLIT);
    // U12 = X11' H12: rows of the left operand are the columns of X11, rows of the right
    // operand the columns of H12
    ozaki_gemm(oz, st, n1, n2, n1, sub1_.Uinv, n1, 1, Hsave_.p + (long)n1 * ldn, ldn, 1, 1.0, 0.0, U12, ldn, 0);
    // S = H22 - U12' U12 (full, exactly symmetric: the integer product of an operand with itself)
    ozaki_gemm(oz, st, n2, n2, n1, U12, ldn, 1, U12, ldn, 1, -1.0, 1.0, sub2_.H, n2, 0);
    tend(KT_SPLIT);
    // the pivot rule's original diagonal is that of H22 + eps I, as in the plain form
    tbegin(KT_FACTOR);
    launch_chol(sub2_.b, eps, dynamic, dyn_eps, dyn_delta, Hsave_.p + (long)n1 * ldn + n1, ldn + 1);
    tend(KT_FACTOR);
    tbegin(KT_TRINV);
    launch_trinv(sub2_.b);
    tend(KT_TRINV);
    tbegin(KT_SPLIT);
    // X12 = -(X11 U12) X22
    ozaki_gemm(oz, st, n1, n2, n1, sub1_.Uinv, 1, n1, U12, ldn, 1, 1.0, 0.0, Tmp_, n1, 0);
    ozaki_gemm(oz, st, n1, n2, n2, Tmp_, 1, n1, sub2_.Uinv, n2, 1, -1.0, 0.0, Uinv_.p + (long)n1 * ldn, ldn, 0);
    // assemble U, X and X'
    copy_block(F_, ldn, sub1_.F, n1, n1, n1);
    copy_block(F_.p + (long)n1 * ldn + n1, ldn, sub2_.F, n2, n2, n2);
    copy_block(Uinv_, ldn, sub1_.Uinv, n1, n1, n1);
    copy_block(Uinv_.p + (long)n1 * ldn + n1, ldn, sub2_.Uinv, n2, n2, n2);
    copy_block(UinvT_, ldn, sub1_.UinvT, n1, n1, n1);
    copy_block(UinvT_.p + (long)n1 * ldn + n1, ldn, sub2_.UinvT, n2, n2, n2);
    ++g_launches, k_transpose_block<<<dim3((n2 + 31) / 32, (n1 + 31) / 32), dim3(32, 8), 0, st>>>(
        Uinv_.p + (long)n1 * ldn, ldn, n1, n2, UinvT_.p + n1, ldn);
    launched("split factor");
    tend(KT_SPLIT);
    uint32_t s = read_status();
    if (s & SDPXG_ST_SYNC_TIMEOUT) throw CudaError("factorization: a bounded inter-CTA wait gave up");
    uint32_t hs[2] = {0, 0};
    copy_d2h(&hs[0], oz.status.p, sizeof(uint32_t), st);
    copy_d2h(&hs[1], oz.err.p, sizeof(uint32_t), st);
    check(cudaStreamSynchronize(st), "split status");
    if (hs[1]) throw CudaError("split-precision GEMM: a bounded wait gave up");
    factor_ok_ = (s == 0 && hs[0] == 0);
    return factor_ok_;
  }
  uint32_t* oz_status_word() {
    if (!oz.status.p) oz.status.alloc(1);
    return oz.status.p;
  }
  // x = F^-1 r = U^-1 (U^-T r) through the explicit inverse: two coalesced GEMVs.
  void trisolve(const double* r, double* x) {
    need(r, "trisolve r");
    need(x, "trisolve x");
    tbegin(KT_TRISOLVE);
    // y = X' b: column dots on X (upper); x = X y: column dots on the stored X' (lower)
    const dim3 grid((n + 7) / 8, (n + 255) / 256);
    ++g_launches, k_coldot_seg<<<grid, 256, 0, st>>>(Uinv_, n, 1, r, nullptr, 1.0, tri_y_, gv_part_,
                                                     gv_cnt_);
    ++g_launches, k_coldot_seg<<<grid, 256, 0, st>>>(UinvT_, n, 2, tri_y_, nullptr, 1.0, x, gv_part_,
                                                     gv_cnt_);
    launched("trisolve");
    tend(KT_TRISOLVE);
  }
  // e = r - Hsave x
  void schur_residual(const double* r, const double* x, double* e) {
    need(r, "schur_residual r");
    need(x, "schur_residual x");
    need(e, "schur_residual e");
    if (!n) return;
    tbegin(KT_SYMV);
    const dim3 grid((n + 7) / 8, (n + 255) / 256);  // H symmetric: column i . x = (H x)_i
    ++g_launches, k_coldot_seg<<<grid, 256, 0, st>>>(Hsave_, n, 0, x, r, -1.0, e, gv_part_, gv_cnt_);
    launched("schur_residual");
    tend(KT_SYMV);
  }

  void lincomb(long len, double a, const double* x, double b, const double* y, double c,
               const double* w, double* out) {
    if (len <= 0) return;
    need(out, "lincomb out");
    int grid = (int)std::min<long>((len + 255) / 256, 1184);
    ++g_launches, k_lincomb<<<grid, 256, 0, st>>>(len, a, x, b, y, c, w, out);
  }
  // Independent updates out = a x + b y + c w in one launch (the same values as one lincomb
  // each).  A copy is {len, 1.0, 0.0, 0.0, src, nullptr, nullptr, dst}.  The outputs must not
  // be read by another request of the same batch.
  void lincomb_batch(std::initializer_list<LinReq> reqs) {
    const int k = (int)reqs.size();
    if (k == 0 || k > kLinBatchMax) throw std::invalid_argument("update batch size");
    LinBatch b{};
    long mx = 0;
    int i = 0;
    for (const LinReq& q : reqs) {
      if (q.n > 0) need(q.out, "lincomb out");
      b.r[i++] = q;
      mx = std::max(mx, q.n);
    }
    if (mx <= 0) return;
    const int grid = (int)std::min<long>((mx + 255) / 256, 1184);
    ++g_launches, k_lincomb_batch<<<dim3(grid, k), 256, 0, st>>>(b);
  }
  static LinReq cp(double* dst, const double* src, long len) {
    return LinReq{len, 1.0, 0.0, 0.0, src, nullptr, nullptr, dst};
  }
  void copy(double* dst, const double* src, long len) {
    if (len > 0) {
      need(dst, "copy dst");
      need(src, "copy src");
    }
    if (len > 0)
      check(cudaMemcpyAsync(dst, src, len * sizeof(double), cudaMemcpyDeviceToDevice, st), "d2d");
  }

  double* Hsave() { return Hsave_.p; }
  const double* uinv() const { return Uinv_.p; }
  const double* uinvT() const { return UinvT_.p; }
  bool factored() const { return factor_ok_; }
  double* F() { return F_.p; }
  const BlockDesc* blocks() const { return blocks_.p; }

 private:
  static void set_smem(const void* fn, size_t bytes) {
    check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
          "cudaFuncSetAttribute");
  }
  void launched(const char* what) { check(cudaGetLastError(), what); }

  double up_t_[3] = {0, 0, 0};
  int matlen_ = 0, veclen_ = 0, nwork_ = 0, ntiles_ = 0, p_nnz_ = 0, pup_nnz_ = 0;
  bool factor_ok_ = false;
  DevBuf<BlockDesc> blocks_;
  DevBuf<double> R_, Rinv_, Ginv_, lam_, lisqrt_;
  DevBuf<double> acol_, tcol_, S_;
  DevBuf<long> acol_off_, s_off_;
  DevBuf<int> kcount_, col_ptr_, col_idx_, c2b_ptr_, c2b_blk_, c2b_loc_, wblk_, wloc_, tiles_;
  DevBuf<int> ftile_blk_, ftile_r0_;
  int nftile_ = 0;
  // nonnegative-orthant rows
  int nnn_ = 0;
  DevBuf<int> nn_idx_;
  DevBuf<double> nnw_, nnlam_, Ann_;
  // rank-one (Gram) blocks
  DevBuf<double> gU_, gV_, gsig_;
  DevBuf<long> gu_off_;
  DevBuf<int> gtiles_, gitem_blk_, gitem_c0_, gblk_;
  DevBuf<double> gf_part_;  // k_gram_forward chunk partials (64 x 64 per item)
  DevBuf<unsigned> gf_cnt_;  // its per-block arrival tickets (self-resetting)
  int ngram_ = 0, ngtiles_ = 0, ngitem_ = 0, ngblk_ = 0, ncol_ = 0;
  // matrix-valued sampled blocks (dim > 1)
  int nms_ = 0, ms_rmax_ = 0, ms_kmax_ = 0, ms_tnmax_ = 0;
  DevBuf<MsDesc> ms_desc_;
  DevBuf<double> ms_q_, ms_w_, ms_v_, ms_k_;
  DevBuf<int> ms_pairs_;
  DevBuf<int> prp_, pci_, pup_ptr_, pup_row_;
  DevBuf<double> pv_, pup_val_;
  DevBuf<double> adj_part_;
  DevBuf<double> Hsave_, F_, Dinv_, diag0_, tri_y_, Uinv_, UinvT_, Tmp_;
  DevBuf<double> gv_part_;   // k_coldot_seg segment sums (segments x n)
  DevBuf<unsigned> gv_cnt_;  // k_coldot_seg column tickets (self-resetting)
  DevBuf<double> step_out_, marg_out_, scal_;
  DevBuf<uint32_t> status_;
  PinnedBuf<uint32_t> hstat_;
  PinnedBuf<double> hblk_;  // per-block scalars read back (step bounds, margins)
  DevBuf<unsigned> df_list_;
  DevBuf<int> df_sync_;
  int df_items_ = 0, df_grid_ = 0;
  SubFactor sub1_, sub2_;  // diagonal blocks of the split form
  cudaEvent_t ev_[2 * KT_N] = {};
  struct GraphEntry {
    cudaGraphExec_t exec;
    int red_count;
    uint64_t launches;
  };
  static constexpr size_t kMaxGraphs = 256;
  std::unordered_map<std::string, GraphEntry> graphs_;
  std::unordered_map<std::string, Program> programs_;
};

}  // namespace sdpxg
