// Host driver of the homogeneous self-dual interior-point iteration over the device engine.
//
// A restatement of the reference's binary64 predictor/corrector
// (crates/solver/src/solver/core/solver.rs:285-1472, default/variables.rs:148-788,
// default/kktsystem.rs:186-655, default/residuals.rs:340-490, default/info.rs:89-537) with
// the condensed KKT system of kkt/condensed/* and the refinement of kkt/refinement.rs.
// Vectors live on the device; the host keeps tau, kappa and the scalar summaries.
#pragma once
#include <chrono>
#include <cmath>
#include <limits>

#include "engine.cuh"

namespace sdpxg {

constexpr double kEps = 2.220446049250313e-16;

// Solver status codes of the reference C ABI (include/sdpx.h:76-80).
enum Status {
  ST_UNSOLVED = 0, ST_SOLVED = 1, ST_PRIMAL_INFEASIBLE = 2, ST_DUAL_INFEASIBLE = 3,
  ST_ALMOST_SOLVED = 4, ST_ALMOST_PRIMAL_INFEASIBLE = 5, ST_ALMOST_DUAL_INFEASIBLE = 6,
  ST_MAX_ITERATIONS = 7, ST_MAX_TIME = 8, ST_NUMERICAL_ERROR = 9, ST_INSUFFICIENT_PROGRESS = 10,
};

// Binary64 defaults of default/settings.rs:17-314.
struct Settings {
  int max_iter = 200;
  double time_limit = std::numeric_limits<double>::infinity();
  double max_step_fraction = 0.99;
  double tol_gap_abs = 1e-8, tol_gap_rel = 1e-8, tol_feas = 1e-8;
  double tol_infeas_abs = 1e-8, tol_infeas_rel = 1e-8, tol_ktratio = 1e-6;
  double reduced_tol_gap_abs = 5e-5, reduced_tol_gap_rel = 5e-5, reduced_tol_feas = 1e-4;
  double reduced_tol_infeas_abs = 5e-12, reduced_tol_infeas_rel = 5e-5, reduced_tol_ktratio = 1e-4;
  double tol_original = 1e-6;  // <= 0 disables the original-coordinate test
  bool equilibrate_enable = true;
  int equilibrate_max_iter = 10;
  double equilibrate_min_scaling = 1e-4, equilibrate_max_scaling = 1e4;
  bool static_reg_enable = true;
  double static_reg_constant = 1e-8, static_reg_proportional = kEps * kEps;
  bool dynamic_reg_enable = true;
  double dynamic_reg_eps = 1e-13, dynamic_reg_delta = 2e-7;
  bool ir_enable = true;
  double ir_reltol = 1e-13, ir_abstol = 1e-12;
  int ir_max_iter = 10;
  double ir_stop_ratio = 5.0;
};

struct Equilibration {
  std::vector<double> d, dinv, e, einv;
  double c = 1.0;
};

struct Info {
  int status = ST_UNSOLVED;
  int iterations = 0;
  double cost_primal = 0, cost_dual = 0, res_primal = 0, res_dual = 0;
  double res_primal_inf = 0, res_dual_inf = 0, gap_abs = 0, gap_rel = 0, ktratio = 0;
  double solve_time = 0;
  double rz_ns = 0, rx_ns = 0;
};

struct PhaseTimes {
  double residual = 0, scale = 0, assemble = 0, factor = 0, solve = 0, step = 0, other = 0;
  int factorizations = 0, kkt_solves = 0, outer_refinements = 0, inner_refinements = 0;
  int device_kkt_solves = 0;  // KKT solves whose refinement ran as one device-driven graph
};

class HsdSolver {
 public:
  HsdSolver(Engine& eng, const HostProblem& p, const Equilibration& eq, const Settings& st)
      : E(eng), eq_(eq), st_(st), n_(p.n), m_(p.m) {
    reset(p, eq, st);
  }

  // Take a new problem (other dimensions, equilibration or settings) on the same engine: the
  // work vectors grow if needed and are otherwise reused.
  void reset(const HostProblem& p, const Equilibration& eq, const Settings& st) {
    eq_ = eq;
    st_ = st;
    n_ = p.n;
    m_ = p.m;
    const int n = n_, m = m_;
    E.clear_graphs();  // segments captured for earlier work vectors must not be replayed
    ctl_.alloc(1);
    hctl_.alloc(1);
    auto vn = [&](DevBuf<double>& b) { b.alloc(std::max(n, 1)); };
    auto vm = [&](DevBuf<double>& b) { b.alloc(std::max(m, 1)); };
    for (auto* b : {&x_, &px_, &bx_, &rx_, &rxinf_, &Px_, &x2_, &dx_, &ax_, &tx_, &prevx_, &bestx_,
                    &rhsx_, &x1_, &xhat_, &en_, &dxn_, &candn_, &e2n_, &ex_, &cx_, &candx_, &ex2_,
                    &negq_, &q_, &d_, &dinv_, &wn_})
      vn(*b);
    for (auto* b : {&s_, &z_, &ps_, &pz_, &rz_, &rzinf_, &z2_, &ds_, &dz_, &as_, &az_, &ts_, &tz_,
                    &prevs_, &prevz_, &bests_, &bestz_, &rhsz_, &rhss_, &cvec_, &workz_, &z1_,
                    &tm_, &ez_, &cz_, &candz_, &ez2_, &wm1_, &wm2_, &wm3_, &b_, &e_, &einv_, &nn_e_,
                    &nn_einv_})
      vm(*b);
    load(p);
  }

  // (Re)load the problem vectors; the device work vectors stay allocated across solves, so a
  // handle that solves repeatedly (sdpx_update, parameter sweeps) allocates nothing per solve.
  void load(const HostProblem& p) {
    const int n = n_, m = m_;
    const Equilibration& eq = eq_;
    if (p.n != n || p.m != m) throw std::invalid_argument("problem dimensions changed");
    q_.upload(p.q.data(), n, E.st);
    b_.upload(p.b.data(), m, E.st);
    std::vector<double> nq(p.q);
    for (auto& v : nq) v = -v;
    negq_.upload(nq.data(), n, E.st);
    d_.upload(eq.d.data(), n, E.st);
    dinv_.upload(eq.dinv.data(), n, E.st);
    e_.upload(eq.e.data(), m, E.st);
    einv_.upload(eq.einv.data(), m, E.st);
    degree_ = 0;
    for (int d : p.psd) degree_ += d;
    degree_ += E.nn_count();  // an orthant of dimension d has degree d
    {  // original-coordinate scales of the orthant rows (zero on PSD rows: a row mask)
      std::vector<double> ne(m, 0.0), nei(m, 0.0);
      for (int r : E.nn_rows) {
        ne[r] = eq.e[r];
        nei[r] = eq.einv[r];
      }
      nn_e_.upload(ne.data(), m, E.st);
      nn_einv_.upload(nei.data(), m, E.st);
    }
    // scaled norms of the data (default/problemdata.rs:444-465)
    normq_ = 0;
    for (int i = 0; i < n; ++i) normq_ = std::max(normq_, std::fabs(p.q[i] * eq.dinv[i]));
    normq_ /= eq.c;
    normb_ = 0;
    for (int i = 0; i < m; ++i) normb_ = std::max(normb_, std::fabs(p.b[i] * eq.einv[i]));
    data_scale_ = 1.0;
    for (double v : p.b) data_scale_ = std::max(data_scale_, std::fabs(v));
    for (double v : p.q) data_scale_ = std::max(data_scale_, std::fabs(v));
    for (double v : p.Aval) data_scale_ = std::max(data_scale_, std::fabs(v));
    dmax_ = 1.0;
    for (double v : eq.d) dmax_ = std::max(dmax_, v);
  }

  Info info;
  PhaseTimes times;
  std::vector<double> hx, hs, hz;  // unscaled solution

  void solve();
  // (u, v) = K^-1 [gx; gz - Hs gs] in original coordinates, K = [P A'; A -Hs] re-factored at the
  // NT scaling of the final point (the solution's sensitivities; see sdpx_b200_adjoint).
  bool adjoint(const std::vector<double>& gx, const std::vector<double>& gz,
               const std::vector<double>& gs, std::vector<double>& u, std::vector<double>& v);

  // ---------------- KKT system (also driven directly by the kernel-level ABI) ----------------
  bool kkt_update();
  bool reduced_solve(const double* r, double* x);
  void reduced_first(const double* r, double* x);
  bool reduced_refine(const double* r, double* x, double normb, double norme);
  void condense_first(const double* bx, const double* bz, double* x);
  void recover(const double* bz, const double* x, double* z);
  bool solve_raw(const double* bx, const double* bz, double* x, double* z);
  bool kkt_solve(const double* bx, const double* bz, double* x, double* z);
  // The same refined solve as ONE CUDA graph whose refinement loops run on the device (WHILE
  // nodes driven by the control kernels of refine_ctl.cu): one host read per solve.
  bool kkt_solve_graph(const double* bx, const double* bz, double* x, double* z);
  void residual_full(const double* bx, const double* bz, const double* x, const double* z,
                     double* ex, double* ez);

 private:
  using clock = std::chrono::steady_clock;
  static double secs(clock::time_point a) {
    return std::chrono::duration<double>(clock::now() - a).count();
  }
  cudaStream_t st() const { return E.st; }
  // ---------------- HSD pieces ----------------
  struct Resid { double qx, bz, sz, xPx, rtau; double norms[8]; };
  Resid residuals();
  void update_info(const Resid& r);
  bool is_solved(double ga, double gr, double feas) const;
  void check_convergence(const Resid& r, bool full);
  bool check_termination(const Resid& r, int iter);
  double original_ratio(bool reduced);
  bool hsd_direction(const double* rhs_x, const double* workz, double rhs_tau, double rhs_kappa,
                     const double* rhs_z, const double* x1, const double* z1, double* dtau,
                     double* dkappa);
  double step_bounds(const double* dz, const double* ds, double dtau, double dkappa, int mode,
                     double amax_cap);
  bool default_start();
  double tolerance_multiple(const Info& in) const {
    double gap = std::min(in.gap_abs / st_.tol_gap_abs, in.gap_rel / st_.tol_gap_rel);
    return std::max(std::max(in.res_primal, in.res_dual) / st_.tol_feas, gap);
  }

  Engine& E;
  Equilibration eq_;
  Settings st_;
  int n_, m_, degree_ = 0;
  double normq_ = 0, normb_ = 0, data_scale_ = 1, dmax_ = 1;
  double tau_ = 1, kappa_ = 1;
  double best_tau_ = 1, best_kappa_ = 1;
  int reg_boost_ = 0;
  Info prev_;
  bool have_prev_ = false;
  // device vectors (n-length then m-length groups)
  DevBuf<RefineCtl> ctl_;
  PinnedBuf<RefineCtl> hctl_;
  bool program_failed_ = false;  // building the device-driven solve failed once: host-driven
  DevBuf<double> x_, px_, bx_, rx_, rxinf_, Px_, x2_, dx_, ax_, tx_, prevx_, bestx_, rhsx_, x1_,
      xhat_, en_, dxn_, candn_, e2n_, ex_, cx_, candx_, ex2_, negq_, q_, d_, dinv_, wn_;
  DevBuf<double> s_, z_, ps_, pz_, rz_, rzinf_, z2_, ds_, dz_, as_, az_, ts_, tz_, prevs_, prevz_,
      bests_, bestz_, rhsz_, rhss_, cvec_, workz_, z1_, tm_, ez_, cz_, candz_, ez2_, wm1_, wm2_, wm3_,
      b_, e_, einv_, nn_e_, nn_einv_;
};

// ------------------------------------------------------------------------------------------
// KKT: assemble + factor with the static shift and its escalation (kkt/direct/solver.rs:758-877,
// 511-520, 1473-1485)
// ------------------------------------------------------------------------------------------
inline bool HsdSolver::kkt_update() {
  auto t0 = clock::now();
  bool ok = E.assemble();
  times.assemble += secs(t0);
  if (!ok) return false;
  auto t1 = clock::now();
  double diag = E.schur_diag_absmax();
  for (;;) {
    double eps = 0.0;
    if (st_.static_reg_enable) {
      eps = st_.static_reg_constant + st_.static_reg_proportional * diag;
      if (reg_boost_ > 0) eps *= std::pow(100.0, reg_boost_);
    }
    times.factorizations++;
    ok = E.factor(eps, st_.dynamic_reg_enable, st_.dynamic_reg_eps, st_.dynamic_reg_delta);
    if (ok || !st_.static_reg_enable || reg_boost_ >= 3) break;
    reg_boost_++;
  }
  times.factor += secs(t1);
  return ok;
}

// Captured segments of the KKT solve (Engine::segment): ids of the straight runs between the
// host reads of the refinement norms.
enum : int { SEG_RS_HEAD = 1, SEG_RS_STEP = 2, SEG_RAW_HEAD = 3, SEG_RAW_TAIL = 4,
             SEG_KKT_HEAD = 5, SEG_KKT_TAIL = 6, SEG_OUT_HEAD = 7, SEG_OUT_TAIL = 8 };

// First pass of the reduced solve: x = F^-1 r and e = r - H x (unshifted Schur).
// Queues |r|max, |e|max and finite(x).
inline void HsdSolver::reduced_first(const double* r, double* x) {
  const int n = n_;
  E.trisolve(r, x);
  E.schur_residual(r, x, en_);
  E.red.add_batch(st(), {{RED_MAXABS, n, r, nullptr}, {RED_MAXABS, n, en_, nullptr}, {RED_FINITE, n, x, nullptr}});
}

// Stationary refinement of the reduced system against the unshifted Schur complement, from the
// norms of the first pass (kkt/refinement.rs:118-191 stopping rules).
inline bool HsdSolver::reduced_refine(const double* r, double* x, double normb, double norme) {
  const int n = n_;
  const double tol = st_.ir_abstol + st_.ir_reltol * normb;
  bool converged = norme <= tol;
  for (int it = 0; it < st_.ir_max_iter && !converged; ++it) {
    double previous = norme;
    times.inner_refinements++;
    E.segment(SEG_RS_STEP, {r, x}, [&] {
      E.trisolve(en_, dxn_);
      E.lincomb(n, 1.0, x, 1.0, dxn_, 0.0, nullptr, candn_);
      E.schur_residual(r, candn_, e2n_);
      E.red.add(st(), RED_MAXABS, n, e2n_, nullptr);
    });
    norme = E.red.fetch(st())[0];
    if (!std::isfinite(norme)) return false;
    double ratio = previous / norme;
    if (ratio < st_.ir_stop_ratio) {
      if (ratio > 1.0) E.copy(x, candn_, n);
      break;
    }
    E.copy(x, candn_, n);
    E.copy(en_, e2n_, n);
    converged = norme <= tol;
  }
  return true;
}

inline bool HsdSolver::reduced_solve(const double* r, double* x) {
  if (!st_.ir_enable) {
    E.trisolve(r, x);
    return true;
  }
  E.segment(SEG_RS_HEAD, {r, x}, [&] { reduced_first(r, x); });
  auto& h = E.red.fetch(st());
  const double normb = h[0], norme = h[1];
  if (h[2] != 1.0 || !std::isfinite(norme)) return false;
  return reduced_refine(r, x, normb, norme);
}

// Condense: xhat = bx + A' Hs^-1 bz (kkt/condensed/mod.rs:2416-2507), then the first pass.
inline void HsdSolver::condense_first(const double* bx, const double* bz, double* x) {
  E.cone_apply(CM_HINV, bz, tm_);     // Hs^-1 bz
  E.copy(xhat_, bx, n_);
  E.A_adjoint(tm_, 1.0, 1.0, xhat_);  // bx + A' Hs^-1 bz
  reduced_first(xhat_, x);
}

// Recover z = Hs^-1 (A x - bz) (kkt/condensed/mod.rs:2511-2604).
inline void HsdSolver::recover(const double* bz, const double* x, double* z) {
  E.lincomb(m_, -1.0, bz, 0.0, nullptr, 0.0, nullptr, tm_);
  E.A_forward(x, 1.0, 1.0, tm_);  // A x - bz
  E.cone_apply(CM_HINV, tm_, z);
}

// Condense, reduced solve, recover (kkt/condensed/mod.rs:2416-2622).
inline bool HsdSolver::solve_raw(const double* bx, const double* bz, double* x, double* z) {
  if (!st_.ir_enable) {
    E.cone_apply(CM_HINV, bz, tm_);
    E.copy(xhat_, bx, n_);
    E.A_adjoint(tm_, 1.0, 1.0, xhat_);
    E.trisolve(xhat_, x);
    recover(bz, x, z);
    return true;
  }
  E.segment(SEG_RAW_HEAD, {bx, bz, x}, [&] { condense_first(bx, bz, x); });
  auto& h = E.red.fetch(st());
  if (h[2] != 1.0 || !std::isfinite(h[1])) return false;
  if (!reduced_refine(xhat_, x, h[0], h[1])) return false;
  E.segment(SEG_RAW_TAIL, {bz, x, z}, [&] { recover(bz, x, z); });
  return true;
}

// e = b - [P A'; A -Hs] [x; z] against the unshifted original operator.
inline void HsdSolver::residual_full(const double* bx, const double* bz, const double* x,
                                     const double* z, double* ex, double* ez) {
  E.P_mult(x, -1.0, 0.0, wn_);
  E.lincomb(n_, 1.0, bx, 1.0, wn_, 0.0, nullptr, ex);
  E.A_adjoint(z, -1.0, 1.0, ex);
  E.cone_apply(CM_HS, z, wm3_);
  E.lincomb(m_, 1.0, bz, 1.0, wm3_, 0.0, nullptr, ez);
  E.A_forward(x, -1.0, 1.0, ez);
}

// Solve with outer refinement on the original operator (kkt/condensed/kkt.rs:275-318,
// kkt/refinement.rs:118-191).  The work between two host reads of refinement norms runs as one
// captured segment: right-hand-side check + condense + first reduced pass; recover + full
// residual; and the same pair for every outer correction.
inline bool HsdSolver::kkt_solve(const double* bx, const double* bz, double* x, double* z) {
  auto t0 = clock::now();
  times.kkt_solves++;
  const int n = n_, m = m_;
  if (!st_.ir_enable) {
    const int a = E.red.add_batch(st(), {{RED_FINITE, n, bx, nullptr}, {RED_FINITE, m, bz, nullptr}});
    auto& h = E.red.fetch(st());
    if (h[a] != 1.0 || h[a + 1] != 1.0) return false;
    const bool ok = solve_raw(bx, bz, x, z);
    times.solve += secs(t0);
    return ok;
  }
  if (E.graphs_enabled && !E.timing && !program_failed_ && n > 0 && m > 0 &&
      st_.ir_max_iter >= 0 && st_.ir_max_iter <= 64) {
    const bool ok = kkt_solve_graph(bx, bz, x, z);
    times.solve += secs(t0);
    return ok;
  }
  E.segment(SEG_KKT_HEAD, {bx, bz, x}, [&] {
    E.red.add_batch(st(), {{RED_FINITE, n, bx, nullptr}, {RED_FINITE, m, bz, nullptr}});
    condense_first(bx, bz, x);
  });
  {
    auto& h = E.red.fetch(st());
    if (h[0] != 1.0 || h[1] != 1.0) return false;  // non-finite right-hand side
    if (h[4] != 1.0 || !std::isfinite(h[3])) return false;
    const double normb = h[2], norme = h[3];
    if (!reduced_refine(xhat_, x, normb, norme)) return false;
  }
  E.segment(SEG_KKT_TAIL, {bx, bz, x, z}, [&] {
    recover(bz, x, z);
    residual_full(bx, bz, x, z, ex_, ez_);
    E.red.add_batch(st(), {{RED_MAXABS, n, bx, nullptr}, {RED_MAXABS, m, bz, nullptr},
                           {RED_MAXABS, n, ex_, nullptr}, {RED_MAXABS, m, ez_, nullptr}});
  });
  bool ok = true;
  auto& h = E.red.fetch(st());
  const double normb = std::max(h[0], h[1]);
  double norme = std::max(h[2], h[3]);
  if (!std::isfinite(norme)) {
    ok = false;
  } else {
    const double tol = st_.ir_abstol + st_.ir_reltol * normb;
    bool converged = norme <= tol;
    for (int it = 0; it < st_.ir_max_iter && !converged; ++it) {
      double previous = norme;
      times.outer_refinements++;
      // correction (cx, cz) = K^-1 (ex, ez), same steps as solve_raw
      E.segment(SEG_OUT_HEAD, {ex_.p, ez_.p, cx_.p}, [&] { condense_first(ex_, ez_, cx_); });
      {
        auto& hc = E.red.fetch(st());
        if (hc[2] != 1.0 || !std::isfinite(hc[1]) || !reduced_refine(xhat_, cx_, hc[0], hc[1])) {
          ok = false;
          break;
        }
      }
      E.segment(SEG_OUT_TAIL, {bx, bz, x, z}, [&] {
        recover(ez_, cx_, cz_);
        E.lincomb_batch({LinReq{n, 1.0, 1.0, 0.0, x, cx_, nullptr, candx_},
                         LinReq{m, 1.0, 1.0, 0.0, z, cz_, nullptr, candz_}});
        residual_full(bx, bz, candx_, candz_, ex2_, ez2_);
        E.red.add_batch(st(), {{RED_MAXABS, n, ex2_, nullptr}, {RED_MAXABS, m, ez2_, nullptr}});
      });
      auto& hh = E.red.fetch(st());
      norme = std::max(hh[0], hh[1]);
      if (!std::isfinite(norme)) { ok = false; break; }
      double ratio = previous / norme;
      if (ratio < st_.ir_stop_ratio) {
        if (ratio > 1.0) {
          E.copy(x, candx_, n);
          E.copy(z, candz_, m);
        }
        break;
      }
      E.copy(x, candx_, n);
      E.copy(z, candz_, m);
      E.copy(ex_, ex2_, n);
      E.copy(ez_, ez2_, m);
      converged = norme <= tol;
    }
  }
  times.solve += secs(t0);
  return ok;
}

// Graph of one refined KKT solve (kkt_solve's steps, in its order):
//   head run (finite bx, bz; condense; first reduced pass) -> k_refine_head
//   WHILE inner: [trisolve e, candidate, reduced residual] -> k_refine_step -> keep candidate
//   tail run (recover; full residual; norms) -> k_refine_outer_init
//   WHILE outer: [condense (ex, ez); first pass] -> k_refine_head -> WHILE inner (on cx)
//                -> [recover; candidate (x, z); full residual] -> k_refine_outer_step -> keep
// Runs are captured once from the same Engine calls as the host-driven path; the graph is cached
// per (bx, bz, x, z, refinement settings) and replayed.
inline bool HsdSolver::kkt_solve_graph(const double* bx, const double* bz, double* x, double* z) {
  const int n = n_, m = m_;
  RefineParams prm{st_.ir_abstol, st_.ir_reltol, st_.ir_stop_ratio, st_.ir_max_iter, 0};
  prm.guard_max = (prm.max_iter + 1) * (prm.max_iter + 2) + 2;
  std::string key("KKT");
  for (const void* ptr : {(const void*)bx, (const void*)bz, (const void*)x, (const void*)z})
    key.append(reinterpret_cast<const char*>(&ptr), sizeof ptr);
  key.append(reinterpret_cast<const char*>(&prm), sizeof prm);
  Engine::Program* pg = E.find_program(key);
  if (!pg) {
    if (E.red.count() != 0) throw CudaError("a captured program must start with an empty reducer");
    const uint64_t launches0 = g_launches;  // capture counts launches that do not run
    RefineCtl* c = ctl_.p;
    const int* accept = &c->accept;
    const int* cont = &c->cont;
    const int* oaccept = &c->oaccept;
    const int* ocont = &c->ocont;
    cudaGraph_t G = nullptr;
    std::vector<cudaGraph_t> runs;  // captured runs, destroyed once cloned into G
    Engine::Program built;
    try {
      check(cudaGraphCreate(&G, 0), "graph create");
      auto child = [&](cudaGraph_t g, std::initializer_list<cudaGraphNode_t> deps,
                       cudaGraph_t run) {
        cudaGraphNode_t nd;
        std::vector<cudaGraphNode_t> d(deps);
        check(cudaGraphAddChildGraphNode(&nd, g, d.data(), d.size(), run), "child node");
        return nd;
      };
      auto kernel = [&](cudaGraph_t g, cudaGraphNode_t dep, const void* fn, void** args,
                        unsigned grid) {
        cudaKernelNodeParams kp{};
        kp.func = const_cast<void*>(fn);
        kp.gridDim = dim3(grid);
        kp.blockDim = dim3(grid > 1 ? 256 : 32);
        kp.kernelParams = args;
        cudaGraphNode_t nd;
        check(cudaGraphAddKernelNode(&nd, g, &dep, 1, &kp), "kernel node");
        return nd;
      };
      auto loop = [&](cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h,
                      cudaGraph_t* body) {
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t nd;
        check(cudaGraphAddNode(&nd, g, &dep, 1, &np), "while node");
        *body = np.conditional.phGraph_out[0];
        return nd;
      };
      auto run = [&](uint64_t* kernels, auto&& f) {
        E.red.set_count(0);
        cudaGraph_t g = E.capture(f, kernels);
        E.red.set_count(0);
        runs.push_back(g);
        return g;
      };
      const unsigned cgrid = (unsigned)std::min<long>((2L * std::max(n, m) + 255) / 256, 592);
      // inner refinement loop on (r, xx): body of a WHILE node
      uint64_t k_step = 0;
      auto inner = [&](cudaGraph_t body, const double* r, double* xx,
                       cudaGraphConditionalHandle h) {
        int se = 0;
        cudaGraph_t g = run(&k_step, [&] {
          E.trisolve(en_, dxn_);
          E.lincomb(n, 1.0, xx, 1.0, dxn_, 0.0, nullptr, candn_);
          E.schur_residual(r, candn_, e2n_);
          se = E.red.add(st(), RED_MAXABS, n, e2n_, nullptr);
        });
        cudaGraphNode_t a = child(body, {}, g);
        const double* p_se = E.red.slot(se);
        void* sa[] = {&p_se, &c, &prm, &h};
        cudaGraphNode_t b = kernel(body, a, (const void*)k_refine_step, sa, 1);
        long nn = n;
        double* d1 = xx;
        const double* s1 = candn_.p;
        double* d2 = en_.p;
        const double* s2 = e2n_.p;
        void* ca[] = {&accept, &nn, &d1, &s1, &cont, &nn, &d2, &s2};
        kernel(body, b, (const void*)k_refine_copy, ca, cgrid);
      };
      // head
      int h0 = 0, h1 = 0, hb = 0;
      uint64_t k_head = 0;
      cudaGraph_t g_head = run(&k_head, [&] {
        h0 = E.red.add_batch(st(), {{RED_FINITE, n, bx, nullptr}, {RED_FINITE, m, bz, nullptr}});
        h1 = h0 + 1;
        hb = E.red.count();
        condense_first(bx, bz, x);
      });
      cudaGraphNode_t nh = child(G, {}, g_head);
      cudaGraphConditionalHandle hin;
      check(cudaGraphConditionalHandleCreate(&hin, G, 0, 0), "conditional handle");
      {
        const double *a0 = E.red.slot(h0), *a1 = E.red.slot(h1), *a2 = E.red.slot(hb),
                     *a3 = E.red.slot(hb + 1), *a4 = E.red.slot(hb + 2);
        int reset = 1;
        void* args[] = {&a0, &a1, &a2, &a3, &a4, &reset, &c, &prm, &hin};
        nh = kernel(G, nh, (const void*)k_refine_head, args, 1);
      }
      cudaGraph_t body1;
      cudaGraphNode_t w1 = loop(G, nh, hin, &body1);
      inner(body1, xhat_, x, hin);
      // tail
      int t0 = 0;
      uint64_t k_tail = 0;
      cudaGraph_t g_tail = run(&k_tail, [&] {
        recover(bz, x, z);
        residual_full(bx, bz, x, z, ex_, ez_);
        t0 = E.red.add_batch(st(), {{RED_MAXABS, n, bx, nullptr}, {RED_MAXABS, m, bz, nullptr},
                                    {RED_MAXABS, n, ex_, nullptr}, {RED_MAXABS, m, ez_, nullptr}});
      });
      cudaGraphNode_t nt = child(G, {w1}, g_tail);
      cudaGraphConditionalHandle hout;
      check(cudaGraphConditionalHandleCreate(&hout, G, 0, 0), "conditional handle");
      {
        const double *a0 = E.red.slot(t0), *a1 = E.red.slot(t0 + 1), *a2 = E.red.slot(t0 + 2),
                     *a3 = E.red.slot(t0 + 3);
        void* args[] = {&a0, &a1, &a2, &a3, &c, &prm, &hout};
        nt = kernel(G, nt, (const void*)k_refine_outer_init, args, 1);
      }
      cudaGraph_t body2;
      loop(G, nt, hout, &body2);
      // outer body: correction (cx, cz) = K^-1 (ex, ez), candidate, full residual
      int ob = 0;
      uint64_t k_ohead = 0;
      cudaGraph_t g_oh = run(&k_ohead, [&] {
        ob = E.red.count();
        condense_first(ex_, ez_, cx_);
      });
      cudaGraphNode_t no = child(body2, {}, g_oh);
      cudaGraphConditionalHandle hin2;
      check(cudaGraphConditionalHandleCreate(&hin2, body2, 0, 0), "conditional handle");
      {
        const double* nul = nullptr;
        const double *a2 = E.red.slot(ob), *a3 = E.red.slot(ob + 1), *a4 = E.red.slot(ob + 2);
        int reset = 0;
        void* args[] = {&nul, &nul, &a2, &a3, &a4, &reset, &c, &prm, &hin2};
        no = kernel(body2, no, (const void*)k_refine_head, args, 1);
      }
      cudaGraph_t body3;
      cudaGraphNode_t w3 = loop(body2, no, hin2, &body3);
      inner(body3, xhat_, cx_, hin2);
      int u0 = 0;
      uint64_t k_otail = 0;
      cudaGraph_t g_ot = run(&k_otail, [&] {
        recover(ez_, cx_, cz_);
        E.lincomb_batch({LinReq{n, 1.0, 1.0, 0.0, x, cx_, nullptr, candx_},
                         LinReq{m, 1.0, 1.0, 0.0, z, cz_, nullptr, candz_}});
        residual_full(bx, bz, candx_, candz_, ex2_, ez2_);
        u0 = E.red.add_batch(st(), {{RED_MAXABS, n, ex2_, nullptr}, {RED_MAXABS, m, ez2_, nullptr}});
      });
      cudaGraphNode_t nq = child(body2, {w3}, g_ot);
      {
        const double *a0 = E.red.slot(u0), *a1 = E.red.slot(u0 + 1);
        void* args[] = {&a0, &a1, &c, &prm, &hout};
        nq = kernel(body2, nq, (const void*)k_refine_outer_step, args, 1);
      }
      {
        long nn = n, mm = m;
        double *d1 = x, *d2 = z;
        const double *s1 = candx_.p, *s2 = candz_.p;
        void* args[] = {&oaccept, &nn, &d1, &s1, &oaccept, &mm, &d2, &s2};
        nq = kernel(body2, nq, (const void*)k_refine_copy, args, cgrid);
        double *e1 = ex_.p, *e2 = ez_.p;
        const double *f1 = ex2_.p, *f2 = ez2_.p;
        void* args2[] = {&ocont, &nn, &e1, &f1, &ocont, &mm, &e2, &f2};
        kernel(body2, nq, (const void*)k_refine_copy, args2, cgrid);
      }
      check(cudaGraphInstantiate(&built.exec, G, 0), "cudaGraphInstantiate");
      built.fixed = k_head + 1 + k_tail + 1;
      built.per_inner = k_step + 2;
      built.per_outer = k_ohead + 1 + k_otail + 1 + 2;
    } catch (...) {
      for (cudaGraph_t g : runs) cudaGraphDestroy(g);
      if (G) cudaGraphDestroy(G);
      if (built.exec) cudaGraphExecDestroy(built.exec);
      g_launches = launches0;
      E.red.set_count(0);
      cudaGetLastError();
      program_failed_ = true;  // the host-driven refinement takes over for this handle
      if (std::getenv("SDPX_B200_VERBOSE"))
        std::fprintf(stderr, "sdpx_b200: device-driven KKT solve unavailable, host-driven\n");
      times.kkt_solves--;  // counted again by kkt_solve
      return kkt_solve(bx, bz, x, z);
    }
    for (cudaGraph_t g : runs) cudaGraphDestroy(g);
    cudaGraphDestroy(G);
    g_launches = launches0;
    pg = E.add_program(key, built);
  }
  check(cudaGraphLaunch(pg->exec, st()), "cudaGraphLaunch");
  copy_d2h(hctl_.p, ctl_.p, sizeof(RefineCtl), st());
  check(cudaStreamSynchronize(st()), "refined solve sync");
  const RefineCtl& hc = hctl_.p[0];
  times.device_kkt_solves++;
  times.inner_refinements += hc.inner_steps;
  times.outer_refinements += hc.outer_steps;
  g_launches += pg->fixed + pg->per_inner * (uint64_t)hc.inner_steps +
                pg->per_outer * (uint64_t)hc.outer_steps;
  return hc.ok != 0;
}

// ------------------------------------------------------------------------------------------
// Residuals and info (default/residuals.rs:340-490, default/info.rs:89-192)
// ------------------------------------------------------------------------------------------
inline HsdSolver::Resid HsdSolver::residuals() {
  auto t0 = clock::now();
  const int n = n_, m = m_;
  E.P_mult(x_, 1.0, 0.0, Px_);
  E.A_adjoint(z_, -1.0, 0.0, rxinf_);
  E.copy(rzinf_, s_, m);
  E.A_forward(x_, 1.0, 1.0, rzinf_);
  E.lincomb(n, -1.0, Px_, -tau_, q_, 1.0, rxinf_, rx_);
  E.lincomb(m, 1.0, rzinf_, -tau_, b_, 0.0, nullptr, rz_);
  const int sq = E.red.add_batch(st(), {{RED_DOT, n, q_, x_},
                                        {RED_DOT, m, b_, z_},
                                        {RED_DOT, m, s_, z_},
                                        {RED_DOT, n, x_, Px_},
                                        {RED_SUMSQ, n, x_, d_},
                                        {RED_SUMSQ, m, z_, e_},
                                        {RED_SUMSQ, m, s_, einv_},
                                        {RED_SUMSQ, n, rxinf_, dinv_},
                                        {RED_SUMSQ, n, Px_, dinv_},
                                        {RED_SUMSQ, m, rzinf_, einv_},
                                        {RED_SUMSQ, m, rz_, einv_},
                                        {RED_SUMSQ, n, rx_, dinv_}});
  const int sb = sq + 1, ss = sq + 2, sp = sq + 3;
  int nr[8];
  for (int k = 0; k < 8; ++k) nr[k] = sq + 4 + k;
  auto& h = E.red.fetch(st());
  Resid r;
  r.qx = h[sq];
  r.bz = h[sb];
  r.sz = h[ss];
  r.xPx = h[sp];
  for (int k = 0; k < 8; ++k) r.norms[k] = std::sqrt(h[nr[k]]);
  r.rtau = r.qx + r.bz + kappa_ + r.xPx / tau_;
  times.residual += secs(t0);
  return r;
}

inline void HsdSolver::update_info(const Resid& r) {
  const double tinv = 1.0 / tau_, cinv = 1.0 / eq_.c;
  const double xpx = r.xPx * tinv * tinv / 2.0;
  Info& in = info;
  in.cost_primal = (r.qx * tinv + xpx) * cinv;
  in.cost_dual = (-r.bz * tinv - xpx) * cinv;
  double normx = r.norms[0], normz = r.norms[1] * cinv, norms = r.norms[2];
  in.res_primal_inf = (r.norms[3] * cinv) / std::max(1.0, normz);
  in.res_dual_inf = std::max(r.norms[4] / std::max(1.0, normx), r.norms[5] / std::max(1.0, normx + norms));
  normx *= tinv;
  normz *= tinv;
  norms *= tinv;
  in.rz_ns = r.norms[6];
  in.rx_ns = r.norms[7];
  in.res_primal = r.norms[6] * tinv / std::max(1.0, normb_ + normx + norms);
  in.res_dual = r.norms[7] * tinv * cinv / std::max(1.0, normq_ + normx + normz);
  in.gap_abs = std::fabs(in.cost_primal - in.cost_dual);
  in.gap_rel = in.gap_abs / std::max(1.0, std::min(std::fabs(in.cost_primal), std::fabs(in.cost_dual)));
  in.ktratio = kappa_ * tinv;
}

inline bool HsdSolver::is_solved(double ga, double gr, double feas) const {
  return (info.gap_abs < ga || info.gap_rel < gr) && info.res_primal < feas && info.res_dual < feas;
}

inline void HsdSolver::check_convergence(const Resid& r, bool full) {
  double ga, gr, fe, ia, ir, kt;
  int c0, c1, c2;
  if (full) {
    ga = st_.tol_gap_abs; gr = st_.tol_gap_rel; fe = st_.tol_feas;
    ia = st_.tol_infeas_abs; ir = st_.tol_infeas_rel; kt = st_.tol_ktratio;
    c0 = ST_SOLVED; c1 = ST_PRIMAL_INFEASIBLE; c2 = ST_DUAL_INFEASIBLE;
  } else {
    ga = st_.reduced_tol_gap_abs; gr = st_.reduced_tol_gap_rel; fe = st_.reduced_tol_feas;
    ia = st_.reduced_tol_infeas_abs; ir = st_.reduced_tol_infeas_rel; kt = st_.reduced_tol_ktratio;
    c0 = ST_ALMOST_SOLVED; c1 = ST_ALMOST_PRIMAL_INFEASIBLE; c2 = ST_ALMOST_DUAL_INFEASIBLE;
  }
  if (info.ktratio <= 1.0 && is_solved(ga, gr, fe)) {
    info.status = c0;
  } else if (info.ktratio > (1.0 / kt) * 1000.0) {
    if (r.bz < -ia && info.res_primal_inf < -ir * r.bz) info.status = c1;
    else if (r.qx < -ia && info.res_dual_inf < -ir * r.qx) info.status = c2;
  }
}

// default/info.rs:263-327
inline bool HsdSolver::check_termination(const Resid& r, int iter) {
  check_convergence(r, true);
  if (info.status == ST_UNSOLVED && iter > 1 && have_prev_ &&
      (info.res_dual > prev_.res_dual || info.res_primal > prev_.res_primal)) {
    if (info.ktratio < kEps * 100.0 &&
        (prev_.gap_abs < st_.tol_gap_abs || prev_.gap_rel < st_.tol_gap_rel))
      info.status = ST_INSUFFICIENT_PROGRESS;
    if (info.ktratio < 1.0) {
      if ((info.res_dual > st_.tol_feas * 100.0 && info.res_dual > prev_.res_dual * 100.0) ||
          (info.res_primal > st_.tol_feas * 100.0 && info.res_primal > prev_.res_primal * 100.0))
        info.status = ST_INSUFFICIENT_PROGRESS;
    }
  }
  if (info.status == ST_UNSOLVED) {
    if (st_.max_iter == iter) info.status = ST_MAX_ITERATIONS;
    else if (info.solve_time > st_.time_limit) info.status = ST_MAX_TIME;
  }
  return info.status != ST_UNSOLVED;
}

// Original-coordinate acceptance (default/original_check.rs, default/solution.rs:169-193).
// PSD equilibration is one scalar per cone, so the cone distances scale exactly.
inline double HsdSolver::original_ratio(bool reduced) {
  if (!(st_.tol_original > 0)) return -1.0;
  const int n = n_, m = m_;
  const double tinv = 1.0 / tau_, cinv = 1.0 / eq_.c;
  const int a = E.red.add_batch(st(), {{RED_MAXABS, m, rz_, einv_}, {RED_MAXABS, n, rx_, dinv_}});
  auto& h = E.red.fetch(st());
  double prim = h[a] * tinv, dual = h[a + 1] * tinv * cinv;
  E.lincomb(m, tau_, b_, 0.0, nullptr, 0.0, nullptr, wm1_);
  E.A_forward(x_, -1.0, 1.0, wm1_);  // b tau - A x
  std::vector<double> mr, ms, mz;
  E.margins(wm1_, mr, true);
  E.margins(s_, ms, true);
  E.margins(z_, mz, true);
  for (int j = 0; j < E.nblk; ++j) {
    double ej = eq_.e[E.hblocks[j].svec_off];
    prim = std::max(prim, std::max(0.0, -mr[2 * j]) * tinv / ej);
    prim = std::max(prim, std::max(0.0, -ms[2 * j]) * tinv / ej);
    dual = std::max(dual, std::max(0.0, -mz[2 * j]) * tinv * cinv * ej);
  }
  if (E.nn_count()) {  // orthant rows, entrywise in original coordinates
    const int ra = E.red.add_batch(st(), {{RED_NEGMAX, m, wm1_, nn_einv_}, {RED_NEGMAX, m, s_, nn_einv_},
                                          {RED_NEGMAX, m, z_, nn_e_}});
    const int rb = ra + 1, rc = ra + 2;
    auto& hn = E.red.fetch(st());
    prim = std::max(prim, std::max(hn[ra], hn[rb]) * tinv);
    dual = std::max(dual, hn[rc] * tinv * cinv);
  }
  prim /= (1.0 + normb_);
  dual /= (1.0 + normq_);
  double gap_abs = std::fabs(info.cost_primal - info.cost_dual);
  double gap_rel = gap_abs / (1.0 + std::fabs(info.cost_primal));
  double tf = st_.tol_original, ta = st_.tol_original, tr = st_.tol_original;
  if (reduced) {
    tf = std::max(tf, st_.reduced_tol_feas);
    ta = std::max(ta, st_.reduced_tol_gap_abs);
    tr = std::max(tr, st_.reduced_tol_gap_rel);
  }
  double gap = std::min(gap_abs / ta, gap_rel / tr);
  double r = std::max(std::max(prim / tf, dual / tf), gap);
  return std::isnan(r) ? std::numeric_limits<double>::infinity() : r;
}

// Homogeneous direction from a solved column (x1, z1) and the constant column (x2, z2):
// dtau (default/kktsystem.rs:550-655), dx, dz, ds from the linear row (403-418), dkappa.
inline bool HsdSolver::hsd_direction(const double* rhs_x, const double* workz, double rhs_tau,
                                     double rhs_kappa, const double* rhs_z, const double* x1,
                                     const double* z1, double* dtau, double* dkappa) {
  (void)rhs_x; (void)workz;
  const int n = n_, m = m_;
  const int a = E.red.add_batch(st(), {{RED_DOT, n, q_, x1}, {RED_DOT, m, b_, z1},
                                       {RED_DOT, n, q_, x2_}, {RED_DOT, m, b_, z2_}});
  const int b = a + 1, c = a + 2, d = a + 3;
  int f1 = -1, f2 = -1, f3 = -1;
  if (E.has_P()) {
    // xi = x / tau; quad1 = xi' P x1; delta = (xi - x2)' P (xi - x2); quad2 = x2' P x2
    E.P_mult(x1, 1.0, 0.0, wn_);
    E.lincomb(n, 1.0 / tau_, x_, 0.0, nullptr, 0.0, nullptr, tx_);
    f1 = E.red.add(st(), RED_DOT, n, tx_, wn_);
    E.lincomb(n, 1.0 / tau_, x_, -1.0, x2_, 0.0, nullptr, tx_);
    E.P_mult(tx_, 1.0, 0.0, candn_);
    f2 = E.red.add(st(), RED_DOT, n, tx_, candn_);
    E.P_mult(x2_, 1.0, 0.0, e2n_);
    f3 = E.red.add(st(), RED_DOT, n, x2_, e2n_);
  }
  auto& h = E.red.fetch(st());
  double q1 = h[a], b1 = h[b], q2 = h[c], b2 = h[d];
  double quad1 = f1 >= 0 ? h[f1] : 0.0, delta = f2 >= 0 ? h[f2] : 0.0, quad2 = f3 >= 0 ? h[f3] : 0.0;
  double num = rhs_tau - rhs_kappa / tau_ + q1 + b1 + 2.0 * quad1;
  double den = kappa_ / tau_ - q2 - b2;
  den += delta - quad2;
  double dt = num / den;
  if (!std::isfinite(dt)) return false;
  E.lincomb_batch({LinReq{n, 1.0, dt, 0.0, x1, x2_, nullptr, dx_}, LinReq{m, 1.0, dt, 0.0, z1, z2_, nullptr, dz_},
                   LinReq{m, -1.0, dt, 0.0, rhs_z, b_, nullptr, ds_}});
  E.A_forward(dx_, -1.0, 1.0, ds_);
  *dtau = dt;
  *dkappa = -(rhs_kappa + kappa_ * dt) / tau_;
  return true;
}

// min(alpha_tau, alpha_kappa, cap, cone bounds) (default/variables.rs:697-750)
inline double HsdSolver::step_bounds(const double* dz, const double* ds, double dtau, double dkappa,
                                     int mode, double cap) {
  auto t0 = clock::now();
  double at = dtau < 0 ? -tau_ / dtau : std::numeric_limits<double>::max();
  double ak = dkappa < 0 ? -kappa_ / dkappa : std::numeric_limits<double>::max();
  double a = std::min(std::min(at, ak), cap);
  double az, as;
  bool ok = E.step_bounds(dz, ds, a, mode, &az, &as);
  times.step += secs(t0);
  if (!ok) return 0.0;
  return std::min(az, as);
}

// core/solver.rs:1209-1322 and default/kktsystem.rs:462-527, variables.rs:577-620
inline bool HsdSolver::default_start() {
  const int n = n_, m = m_;
  E.identity_scaling();
  reg_boost_ = 0;
  bool ok = kkt_update();
  E.lincomb(n, 0.0, nullptr, 0.0, nullptr, 0.0, nullptr, x_);
  if (ok) {
    if (!E.has_P()) {
      E.lincomb(n, 0.0, nullptr, 0.0, nullptr, 0.0, nullptr, wn_);
      ok = kkt_solve(wn_, b_, x_, wm2_);
      if (ok) {
        E.lincomb(m, -1.0, wm2_, 0.0, nullptr, 0.0, nullptr, s_);
        E.lincomb(m, 0.0, nullptr, 0.0, nullptr, 0.0, nullptr, wm1_);
        ok = kkt_solve(negq_, wm1_, wn_, z_);
      }
    } else {
      ok = kkt_solve(negq_, b_, x_, z_);
      if (ok) E.lincomb(m, -1.0, z_, 0.0, nullptr, 0.0, nullptr, s_);
    }
  }
  if (ok) {
    const int a = E.red.add_batch(st(), {{RED_MAXABS, n, x_, nullptr}, {RED_MAXABS, m, z_, nullptr}});
    const int b = a + 1;
    auto& h = E.red.fetch(st());
    double bound = 1e12 * data_scale_;
    if (!(h[a] <= bound && h[b] <= bound)) ok = false;
  }
  if (ok) {
    for (double* v : {s_.p, z_.p}) {
      std::vector<double> mg;
      if (!E.margins(v, mg)) return false;
      double mn = std::numeric_limits<double>::max(), pos = 0.0;
      for (size_t j = 0; j + 1 < mg.size(); j += 2) {  // PSD blocks, then the orthant rows
        mn = std::min(mn, mg[j]);
        pos += mg[j + 1];
      }
      double target = std::max(1.0, (pos * 0.1) / std::max(degree_, 1));
      if (mn <= 0) {
        E.shift_unit(v, -mn);
        E.shift_unit(v, target);
      } else if (mn < target) {
        E.shift_unit(v, target - mn);
      }
    }
    tau_ = 1.0;
    kappa_ = 1.0;
  } else {
    // unit start (core/solver.rs:1259-1290)
    E.lincomb(n, 0.0, nullptr, 0.0, nullptr, 0.0, nullptr, x_);
    E.lincomb(m, 0.0, nullptr, 0.0, nullptr, 0.0, nullptr, s_);
    E.shift_unit(s_, 1.0);
    E.copy(z_, s_, m);
    double t0 = std::min(1.0, 1.0 / dmax_);
    tau_ = t0;
    kappa_ = 1.0 / t0;
  }
  return true;
}

// ------------------------------------------------------------------------------------------
// The iteration (core/solver.rs:285-505, 831-1012)
// ------------------------------------------------------------------------------------------
inline void HsdSolver::solve() {
  auto tstart = clock::now();
  const int n = n_, m = m_;
  info = Info();
  times = PhaseTimes();
  have_prev_ = false;
  default_start();
  int it = 0;
  double mu = 0.0, sigma = 1.0, alpha = 0.0;
  bool have_best = false;
  double best_tm = 0.0;
  double prev_tau = tau_, prev_kappa = kappa_;
  E.copy(prevx_, x_, n);
  E.copy(prevs_, s_, m);
  E.copy(prevz_, z_, m);
  double orig_best = -1.0;
  int orig_stale = 0;
  Resid r{};
  for (;;) {
    r = residuals();
    mu = (r.sz + tau_ * kappa_) / (degree_ + 1);
    update_info(r);
    info.iterations = it;
    info.solve_time = secs(tstart);
    bool stop = check_termination(r, it);
    if (stop && info.status == ST_SOLVED) {
      double ratio = original_ratio(false);
      if (ratio >= 0 && !(ratio <= 1.0)) {
        if (orig_best < 0 || ratio < orig_best * 0.5) {
          orig_best = ratio;
          orig_stale = 0;
        } else {
          orig_stale++;
        }
        if (orig_stale >= 3) info.status = ST_INSUFFICIENT_PROGRESS;
        else if (it >= st_.max_iter) info.status = ST_MAX_ITERATIONS;
        else {
          info.status = ST_UNSOLVED;
          stop = false;
        }
      }
    }
    if (stop) {
      if (info.status == ST_INSUFFICIENT_PROGRESS) {
        E.copy(x_, prevx_, n);
        E.copy(s_, prevs_, m);
        E.copy(z_, prevz_, m);
        tau_ = prev_tau;
        kappa_ = prev_kappa;
      }
      break;
    }
    // scale
    auto t0 = clock::now();
    bool sok = E.nt_scale(s_, z_);
    times.scale += secs(t0);
    if (!sok) {
      info.status = ST_NUMERICAL_ERROR;
      break;
    }
    ++it;
    // ---------------- predictor ----------------
    bool ok = kkt_update();
    if (ok) {
      ok = kkt_solve(negq_, b_, x2_, z2_);
      while (!ok && st_.static_reg_enable && reg_boost_ < 3) {
        reg_boost_++;
        ok = kkt_update() && kkt_solve(negq_, b_, x2_, z2_);
      }
    }
    double dtau = 0, dkappa = 0;
    if (ok) {
      E.lincomb(m, 1.0, s_, -1.0, rz_, 0.0, nullptr, workz_);
      ok = kkt_solve(rx_, workz_, x1_, z1_) &&
           hsd_direction(rx_, workz_, r.rtau, tau_ * kappa_, rz_, x1_, z1_, &dtau, &dkappa);
    }
    if (!ok) {
      info.status = ST_NUMERICAL_ERROR;
      alpha = 0.0;
      break;
    }
    // keep the raw affine direction for the curve search
    E.lincomb_batch({E.cp(ax_, dx_, n), E.cp(as_, ds_, m), E.cp(az_, dz_, m)});
    double adtau = dtau, adkappa = dkappa;
    alpha = step_bounds(dz_, ds_, dtau, dkappa, 0, 1.0);
    sigma = std::max(std::pow(1.0 - alpha, 3), 0.0);
    const double mfac = (it == 1) ? alpha : 1.0;
    // ---------------- combined rhs ----------------
    auto tc = clock::now();
    E.lincomb_batch({LinReq{n, 1.0 - sigma, 0.0, 0.0, rx_, nullptr, nullptr, rhsx_},
                     LinReq{m, mfac, 0.0, 0.0, dz_, nullptr, nullptr, wm1_}});
    double rhs_tau = (1.0 - sigma) * r.rtau;
    double rhs_kappa = -sigma * mu + mfac * dtau * dkappa + tau_ * kappa_;
    E.cone_apply(CM_W, wm1_, wm2_);       // W dz
    E.cone_apply(CM_WINVT, ds_, wm3_);    // W^-T ds
    E.circ_op(wm3_, wm2_, wm1_);
    E.shift_unit(wm1_, -sigma * mu);
    E.affine_ds(rhss_);
    E.lincomb(m, 1.0, rhss_, 1.0, wm1_, 0.0, nullptr, rhss_);
    E.lincomb(m, 1.0 - sigma, rz_, 0.0, nullptr, 0.0, nullptr, rhsz_);
    E.lam_inv_circ(rhss_, wm2_);
    E.cone_apply(CM_WT, wm2_, cvec_);     // W'(lambda \ ds)
    E.lincomb(m, 1.0, cvec_, -1.0, rhsz_, 0.0, nullptr, workz_);
    times.other += secs(tc);
    ok = kkt_solve(rhsx_, workz_, x1_, z1_) &&
         hsd_direction(rhsx_, workz_, rhs_tau, rhs_kappa, rhsz_, x1_, z1_, &dtau, &dkappa);
    if (!ok) {
      info.status = ST_NUMERICAL_ERROR;
      alpha = 0.0;
      break;
    }
    // ---------------- step length and curve search ----------------
    alpha = step_bounds(dz_, ds_, dtau, dkappa, 0, 1.0) * st_.max_step_fraction;
    if (alpha > 0.0 && alpha < 0.9) {
      for (double frac : {0.5, 0.25}) {
        double t = alpha + (1.0 - alpha) * frac;
        if (t * (1.0 - sigma * t) <= 1.01 * alpha * (1.0 - sigma)) continue;
        E.lincomb_batch({LinReq{n, 1.0 - t, t, 0.0, ax_, dx_, nullptr, tx_},
                         LinReq{m, 1.0 - t, t, 0.0, as_, ds_, nullptr, ts_},
                         LinReq{m, 1.0 - t, t, 0.0, az_, dz_, nullptr, tz_}});
        double ttau = (1.0 - t) * adtau + t * dtau, tkap = (1.0 - t) * adkappa + t * dkappa;
        double a = t / st_.max_step_fraction;
        bool admitted = a <= 1.0 && tau_ + a * ttau >= 0 && kappa_ + a * tkap >= 0;
        if (admitted) {
          double az, as;
          auto t1 = clock::now();
          bool eok = E.step_bounds(tz_, ts_, a, 1, &az, &as);
          times.step += secs(t1);
          admitted = eok && az >= a && as >= a;
        }
        if (admitted) {
          E.lincomb_batch({E.cp(dx_, tx_, n), E.cp(ds_, ts_, m), E.cp(dz_, tz_, m)});
          dtau = ttau;
          dkappa = tkap;
          alpha = t;
          break;
        }
      }
    }
    if (alpha <= 0.0) {
      info.status = ST_INSUFFICIENT_PROGRESS;
      break;
    }
    prev_ = info;
    have_prev_ = true;
    double tm = tolerance_multiple(info);
    if (!have_best || tm < best_tm) {
      have_best = true;
      best_tm = tm;
      E.lincomb_batch({E.cp(bestx_, x_, n), E.cp(bests_, s_, m), E.cp(bestz_, z_, m),
                       E.cp(prevx_, x_, n), E.cp(prevs_, s_, m), E.cp(prevz_, z_, m)});
      best_tau_ = tau_;
      best_kappa_ = kappa_;
    } else {
      E.lincomb_batch({E.cp(prevx_, x_, n), E.cp(prevs_, s_, m), E.cp(prevz_, z_, m)});
    }
    prev_tau = tau_;
    prev_kappa = kappa_;
    E.lincomb_batch({LinReq{n, 1.0, alpha, 0.0, x_, dx_, nullptr, x_}, LinReq{m, 1.0, alpha, 0.0, s_, ds_, nullptr, s_},
                     LinReq{m, 1.0, alpha, 0.0, z_, dz_, nullptr, z_}});
    tau_ += alpha * dtau;
    kappa_ += alpha * dkappa;
  }
  // finish (core/solver.rs:1128-1207)
  const int before = info.status;
  if (before == ST_NUMERICAL_ERROR || before == ST_INSUFFICIENT_PROGRESS ||
      before == ST_MAX_ITERATIONS || before == ST_MAX_TIME) {
    r = residuals();
    update_info(r);
    if (have_best && best_tm < tolerance_multiple(info)) {
      E.copy(x_, bestx_, n);
      E.copy(s_, bests_, m);
      E.copy(z_, bestz_, m);
      tau_ = best_tau_;
      kappa_ = best_kappa_;
      r = residuals();
      update_info(r);
    }
    info.status = before;
    check_convergence(r, false);
    if (info.status == ST_ALMOST_SOLVED && before != ST_ALMOST_SOLVED) {
      double ratio = original_ratio(true);
      if (ratio >= 0 && !(ratio <= 1.0)) info.status = before;
    }
  }
  info.iterations = it;
  // unscale (default/variables.rs:640-665)
  hx.resize(n);
  hs.resize(m);
  hz.resize(m);
  copy_d2h(hx.data(), x_.p, n * sizeof(double), st());
  copy_d2h(hs.data(), s_.p, m * sizeof(double), st());
  copy_d2h(hz.data(), z_.p, m * sizeof(double), st());
  check(cudaStreamSynchronize(st()), "result sync");
  const double tinv = 1.0 / tau_;
  for (int i = 0; i < n; ++i) hx[i] = hx[i] * eq_.d[i] * tinv;
  for (int i = 0; i < m; ++i) {
    hs[i] = hs[i] * eq_.einv[i] * tinv;
    hz[i] = hz[i] * eq_.e[i] * tinv / eq_.c;
  }
  info.solve_time = secs(tstart);
}

// Cyclic Jacobi eigen-decomposition of a small symmetric matrix (host, n <= 64, column-major):
// A = Q diag(w) Q'.  Used once per adjoint call per PSD block.
inline void host_sym_eig(int n, std::vector<double> A, std::vector<double>& Q, std::vector<double>& w) {
  Q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Q[i + (size_t)i * n] = 1.0;
  auto a = [&](int i, int j) -> double& { return A[i + (size_t)j * n]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        tot += a(i, j) * a(i, j);
        if (i != j) off += a(i, j) * a(i, j);
      }
    if (off <= 1e-30 * tot) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a(p, q);
        if (apq == 0.0) continue;
        const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < n; ++k) {  // A <- J' A J
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - sn * akq;
          a(k, q) = sn * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - sn * aqk;
          a(q, k) = sn * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double qkp = Q[k + (size_t)p * n], qkq = Q[k + (size_t)q * n];
          Q[k + (size_t)p * n] = c * qkp - sn * qkq;
          Q[k + (size_t)q * n] = sn * qkp + c * qkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = a(i, i);
}

// Adjoint of the solution map.  At a strictly complementary solution, perturbing (q, b, A) moves
// (x, z, s) along
//   [P A'; A -Hs] [dx; dz] = [-dq - dA' z; db - dA x],  ds = -Hs dz,
// with Hs the limit of the NT scaling as the iterates approach the solution (the KKT rows plus
// the linearised complementarity, the system the last iterations solved).  For a loss with
// gradients (gx, gz, gs) the one solve K [u; v] = [gx; gz - Hs gs] gives dL/dq = -u,
// dL/db = v, dL/dA = -(z u' + v x').
// The final iterate's own scaling is too close to that limit to solve with (entries of Hs span
// ~1e20 at gap 1e-10: the solve loses most digits), so the system is formed at the solution
// re-centred on the central path at a small relative mu: per PSD block, S - Z = Q diag(l) Q'
// (complementary ranges), S_c = Q diag(l+ or d |l|) Q', Z_c = Q diag(l- or d |l|) Q' with
// d = 1e-9 relative to the block scale; per orthant row the smaller of (s, z) becomes d times
// the larger.  That keeps the O(d) bias of the linearisation and a Schur conditioning of ~1/d.
// The solve runs on the equilibrated engine: with x = D xb / tau, s = E^-1 sb / tau,
// z = E zb / (c tau), Kb [ub; vb] = [D gx; E gz / c - Hb (E^-1 gs)] and u = c D ub, v = E vb.
inline bool HsdSolver::adjoint(const std::vector<double>& gx, const std::vector<double>& gz,
                               const std::vector<double>& gs, std::vector<double>& u,
                               std::vector<double>& v) {
  const int n = n_, m = m_;
  const double tinv = 1.0 / tau_, rel = 1e-9;
  std::vector<double> sb(m), zb(m);
  copy_d2h(sb.data(), s_.p, m * sizeof(double), st());
  copy_d2h(zb.data(), z_.p, m * sizeof(double), st());
  check(cudaStreamSynchronize(st()), "adjoint sync");
  for (int i = 0; i < m; ++i) {
    sb[i] *= tinv;
    zb[i] *= tinv;
  }
  std::vector<double> sc(sb), zc(zb);
  for (const BlockDesc& bd : E.hblocks) {  // PSD blocks: re-centre in the eigenbasis of S - Z
    const int nb = bd.n;
    std::vector<double> X((size_t)nb * nb), Q, w;
    auto at = [&](const std::vector<double>& v, int i, int j) {
      const int a = std::min(i, j), b = std::max(i, j);
      const double x = v[bd.svec_off + b * (b + 1) / 2 + a];
      return a == b ? x : x * SDPXG_RSQRT2;
    };
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) X[i + (size_t)j * nb] = at(sb, i, j) - at(zb, i, j);
    host_sym_eig(nb, X, Q, w);
    double scale = 0.0;
    for (double l : w) scale = std::max(scale, std::fabs(l));
    if (!(scale > 0.0)) scale = 1.0;
    std::vector<double> ls(nb), lz(nb);
    for (int i = 0; i < nb; ++i) {
      const double l = std::fabs(w[i]) > rel * scale ? w[i] : (w[i] >= 0 ? rel * scale : -rel * scale);
      if (l > 0) {
        ls[i] = l;
        lz[i] = rel * scale * scale / l;
      } else {
        lz[i] = -l;
        ls[i] = rel * scale * scale / (-l);
      }
    }
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i <= j; ++i) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < nb; ++k) {
          const double qq = Q[i + (size_t)k * nb] * Q[j + (size_t)k * nb];
          a += qq * ls[k];
          b += qq * lz[k];
        }
        const double f = (i == j) ? 1.0 : SDPXG_SQRT2;
        sc[bd.svec_off + j * (j + 1) / 2 + i] = a * f;
        zc[bd.svec_off + j * (j + 1) / 2 + i] = b * f;
      }
  }
  for (int r : E.nn_rows) {  // orthant rows: the smaller partner becomes rel x the larger
    const double big = std::max(std::fabs(sb[r]), std::fabs(zb[r]));
    if (!(big > 0.0)) return false;
    if (sb[r] >= zb[r]) {
      sc[r] = big;
      zc[r] = rel * big;
    } else {
      zc[r] = big;
      sc[r] = rel * big;
    }
  }
  ts_.upload(sc.data(), m, st());
  tz_.upload(zc.data(), m, st());
  if (!E.nt_scale(ts_, tz_)) return false;
  reg_boost_ = 0;
  if (!kkt_update()) return false;
  std::vector<double> bx(n), bz(m), gsi(m);
  for (int i = 0; i < n; ++i) bx[i] = eq_.d[i] * gx[i];
  for (int i = 0; i < m; ++i) {
    bz[i] = eq_.e[i] * gz[i] / eq_.c;
    gsi[i] = eq_.einv[i] * gs[i];
  }
  rhsx_.upload(bx.data(), n, st());
  rhsz_.upload(bz.data(), m, st());
  wm1_.upload(gsi.data(), m, st());
  E.cone_apply(CM_HS, wm1_, wm2_);
  E.lincomb(m, 1.0, rhsz_, -1.0, wm2_, 0.0, nullptr, rhsz_);
  if (!kkt_solve(rhsx_, rhsz_, x1_, z1_)) return false;
  u.resize(n);
  v.resize(m);
  copy_d2h(u.data(), x1_.p, n * sizeof(double), st());
  copy_d2h(v.data(), z1_.p, m * sizeof(double), st());
  check(cudaStreamSynchronize(st()), "adjoint sync");
  for (int i = 0; i < n; ++i) u[i] *= eq_.c * eq_.d[i];
  for (int i = 0; i < m; ++i) v[i] *= eq_.e[i];
  for (double t : u)
    if (!std::isfinite(t)) return false;
  for (double t : v)
    if (!std::isfinite(t)) return false;
  return true;
}

}  // namespace sdpxg
