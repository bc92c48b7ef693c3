// C ABI of libsdpx_b200: the reference's solver ABI (include/sdpx.h) over the GPU engine and
// the kernel-level sdpxg_* entry points.  Exceptions never cross the boundary: they become
// return code 5 (the reference's "panic" code) with the message kept thread-locally, and a
// handle whose solve threw is poisoned (crates/ffi/src/lib.rs:29-42, 567-584).
#include <chrono>
#include <climits>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/sdpx_b200.h"
#include "hsd.cuh"
#include "sampled.cuh"
#include "i8_gemm.cuh"
#include "host_parallel.h"

using namespace sdpxg;

namespace sdpxg {
thread_local std::string g_last_error;  // shared by both ABI levels
}

namespace {


struct AbiError {
  int32_t code;
  std::string msg;
};

template <typename F>
int32_t boundary(F&& f) {
  try {
    f();
    return 0;
  } catch (const AbiError& e) {
    sdpxg::g_last_error = e.msg;
    return e.code;
  } catch (const sdpxg::SampledUnsupported& e) {
    sdpxg::g_last_error = e.what();
    return 2;
  } catch (const std::invalid_argument& e) {
    sdpxg::g_last_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    sdpxg::g_last_error = std::string("internal error: ") + e.what();
    return 5;
  } catch (...) {
    sdpxg::g_last_error = "internal error at ABI boundary";
    return 5;
  }
}

[[noreturn]] void invalid(const std::string& s) { throw AbiError{1, s}; }
[[noreturn]] void unsupported(const std::string& s) { throw AbiError{2, s}; }

template <typename T>
const T* ref(const T* p) {
  if (!p) invalid("null pointer");
  return p;
}

std::vector<double> scalars(const sdpx_scalars& a) {
  if (a.reserved != 0) invalid("nonzero scalar reserved field");
  std::vector<double> v(a.count);
  if (a.kind == 0) {
    if (a.count && !a.f64) invalid("null pointer");
    parallel_for((int64_t)a.count, 1 << 16, [&](int64_t b, int64_t e, int) {
      for (int64_t i = b; i < e; ++i) {
        v[i] = a.f64[i];
        if (!std::isfinite(v[i])) invalid("nonfinite input");
      }
    });
    return v;
  } else if (a.kind == 1) {
    if (a.count && !a.decimal) invalid("null pointer");
    for (uint64_t i = 0; i < a.count; ++i) {
      const char* s = a.decimal[i];
      if (!s) invalid("null pointer");
      char* end = nullptr;
      v[i] = std::strtod(s, &end);
      if (end == s || *end != '\0') invalid("invalid decimal scalar");
    }
  } else {
    invalid("unknown scalar encoding");
  }
  for (double x : v)
    if (!std::isfinite(x)) invalid("nonfinite input");
  return v;
}

// Finite binary64 values of a stored-entry array, copied in parallel (no zero fill first).
void values_into(const sdpx_scalars& a, F64Vec& v) {
  if (a.reserved != 0) invalid("nonzero scalar reserved field");
  if (a.kind != 0) {
    std::vector<double> t = scalars(a);
    v.assign(t.begin(), t.end());
    return;
  }
  if (a.count && !a.f64) invalid("null pointer");
  v.resize(a.count);
  parallel_for((int64_t)a.count, 1 << 16, [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; ++i) {
      v[i] = a.f64[i];
      if (!std::isfinite(v[i])) invalid("nonfinite input");
    }
  });
}

struct Csc {
  uint64_t rows = 0, cols = 0;
  I64Vec colptr, rowval;
  F64Vec val;
};

// crates/ffi/src/lib.rs:224-259 validation
Csc matrix(const sdpx_csc& a, bool upper) {
  Csc c;
  c.rows = a.rows;
  c.cols = a.cols;
  if (!a.colptr) invalid("null pointer");
  if (a.nnz && !a.rowval) invalid("null pointer");
  if (a.values.count != a.nnz || a.colptr[0] != 0 || a.colptr[a.cols] != a.nnz)
    invalid("inconsistent CSC lengths");
  c.colptr.resize(a.cols + 1);
  c.rowval.resize(a.nnz);
  for (uint64_t j = 0; j <= a.cols; ++j) c.colptr[j] = (int64_t)a.colptr[j];
  for (uint64_t j = 0; j < a.cols; ++j)
    if (a.colptr[j] > a.colptr[j + 1] || a.colptr[j + 1] > a.nnz)
      invalid("invalid CSC column pointers");
  parallel_for((int64_t)a.cols, col_grain(a.cols, a.nnz), [&](int64_t j0, int64_t j1, int) {
    for (int64_t j = j0; j < j1; ++j)
      for (uint64_t p = a.colptr[j]; p < a.colptr[j + 1]; ++p) {
        uint64_t r = a.rowval[p];
        if (r >= a.rows || (upper && r > (uint64_t)j) || (p > a.colptr[j] && a.rowval[p - 1] >= r))
          invalid("CSC rows must be sorted unique in range; P upper triangular");
        c.rowval[p] = (int64_t)r;
      }
  });
  values_into(a.values, c.val);
  return c;
}

constexpr uint32_t kPreprocessAll = 7u;

void validate_settings(const sdpx_settings& s) {
  if (s.abi_version != SDPX_ABI_VERSION)
    invalid("unsupported SDPX ABI version " + std::to_string(s.abi_version) +
            "; this library requires ABI 4");
  if (s.struct_size != sizeof(sdpx_settings) || s.kkt_form > 2 || s.reserved_0 != 0 ||
      s.verbose > 1 || (s.preprocessing_flags & ~kPreprocessAll) != 0 || std::isnan(s.time_limit) ||
      s.time_limit < 0.0)
    invalid("invalid settings layout or values");
}

double tolerance(const char* p, double dflt) {
  if (!p) return dflt;
  char* end = nullptr;
  double x = std::strtod(p, &end);
  if (end == p || *end != '\0' || !std::isfinite(x) || x <= 0.0)
    invalid("tolerance must be finite positive");
  return x;
}

Settings to_settings(const sdpx_settings& s) {
  validate_settings(s);
  Settings v;
  v.max_iter = (int)s.max_iter;
  v.time_limit = s.time_limit;
  v.equilibrate_enable = (s.preprocessing_flags & SDPX_PREPROCESS_RUIZ) != 0;
  v.tol_gap_abs = tolerance(s.tol_gap_abs, v.tol_feas);
  v.tol_gap_rel = tolerance(s.tol_gap_rel, v.tol_feas);
  double f = v.tol_feas;
  v.tol_feas = tolerance(s.tol_feas, f);
  v.tol_infeas_abs = tolerance(s.tol_infeas_abs, f);
  v.tol_infeas_rel = tolerance(s.tol_infeas_rel, f);
  return v;
}

// --------------------------------------------------------------------------------------
// Ruiz equilibration on the host (default/problemdata.rs:639-735), restated on CSC data.
// --------------------------------------------------------------------------------------
// Ruiz equilibration (default/problemdata.rs:639-760).  The reference rescales A in place in
// every pass; here the passes read A against the accumulated scales instead -- the maxima of
// |e_i a_ij d_j| per column and row of the current iterate -- and A is rescaled once at the end
// (E A D with the PSD rectification folded in): one read pass over the stored entries per
// iteration instead of a read and a write pass, the same scalings up to rounding.  P, q, b and
// the cost scale c are small and are updated in place as in the reference.
void equilibrate(HostProblem& p, const Settings& st, Equilibration& eq) {
  const int n = p.n, m = p.m;
  eq.d.assign(n, 1.0);
  eq.e.assign(m, 1.0);
  eq.c = 1.0;
  if (st.equilibrate_enable) {
    const double smin = st.equilibrate_min_scaling, smax = st.equilibrate_max_scaling;
    std::vector<double> dw(n), ew(m);
    const int nt = host_threads();
    std::vector<std::vector<double>> ewp((size_t)nt);
    std::vector<char> used((size_t)nt, 0);
    for (int it = 0; it < st.equilibrate_max_iter; ++it) {
      std::fill(dw.begin(), dw.end(), 0.0);
      std::fill(ew.begin(), ew.end(), 0.0);
      for (int j = 0; j < n; ++j)
        for (int64_t q = p.Pcolptr[j]; q < p.Pcolptr[j + 1]; ++q) {
          double a = std::fabs(p.Pval[q]);
          dw[j] = std::max(dw[j], a);
          dw[p.Prow[q]] = std::max(dw[p.Prow[q]], a);
        }
      {  // column maxima, and row maxima through per-chunk partial arrays, of E A D
        const double* e = eq.e.data();
        const double* d = eq.d.data();
        std::fill(used.begin(), used.end(), 0);
        parallel_for(n, col_grain(n, p.Aval.size()), [&](int64_t j0, int64_t j1, int t) {
          std::vector<double>& er = ewp[(size_t)t];
          er.assign(m, 0.0);
          used[(size_t)t] = 1;
          for (int64_t j = j0; j < j1; ++j) {
            const double dj = d[j];
            double cmax = 0.0;
            for (int64_t q = p.Acolptr[j]; q < p.Acolptr[j + 1]; ++q) {
              const int64_t r = p.Arow[q];
              const double a = std::fabs(p.Aval[q]) * dj;  // |a_ij| d_j
              const double v = e[r] * a;                   // |e_i a_ij d_j|
              cmax = std::max(cmax, v);
              er[r] = std::max(er[r], a);
            }
            dw[j] = std::max(dw[j], cmax);
          }
        });
        parallel_for(m, std::max<int64_t>(1 << 12, (int64_t)m * nt / 4), [&](int64_t i0, int64_t i1, int) {
          for (int t = 0; t < nt; ++t)
            if (used[(size_t)t])
              for (int64_t i = i0; i < i1; ++i) ew[i] = std::max(ew[i], ewp[(size_t)t][i]);
          for (int64_t i = i0; i < i1; ++i) ew[i] *= e[i];
        });
      }
      for (int j = 0; j < n; ++j) {
        double w = dw[j] == 0.0 ? 1.0 : dw[j];
        w = 1.0 / std::sqrt(w);
        dw[j] = std::min(std::max(w, smin / eq.d[j]), smax / eq.d[j]);
      }
      for (int i = 0; i < m; ++i) {
        double w = ew[i] == 0.0 ? 1.0 : ew[i];
        w = 1.0 / std::sqrt(w);
        ew[i] = std::min(std::max(w, smin / eq.e[i]), smax / eq.e[i]);
      }
      for (int j = 0; j < n; ++j)
        for (int64_t q = p.Pcolptr[j]; q < p.Pcolptr[j + 1]; ++q) p.Pval[q] *= dw[p.Prow[q]] * dw[j];
      for (int j = 0; j < n; ++j) {
        p.q[j] *= dw[j];
        eq.d[j] *= dw[j];
      }
      for (int i = 0; i < m; ++i) {
        p.b[i] *= ew[i];
        eq.e[i] *= ew[i];
      }
      if (!p.Pval.empty()) {
        std::vector<double> cn(n, 0.0);
        for (int j = 0; j < n; ++j)
          for (int64_t q = p.Pcolptr[j]; q < p.Pcolptr[j + 1]; ++q) cn[j] = std::max(cn[j], std::fabs(p.Pval[q]));
        double mean = 0.0;
        for (double v : cn) mean += v;
        mean /= std::max(n, 1);
        double qn = 0.0;
        for (double v : p.q) qn = std::max(qn, std::fabs(v));
        if (mean != 0.0 && qn != 0.0) {
          double ct = 1.0 / std::max(qn, mean);
          ct = std::min(std::max(ct, smin / eq.c), smax / eq.c);
          for (double& v : p.Pval) v *= ct;
          for (double& v : p.q) v *= ct;
          eq.c *= ct;
        }
      }
    }
    // rectify: one scalar per PSD cone, mean(e) (cones/psdtrianglecone.rs:252-255)
    int row = 0;
    std::vector<std::pair<int, int>> cl = p.cones;
    if (cl.empty())
      for (int d : p.psd) cl.push_back({3, d});
    for (const auto& c : cl) {
      if (c.first != 3) {  // orthant rows keep their own scaling
        row += c.second;
        continue;
      }
      const int d = c.second, tn = d * (d + 1) / 2;
      double mean = 0.0;
      for (int i = row; i < row + tn; ++i) mean += eq.e[i];
      mean /= std::max(tn, 1);
      for (int i = row; i < row + tn; ++i) {
        p.b[i] *= mean / eq.e[i];
        eq.e[i] = mean;
      }
      row += tn;
    }
    // A := E A D with the final (rectified) scales, one pass
    const double* e = eq.e.data();
    const double* d = eq.d.data();
    parallel_for(n, col_grain(n, p.Aval.size()), [&](int64_t j0, int64_t j1, int) {
      for (int64_t j = j0; j < j1; ++j)
        for (int64_t q = p.Acolptr[j]; q < p.Acolptr[j + 1]; ++q)
          p.Aval[q] = e[p.Arow[q]] * p.Aval[q] * d[j];
    });
  }
  eq.dinv.resize(n);
  eq.einv.resize(m);
  for (int j = 0; j < n; ++j) eq.dinv[j] = 1.0 / eq.d[j];
  for (int i = 0; i < m; ++i) eq.einv[i] = 1.0 / eq.e[i];
}

// SDPX_B200_VERBOSE=1 prints the host-side prepare breakdown to stderr.
bool verbose_from_env() {
  const char* s = std::getenv("SDPX_B200_VERBOSE");
  return s && s[0] == '1';
}

int device_from_env() {
  const char* s = std::getenv("SDPX_B200_DEVICE");
  return s ? std::atoi(s) : 0;
}

}  // namespace

// --------------------------------------------------------------------------------------
// Handle
// --------------------------------------------------------------------------------------
struct sdpx_handle {
  std::mutex mu;
  bool poisoned = false;
  Settings settings;
  HostProblem orig;   // copied user data
  HostProblem equil;  // equilibrated data
  Equilibration eq;
  std::unique_ptr<Engine> eng;
  std::unique_ptr<HsdSolver> hsd;  // device work vectors, allocated by the first solve
  bool solved = false;
  Info info;
  PhaseTimes times;
  std::vector<double> x, s, z;
};

namespace {

template <typename F>
int32_t operate(sdpx_handle* h, F&& f) {
  if (!h) throw AbiError{1, "null handle"};
  std::unique_lock<std::mutex> lk(h->mu, std::try_to_lock);
  if (!lk.owns_lock()) throw AbiError{3, "handle is busy"};
  if (h->poisoned) throw AbiError{4, "handle is poisoned"};
  try {
    f(*h);
  } catch (const AbiError&) {
    throw;
  } catch (...) {
    h->poisoned = true;
    throw;
  }
  return 0;
}

void output_bytes(const void* src, uint64_t count, size_t elem, void* out, uint64_t capacity,
                  uint64_t* required) {
  if (!required) invalid("null pointer");
  *required = count;
  if (!out && capacity == 0) return;
  if (capacity < count) throw AbiError{6, "insufficient output capacity"};
  if (count) {
    if (!out) invalid("null pointer");
    std::memcpy(out, src, count * elem);
  }
}

std::vector<double> result_vector(const sdpx_handle& h) {
  if (!h.solved) throw AbiError{7, "solve required before reading result"};
  std::vector<double> r;
  r.reserve(h.x.size() + 2 * h.z.size() + 6);
  r.insert(r.end(), h.x.begin(), h.x.end());
  r.insert(r.end(), h.z.begin(), h.z.end());
  r.insert(r.end(), h.s.begin(), h.s.end());
  r.push_back(h.info.cost_primal);
  r.push_back(h.info.cost_dual);
  r.push_back(h.info.res_primal);
  r.push_back(h.info.res_dual);
  r.push_back(h.info.gap_abs);
  r.push_back(h.info.gap_rel);
  return r;
}

// Rust `{:.19e}` formatting of the reference's decimal output (ffi/src/lib.rs:511-526).
std::string rust_exp(double x) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.19e", x);
  std::string s(buf);
  size_t e = s.find('e');
  if (e == std::string::npos) return s;  // inf / nan
  std::string mant = s.substr(0, e);
  int ex = std::atoi(s.c_str() + e + 1);
  return mant + "e" + std::to_string(ex);
}

// Validated, equilibrated copy of a problem, without device state (shared by prepare and
// reprepare).
std::unique_ptr<sdpx_handle> build_problem(const sdpx_csc* P, const sdpx_scalars* q,
                                           const sdpx_csc* A, const sdpx_scalars* b,
                                           const sdpx_cone* cones, uint64_t nc,
                                           const sdpx_settings* s, double* t_validate,
                                           double* t_equil) {
  const auto t0 = std::chrono::steady_clock::now();
  ref(q); ref(A); ref(b); ref(s);
  if (nc && !cones) invalid("null pointer");
  validate_settings(*s);
  if (s->precision_bits != 53)
    unsupported("unsupported precision: this GPU build solves binary64 (precision_bits 53)");
  if (s->kkt_form == 1) unsupported("augmented KKT form is not implemented on the GPU path");
  uint64_t n = A->cols;
  if ((P && (P->rows != P->cols || P->cols != n)) || q->count != n || b->count != A->rows)
    invalid("inconsistent problem dimensions");
  auto h = std::make_unique<sdpx_handle>();
  h->settings = to_settings(*s);
  HostProblem& p = h->orig;
  p.n = (int)n;
  p.m = (int)A->rows;
  if (P) {
    Csc pm = matrix(*P, true);
    p.Pcolptr.assign(pm.colptr.begin(), pm.colptr.end());
    p.Prow.assign(pm.rowval.begin(), pm.rowval.end());
    p.Pval.assign(pm.val.begin(), pm.val.end());
  } else {
    p.Pcolptr.assign(n + 1, 0);
  }
  Csc am = matrix(*A, false);
  p.Acolptr = std::move(am.colptr);
  p.Arow = std::move(am.rowval);
  p.Aval = std::move(am.val);
  p.q = scalars(*q);
  p.b = scalars(*b);
  uint64_t rows = 0;
  for (uint64_t i = 0; i < nc; ++i) {
    const sdpx_cone& c = cones[i];
    if (c.reserved != 0 && c.kind != 8) invalid("nonzero cone reserved field");
    if (c.dim == 0) invalid("cone dimension must be positive");
    if (c.kind > 8) invalid("invalid cone kind/dimension/parameters");
    if (c.kind != 3 && c.kind != 1)
      unsupported("only nonnegative (kind 1) and PSD triangle (kind 3) cones run on the GPU path");
    if (c.alpha.count != 0) invalid("unexpected cone alpha");
    if (c.kind == 1) {
      if (c.dim > (uint64_t)INT32_MAX) invalid("invalid cone kind/dimension/parameters");
      p.cones.push_back({1, (int)c.dim});
      rows += c.dim;
      continue;
    }
    if (c.dim > SDPXG_NMAX) unsupported("PSD cone order above 64 is not supported on the GPU path");
    p.psd.push_back((int)c.dim);
    p.cones.push_back({3, (int)c.dim});
    rows += c.dim * (c.dim + 1) / 2;
  }
  if (rows != A->rows) invalid("cone dimensions do not match the rows of A");
  const auto t1 = std::chrono::steady_clock::now();
  // the equilibrated copy takes the matrices; the original keeps what sdpx_update and the
  // info need (dimensions, q, b, cone orders)
  h->equil = std::move(h->orig);
  h->orig = HostProblem();
  h->orig.n = h->equil.n;
  h->orig.m = h->equil.m;
  h->orig.q = h->equil.q;
  h->orig.b = h->equil.b;
  h->orig.psd = h->equil.psd;
  h->orig.cones = h->equil.cones;
  equilibrate(h->equil, h->settings, h->eq);
  const auto t2 = std::chrono::steady_clock::now();
  auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
  *t_validate = sec(t0, t1);
  *t_equil = sec(t1, t2);
  return h;
}

void prepare_impl(const sdpx_csc* P, const sdpx_scalars* q, const sdpx_csc* A, const sdpx_scalars* b,
                  const sdpx_cone* cones, uint64_t nc, const sdpx_settings* s, sdpx_handle** out) {
  if (!out) invalid("null pointer");
  *out = nullptr;
  double tv = 0, te = 0;
  auto h = build_problem(P, q, A, b, cones, nc, s, &tv, &te);
  if (verbose_from_env())
    std::fprintf(stderr, "sdpx_b200 prepare: copy+validate %.3f s, equilibrate %.3f s\n", tv, te);
  const auto t2 = std::chrono::steady_clock::now();
  h->eng = std::make_unique<Engine>();
  h->eng->init(device_from_env());
  const auto t3 = std::chrono::steady_clock::now();
  h->eng->upload(h->equil);
  const auto t4 = std::chrono::steady_clock::now();
  if (verbose_from_env()) {
    auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    std::fprintf(stderr,
                 "sdpx_b200 prepare: device init %.3f s, upload %.3f s (%s)\n", sec(t2, t3),
                 sec(t3, t4), h->eng->upload_report().c_str());
  }
  *out = h.release();
}

// Factor-authoritative sampled input (ffi/src/lib.rs:608-658): the columns are materialised
// into A for validation, equilibration and the residuals (materialize_sampled), and the factors
// -- basis and weights scaled by the equilibration (one scalar per PSD cone after rectification,
// times the column scale) -- drive the Schur complement and the operator on the GPU.
void prepare_sampled_impl(const sdpx_csc* P, const sdpx_scalars* q, const sdpx_csc* A_linear,
                          const sdpx_scalars* b, const sdpx_cone* cones, uint64_t nc,
                          const sdpx_settings* s, const sdpx_sampled_block* blocks, uint64_t nb,
                          sdpx_handle** out) {
  if (!out) invalid("null pointer");
  *out = nullptr;
  ref(A_linear);
  if (nc && !cones) invalid("null pointer");
  Csc lin = matrix(*A_linear, false);
  std::vector<std::pair<uint64_t, uint64_t>> psd_rows;  // (row start, order) of the PSD cones
  uint64_t row = 0;
  for (uint64_t i = 0; i < nc; ++i) {
    const uint64_t d = cones[i].dim;
    if (cones[i].kind == 3) {
      psd_rows.push_back({row, d});
      row += d * (d + 1) / 2;
    } else {
      row += d;
    }
  }
  SampledCsc merged = materialize_sampled(A_linear->rows, A_linear->cols, lin.colptr, lin.rowval, lin.val,
                                          psd_rows, blocks, nb);
  sdpx_csc A{};
  A.rows = A_linear->rows;
  A.cols = A_linear->cols;
  A.nnz = merged.rowval.size();
  A.colptr = merged.colptr.data();
  A.rowval = merged.rowval.data();
  A.values.kind = 0;
  A.values.count = merged.val.size();
  A.values.f64 = merged.val.data();
  double tv = 0, te = 0;
  auto h = build_problem(P, q, &A, b, cones, nc, s, &tv, &te);
  for (auto& r : merged.recs) {  // the factors in the equilibrated coordinates: one weight per column
    const double e = h->eq.e[(size_t)r.row_start];
    for (size_t k = 0; k < r.weight.size(); ++k) r.weight[k] = r.weight[k] * h->eq.d[(size_t)r.col0 + k] * e;
  }
  h->equil.sampled = std::move(merged.recs);
  h->eng = std::make_unique<Engine>();
  h->eng->init(device_from_env());
  h->eng->upload(h->equil);
  *out = h.release();
}

}  // namespace

extern "C" {

int32_t sdpx_default_settings_v4(sdpx_settings* out) {
  return boundary([&] {
    if (!out) invalid("null pointer");
    sdpx_settings s{};
    s.abi_version = SDPX_ABI_VERSION;
    s.struct_size = sizeof(sdpx_settings);
    s.precision_bits = 53;
    s.max_iter = 200;
    s.verbose = 0;
    s.preprocessing_flags = kPreprocessAll;
    s.max_threads = 1;
    s.kkt_form = 0;
    s.reserved_0 = 0;
    s.time_limit = std::numeric_limits<double>::infinity();
    *out = s;
  });
}

int32_t sdpx_mpi_world_size(void) { return 1; }

int32_t sdpx_prepare(const sdpx_csc* P, const sdpx_scalars* q, const sdpx_csc* A,
                     const sdpx_scalars* b, const sdpx_cone* cones, uint64_t cone_count,
                     const sdpx_settings* settings, sdpx_handle** out) {
  return boundary([&] { prepare_impl(P, q, A, b, cones, cone_count, settings, out); });
}

int32_t sdpx_prepare_sampled(const sdpx_csc* P, const sdpx_scalars* q, const sdpx_csc* A_linear,
                             const sdpx_scalars* b, const sdpx_cone* cones, uint64_t cone_count,
                             const sdpx_settings* settings, const sdpx_sampled_block* blocks,
                             uint64_t block_count, sdpx_handle** out) {
  return boundary([&] { prepare_sampled_impl(P, q, A_linear, b, cones, cone_count, settings, blocks, block_count, out); });
}

int32_t sdpx_b200_reprepare(sdpx_handle* h, const sdpx_csc* P, const sdpx_scalars* q,
                            const sdpx_csc* A, const sdpx_scalars* b, const sdpx_cone* cones,
                            uint64_t cone_count, const sdpx_settings* settings) {
  return boundary([&] {
    double tv = 0, te = 0;
    auto fresh = build_problem(P, q, A, b, cones, cone_count, settings, &tv, &te);
    operate(h, [&](sdpx_handle& hh) {
      hh.solved = false;
      hh.settings = fresh->settings;
      hh.orig = std::move(fresh->orig);
      hh.equil = std::move(fresh->equil);
      hh.eq = std::move(fresh->eq);
      hh.eng->upload(hh.equil);  // buffers grow only; cached graphs are dropped
      if (hh.hsd) hh.hsd->reset(hh.equil, hh.eq, hh.settings);
    });
  });
}

int32_t sdpx_solve(sdpx_handle* h) {
  return boundary([&] {
    operate(h, [](sdpx_handle& hh) {
      hh.solved = false;
      if (hh.hsd) hh.hsd->load(hh.equil);
      else hh.hsd = std::make_unique<HsdSolver>(*hh.eng, hh.equil, hh.eq, hh.settings);
      HsdSolver& solver = *hh.hsd;
      solver.solve();
      hh.info = solver.info;
      hh.times = solver.times;
      hh.x = solver.hx;
      hh.s = solver.hs;
      hh.z = solver.hz;
      hh.solved = true;
    });
  });
}

int32_t sdpx_update(sdpx_handle* h, const sdpx_scalars* q, const sdpx_scalars* b) {
  return boundary([&] {
    ref(q); ref(b);
    operate(h, [&](sdpx_handle& hh) {
      if (q->count != (uint64_t)hh.orig.n || b->count != (uint64_t)hh.orig.m)
        invalid("update dimensions differ from prepared problem");
      std::vector<double> qv = scalars(*q), bv = scalars(*b);
      hh.orig.q = qv;
      hh.orig.b = bv;
      // the prepared equilibration stays: q_eq = c d q, b_eq = e b
      for (int j = 0; j < hh.orig.n; ++j) hh.equil.q[j] = hh.eq.c * hh.eq.d[j] * qv[j];
      for (int i = 0; i < hh.orig.m; ++i) hh.equil.b[i] = hh.eq.e[i] * bv[i];
      hh.solved = false;
    });
  });
}

int32_t sdpx_get_info(sdpx_handle* h, sdpx_info* out) {
  return boundary([&] {
    if (!out) invalid("null pointer");
    operate(h, [&](sdpx_handle& hh) {
      sdpx_info i{};
      i.abi_version = SDPX_ABI_VERSION;
      i.struct_size = sizeof(sdpx_info);
      i.status = hh.solved ? (uint32_t)hh.info.status : 0;
      i.iterations = hh.solved ? (uint32_t)hh.info.iterations : 0;
      i.working_bits = 53;
      i.backend_threads = 1;
      i.cone_threads = 1;
      i.kkt_form = 2;
      i.n = (uint64_t)hh.orig.n;
      i.m = (uint64_t)hh.orig.m;
      i.solve_time = hh.solved ? hh.info.solve_time : 0.0;
      i.objective = hh.info.cost_primal;
      i.dual_objective = hh.info.cost_dual;
      i.primal_residual = hh.info.res_primal;
      i.dual_residual = hh.info.res_dual;
      i.gap_abs = hh.info.gap_abs;
      i.gap_rel = hh.info.gap_rel;
      *out = i;
    });
  });
}

int32_t sdpx_get_solver_name(sdpx_handle* h, char* out, uint64_t capacity, uint64_t* required) {
  return boundary([&] {
    operate(h, [&](sdpx_handle&) {
      static const char name[] = "condensed_b200_dense";
      output_bytes(name, sizeof(name), 1, out, capacity, required);
    });
  });
}

int32_t sdpx_result_f64(sdpx_handle* h, double* out, uint64_t capacity, uint64_t* required) {
  return boundary([&] {
    operate(h, [&](sdpx_handle& hh) {
      std::vector<double> r = result_vector(hh);
      output_bytes(r.data(), r.size(), sizeof(double), out, capacity, required);
    });
  });
}

int32_t sdpx_result_decimal(sdpx_handle* h, char* out, uint64_t capacity, uint64_t* required) {
  return boundary([&] {
    operate(h, [&](sdpx_handle& hh) {
      std::vector<double> r = result_vector(hh);
      std::string bytes;
      for (double x : r) {
        bytes += rust_exp(x);
        bytes.push_back('\0');
      }
      output_bytes(bytes.data(), bytes.size(), 1, out, capacity, required);
    });
  });
}

uint64_t sdpx_last_error(char* out, uint64_t capacity) {
  const std::string& e = sdpxg::g_last_error;
  uint64_t n = e.size() + 1;
  if (out && capacity > 0) {
    uint64_t k = std::min<uint64_t>(e.size(), capacity - 1);
    std::memcpy(out, e.data(), k);
    out[k] = 0;
  }
  return n;
}

int32_t sdpx_destroy(sdpx_handle* h) {
  return boundary([&] {
    if (!h) return;
    {
      std::unique_lock<std::mutex> lk(h->mu, std::try_to_lock);
      if (!lk.owns_lock()) throw AbiError{3, "handle is busy"};
    }
    delete h;
  });
}

uint64_t sdpx_b200_launch_count(void) { return sdpxg::g_launches; }
uint64_t sdpx_b200_device_allocations(void) { return sdpxg::g_dev_allocs; }

int32_t sdpx_b200_set_i8_timing(int32_t on) {
  return boundary([&] { sdpxg::i8_timing(on != 0); });
}

int32_t sdpx_b200_i8_config(int32_t variant) {
  return boundary([&] {
    if (variant < -1 || variant > 2) invalid("variant must be -1 (autotuned), 0, 1 or 2");
    sdpxg::i8_set_config(variant);
  });
}

int32_t sdpx_b200_i8_tuning(char* out, uint64_t capacity, uint64_t* required) {
  return boundary([&] {
    const std::string t = sdpxg::i8_tuning_table();
    output_bytes(t.c_str(), t.size() + 1, 1, out, capacity, required);
  });
}

int32_t sdpx_b200_i8_times(double* ms, double* ops, double* alg_ops, uint64_t* launches) {
  return boundary([&] {
    if (!ms || !ops || !alg_ops || !launches) invalid("null pointer");
    sdpxg::i8_times(ms, ops, alg_ops, launches);
  });
}

int32_t sdpx_b200_transfer_bytes(uint64_t* h2d, uint64_t* d2h) {
  return boundary([&] {
    if (!h2d || !d2h) invalid("null pointer");
    *h2d = sdpxg::g_h2d_bytes;
    *d2h = sdpxg::g_d2h_bytes;
  });
}

int32_t sdpx_b200_set_kernel_timing(sdpx_handle* h, int32_t on) {
  return boundary([&] {
    operate(h, [&](sdpx_handle& hh) {
      hh.eng->timing = on != 0;
      hh.eng->reset_timers();
    });
  });
}

int32_t sdpx_b200_kernel_times(sdpx_handle* h, double* ms, uint64_t* counts) {
  return boundary([&] {
    if (!ms || !counts) invalid("null pointer");
    operate(h, [&](sdpx_handle& hh) {
      for (int k = 0; k < KT_N; ++k) {
        ms[k] = hh.eng->kt_ms[k];
        counts[k] = hh.eng->kt_count[k];
      }
    });
  });
}

int32_t sdpx_b200_adjoint(sdpx_handle* h, const double* dl_dx, const double* dl_dz,
                          const double* dl_ds, double* dq, double* db, double* dA, uint64_t nnz) {
  return boundary([&] {
    if (!dl_dx || !dq || !db) invalid("null pointer");
    operate(h, [&](sdpx_handle& hh) {
      if (!hh.solved || !hh.hsd) throw AbiError{7, "no result: solve the handle first"};
      const int st = (int)hh.info.status;
      if (st != ST_SOLVED && st != ST_ALMOST_SOLVED)
        throw AbiError{7, "no optimal solution to differentiate (status " + std::to_string(st) + ")"};
      const int n = hh.orig.n, m = hh.orig.m;
      const HostProblem& p = hh.equil;  // same sparsity pattern as the input A
      if (dA && nnz != (uint64_t)p.Aval.size()) invalid("dA needs one value per stored entry of A");
      std::vector<double> gx(dl_dx, dl_dx + n), gz(m, 0.0), gs(m, 0.0), u, v;
      if (dl_dz) gz.assign(dl_dz, dl_dz + m);
      if (dl_ds) gs.assign(dl_ds, dl_ds + m);
      for (double t : gx)
        if (!std::isfinite(t)) invalid("nonfinite input");
      if (!hh.hsd->adjoint(gx, gz, gs, u, v))
        throw AbiError{5, "adjoint: the KKT system at the solution could not be factored or solved"};
      for (int j = 0; j < n; ++j) dq[j] = -u[j];
      for (int i = 0; i < m; ++i) db[i] = v[i];
      if (dA)
        for (int j = 0; j < n; ++j)
          for (int64_t q = p.Acolptr[j]; q < p.Acolptr[j + 1]; ++q) {
            const int64_t i = p.Arow[q];
            dA[q] = -(hh.z[i] * u[j] + v[i] * hh.x[j]);
          }
    });
  });
}

int32_t sdpx_b200_set_graphs(sdpx_handle* h, int32_t on) {
  return boundary([&] {
    operate(h, [&](sdpx_handle& hh) {
      hh.eng->clear_graphs();
      hh.eng->graphs_enabled = on != 0;
    });
  });
}

int32_t sdpx_b200_set_form(sdpx_handle* h, uint32_t form) {
  return boundary([&] {
    if (form > 1) invalid("form must be 0 (plain) or 1 (split precision)");
    operate(h, [&](sdpx_handle& hh) { hh.eng->factor_form = (int)form; });
  });
}

int32_t sdpx_b200_schur_forms(sdpx_handle* h, uint32_t* gram_blocks, uint32_t* ordinary_blocks) {
  return boundary([&] {
    if (!gram_blocks || !ordinary_blocks) invalid("null pointer");
    operate(h, [&](sdpx_handle& hh) {
      *gram_blocks = (uint32_t)hh.eng->gram_blocks();
      *ordinary_blocks = (uint32_t)(hh.eng->nblk - hh.eng->gram_blocks());
    });
  });
}

int32_t sdpx_b200_phase_times(sdpx_handle* h, double* times, uint64_t* counts) {
  return boundary([&] {
    if (!times || !counts) invalid("null pointer");
    operate(h, [&](sdpx_handle& hh) {
      const PhaseTimes& t = hh.times;
      double v[7] = {t.scale, t.assemble, t.factor, t.solve, t.step, t.residual, t.other};
      std::memcpy(times, v, sizeof v);
      counts[0] = (uint64_t)t.factorizations;
      counts[1] = (uint64_t)t.kkt_solves;
      counts[2] = (uint64_t)t.outer_refinements;
      counts[3] = (uint64_t)t.inner_refinements;
    });
  });
}

int32_t sdpx_b200_kkt_paths(sdpx_handle* h, uint64_t* device_driven, uint64_t* host_driven) {
  return boundary([&] {
    if (!device_driven || !host_driven) invalid("null pointer");
    operate(h, [&](sdpx_handle& hh) {
      const PhaseTimes& t = hh.times;
      *device_driven = (uint64_t)t.device_kkt_solves;
      *host_driven = (uint64_t)(t.kkt_solves - t.device_kkt_solves);
    });
  });
}

}  // extern "C"
