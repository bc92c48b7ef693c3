// Kernel-level C ABI (sdpxg_*): one hot-path operation per call, host pointers in and out.
// These are the entry points a host that keeps its own interior-point driver binds in place
// of its CPU kernels; each copies its inputs to the device, runs on the context's stream and
// copies the outputs back before returning.
#include <memory>
#include <string>

#include "../../include/sdpx_b200.h"
#include "hsd.cuh"
#include "sampled.cuh"

using namespace sdpxg;

namespace sdpxg {
extern thread_local std::string g_last_error;
}

namespace {

template <typename F>
int32_t guard(F&& f) {
  try {
    return f();
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
    sdpxg::g_last_error = "internal error";
    return 5;
  }
}
}  // namespace

struct sdpxg_ctx {
  int device = 0;
  std::unique_ptr<Engine> eng;
  HostProblem prob;
  Equilibration eq;
  std::unique_ptr<HsdSolver> kkt;  // owns the refinement scratch
  DevBuf<double> a, b, c, d, e, f;
  bool uploaded = false;
  std::shared_ptr<void> rns_ws;  // workspace of the exact (RNS) products, created on first use
};

namespace sdpxg {
// The engine of a context with an uploaded problem (nullptr otherwise).
Engine* ctx_engine(sdpxg_ctx* c) { return (c && c->uploaded) ? c->eng.get() : nullptr; }
// The engine of any context (no problem needed) and its RNS workspace slot.
Engine* ctx_engine_any(sdpxg_ctx* c) { return c ? c->eng.get() : nullptr; }
std::shared_ptr<void>* ctx_rns_slot(sdpxg_ctx* c) { return c ? &c->rns_ws : nullptr; }
}  // namespace sdpxg

namespace {
void need(sdpxg_ctx* c) {
  if (!c) throw std::invalid_argument("null context");
  if (!c->uploaded) throw std::invalid_argument("no problem uploaded");
}
// Ensure buf holds n doubles; copy h into it when h is given (h == nullptr: allocate only).
void to_dev(DevBuf<double>& buf, const double* h, size_t n, cudaStream_t st) {
  if (buf.n < std::max<size_t>(n, 1)) buf.alloc(std::max<size_t>(n, 1));
  if (n && h) buf.upload(h, n, st);
}
void in_dev(DevBuf<double>& buf, const double* h, size_t n, cudaStream_t st) {
  if (n && !h) throw std::invalid_argument("null pointer");
  to_dev(buf, h, n, st);
}
void to_host(double* h, const DevBuf<double>& buf, size_t n, cudaStream_t st) {
  if (!n) return;
  if (!h) throw std::invalid_argument("null pointer");
  check(cudaMemcpyAsync(h, buf.p, n * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
  check(cudaStreamSynchronize(st), "sync");
}
template <class IC, class IR, class DV>
void csc_into(const sdpx_csc* m, IC& cp, IR& rv, DV& v, uint64_t cols) {
  cp.assign(cols + 1, 0);
  rv.clear();
  v.clear();
  if (!m) return;
  if (m->cols != cols || m->values.kind != 0 || !m->colptr) throw std::invalid_argument("bad CSC");
  for (uint64_t j = 0; j <= cols; ++j) cp[j] = (int64_t)m->colptr[j];
  for (uint64_t p = 0; p < m->nnz; ++p) {
    rv.push_back((int64_t)m->rowval[p]);
    v.push_back(m->values.f64[p]);
  }
}
}  // namespace

extern "C" {

int32_t sdpxg_ctx_create(int32_t device, uint32_t flags, sdpxg_ctx** out) {
  return guard([&] {
    if (!out) throw std::invalid_argument("null pointer");
    *out = nullptr;
    if (flags != 0) throw std::invalid_argument("flags must be 0");
    auto c = std::make_unique<sdpxg_ctx>();
    c->device = device;
    c->eng = std::make_unique<Engine>();
    c->eng->init(device);
    *out = c.release();
    return 0;
  });
}

int32_t sdpxg_ctx_destroy(sdpxg_ctx* ctx) {
  return guard([&] {
    delete ctx;
    return 0;
  });
}

int32_t sdpxg_problem_upload(sdpxg_ctx* ctx, const sdpx_csc* P, const sdpx_csc* A,
                             const uint64_t* psd_orders, uint64_t block_count) {
  return guard([&] {
    if (!ctx || !A) throw std::invalid_argument("null pointer");
    if (block_count && !psd_orders) throw std::invalid_argument("null pointer");
    HostProblem& p = ctx->prob;
    p = HostProblem();
    p.n = (int)A->cols;
    p.m = (int)A->rows;
    csc_into(A, p.Acolptr, p.Arow, p.Aval, A->cols);
    csc_into(P, p.Pcolptr, p.Prow, p.Pval, A->cols);
    for (uint64_t j = 0; j < block_count; ++j) p.psd.push_back((int)psd_orders[j]);
    p.q.assign(p.n, 0.0);
    p.b.assign(p.m, 0.0);
    ctx->eq.d.assign(p.n, 1.0);
    ctx->eq.dinv.assign(p.n, 1.0);
    ctx->eq.e.assign(p.m, 1.0);
    ctx->eq.einv.assign(p.m, 1.0);
    ctx->eq.c = 1.0;
    ctx->eng->upload(p);
    ctx->kkt = std::make_unique<HsdSolver>(*ctx->eng, p, ctx->eq, Settings());
    ctx->uploaded = true;
    return 0;
  });
}

int32_t sdpxg_problem_upload_sampled(sdpxg_ctx* ctx, const sdpx_csc* P, const sdpx_csc* A_linear,
                                     const uint64_t* psd_orders, uint64_t block_count,
                                     const sdpx_sampled_block* blocks, uint64_t nblocks) {
  return guard([&] {
    if (!ctx || !A_linear) throw std::invalid_argument("null pointer");
    if (block_count && !psd_orders) throw std::invalid_argument("null pointer");
    std::vector<int64_t> cp, rv;
    std::vector<double> v;
    csc_into(A_linear, cp, rv, v, A_linear->cols);
    std::vector<std::pair<uint64_t, uint64_t>> psd_rows;
    uint64_t row = 0;
    for (uint64_t j = 0; j < block_count; ++j) {
      psd_rows.push_back({row, psd_orders[j]});
      row += psd_orders[j] * (psd_orders[j] + 1) / 2;
    }
    SampledCsc merged = materialize_sampled(A_linear->rows, A_linear->cols, cp, rv, v, psd_rows, blocks, nblocks);
    sdpx_csc A{};
    A.rows = A_linear->rows;
    A.cols = A_linear->cols;
    A.nnz = merged.rowval.size();
    A.colptr = merged.colptr.data();
    A.rowval = merged.rowval.data();
    A.values.kind = 0;
    A.values.count = merged.val.size();
    A.values.f64 = merged.val.data();
    const int32_t rc = sdpxg_problem_upload(ctx, P, &A, psd_orders, block_count);
    if (rc) return rc;
    // the given factors replace the rank-one test of the materialised columns
    ctx->prob.sampled = std::move(merged.recs);
    ctx->eng->upload(ctx->prob);
    ctx->kkt = std::make_unique<HsdSolver>(*ctx->eng, ctx->prob, ctx->eq, Settings());
    return 0;
  });
}

int32_t sdpxg_set_scaling(sdpxg_ctx* ctx, const double* R, const double* Rinv) {
  return guard([&] {
    need(ctx);
    ctx->eng->set_scaling(R, Rinv);
    return 0;
  });
}

int32_t sdpxg_identity_scaling(sdpxg_ctx* ctx) {
  return guard([&] {
    need(ctx);
    ctx->eng->identity_scaling();
    check(cudaStreamSynchronize(ctx->eng->st), "sync");
    return 0;
  });
}

int32_t sdpxg_nt_scale(sdpxg_ctx* ctx, const double* s, const double* z, double* out_lambda,
                       uint32_t* status) {
  return guard([&] {
    need(ctx);
    Engine& E = *ctx->eng;
    in_dev(ctx->a, s, E.m, E.st);
    in_dev(ctx->b, z, E.m, E.st);
    bool ok = E.nt_scale(ctx->a, ctx->b);
    if (status) *status = ok ? 0u : 1u;
    if (out_lambda && ok) {
      // lambda is the diagonal of W^-T s = svec(diag(lambda)) per block
      to_dev(ctx->c, nullptr, E.m, E.st);
      E.cone_apply(CM_WINVT, ctx->a, ctx->c);
      std::vector<double> h(E.m);
      to_host(h.data(), ctx->c, E.m, E.st);
      size_t k = 0;
      for (const BlockDesc& bd : E.hblocks)
        for (int i = 0; i < bd.n; ++i) out_lambda[k++] = h[bd.svec_off + i * (i + 1) / 2 + i];
    }
    return 0;
  });
}

int32_t sdpxg_schur_assemble(sdpxg_ctx* ctx, double* out_schur) {
  return guard([&] {
    need(ctx);
    Engine& E = *ctx->eng;
    if (!E.assemble()) throw std::runtime_error("non-finite Schur complement");
    if (out_schur) {
      check(cudaMemcpyAsync(out_schur, E.Hsave(), (size_t)E.n * E.n * sizeof(double),
                            cudaMemcpyDeviceToHost, E.st), "schur D2H");
      check(cudaStreamSynchronize(E.st), "sync");
    }
    return 0;
  });
}

int32_t sdpxg_factor(sdpxg_ctx* ctx, double shift, uint32_t dynamic, double eps, double delta,
                     uint32_t* status) {
  return guard([&] {
    need(ctx);
    bool ok = ctx->eng->factor(shift, dynamic != 0, eps, delta);
    if (status) *status = ok ? 0u : (uint32_t)SDPXG_ST_PIVOT_FAIL;
    return 0;
  });
}

int32_t sdpxg_set_factor_form(sdpxg_ctx* ctx, uint32_t form) {
  return guard([&] {
    if (!ctx) throw std::invalid_argument("null context");
    if (form > 1) throw std::invalid_argument("form must be 0 (plain) or 1 (split precision)");
    ctx->eng->factor_form = (int)form;
    return 0;
  });
}

int32_t sdpxg_split_dgemm_device(sdpxg_ctx* ctx, char ta, char tb, uint64_t m, uint64_t n, uint64_t k,
                                 double alpha, const double* d_A, uint64_t lda, const double* d_B, uint64_t ldb,
                                 double beta, double* d_C, uint64_t ldc, uint32_t* status) {
  return guard([&] {
    if (!ctx) throw std::invalid_argument("null context");
    if ((ta != 'N' && ta != 'T') || (tb != 'N' && tb != 'T')) throw std::invalid_argument("bad transpose flag");
    if (m > (1u << 30) || n > (1u << 30) || k > (1u << 16)) throw std::invalid_argument("size out of range");
    if (m == 0 || n == 0) return 0;
    const uint64_t ar = ta == 'N' ? m : k, br = tb == 'N' ? k : n;
    if (lda < std::max<uint64_t>(ar, 1) || ldb < std::max<uint64_t>(br, 1) || ldc < m)
      throw std::invalid_argument("leading dimension too small");
    if (!d_A || !d_B || !d_C) throw std::invalid_argument("null pointer");
    Engine& E = *ctx->eng;
    check(cudaSetDevice(E.device), "cudaSetDevice");
    // the left operand's row i is row i of op(A); the right operand's row j is column j of op(B)
    const long l_sr = ta == 'N' ? 1 : (long)lda, l_sk = ta == 'N' ? (long)lda : 1;
    const long r_sr = tb == 'N' ? (long)ldb : 1, r_sk = tb == 'N' ? 1 : (long)ldb;
    if (!E.oz.status.p) E.oz.status.alloc(1);
    check(cudaMemsetAsync(E.oz.status.p, 0, sizeof(uint32_t), E.st), "memset");
    ozaki_gemm(E.oz, E.st, (int)m, (int)n, (int)k, d_A, l_sr, l_sk, d_B, r_sr, r_sk, alpha, beta, d_C, (long)ldc, 0);
    uint32_t hs[2] = {0, 0};
    copy_d2h(&hs[0], E.oz.status.p, sizeof(uint32_t), E.st);
    copy_d2h(&hs[1], E.oz.err.p, sizeof(uint32_t), E.st);
    check(cudaStreamSynchronize(E.st), "sync");
    if (hs[1]) throw std::runtime_error("split-precision GEMM: a bounded wait gave up");
    if (status) *status = hs[0];
    return 0;
  });
}

int32_t sdpxg_solve_many(sdpxg_ctx* ctx, const double* rhs, double* out, uint32_t ncols) {
  return guard([&] {
    need(ctx);
    Engine& E = *ctx->eng;
    for (uint32_t c = 0; c < ncols; ++c) {
      in_dev(ctx->a, rhs + (size_t)c * E.n, E.n, E.st);
      to_dev(ctx->b, nullptr, E.n, E.st);
      if (!ctx->kkt->reduced_solve(ctx->a, ctx->b)) throw std::runtime_error("reduced solve failed");
      to_host(out + (size_t)c * E.n, ctx->b, E.n, E.st);
    }
    return 0;
  });
}

int32_t sdpxg_kkt_solve(sdpxg_ctx* ctx, const double* bx, const double* bz, double* x, double* z) {
  return guard([&] {
    need(ctx);
    Engine& E = *ctx->eng;
    in_dev(ctx->a, bx, E.n, E.st);
    in_dev(ctx->b, bz, E.m, E.st);
    to_dev(ctx->c, nullptr, E.n, E.st);
    to_dev(ctx->d, nullptr, E.m, E.st);
    if (!ctx->kkt->kkt_solve(ctx->a, ctx->b, ctx->c, ctx->d)) throw std::runtime_error("KKT solve failed");
    to_host(x, ctx->c, E.n, E.st);
    to_host(z, ctx->d, E.m, E.st);
    return 0;
  });
}

int32_t sdpxg_residual(sdpxg_ctx* ctx, const double* bx, const double* bz, const double* x,
                       const double* z, double* ex, double* ez, double* norm) {
  return guard([&] {
    need(ctx);
    Engine& E = *ctx->eng;
    in_dev(ctx->a, bx, E.n, E.st);
    in_dev(ctx->b, bz, E.m, E.st);
    in_dev(ctx->c, x, E.n, E.st);
    in_dev(ctx->d, z, E.m, E.st);
    to_dev(ctx->e, nullptr, E.n, E.st);
    to_dev(ctx->f, nullptr, E.m, E.st);
    ctx->kkt->residual_full(ctx->a, ctx->b, ctx->c, ctx->d, ctx->e, ctx->f);
    int s0 = E.red.add(E.st, RED_MAXABS, E.n, ctx->e, nullptr);
    int s1 = E.red.add(E.st, RED_MAXABS, E.m, ctx->f, nullptr);
    auto& h = E.red.fetch(E.st);
    if (norm) *norm = std::max(h[s0], h[s1]);
    if (ex) to_host(ex, ctx->e, E.n, E.st);
    if (ez) to_host(ez, ctx->f, E.m, E.st);
    return 0;
  });
}

int32_t sdpxg_step_length(sdpxg_ctx* ctx, const double* dz, const double* ds, double amax,
                          uint32_t mode, double* out_alpha, uint32_t* status) {
  return guard([&] {
    need(ctx);
    if (!out_alpha) throw std::invalid_argument("null pointer");
    Engine& E = *ctx->eng;
    in_dev(ctx->a, dz, E.m, E.st);
    in_dev(ctx->b, ds, E.m, E.st);
    double az, as;
    bool ok = E.step_bounds(ctx->a, ctx->b, amax, mode ? 1 : 0, &az, &as);
    *out_alpha = std::min(az, as);
    if (status) *status = ok ? 0u : (uint32_t)SDPXG_ST_EIG_FAIL;
    return 0;
  });
}

int32_t sdpxg_cone_apply(sdpxg_ctx* ctx, uint32_t op, const double* x, double* y) {
  return guard([&] {
    need(ctx);
    if (op > 5) throw std::invalid_argument("unknown cone operator");
    Engine& E = *ctx->eng;
    in_dev(ctx->a, x, E.m, E.st);
    to_dev(ctx->b, nullptr, E.m, E.st);
    E.cone_apply((int)op, ctx->a, ctx->b);
    to_host(y, ctx->b, E.m, E.st);
    return 0;
  });
}

}  // extern "C"
