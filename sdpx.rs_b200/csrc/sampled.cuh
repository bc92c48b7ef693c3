// Factor-authoritative sampled PSD blocks (the reference's SampledBlock,
// crates/solver/src/solver/sampled/mod.rs:9-29; C ABI include/sdpx.h:40-50): validation and
// materialisation of their primitive columns.
//
// A block sits on one PSD cone of order dim * basis_rows starting at row row_start and owns the
// variables column_start .. column_start + tri(dim) basis_cols - 1, in the order (s, r, k),
// r <= s < dim, k fastest; variable (s, r, k) is weights[t] svec(sym(e_r e_s') (x) q_k q_k'), q_k
// column k of the column-major basis (dim = 1: weights[k] svec(q_k q_k')).  Its materialised
// column keeps every entry of the blocks it touches (explicit zeros included) so each primitive
// stays present in A.
#pragma once
#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <utility>
#include <vector>

#include "../../include/sdpx_b200.h"
#include "engine.cuh"

namespace sdpxg {

struct SampledCsc {
  std::vector<uint64_t> colptr, rowval;
  std::vector<double> val;
  std::vector<HostProblem::Sampled> recs;  // weights as given (unscaled)
};

// Unsupported inputs throw SampledUnsupported (mapped to return code 2 by the callers); invalid
// ones std::invalid_argument.
struct SampledUnsupported : std::runtime_error {
  using std::runtime_error::runtime_error;
};

template <class IV, class FV>
SampledCsc materialize_sampled(uint64_t m, uint64_t n, const IV& colptr, const IV& rowval, const FV& val,
                               const std::vector<std::pair<uint64_t, uint64_t>>& psd_rows,
                               const sdpx_sampled_block* blocks, uint64_t nb) {
  if (nb && !blocks) throw std::invalid_argument("null pointer");
  struct Prim {
    uint64_t row0, h;   // cone rows start, basis rows
    int r, s;           // block pair, r <= s
    const double* q;    // basis column
    double w;
  };
  std::vector<int64_t> owner(n, -1);
  std::vector<Prim> prims;
  SampledCsc out;
  std::vector<char> cone_used(psd_rows.size(), 0);
  for (uint64_t bi = 0; bi < nb; ++bi) {
    const sdpx_sampled_block& B = blocks[bi];
    if (B.dim == 0 || B.basis_rows == 0) throw std::invalid_argument("sampled block dim and basis_rows must be positive");
    if (B.dim * B.basis_rows > SDPXG_NMAX)
      throw SampledUnsupported("sampled block order dim * basis_rows above 64 is not supported on the GPU path");
    if (B.basis.kind != 0 || B.weights.kind != 0)
      throw SampledUnsupported("decimal sampled data needs precision_bits > 53");
    const uint64_t prims_n = B.dim * (B.dim + 1) / 2 * B.basis_cols;
    if (B.basis.count != B.basis_rows * B.basis_cols || B.weights.count != prims_n)
      throw std::invalid_argument("sampled block basis or weights have the wrong length");
    if (B.basis_cols && (!B.basis.f64 || !B.weights.f64)) throw std::invalid_argument("null pointer");
    size_t c = 0;
    while (c < psd_rows.size() && psd_rows[c].first != B.row_start) ++c;
    if (c == psd_rows.size() || psd_rows[c].second != B.dim * B.basis_rows)
      throw std::invalid_argument("sampled block is not aligned with a PSD cone of order dim * basis_rows");
    if (cone_used[c]) throw std::invalid_argument("two sampled blocks share a PSD cone");
    cone_used[c] = 1;
    if (B.column_start + prims_n > n) throw std::invalid_argument("sampled block columns exceed the variables");
    const uint64_t order = B.dim * B.basis_rows, tn = order * (order + 1) / 2;
    for (uint64_t j = 0; j < n; ++j)  // A_linear must be zero on the block's rows
      for (int64_t p = (int64_t)colptr[j]; p < (int64_t)colptr[j + 1]; ++p)
        if ((uint64_t)rowval[p] >= B.row_start && (uint64_t)rowval[p] < B.row_start + tn && val[p] != 0.0)
          throw std::invalid_argument("A_linear must be zero on the rows of a sampled block");
    HostProblem::Sampled rec;
    rec.row_start = (int)B.row_start;
    rec.col0 = (int)B.column_start;
    rec.count = (int)B.basis_cols;
    rec.dim = (int)B.dim;
    rec.order = (int)order;
    rec.basis.assign(B.basis.f64, B.basis.f64 + B.basis.count);
    rec.weight.assign(B.weights.f64, B.weights.f64 + B.weights.count);
    uint64_t t = 0;
    for (uint64_t ss = 0; ss < B.dim; ++ss)
      for (uint64_t rr = 0; rr <= ss; ++rr)
        for (uint64_t k = 0; k < B.basis_cols; ++k, ++t) {  // primitive order (s, r, k), k fastest
          const uint64_t col = B.column_start + t;
          if (owner[col] >= 0) throw std::invalid_argument("two sampled blocks share a primitive column");
          owner[col] = (int64_t)prims.size();
          prims.push_back({B.row_start, B.basis_rows, (int)rr, (int)ss, B.basis.f64 + k * B.basis_rows,
                           B.weights.f64[t]});
        }
    out.recs.push_back(std::move(rec));
  }
  out.colptr.assign(n + 1, 0);
  std::vector<std::pair<uint64_t, double>> e;
  for (uint64_t j = 0; j < n; ++j) {
    e.clear();
    for (int64_t p = (int64_t)colptr[j]; p < (int64_t)colptr[j + 1]; ++p) e.push_back({(uint64_t)rowval[p], val[p]});
    if (owner[j] >= 0) {
      // w svec(sym(e_r e_s') (x) q q'): the (r, s) and (s, r) h x h blocks hold q q' / 2 (q q' on the
      // diagonal when r = s); every entry of those blocks is kept, zeros included
      const Prim& pr = prims[(size_t)owner[j]];
      uint64_t r1 = pr.row0;
      {  // the block's rows end where its cone ends
        size_t c = 0;
        while (c < psd_rows.size() && psd_rows[c].first != pr.row0) ++c;
        r1 = pr.row0 + psd_rows[c].second * (psd_rows[c].second + 1) / 2;
      }
      e.erase(std::remove_if(e.begin(), e.end(),
                             [&](const std::pair<uint64_t, double>& x) { return x.first >= pr.row0 && x.first < r1; }),
              e.end());
      const double f = pr.r == pr.s ? 1.0 : 0.5;
      for (uint64_t tj = 0; tj < pr.h; ++tj) {
        const uint64_t cj = pr.s * pr.h + tj;  // column in block s
        for (uint64_t ti = 0; ti < pr.h; ++ti) {
          const uint64_t ci = pr.r * pr.h + ti;  // row in block r
          if (pr.r == pr.s && ci > cj) continue;  // diagonal block: upper triangle only
          e.push_back({pr.row0 + cj * (cj + 1) / 2 + ci,
                       pr.w * f * pr.q[ti] * pr.q[tj] * (ci == cj ? 1.0 : SDPXG_SQRT2)});
        }
      }
      std::sort(e.begin(), e.end());
    }
    for (auto& x : e) {
      out.rowval.push_back(x.first);
      out.val.push_back(x.second);
    }
    out.colptr[j + 1] = out.rowval.size();
  }
  (void)m;
  return out;
}

}  // namespace sdpxg
