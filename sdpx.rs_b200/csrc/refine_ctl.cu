// Control kernels of the device-driven KKT solve.  One refined solve (condense, reduced solve
// with inner refinement against the unshifted Schur complement, recover, outer refinement against
// the original operator: kkt/condensed/kkt.rs:275-318 with kkt/refinement.rs:118-191) runs as ONE
// CUDA graph whose two refinement loops are WHILE conditional nodes.  After each straight run of
// the graph a single thread reads the run's reduction slots, applies the reference's stopping
// rule (tolerance abstol + reltol |b|, stop when the residual ratio falls below stop_ratio,
// keep the candidate only when it improved, at most max_iter steps) and sets the loop's
// condition.  Every loop also stops once `guard` body executions have run, so no condition can
// stay set.  The arithmetic is the host driver's, operation for operation, so the graph's
// results equal the host-driven refinement's bit for bit.
#include "common.cuh"

// std::max(a, b) of the host driver: (a < b) ? b : a (a NaN in b is ignored, one in a is kept)
__device__ __forceinline__ double host_max(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ void ctl_set(cudaGraphConditionalHandle h, bool go) {
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// Start of a reduced solve: slots |r|max, |e|max, finite(x) of the first pass (and, at the head
// of a KKT solve, finite(bx), finite(bz)).  reset != 0 starts a new KKT solve.
extern "C" __global__ void k_refine_head(const double* fin_bx, const double* fin_bz,
                                         const double* nr, const double* ne, const double* fin_x,
                                         int reset, RefineCtl* c, RefineParams p,
                                         cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (reset) {
    RefineCtl z{};
    z.ok = 1;
    *c = z;
  }
  bool ok = c->ok != 0;
  if (fin_bx && *fin_bx != 1.0) ok = false;
  if (fin_bz && *fin_bz != 1.0) ok = false;
  if (*fin_x != 1.0 || !isfinite(*ne)) ok = false;
  c->ok = ok ? 1 : 0;
  c->normb = *nr;
  c->norme = *ne;
  c->tol = p.abstol + p.reltol * c->normb;
  c->it = 0;
  c->accept = c->cont = 0;
  ctl_set(h, ok && !(c->norme <= c->tol) && p.max_iter > 0);
}

// After one inner step: slot |e2|max of the candidate's reduced residual.
extern "C" __global__ void k_refine_step(const double* ne2, RefineCtl* c, RefineParams p,
                                         cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  c->inner_steps++;
  c->guard++;
  bool go = false;
  int acc = 0;
  const double e = *ne2;
  if (!isfinite(e)) {
    c->ok = 0;
  } else {
    const double ratio = c->norme / e;
    if (ratio < p.stop_ratio) {
      acc = ratio > 1.0;
    } else {
      acc = 1;
      c->norme = e;
      c->it++;
      go = !(e <= c->tol) && c->it < p.max_iter;
    }
  }
  if (c->guard >= p.guard_max) {
    go = false;
    c->ok = 0;
  }
  c->accept = acc;
  c->cont = go;
  ctl_set(h, go);
}

// After recover + full residual: slots |bx|, |bz|, |ex|, |ez|.
extern "C" __global__ void k_refine_outer_init(const double* nbx, const double* nbz,
                                               const double* nex, const double* nez, RefineCtl* c,
                                               RefineParams p, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  c->onormb = host_max(*nbx, *nbz);
  const double e = host_max(*nex, *nez);
  c->onorme = e;
  c->oit = 0;
  c->oaccept = c->ocont = 0;
  bool go = false;
  if (!isfinite(e)) {
    c->ok = 0;
  } else if (c->ok) {
    c->otol = p.abstol + p.reltol * c->onormb;
    go = !(e <= c->otol) && p.max_iter > 0;
  }
  ctl_set(h, go);
}

// After one outer correction: slots |ex2|, |ez2| of the candidate's full residual.
extern "C" __global__ void k_refine_outer_step(const double* nex2, const double* nez2,
                                               RefineCtl* c, RefineParams p,
                                               cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  c->outer_steps++;
  c->guard++;
  bool go = false;
  int acc = 0;
  if (c->ok) {  // the correction's own solve passed its checks
    const double e = host_max(*nex2, *nez2);
    if (!isfinite(e)) {
      c->ok = 0;
    } else {
      const double ratio = c->onorme / e;
      if (ratio < p.stop_ratio) {
        acc = ratio > 1.0;
      } else {
        acc = 1;
        c->onorme = e;
        c->oit++;
        go = !(e <= c->otol) && c->oit < p.max_iter;
      }
    }
  }
  if (c->guard >= p.guard_max) {
    go = false;
    c->ok = 0;
  }
  c->oaccept = acc;
  c->ocont = go;
  ctl_set(h, go);
}

// d1 = s1 (n1 entries) when *f1 is set, d2 = s2 (n2 entries) when *f2 is set.
extern "C" __global__ void k_refine_copy(const int* f1, long n1, double* d1, const double* s1,
                                         const int* f2, long n2, double* d2, const double* s2) {
  const bool a = *f1 != 0, b = *f2 != 0;
  if (!a && !b) return;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n1 + n2; i += stride) {
    if (i < n1) {
      if (a) d1[i] = s1[i];
    } else if (b) {
      d2[i - n1] = s2[i - n1];
    }
  }
}
