"""Adjoint of the conic QP solution map -- TEST ORACLE (test infrastructure only).

The reference has no differentiation feature, so gradients have no reference to pin against
("parity unpinned" for gradients): this restatement is checked against central finite
differences of whole solves (``tests/test_adjoint.py``) and serves as the FP64 checker of the
library's adjoint.  It solves the reference's KKT system, the quasi-definite matrix
``[P A'; A -Hs]`` of crates/solver/src/solver/kkt/direct/kkt_assembly.rs:31-246, with ``Hs`` the
NT scaling of cones/psdtrianglecone.rs:311-439 (PSD blocks) and cones/nonnegativecone.rs
(orthant rows, Hs = s / z), all in dense binary64.

Solution map and its adjoint.  At a solution (x, s, z) of  min 1/2 x'Px + q'x  s.t.
A x + s = b, s in K, the directions satisfy  P dx + A'dz = -dq - dA'z,  A dx - Hs dz =
db - dA x  once the complementarity block is linearised in the scaled coordinates.  For a loss
with gradient g = dL/dx, solve  [P A'; A -Hs] [u; v] = [g; 0]; then
    dL/dq = -u,  dL/db = v,  dL/dA = -(z u' + v x').
At an exactly complementary solution Hs is singular or unbounded on the active/inactive split;
the solution is first moved onto the central path at a small relative mu (``recentre``), in the
equilibrated coordinates the library works in.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import ipm


def recentre(cones, s, z, rel=1e-9):
    """(s, z) moved onto the central path at a small relative mu: per PSD block the eigenbasis
    of S - Z, the larger of each complementary eigenvalue pair kept and its partner set to
    rel * scale^2 / |lambda| (scale = the block's largest |lambda|); per orthant row the larger
    of s_i, z_i kept and the other set to rel times it."""
    sc, zc, r = s.copy(), z.copy(), 0
    for kind, d in cones:
        if kind == "nonneg":
            for i in range(r, r + d):
                big = max(abs(s[i]), abs(z[i]))
                if s[i] >= z[i]:
                    sc[i], zc[i] = big, rel * big
                else:
                    sc[i], zc[i] = rel * big, big
            r += d
        else:
            k = d * (d + 1) // 2
            w, Q = np.linalg.eigh(ipm.svec_to_mat(s[r:r + k], d) - ipm.svec_to_mat(z[r:r + k], d))
            top = np.abs(w).max()
            ls = np.where(w > 0, w, rel * top * top / np.abs(w))
            lz = np.where(w > 0, rel * top * top / np.abs(w), -w)
            sc[r:r + k] = ipm.mat_to_svec(Q @ np.diag(ls) @ Q.T)
            zc[r:r + k] = ipm.mat_to_svec(Q @ np.diag(lz) @ Q.T)
            r += k
    return sc, zc


def dense_hs(cones, s, z):
    """Hs of the NT scaling at (s, z): block diagonal over the cones, in svec coordinates."""
    objs = ipm.make_cones(cones)
    m = sum(c.numel for c in objs)
    out = np.zeros((m, m))
    r = 0
    for c in objs:
        k = c.numel
        if not c.update_scaling(s[r:r + k], z[r:r + k]):
            raise ValueError("recentred point is not interior")
        out[r:r + k, r:r + k] = np.column_stack([c.mul_Hs(e) for e in np.eye(k)])
        r += k
    return out


def adjoint(prob, x, s, z, gx, rel=1e-9, equilibrated=True):
    """(dL/dq, dL/db, dL/dA on the CSC pattern of A) for dL/dx = gx at the solution (x, s, z).

    ``equilibrated``: re-centre (s, z) in the coordinates of the reference's Ruiz equilibration
    (problemdata.rs:639-900; s_bar = E s, z_bar = c E^-1 z) and solve the equilibrated system
    [P_bar A_bar'; A_bar -Hs_bar][u_bar; v_bar] = [D gx; 0], mapping back u = c D u_bar,
    v = E v_bar -- the point and system the library differentiates.  Both choices define the
    same limit as rel -> 0; at rel = 1e-9 they differ by about 1e-5 relative, the distance of the
    re-centred point from that limit."""
    A = sp.csc_matrix(prob.A)
    n, m = A.shape[1], A.shape[0]
    Pm = np.zeros((n, n)) if prob.P is None else sp.csc_matrix(prob.P).toarray()
    if not np.allclose(Pm, Pm.T):  # upper triangle given
        Pm = np.triu(Pm) + np.triu(Pm, 1).T
    if equilibrated:
        dat = ipm.Data(prob, ipm.Settings())
        d, e, c = dat.d, dat.e, dat.c
    else:
        d, e, c = np.ones(n), np.ones(m), 1.0
    Pb = c * (d[:, None] * Pm * d[None, :])
    Ab = e[:, None] * A.toarray() * d[None, :]
    Hs = dense_hs(prob.cones, *recentre(prob.cones, e * s, c * z / e, rel))
    K = np.block([[Pb, Ab.T], [Ab, -Hs]])
    uv = np.linalg.solve(K, np.concatenate([d * gx, np.zeros(m)]))
    u, v = c * d * uv[:n], e * uv[n:]
    rows = A.indices
    cols = np.repeat(np.arange(n), np.diff(A.indptr))
    dA = sp.csc_matrix((-(z[rows] * u[cols] + v[rows] * x[cols]), A.indices, A.indptr), shape=A.shape)
    return -u, v, dA
