"""FP64 reference gradient of a single-particle Green's function with respect
to the coefficients of the Hamiltonian's terms.

Test infrastructure only: the checker of pgx_gf_vjp, never a product path.

The reference computes no derivatives.  The function differentiated is the
forward chain it does compute, restated in numpy:
  block Hamiltonians   H_b = sum_t c_t <b|O_t|b>     (HamiltonianPart.cpp:56-76)
  eigensolve           H_b = U_b diag(E_b) U_b^T     (HamiltonianPart.cpp:90-102)
  weights              w_s = exp(-beta E_s) / Z      (DensityMatrixPart.cpp:23-50)
  rotation             O'_LR = U_L^T O U_R           (MonomialOperatorPart.cpp:48-92)
  Lehmann sum          G(z) = sum_{o,i} A_oi B_io (w_o + w_i) / (z - E_i + E_o)
                                                     (GreensFunctionPart.cpp:65-110)
without the reference's coefficient filter and pole merge (both are
discontinuous in the parameters).  A = <o|c_i|i> is the adjoint of the
rotated c^+_i, as FieldOperatorContainer forms it; B = <i|c^+_j|o>.

The reverse pass follows the chain rule stage by stage: the Lehmann sum
(dL/dA, dL/dB, dL/dw, dL/dE), the normalised weights, the rotation (dL/dU
through the Fock action of c^+), the symmetric eigendecomposition (Giles,
"Collected matrix derivative results for forward and reverse mode
algorithmic differentiation", 2008, sec. 3.1, with the degenerate-pair terms
set to zero: G does not depend on the basis of a degenerate subspace), and
the assembly (dL/dc_t = sum of the symmetrised dL/dH over the term's
matrix elements).
"""
from __future__ import annotations

import numpy as np

from . import ed as EDm
from . import model as M


def _rotated_cdag(m: M.Model, ed: EDm.ED, ix):
    """{right block: (left block, O' = U_L^T C U_R, target rows, signs)} of c^+_ix."""
    out = {}
    for R, (Lb, tgt, sg) in m.monomial_parts(((True, m.info.tuples[ix]),)).items():
        sg = np.real(sg).astype(float)
        ok = tgt >= 0
        C = np.zeros((ed.U[Lb].shape[0], ed.U[R].shape[1]))
        np.add.at(C, tgt[ok], sg[ok, None] * ed.U[R][ok, :])
        out[R] = (Lb, ed.U[Lb].T @ C, tgt, sg)
    return out


def _pairs(cd_i, cd_j):
    """(outer, inner, A = <o|c_i|i>, B = <i|c^+_j|o>, right block of c^+_i's part)."""
    out = []
    for Ri, (Li, Oi, _, _) in sorted(cd_i.items()):
        # c^+_i maps Ri -> Li, so its adjoint c_i has left block Ri (the outer
        # block of G's first operator), right block Li and matrix Oi^T
        o, inner, A = Ri, Li, Oi.T
        if o not in cd_j:
            continue
        Lj, Oj, _, _ = cd_j[o]
        if Lj != inner:
            continue
        out.append((o, inner, A, Oj, Ri))
    return out


def gf_exact(m: M.Model, beta, i, j, z, ed: EDm.ED | None = None):
    """<c_i c^+_j>(z) with every residue kept."""
    ed = ed or EDm.ED(m, beta)
    z = np.asarray(z, dtype=complex)
    G = np.zeros(len(z), dtype=complex)
    for o, inner, A, B, _ in _pairs(_rotated_cdag(m, ed, i), _rotated_cdag(m, ed, j)):
        R = A * B.T * (ed.w[o][:, None] + ed.w[inner][None, :])
        P = ed.E[inner][None, :] - ed.E[o][:, None]
        nz = R != 0.0
        G += (R[nz][None, :] / (z[:, None] - P[nz][None, :])).sum(1)
    return G


def term_coefficients(expr, keys):
    """Real parts of the coefficients of the given monomials in expr."""
    terms = expr.terms
    missing = [k for k in keys if k not in terms]
    if missing or len(terms) != len(keys):
        raise ValueError("the expression's monomials differ from the given keys")
    return np.array([complex(terms[k]).real for k in keys])


def gf_term_gradient(m: M.Model, beta, i, j, z, lam, degeneracy_tol=1e-10):
    """dL/dc_t for every monomial of m.expr (in m.expr.terms order) and dL/dE
    (one array per block), for dL = Re sum_n lam[n] dG(z_n), G = <c_i c^+_j>."""
    if m.complex:
        raise ValueError("real Hamiltonians only")
    z = np.asarray(z, dtype=complex)
    lam = np.asarray(lam, dtype=complex)
    ed = EDm.ED(m, beta)
    nb = len(m.blocks)
    cd_i = _rotated_cdag(m, ed, i)
    cd_j = _rotated_cdag(m, ed, j)
    # ---- Lehmann sum
    gi = {R: np.zeros_like(v[1]) for R, v in cd_i.items()}  # dL/d(c^+_i part)
    gj = {R: np.zeros_like(v[1]) for R, v in cd_j.items()}
    Eb = [np.zeros_like(e) for e in ed.E]
    wb = [np.zeros_like(e) for e in ed.E]
    for o, inner, A, B, Ri in _pairs(cd_i, cd_j):
        s = ed.w[o][:, None] + ed.w[inner][None, :]
        pole = ed.E[inner][None, :] - ed.E[o][:, None]
        Px = np.zeros_like(pole)
        Qx = np.zeros_like(pole)
        for zn, ln in zip(z, lam):
            r = 1.0 / (zn - pole)
            Px += np.real(ln * r)
            Qx += np.real(ln * r * r)
        ab = A * B.T
        gi[Ri] += (B.T * s * Px).T  # A = (c^+_i part)^T
        gj[o] += (A * s * Px).T
        wb[o] += (ab * Px).sum(1)
        wb[inner] += (ab * Px).sum(0)
        de = ab * s * Qx
        Eb[inner] += de.sum(0)
        Eb[o] -= de.sum(1)
    # ---- normalised weights
    S = sum(float(w @ g) for w, g in zip(ed.w, wb))
    for b in range(nb):
        Eb[b] += -beta * ed.w[b] * (wb[b] - S)
    # ---- rotation O' = U_L^T C U_R with C[t_k, k] = s_k
    Ub = [np.zeros_like(u) for u in ed.U]
    for parts, grads in ((cd_i, gi), (cd_j, gj)):
        for R, (Lb, _, tgt, sg) in parts.items():
            Ob = grads[R]
            ok = tgt >= 0
            k = np.nonzero(ok)[0]
            t = tgt[ok]
            np.add.at(Ub[Lb], t, sg[ok, None] * (ed.U[R] @ Ob.T)[k])
            np.add.at(Ub[R], k, sg[ok, None] * (ed.U[Lb] @ Ob)[t])
    # ---- eigendecomposition
    emax = max(1.0, max(float(np.abs(e).max()) for e in ed.E))
    Hb = []
    for b in range(nb):
        U, E = ed.U[b], ed.E[b]
        gap = E[None, :] - E[:, None]
        keep = np.abs(gap) > degeneracy_tol * emax
        F = np.where(keep, 1.0 / np.where(keep, gap, 1.0), 0.0)
        X = F * (U.T @ Ub[b]) + np.diag(Eb[b])
        H = U @ X @ U.T
        Hb.append(0.5 * (H + H.T))
    # ---- assembly
    keys = list(m.expr.terms)
    dterm = np.zeros(len(keys))
    for t, key in enumerate(keys):
        for R, (Lb, tgt, sg) in m.monomial_parts(key).items():
            if Lb != R:
                raise ValueError("a Hamiltonian term connects different blocks")
            ok = tgt >= 0
            k = np.nonzero(ok)[0]
            dterm[t] += float((np.real(sg)[ok] * Hb[R][tgt[ok], k]).sum())
    return dterm, Eb
