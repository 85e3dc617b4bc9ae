"""CPU oracle, part 4: three-point fermion-boson susceptibility (test
infrastructure).

Reference lines restated:
  ThreePointSusceptibility::getF1/F2/B1/B2   ThreePointSusceptibility.cpp:37-66
  ThreePointSusceptibility::prepare          ThreePointSusceptibility.cpp:68-142
  ThreePointSusceptibilityPart::computeImpl  ThreePointSusceptibilityPart.cpp:243-296
  ThreePointSusceptibilityPart::addMultiterm ThreePointSusceptibilityPart.cpp:298-342
  term evaluation                            ThreePointSusceptibilityPart.hpp:516-538
  term merges (weight-averaged poles)        ThreePointSusceptibilityPart.cpp:34-43, 85-95, 141-149
  Channel enum (PP, PH, xPH = 0, 1, 2)        Misc.hpp:160-164

Two modes:
  * chi3_direct: the reference's term lists (coefficient filter, pole merge)
    evaluated term by term, for small blocks;
  * chi3_exact: every state triple, no filter or merge, factorised over
    matrix products.  The resonance rules (|E_i - E_k| <= PoleResolution for
    the term type, |z1 - xi z2| <= PoleResolution for the resonant delta) are
    kept in both.
"""
from __future__ import annotations

import numpy as np

from .ed import ED, left_index
from .lehmann import TermList

PP, PH, XPH = 0, 1, 2


def channel_ops(channel, CX1, C2, CX3, C4):
    """(F1, F2, B1, B2) of a channel (ThreePointSusceptibility.cpp:37-66)."""
    if channel == PP:
        return CX1, CX3, C2, C4
    if channel == PH:
        return CX1, C2, CX3, C4
    if channel == XPH:
        return CX1, C4, CX3, C2
    raise ValueError("bad channel")


def chi3_parts(ed: ED, channel, CX1, C2, CX3, C4):
    """Block triples of ThreePointSusceptibility::prepare.  Operators are
    dicts right_block -> (left_block, matrix).  Each part: blocks (i, j, k)
    = (B2 right, middle, B1 left), the matrices <i|F|j>, <j|F'|k>,
    B = <k|B1 B2|i>, and the swapped flag."""
    F1, F2, B1, B2 = channel_ops(channel, CX1, C2, CX3, C4)
    F1L, F2L, B1L = left_index(F1), left_index(F2), left_index(B1)
    parts = []
    for b2r in sorted(B2):
        b2l, MB2 = B2[b2r]
        if b2l not in B1:
            continue
        b1l, MB1 = B1[b2l]
        B = MB1 @ MB2  # <b1l|B1|b2l><b2l|B2|b2r>
        # F1, F2, B: <b2r|F1|F1right><F2left|F2|b1l>
        if b2r in F1L and b1l in F2:
            f1r, MF1 = F1L[b2r]
            f2l, MF2 = F2[b1l]
            if f1r == f2l and ed.retained[b2r] and ed.retained[f1r] and ed.retained[b1l]:
                parts.append(dict(b=(b2r, f1r, b1l), F1=MF1, F2=MF2, B=B, swapped=False))
        # F2, F1, B: <b2r|F2|F2right><F1left|F1|b1l>
        if b2r in F2L and b1l in F1:
            f2r, MF2 = F2L[b2r]
            f1l, MF1 = F1[b1l]
            if f2r == f1l and ed.retained[b2r] and ed.retained[f2r] and ed.retained[b1l]:
                parts.append(dict(b=(b2r, f2r, b1l), F1=MF2, F2=MF1, B=B, swapped=True))
    return parts


def _signs(channel, swapped):
    pf = 1.0 if ((channel == PH) == swapped) else -1.0
    spp = -1.0 if channel == PP else 1.0     # sign of the fermion-fermion coefficient
    sig = 1.0 if channel == PP else -1.0     # sign of its second pole
    xi = -1 if channel == PP else 1
    return pf, spp, sig, xi


def chi3_part_terms(ed: ED, p, channel, res=1e-8, tol=1e-16):
    """The three term lists of one part (computeImpl + addMultiterm)."""
    i_, j_, k_ = p["b"]
    Ei, Ej, Ek = ed.E[i_], ed.E[j_], ed.E[k_]
    wi, wj, wk = ed.w[i_], ed.w[j_], ed.w[k_]
    F1, F2, B = p["F1"], p["F2"], p["B"]
    S = p["swapped"]
    pf, spp, sig, xi = _signs(channel, S)
    beta = ed.beta
    ff = TermList(res, tol, 2, True)
    fb = TermList(res, tol, 2, True)
    rs = TermList(res, tol, 1, True)
    for i in range(F1.shape[0]):
        for j in np.nonzero(F1[i])[0]:
            for k in np.nonzero(F2[j] * B[:, i])[0]:
                C = pf * F1[i, j] * F2[j, k] * B[k, i]
                Eij, Ejk, Eik = Ei[i] - Ej[j], Ej[j] - Ek[k], Ei[i] - Ek[k]
                c = C * (wi[i] + wj[j])
                if abs(c) > tol:
                    ff.add(0, (spp * c,), ((Ejk, Eij * sig) if S else (Eij, Ejk * sig)))
                if abs(Eik) <= res:
                    c = -C * beta * wi[i]
                    if abs(c) > tol:
                        rs.add(xi, (-c if S else c,), ((Ejk if S else -Ejk),))
                else:
                    c = C * (wk[k] - wi[i])
                    if abs(c) > tol:
                        fb.add(xi, (-c if S else c,), ((Ejk if S else Eij), Eik))
                        if not S:
                            ff.add(0, (spp * c,), (Eij, sig * Ejk))
    return ff, fb, rs


def chi3_direct(ed: ED, parts, channel, freqs, res=1e-8, tol=1e-16):
    """chi3 at (z1, z2) duplets from the reference's term lists."""
    out = np.zeros(len(freqs), dtype=complex)
    for p in parts:
        ff, fb, rs = chi3_part_terms(ed, p, channel, res, tol)
        for n, (z1, z2) in enumerate(freqs):
            v = 0j
            for c, (P0, P1), _ in ff.d.values():
                v += c[0] / ((z1 - P0) * (z2 - P1))
            for key, (c, (P1, P12), _) in fb.d.items():
                v += c[0] / ((z1 - P1) * (z1 - key[0] * z2 - P12))
            for key, (c, (P,), _) in rs.d.items():
                if abs(z1 - key[0] * z2) <= res:
                    v += c[0] / (z1 - P)
            out[n] += v
    return out


def chi3_part_exact(ed: ED, p, channel, z1, z2, res=1e-8):
    """One part at one duplet, every state triple, factorised."""
    i_, j_, k_ = p["b"]
    Ei, Ej, Ek = ed.E[i_], ed.E[j_], ed.E[k_]
    wi, wj, wk = ed.w[i_], ed.w[j_], ed.w[k_]
    F1, F2, B = p["F1"], p["F2"], p["B"]
    S = p["swapped"]
    pf, spp, sig, xi = _signs(channel, S)
    Eij = Ei[:, None] - Ej[None, :]
    Ejk = Ej[:, None] - Ek[None, :]
    Eik = Ei[:, None] - Ek[None, :]
    nonres = np.abs(Eik) > res                       # (i, k)
    Om = z1 - xi * z2
    # (w_k - w_i) / (Om - E_ik) on the non-resonant (k, i) pairs, zero elsewhere
    den = np.where(nonres.T, Om - Eik.T, 1.0)
    FBk = np.where(nonres.T, B * (wk[:, None] - wi[None, :]) / den, 0.0)
    if not S:
        D1 = F1 / (z1 - Eij)
        D2 = F2 / (z2 - sig * Ejk)
        # weights w_i + w_j + [nonres](w_k - w_i) = (nonres ? w_k : w_i) + w_j
        Wik = np.where(nonres, wk[None, :], wi[:, None])    # (i, k)
        ff = (np.einsum("ki,ij,jk->", B * Wik.T, D1, D2) + np.einsum("ki,ij,j,jk->", B, D1, wj, D2))
        fb = np.einsum("ki,ij,jk->", FBk, D1, F2)
        v = spp * pf * ff + pf * fb
        if abs(Om) <= res:
            v += -ed.beta * pf * np.einsum("ki,ij,jk->", np.where(nonres.T, 0.0, B * wi[None, :]), F1,
                                           F2 / (z1 + Ejk))
    else:
        D1 = F1 / (z2 - sig * Eij)
        D2 = F2 / (z1 - Ejk)
        ff = np.einsum("ki,i,ij,jk->", B, wi, D1, D2) + np.einsum("ki,ij,j,jk->", B, D1, wj, D2)
        fb = np.einsum("ki,ij,jk->", FBk, F1, D2)
        v = spp * pf * ff - pf * fb
        if abs(Om) <= res:
            v += ed.beta * pf * np.einsum("ki,ij,jk->", np.where(nonres.T, 0.0, B * wi[None, :]), F1, D2)
    return v


def chi3_exact(ed: ED, parts, channel, freqs, res=1e-8):
    out = np.zeros(len(freqs), dtype=complex)
    for p in parts:
        for n, (z1, z2) in enumerate(freqs):
            out[n] += chi3_part_exact(ed, p, channel, z1, z2, res)
    return out
