"""CPU oracle, part 3: Lehmann sums for G, chi, <A> and G2 (test infrastructure).

Two modes everywhere:
  * "reference rule": the reference's truncations, merges and filters;
  * "exact": no dropping, no merging (the resonant delta rule is physics and
    is kept in both modes, with PoleResolution as its tolerance).

Reference lines restated:
  GreensFunction::prepare          GreensFunction.cpp:41-86
  GreensFunctionPart::computeImpl  GreensFunctionPart.cpp:65-110, Term :24-32
  Susceptibility::prepare          Susceptibility.cpp:42-92
  SusceptibilityPart::computeImpl  SusceptibilityPart.cpp:76-127, operator() .hpp:212-220
  Susceptibility::operator()       Susceptibility.hpp:143-158
  EnsembleAverage::compute         EnsembleAverage.cpp:27-67
  TermList::add_term               TermList.hpp:65-76
  TwoParticleGF::prepare           TwoParticleGF.cpp:67-120
  TwoParticleGFPart::computeImpl   TwoParticleGFPart.cpp:189-265, addMultiterm :267-298
  TwoParticleGFPart::operator()    TwoParticleGFPart.cpp:300-322, terms .hpp:475-495
  permutations3                    Misc.cpp:41-42
  IndexContainer4 symmetry         IndexContainer4.hpp:138-149, 190-237; permutations4 Misc.cpp:61-66
"""
from __future__ import annotations

import numpy as np

from .ed import ED, left_index

PERMUTATIONS3 = [((0, 1, 2), 1), ((0, 2, 1), -1), ((1, 0, 2), -1),
                 ((1, 2, 0), 1), ((2, 0, 1), 1), ((2, 1, 0), -1)]
PERMUTATIONS4 = [((0, 1, 2, 3), 1), ((0, 1, 3, 2), -1), ((0, 2, 1, 3), -1), ((0, 2, 3, 1), 1),
                 ((0, 3, 1, 2), 1), ((0, 3, 2, 1), -1), ((1, 0, 2, 3), -1), ((1, 0, 3, 2), 1),
                 ((1, 2, 0, 3), 1), ((1, 2, 3, 0), -1), ((1, 3, 0, 2), -1), ((1, 3, 2, 0), 1),
                 ((2, 0, 1, 3), 1), ((2, 0, 3, 1), -1), ((2, 1, 0, 3), -1), ((2, 1, 3, 0), 1),
                 ((2, 3, 0, 1), 1), ((2, 3, 1, 0), -1), ((3, 0, 1, 2), -1), ((3, 0, 2, 1), 1),
                 ((3, 1, 0, 2), 1), ((3, 1, 2, 0), -1), ((3, 2, 0, 1), -1), ((3, 2, 1, 0), 1)]


def fermionic(n, beta):
    return 1j * np.pi * (2 * np.asarray(n) + 1) / beta


def bosonic(n, beta):
    return 1j * np.pi * (2 * np.asarray(n)) / beta


class TermList:
    """Merging term list (TermList.hpp:65-76) keyed by binned poles.

    libstdc++ caches hash codes for this hasher, so a lookup only matches a
    stored term whose binned-pole tuple is identical; the KeyEqual test is then
    implied.  `average` selects the G2 merge (poles weight-averaged,
    TwoParticleGFPart.cpp:35-43) instead of the G/chi merge (first pole kept).
    """

    def __init__(self, res, tol, npoles, average):
        self.res, self.tol, self.np, self.avg = res, tol, npoles, average
        self.d = {}

    def key(self, flag, poles):
        return (flag,) + tuple(int(np.round(p / self.res)) for p in poles)

    def add(self, flag, coeffs, poles):
        k = self.key(flag, poles)
        t = self.d.get(k)
        if t is None:
            self.d[k] = [list(coeffs), list(poles), 1]
            return
        del self.d[k]
        c = [a + b for a, b in zip(t[0], coeffs)]
        if self.avg:
            wsum = t[2] + 1
            p = [(t[2] * a + b) / wsum for a, b in zip(t[1], poles)]
        else:
            wsum, p = t[2] + 1, t[1]
        if all(abs(x) <= self.tol / (len(self.d) + 1) for x in c):
            return
        self.d[self.key(flag, p)] = [c, p, wsum]


# ---------------------------------------------------------------------------
# Single-particle Green's function and susceptibility
# ---------------------------------------------------------------------------
def _pair_parts(ed: ED, F1, F2):
    """Matching blocks of F1 (left=outer) and F2 (right=outer)."""
    F1L = left_index(F1)
    out = []
    # F2 is keyed by its right block: the F2 part needed has right == outer
    # and left == inner.
    for outer in sorted(F1L):
        inner, A = F1L[outer]
        if outer not in F2:
            continue
        L2, B = F2[outer]
        if L2 != inner:
            continue
        if not (ed.retained[outer] or ed.retained[inner]):
            continue
        out.append((outer, inner, A, B))
    return out


def gf_terms(ed: ED, F1, F2, res=1e-8, tol=1e-8, rule=True):
    """Residues and poles of G (GreensFunctionPart.cpp:65-110)."""
    R_all, P_all = [], []
    tl = TermList(res, tol, 1, False) if rule else None
    for outer, inner, A, B in _pair_parts(ed, F1, F2):
        wo, wi = ed.w[outer], ed.w[inner]
        R = A * B.T * (wo[:, None] + wi[None, :])
        P = ed.E[inner][None, :] - ed.E[outer][:, None]
        if rule:
            for i1 in range(R.shape[0]):
                for i2 in range(R.shape[1]):
                    if abs(R[i1, i2]) > tol:
                        tl.add(0, (R[i1, i2],), (P[i1, i2],))
        else:
            R_all.append(R.ravel()); P_all.append(P.ravel())
    if rule:
        vals = list(tl.d.values())
        return (np.array([v[0][0] for v in vals], dtype=complex),
                np.array([v[1][0] for v in vals], dtype=float))
    if not R_all:
        return np.zeros(0, complex), np.zeros(0)
    return np.concatenate(R_all).astype(complex), np.concatenate(P_all)


def gf_eval(terms, z):
    R, P = terms
    z = np.atleast_1d(z)
    return (R[None, :] / (z[:, None] - P[None, :])).sum(1)


def susc_terms(ed: ED, A, B, res=1e-8, tol=1e-8, rule=True):
    """Susceptibility terms and zero-pole weight (SusceptibilityPart.cpp:76-127)."""
    zero = 0.0
    R_all, P_all = [], []
    tl = TermList(res, tol, 1, False) if rule else None
    for outer, inner, Ao, Bo in _pair_parts(ed, A, B):
        wo, wi = ed.w[outer], ed.w[inner]
        AB = Ao * Bo.T
        P = ed.E[inner][None, :] - ed.E[outer][:, None]
        zp = np.abs(P) < res
        zero += (AB * wo[:, None])[zp].sum()
        R = AB * (wo[:, None] - wi[None, :])
        if rule:
            for i1 in range(R.shape[0]):
                for i2 in range(R.shape[1]):
                    if not zp[i1, i2] and abs(R[i1, i2]) > tol:
                        tl.add(0, (R[i1, i2],), (P[i1, i2],))
        else:
            R_all.append(R[~zp]); P_all.append(P[~zp])
    if rule:
        vals = list(tl.d.values())
        return (np.array([v[0][0] for v in vals], dtype=complex),
                np.array([v[1][0] for v in vals], dtype=float), zero)
    if not R_all:
        return np.zeros(0, complex), np.zeros(0), zero
    return np.concatenate(R_all).astype(complex), np.concatenate(P_all), zero


def susc_eval(terms, z, beta, ave_a=None, ave_b=None):
    R, P, zero = terms
    z = np.atleast_1d(z).astype(complex)
    v = (-R[None, :] / (z[:, None] - P[None, :])).sum(1)
    at0 = np.abs(z) <= np.finfo(float).eps
    v = v + np.where(at0, zero * beta, 0)
    if ave_a is not None:
        v = v - np.where(at0, ave_a * ave_b * beta, 0)
    return v


def ensemble_average(ed: ED, A):
    """<A> over diagonal retained blocks (EnsembleAverage.cpp:27-67)."""
    r = 0.0
    for R, (L, O) in A.items():
        if L == R and ed.retained[L]:
            r += (np.diag(O) * ed.w[L]).sum()
    return r


# ---------------------------------------------------------------------------
# Two-particle Green's function
# ---------------------------------------------------------------------------
def g2_parts(ed: ED, C1, C2, CX3, CX4):
    """Block chains of TwoParticleGF::prepare (TwoParticleGF.cpp:67-120).

    Returns a list of dicts with blocks b1..b4, matrices O1, O2, O3, CX4,
    permutation and sign.  Operators are dicts right_block -> (left, O).
    """
    ops = [C1, C2, CX3]
    lefts = [left_index(o) for o in ops]
    parts = []
    for S1 in sorted(CX4):                       # CX4 right block, ascending
        S4, X4 = CX4[S1]
        for perm, sign in PERMUTATIONS3:
            o0, o1, o2 = perm
            if S1 not in lefts[o0]:
                continue
            S2, O1 = lefts[o0][S1]                # <S1|O1|S2>
            # S3 = left block of operator at position 2 with right block S4
            if S4 not in ops[o2]:
                continue
            S3, O3 = ops[o2][S4]                  # <S3|O3|S4>
            if S2 not in lefts[o1] or lefts[o1][S2][0] != S3:
                continue
            O2 = lefts[o1][S2][1]                 # <S2|O2|S3>
            if not any(ed.retained[b] for b in (S1, S2, S3, S4)):
                continue
            parts.append(dict(b=(S1, S2, S3, S4), O1=O1, O2=O2, O3=O3, CX4=X4,
                              perm=perm, sign=sign))
    return parts


def permute_freqs(perm, z1, z2, z3):
    F = (z1, z2, -z3)
    return F[perm[0]], F[perm[1]], F[perm[2]]


def g2_part_exact(ed: ED, p, z1, z2, z3, res):
    """Exact Lehmann sum of one part at one (already permuted) triple,
    factorised over matrix products (gauge invariant, no dropping)."""
    S1, S2, S3, S4 = p["b"]
    E1, E2, E3, E4 = (ed.E[b] for b in p["b"])
    w1, w2, w3, w4 = (ed.w[b] for b in p["b"])
    O1, O2, O3, X4 = p["O1"], p["O2"], p["O3"], p["CX4"]
    beta = ed.beta
    A = O1 / (z1 - (E2[None, :] - E1[:, None]))
    B = O2 / (z2 - (E3[None, :] - E2[:, None]))
    C = O3 / (z3 - (E4[None, :] - E3[:, None]))
    t1 = -np.trace(X4 @ A @ (w2[:, None] * B + B * w3[None, :]) @ C)
    Zs = z1 + z2 + z3
    D = X4 * (w1[None, :] + w4[:, None]) / (Zs - (E4[:, None] - E1[None, :]))
    t2 = np.sum(D.T * (A @ O2 @ C))
    s12 = z1 + z2
    d13 = s12 - (E3[None, :] - E1[:, None])
    delta13 = np.abs(d13) <= res
    F13 = np.where(delta13, beta * w1[:, None],
                   (w3[None, :] - w1[:, None]) / np.where(delta13, 1.0, d13))
    t3 = np.sum((A @ O2) * (C @ X4).T * F13)
    s23 = z2 + z3
    d24 = s23 - (E4[None, :] - E2[:, None])
    delta24 = np.abs(d24) <= res
    F24 = np.where(delta24, -beta * w2[:, None],
                   (w2[:, None] - w4[None, :]) / np.where(delta24, 1.0, d24))
    t4 = np.sum((O2 @ C) * (X4 @ A).T * F24)
    return p["sign"] * (t1 + t2 + t3 + t4)


def g2_exact(ed: ED, parts, freqs, res=1e-8):
    """G2 at a list of (z1, z2, z3) triples, exact mode."""
    out = np.zeros(len(freqs), dtype=complex)
    for p in parts:
        for k, (a, b, c) in enumerate(freqs):
            z1, z2, z3 = permute_freqs(p["perm"], a, b, c)
            out[k] += g2_part_exact(ed, p, z1, z2, z3, res)
    return out


def g2_part_direct(ed: ED, p, freqs, res, tol, rule):
    """Quadruple-by-quadruple evaluation (TwoParticleGFPart.cpp:189-298 and
    .hpp:475-495) for small blocks; rule=True applies the weight and
    coefficient filters (merging changes values only at PoleResolution scale
    and is left to the C++ oracle)."""
    E1, E2, E3, E4 = (ed.E[b] for b in p["b"])
    w1, w2, w3, w4 = (ed.w[b] for b in p["b"])
    M = p["sign"] * np.einsum("ab,bc,cd,da->abcd", p["O1"], p["O2"], p["O3"], p["CX4"])
    P1 = E2[None, :, None, None] - E1[:, None, None, None]
    P2 = E3[None, None, :, None] - E2[None, :, None, None]
    P3 = E4[None, None, None, :] - E3[None, None, :, None]
    W1 = w1[:, None, None, None]; W2 = w2[None, :, None, None]
    W3 = w3[None, None, :, None]; W4 = w4[None, None, None, :]
    keep = np.ones(M.shape, bool)
    if rule:
        keep = (W1 + W2 + W3 + W4 > tol) & (np.abs(M) > 0)
    cz2 = -M * (W2 + W3)
    cz4 = M * (W1 + W4)
    r12, n12 = M * beta_(ed) * W1, M * (W3 - W1)
    r23, n23 = -M * beta_(ed) * W2, M * (W2 - W4)
    if rule:
        k2 = keep & (np.abs(cz2) > tol)
        k4 = keep & (np.abs(cz4) > tol)
        k12 = keep & ((np.abs(r12) > tol) | (np.abs(n12) > tol))
        k23 = keep & ((np.abs(r23) > tol) | (np.abs(n23) > tol))
    else:
        k2 = k4 = k12 = k23 = keep
    out = np.zeros(len(freqs), dtype=complex)
    for k, (a, b, c) in enumerate(freqs):
        z1, z2, z3 = permute_freqs(p["perm"], a, b, c)
        d1, d3 = z1 - P1, z3 - P3
        v = np.where(k2, cz2 / (d1 * (z2 - P2) * d3), 0).sum()
        v += np.where(k4, cz4 / (d1 * (z1 + z2 + z3 - P1 - P2 - P3) * d3), 0).sum()
        D = z1 + z2 - P1 - P2
        dl = np.abs(D) <= res
        v += np.where(k12, np.where(dl, r12, n12 / np.where(dl, 1, D)) / (d1 * d3), 0).sum()
        D = z2 + z3 - P2 - P3
        dl = np.abs(D) <= res
        v += np.where(k23, np.where(dl, r23, n23 / np.where(dl, 1, D)) / (d1 * d3), 0).sum()
        out[k] = v
    return out


def beta_(ed):
    return ed.beta


def g2_direct(ed: ED, parts, freqs, res=1e-8, tol=1e-16, rule=True):
    out = np.zeros(len(freqs), dtype=complex)
    for p in parts:
        out += g2_part_direct(ed, p, freqs, res, tol, rule)
    return out


def container_perm_value(perm4, sign, f, n1, n2, n3):
    """ElementWithPermFreq::operator() (IndexContainer4.hpp:138-149): f(n1,n2,n3)
    of the stored element evaluated at permuted Matsubara indices."""
    ns = (n1, n2, n3, n1 + n2 - n3)
    return f(ns[perm4[0]], ns[perm4[1]], ns[perm4[2]]) * sign
