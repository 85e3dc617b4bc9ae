"""CPU oracle, part 5: the G2 Lehmann sum by weight anchors (test
infrastructure only; never imported by the product).

For models whose blocks hold thousands of states (the 8-site ring: 65536
states, blocks up to 4900) the quadruple enumeration of the reference
(TwoParticleGFPart.cpp:189-265) and the full-matrix factorisation of
lehmann.g2_part_exact (O(d^3) per triple) are out of reach on a CPU.  This
module evaluates the same sum at a SAMPLE of frequency triples in
O(d^2 r) per (z1, z3) pair, r being the number of states whose Boltzmann
weight exceeds `anchor_tol`.

Derivation (own restatement of TwoParticleGFPart.cpp:267-298 and
TwoParticleGFPart.hpp:475-495).  For a quadruple (1,2,3,4) of one part with
M = sign O1_12 O2_23 O3_34 CX4_41 and permuted frequencies (a, b, c), the
four terms of addMultiterm share the factor A_12 C_34 with
A = O1 / (a - (E2 - E1)) and C = O3 / (c - (E4 - E3)):
  NR(z2):   -(w2 + w3)  / (b - (E3 - E2))
  NR(z4):    (w1 + w4)  / (a + b + c - (E4 - E1))
  Res(z1z2): |D| <= res ? beta w1 : (w3 - w1) / D,  D = a + b - (E3 - E1)
  Res(z2z3): |D| <= res ? -beta w2 : (w2 - w4) / D, D = b + c - (E4 - E2)
Every weight sum splits into single weights, and a term carrying w_h of one
index h needs only the states of h's block with w_h > anchor_tol ("anchors";
anchor_tol = 0 keeps every state and the sum is exact).  Per (a, c) the
matrix chains are formed with the anchored index as a column or row slice:
  G = C CX4 A   (S3 x S2)   for NR(z2):  G[:, H2] and G[H3, :]
  Y = A O2 C    (S1 x S4)   for NR(z4):  Y[H1, :] and Y[:, H4]
  P = A O2, Q = C CX4       for Res(z1z2): P[H1, :] Q[:, H1], P[:, H3] Q[H3, :]
  R = O2 C, L = CX4 A       for Res(z2z3): R[H2, :] L[:, H2], R[:, H4] L[H4, :]
and the z2-dependent kernels contract them per triple.  Everything is numpy
FP64 (complex128), with BLAS products.
"""
from __future__ import annotations

import numpy as np

from .lehmann import permute_freqs


def _anchors(w, tol):
    return np.nonzero(w > tol)[0]


def _mm(X, Y):
    """X @ Y with a real factor kept real (two real products instead of one
    complex product of twice the work)."""
    if np.iscomplexobj(X) and not np.iscomplexobj(Y):
        return (X.real @ Y) + 1j * (X.imag @ Y)
    if np.iscomplexobj(Y) and not np.iscomplexobj(X):
        return (X @ Y.real) + 1j * (X @ Y.imag)
    return X @ Y


def _part_pairs(p, freqs):
    """Triples of `freqs` grouped by the part's permuted (a, c):
    {(a, c): [(triple index, b), ...]} in order of first appearance."""
    groups = {}
    for t, (z1, z2, z3) in enumerate(freqs):
        a, b, c = permute_freqs(p["perm"], z1, z2, z3)
        groups.setdefault((a, c), []).append((t, b))
    return groups


def g2_part_anchored(ed, p, freqs, res=1e-8, anchor_tol=0.0):
    """One part at the triples `freqs` ((z1, z2, z3) before the part's
    permutation).  Returns complex values aligned with freqs."""
    E1, E2, E3, E4 = (ed.E[x] for x in p["b"])
    w1, w2, w3, w4 = (ed.w[x] for x in p["b"])
    O1, O2, O3, X4 = p["O1"], p["O2"], p["O3"], p["CX4"]
    H1, H2, H3, H4 = (_anchors(w, anchor_tol) for w in (w1, w2, w3, w4))
    beta, sg = ed.beta, p["sign"]
    out = np.zeros(len(freqs), dtype=complex)
    groups = _part_pairs(p, freqs)
    by_a = {}
    for (a, c), items in groups.items():
        by_a.setdefault(a, []).append((c, items))
    # c-only pieces, formed once per distinct c
    cache_c = {}

    def c_pieces(c):
        if c not in cache_c:
            C = O3 / (c - (E4[None, :] - E3[:, None]))
            cache_c[c] = dict(
                C=C,
                Q_H1=_mm(C, X4[:, H1]),            # Q[:, H1]       d3 x r1
                Q_H3=_mm(C[H3, :], X4),            # Q[H3, :]       r3 x d1
                R_H4=_mm(O2, C[:, H4]),            # R[:, H4]       d2 x r4
                R_H2=_mm(O2[H2, :], C),            # R[H2, :]       r2 x d4
            )
        return cache_c[c]

    for a, lst in by_a.items():
        A = O1 / (a - (E2[None, :] - E1[:, None]))
        L_H2 = _mm(X4, A[:, H2])                   # L[:, H2]       d4 x r2
        L_H4 = _mm(X4[H4, :], A)                   # L[H4, :]       r4 x d2
        P_H1 = _mm(A[H1, :], O2)                   # P[H1, :]       r1 x d3
        P_H3 = _mm(A, O2[:, H3])                   # P[:, H3]       d1 x r3
        for c, items in lst:
            cp = c_pieces(c)
            C = cp["C"]
            G_H2 = C @ L_H2                    # G[:, H2]       d3 x r2
            G_H3 = cp["Q_H3"] @ A              # G[H3, :]       r3 x d2
            Y_H1 = P_H1 @ C                    # Y[H1, :]       r1 x d4
            Y_H4 = A @ cp["R_H4"]              # Y[:, H4]       d1 x r4
            for t, b in items:
                Zs = a + b + c
                v = 0.0j
                # NR(z2), weight w2 (anchor h in S2, summed index 3) and w3 (h in S3, index 2)
                if len(H2):
                    K = w2[H2][:, None] / (b - (E3[None, :] - E2[H2][:, None]))        # r2 x d3
                    v -= np.sum(K * O2[H2, :] * G_H2.T)
                if len(H3):
                    K = w3[H3][:, None] / (b - (E3[H3][:, None] - E2[None, :]))        # r3 x d2
                    v -= np.sum(K * O2[:, H3].T * G_H3)
                # NR(z4), weight w1 (h in S1, index 4) and w4 (h in S4, index 1)
                if len(H1):
                    K = w1[H1][:, None] / (Zs - (E4[None, :] - E1[H1][:, None]))       # r1 x d4
                    v += np.sum(K * Y_H1 * X4[:, H1].T)
                if len(H4):
                    K = w4[H4][:, None] / (Zs - (E4[H4][:, None] - E1[None, :]))       # r4 x d1
                    v += np.sum(K * Y_H4.T * X4[H4, :])
                # Res(z1z2): w1 (h in S1, index 3) and w3 (h in S3, index 1)
                s = a + b
                if len(H1):
                    D = s - (E3[None, :] - E1[H1][:, None])                             # r1 x d3
                    dl = np.abs(D) <= res
                    F = np.where(dl, beta * w1[H1][:, None], -w1[H1][:, None] / np.where(dl, 1.0, D))
                    v += np.sum(P_H1 * cp["Q_H1"].T * F)
                if len(H3):
                    D = s - (E3[H3][:, None] - E1[None, :])                             # r3 x d1
                    dl = np.abs(D) <= res
                    F = np.where(dl, 0.0, w3[H3][:, None] / np.where(dl, 1.0, D))
                    v += np.sum(P_H3.T * cp["Q_H3"] * F)
                # Res(z2z3): w2 (h in S2, index 4) and w4 (h in S4, index 2)
                s = b + c
                if len(H2):
                    D = s - (E4[None, :] - E2[H2][:, None])                             # r2 x d4
                    dl = np.abs(D) <= res
                    F = np.where(dl, -beta * w2[H2][:, None], w2[H2][:, None] / np.where(dl, 1.0, D))
                    v += np.sum(cp["R_H2"] * L_H2.T * F)
                if len(H4):
                    D = s - (E4[H4][:, None] - E2[None, :])                             # r4 x d2
                    dl = np.abs(D) <= res
                    F = np.where(dl, 0.0, -w4[H4][:, None] / np.where(dl, 1.0, D))
                    v += np.sum(cp["R_H4"].T * L_H4 * F)
                out[t] += sg * v
    return out


def g2_anchored(ed, parts, freqs, res=1e-8, anchor_tol=0.0):
    """Sum over parts at the triples `freqs` (list of (z1, z2, z3))."""
    freqs = [tuple(f) for f in freqs]
    out = np.zeros(len(freqs), dtype=complex)
    for p in parts:
        out += g2_part_anchored(ed, p, freqs, res, anchor_tol)
    return out
