"""CPU oracle, part 2: exact-diagonalisation stages (test infrastructure only).

Restates, in numpy FP64, the reference's
  * HamiltonianPart::prepareImpl / computeImpl (HamiltonianPart.cpp:56-102):
    dense block matrix, eigenvalues ascending, eigenvectors as columns.  The
    reference calls Eigen::SelfAdjointEigenSolver (Householder
    tridiagonalisation + implicit QR); numpy.linalg.eigh (LAPACK) solves the
    same problem; only the eigenvector gauge may differ, and every observable
    below is gauge invariant;
  * Hamiltonian::computeGroundEnergy (Hamiltonian.cpp:125-130);
  * DensityMatrixPart::computeUnnormalized / normalize / truncate and
    DensityMatrix::compute / truncateBlocks (DensityMatrixPart.cpp:23-50,
    DensityMatrix.cpp:38-92);
  * MonomialOperator::prepare (MonomialOperator.hpp:160-195) and
    MonomialOperatorPart::computeImpl (MonomialOperatorPart.cpp:48-92):
    O' = U_L^dagger (O U_R), O U_R being a signed row gather;
  * MonomialOperatorPart::setFromAdjoint / FieldOperatorContainer::computeAll
    (MonomialOperatorPart.cpp:94-111, FieldOperatorContainer.cpp:22-37).
The rotated matrices are kept dense: Eigen's sparseView(Tolerance) keeps
entries with |x| > Tolerance * 1e-12 (reference times Eigen's default
dummy_precision), i.e. it only drops entries below ~1e-20.
"""
from __future__ import annotations

import numpy as np

from . import model as M


class ED:
    def __init__(self, mdl: M.Model, beta: float):
        self.m = mdl
        self.beta = float(beta)
        self.E, self.U = [], []
        for b in range(len(mdl.blocks)):
            h = mdl.h_block(b)
            if mdl.complex:
                h = h.astype(complex)
            e, u = np.linalg.eigh(h)
            self.E.append(e)
            self.U.append(u)
        self.E0 = min(e.min() for e in self.E)
        raw = [np.exp(-self.beta * (e - self.E0)) for e in self.E]
        self.Z = sum(r.sum() for r in raw)
        self.w = [r / self.Z for r in raw]
        self.retained = [True] * len(self.E)

    def truncate_blocks(self, tol):
        """DensityMatrix::truncateBlocks (DensityMatrix.cpp:77-92)."""
        self.retained = [bool((w > tol).any()) for w in self.w]

    # -- operators -----------------------------------------------------------
    def rotate(self, mono, coef=1.0):
        """Rotated parts of a monomial: {right_block: (left_block, O' dense)}."""
        out = {}
        for R, (L, tgt, sg) in self.m.monomial_parts(mono, coef).items():
            UR, UL = self.U[R], self.U[L]
            G = np.zeros((UL.shape[0], UR.shape[1]), dtype=np.result_type(UR, UL, float))
            ok = tgt >= 0
            np.add.at(G, tgt[ok], sg[ok, None] * UR[ok, :])
            out[R] = (L, UL.conj().T @ G)
        return out

    def cdag(self, ix):
        return self.rotate(((True, self.m.info.tuples[ix]),))

    def c(self, ix):
        """Annihilator from the adjoint of the creator, as computeAll does."""
        return adjoint(self.cdag(ix))

    def quadratic(self, i, j, dag=(True, False)):
        t = self.m.info.tuples
        return self.rotate(((dag[0], t[i]), (dag[1], t[j])))

    def quartic(self, i, j, k, l, dag=(True, True, False, False)):
        t = self.m.info.tuples
        return self.rotate(((dag[0], t[i]), (dag[1], t[j]), (dag[2], t[k]), (dag[3], t[l])))


def adjoint(parts):
    return {L: (R, O.conj().T) for R, (L, O) in parts.items()}


def left_index(parts):
    """left block -> (right block, matrix)."""
    return {L: (R, O) for R, (L, O) in parts.items()}
