"""Drive libpgx's C ABI from an oracle-built model (test helper).

The oracle model only supplies inputs (block Hamiltonians, Fock actions of
c^+); everything computed here runs on the GPU through the C ABI and is
compared with the oracle by the tests.
"""
import numpy as np

from oracle import lehmann as L
from pomerol_b200.pgx import Engine


class GpuED:
    def __init__(self, mdl, beta, device=0):
        self.m = mdl
        self.beta = beta
        self.eng = Engine(device)
        self.eng.set_blocks(mdl.block_sizes(), mdl.complex)
        self.eng.set_hamiltonian([mdl.h_block(b) for b in range(len(mdl.blocks))])
        self.eng.eigh()
        self.E, self.U = self.eng.eigensystem()
        self.w, self.Z = self.eng.weights(beta)
        self.retained = np.ones(len(mdl.blocks), dtype=bool)
        self._cdag, self._c = {}, {}

    def truncate(self, tol):
        self.retained = self.eng.truncate_blocks(tol)

    def op_from_monomial(self, mono):
        parts = []
        for R, (Lb, tgt, sg) in sorted(self.m.monomial_parts(mono).items()):
            parts.append((R, Lb, tgt.astype(np.int32), np.real(sg).astype(np.float64)))
        op = self.eng.op_define(parts)
        self.eng.op_rotate(op)
        return op

    def cdag(self, ix):
        if ix not in self._cdag:
            self._cdag[ix] = self.op_from_monomial(((True, self.m.info.tuples[ix]),))
        return self._cdag[ix]

    def c(self, ix):
        if ix not in self._c:
            self._c[ix] = self.eng.op_adjoint(self.cdag(ix))
        return self._c[ix]

    def quadratic(self, i, j):
        t = self.m.info.tuples
        return self.op_from_monomial(((True, t[i]), (False, t[j])))

    def maps(self, op):
        """right -> left and left -> right block maps of an operator."""
        info = self.eng.op_info(op)
        return {r: l for r, l in info}, {l: r for r, l in info}

    def pair_parts(self, op1, op2):
        """GreensFunction::prepare / Susceptibility::prepare matching."""
        r1, l1 = self.maps(op1)
        r2, _ = self.maps(op2)
        outer, inner = [], []
        for o in sorted(l1):
            i = l1[o]
            if o in r2 and r2[o] == i and (self.retained[o] or self.retained[i]):
                outer.append(o)
                inner.append(i)
        return outer, inner

    def gf(self, op1, op2, z, coef_tol=1e-8):
        o, i = self.pair_parts(op1, op2)
        return self.eng.gf(op1, op2, o, i, z, coef_tol)

    def susc(self, A, B, z, pole_res=1e-8, coef_tol=1e-8):
        o, i = self.pair_parts(A, B)
        return self.eng.susc(A, B, o, i, z, self.beta, pole_res, coef_tol)

    def g2_parts(self, C1, C2, CX3, CX4):
        """TwoParticleGF::prepare (TwoParticleGF.cpp:67-120) over op block maps."""
        ops = [C1, C2, CX3]
        maps = [self.maps(o) for o in ops]  # (right->left, left->right)
        r4, _ = self.maps(CX4)
        parts = []
        for S1 in sorted(r4):
            S4 = r4[S1]
            for perm, sign in L.PERMUTATIONS3:
                o0, o1, o2 = perm
                S2 = maps[o0][1].get(S1)
                if S2 is None:
                    continue
                S3 = maps[o2][0].get(S4)
                if S3 is None or maps[o1][1].get(S2) != S3:
                    continue
                if not any(self.retained[b] for b in (S1, S2, S3, S4)):
                    continue
                parts.append(((ops[o0], ops[o1], ops[o2], CX4), (S1, S2, S3, S4), perm, sign))
        return parts

    def g2(self, C1, C2, CX3, CX4, triples, pole_res=1e-8):
        parts = self.g2_parts(C1, C2, CX3, CX4)
        return self.eng.g2(parts, triples, pole_res=pole_res), parts
