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

    def chi3_parts(self, channel, CX1, C2, CX3, C4):
        """ThreePointSusceptibility::prepare (ThreePointSusceptibility.cpp:68-142)
        over the operators' block maps."""
        F1, F2, B1, B2 = {0: (CX1, CX3, C2, C4), 1: (CX1, C2, CX3, C4), 2: (CX1, C4, CX3, C2)}[channel]
        f1_rl, f1_lr = self.maps(F1)
        f2_rl, f2_lr = self.maps(F2)
        b1_rl, _ = self.maps(B1)
        b2_rl, _ = self.maps(B2)
        ret = self.retained
        parts = []
        for b2r in sorted(b2_rl):
            b2l = b2_rl[b2r]
            b1l = b1_rl.get(b2l)
            if b1l is None:
                continue
            j = f1_lr.get(b2r)
            if j is not None and f2_rl.get(b1l) == j and ret[b2r] and ret[j] and ret[b1l]:
                parts.append((F1, F2, B1, B2, (b2r, j, b1l, b2l), False))
            j = f2_lr.get(b2r)
            if j is not None and f1_rl.get(b1l) == j and ret[b2r] and ret[j] and ret[b1l]:
                parts.append((F2, F1, B1, B2, (b2r, j, b1l, b2l), True))
        return parts

    def chi3(self, channel, ixs, freqs, pole_res=1e-8):
        i1, i2, i3, i4 = ixs
        parts = self.chi3_parts(channel, self.cdag(i1), self.c(i2), self.cdag(i3), self.c(i4))
        return self.eng.chi3(channel, parts, freqs, pole_res), parts

    def g2(self, C1, C2, CX3, CX4, triples, pole_res=1e-8):
        parts = self.g2_parts(C1, C2, CX3, CX4)
        return self.eng.g2(parts, triples, pole_res=pole_res), parts


class GfTermChain:
    """G(z) = <c_i c^+_j>(z) as a function of the coefficients of the
    Hamiltonian's terms, through the C ABI: pgx_assemble_hamiltonian ->
    pgx_eigh -> pgx_weights -> pgx_op_rotate / pgx_op_adjoint -> pgx_gf
    (forward) and pgx_gf_vjp (backward).  The backward pass uses the device
    state of the last forward call."""

    def __init__(self, mdl, beta, i, j, z, device=0):
        self.m, self.beta, self.z = mdl, float(beta), np.asarray(z, dtype=complex)
        self.keys = list(mdl.expr.terms)
        self.monos = [tuple((dag, mdl.info.index[ix]) for dag, ix in k) for k in self.keys]
        self.fock = np.concatenate([np.asarray(b, dtype=np.uint64) for b in mdl.blocks])
        self.sb, self.si = np.asarray(mdl.block_of), np.asarray(mdl.inner)
        self.eng = Engine(device)
        self.eng.set_blocks(mdl.block_sizes(), mdl.complex)
        self.g = GpuED.__new__(GpuED)  # operator helpers on this engine (no host Hamiltonian upload)
        self.g.m, self.g.beta, self.g.eng = mdl, beta, self.eng
        self.g.retained = np.ones(len(mdl.blocks), dtype=bool)
        self.g._cdag, self.g._c = {}, {}
        self.i, self.j = i, j
        self.op1 = self.op2 = None

    def forward(self, coef):
        terms = [(mono, float(c)) for mono, c in zip(self.monos, coef)]
        self.eng.assemble_hamiltonian(terms, self.m.info.size(), self.fock, self.sb, self.si)
        self.eng.eigh()
        self.eng.weights(self.beta)
        if self.op1 is not None:
            for op in {self.op1, self.op2}:
                self.eng.op_release(op)
            if self.j != self.i:
                self.eng.op_release(self.g._cdag[self.i])
        self.g._cdag, self.g._c = {}, {}
        self.op2 = self.g.cdag(self.j)
        self.op1 = self.g.c(self.i)
        self.outer, self.inner = self.g.pair_parts(self.op1, self.op2)
        return self.eng.gf(self.op1, self.op2, self.outer, self.inner, self.z, coef_tol=0.0)

    def vjp(self, lam):
        return self.eng.gf_vjp(self.op1, self.op2, self.outer, self.inner, self.z, lam)


def gf_of_terms():
    """torch.autograd.Function over GfTermChain: real coefficient tensor ->
    complex G tensor.  For a real loss torch passes dL/dRe G + i dL/dIm G as
    the output gradient, so lambda = conj(grad_output)."""
    import torch

    class GfOfTerms(torch.autograd.Function):
        @staticmethod
        def forward(ctx, coef, chain):
            ctx.chain = chain
            return torch.from_numpy(chain.forward(coef.detach().cpu().numpy()))

        @staticmethod
        def backward(ctx, grad_out):
            dterm, _ = ctx.chain.vjp(np.conj(grad_out.detach().cpu().numpy()))
            return torch.from_numpy(dterm), None

    return GfOfTerms
