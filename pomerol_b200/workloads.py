"""Synthetic workloads of the G2 path, built through the drop-in API.

  plaquette  2x2 Hubbard plaquette: CoulombS(U=4, -mu=-2) on sites A..D,
             nearest-neighbour Hopping(t=-1), beta=10, dim 256
  a5         Anderson impurity + 5 bath sites: CoulombS(U=3, eps_d=-U/2) on
             "C", Level(b_k, eps_k) + Hopping(C, b_k, V_k) with
             rng = numpy.random.default_rng(0), eps = rng.uniform(-2,2,5) then
             V = rng.uniform(0.2,0.8,5); beta=20, dim 4096
  ring8      8-site Hubbard ring, PBC, t=1, U=4, mu=2, beta=5, dim 65536
  b64        64 independent Anderson impurities with 3-6 bath sites (dims
             256-16384): rng = numpy.random.default_rng(1), per model in
             order nb = rng.integers(3, 7), U = rng.uniform(1, 6),
             beta = rng.uniform(5, 50), eps = rng.uniform(-2, 2, nb),
             V = rng.uniform(0.1, 1.0, nb), eps_d = -U/2; G_dn on n = 0..1023
             and chi_dd (n_d = n_up + n_dn) on m = 0..31, each model at its
             own beta, all models in one context (BatchRun)

The G2 component is chi_(u0,d0,u0,d0) (c_up c_down c^+_up c^+_down at the
first site) on the fermionic cube n_k in [-N/2, N/2).  No public dataset is
involved: the inputs are fully specified by these parameters.
"""
from __future__ import annotations

import numpy as np

from . import _pomerol as P

L = P.LatticePresets


def plaquette_expr(t=1.0, U=4.0, mu=2.0):
    sites = ["A", "B", "C", "D"]
    e = P.RealExpr()
    for s in sites:
        e += L.CoulombS(s, U, -mu)
    for a, b in zip(sites, sites[1:] + sites[:1]):
        e += L.Hopping(a, b, -t)
    return e, "A"


def anderson_expr(U, eps_d, eps, V, imp="C"):
    e = L.CoulombS(imp, U, eps_d)
    for k, (ek, vk) in enumerate(zip(eps, V)):
        e += L.Level(f"b{k}", float(ek))
        e += L.Hopping(imp, f"b{k}", float(vk))
    return e, imp


def a5_params(seed=0, nb=5):
    rng = np.random.default_rng(seed)
    eps = rng.uniform(-2, 2, nb)
    V = rng.uniform(0.2, 0.8, nb)
    return 3.0, -1.5, eps, V, 20.0


def ring_expr(L_sites=8, t=1.0, U=4.0, mu=2.0):
    sites = [f"S{i}" for i in range(L_sites)]
    e = P.RealExpr()
    for s in sites:
        e += L.CoulombS(s, U, -mu)
    for i in range(L_sites):
        e += L.Hopping(sites[i], sites[(i + 1) % L_sites], -t)
    return e, "S0"


CONFIGS = {
    "plaquette": dict(beta=10.0, nfreq=8, dm_trunc=None),
    "a5": dict(beta=20.0, nfreq=16, dm_trunc=None),
    "ring8": dict(beta=5.0, nfreq=24, dm_trunc=1e-12),
}


def expr_of(name):
    if name == "plaquette":
        return plaquette_expr()
    if name == "a5":
        U, epsd, eps, V, _ = a5_params(0)
        return anderson_expr(U, epsd, eps, V)
    if name == "ring8":
        return ring_expr()
    raise KeyError(name)


def matsubara_cube(beta, nfreq, shift=0):
    n = np.arange(-nfreq // 2, nfreq // 2) + shift
    idx = np.array([(a, b, c) for a in n for b in n for c in n])
    z = 1j * np.pi * (2 * idx + 1) / beta
    return idx, z


class Problem:
    """One G2 problem set up through the drop-in API (prepare stage)."""

    def __init__(self, name, device=0):
        cfg = CONFIGS[name]
        self.name, self.beta, self.nfreq, self.dm_trunc = name, cfg["beta"], cfg["nfreq"], cfg["dm_trunc"]
        self.HExpr, site = expr_of(name)
        self.ii = P.MakeIndexClassification(self.HExpr)
        self.hs = P.MakeHilbertSpace(self.ii, self.HExpr)
        self.hs.compute()
        self.S = P.StatesClassification()
        self.S.compute(self.hs)
        self.u0 = self.ii.getIndex(site, 0, P.up)
        self.d0 = self.ii.getIndex(site, 0, P.down)
        self.dims = [self.S.getBlockSize(b) for b in range(self.S.getNumberOfBlocks())]
        self.device = device

    def run_api(self, freqs, split=False, anchor_tol=None, slices=6):
        """Full drop-in sequence from the Hamiltonian expression: Hamiltonian
        (eigensolve), DensityMatrix, FieldOperatorContainer (rotation),
        TwoParticleGFContainer.computeAll on the triples (SplitProducts =
        split; AnchorTolerance = anchor_tol when given).  Returns the values."""
        H = P.Hamiltonian(self.S, self.device)
        H.prepare(self.HExpr, self.hs)
        H.compute()
        rho = P.DensityMatrix(self.S, H, self.beta)
        rho.prepare()
        rho.compute()
        if self.dm_trunc:
            rho.truncateBlocks(self.dm_trunc)
        ops = P.FieldOperatorContainer(self.ii, self.hs, self.S, H, {self.u0, self.d0})
        ops.prepareAll(self.hs)
        ops.computeAll()
        chi = P.TwoParticleGFContainer(self.ii, self.S, H, rho, ops)
        chi.SplitProducts = bool(split)
        chi.SplitSlices = int(slices)
        if anchor_tol is not None:
            chi.AnchorTolerance = float(anchor_tol)
        key = (self.u0, self.d0, self.u0, self.d0)
        chi.prepareAll([key])
        out = chi.computeAll(True, [tuple(t) for t in freqs])
        self._last = (H, rho, ops, chi)
        return np.asarray(out[key])

    def engine_inputs(self):
        """Inputs of the C-ABI leg: block Hamiltonians, Fock actions of c^+,
        and the block chains of chi_(u0,d0,u0,d0) as found by TwoParticleGF."""
        H = P.Hamiltonian(self.S, self.device)
        H.prepare(self.HExpr, self.hs)
        blocks = [np.array(H.getPart(b).getMatrix()) for b in range(len(self.dims))]
        H.compute()
        rho = P.DensityMatrix(self.S, H, self.beta)
        rho.prepare()
        rho.compute()
        if self.dm_trunc:
            rho.truncateBlocks(self.dm_trunc)
        ops = P.FieldOperatorContainer(self.ii, self.hs, self.S, H, {self.u0, self.d0})
        ops.prepareAll(self.hs)
        ops.computeAll()
        g2 = P.TwoParticleGF(self.S, H, ops.getAnnihilationOperator(self.u0), ops.getAnnihilationOperator(self.d0),
                             ops.getCreationOperator(self.u0), ops.getCreationOperator(self.d0), rho)
        g2.prepare()
        actions = {i: ops.getCreationOperator(i).fockAction() for i in (self.u0, self.d0)}
        return blocks, actions, g2.parts()


def matsubara_square(beta, n):
    """Fermionic duplets (n1, n2) in [-n/2, n/2)^2 and their frequencies."""
    k = np.arange(-n // 2, n // 2)
    idx = np.array([(a, b) for a in k for b in k])
    return idx, 1j * np.pi * (2 * idx + 1) / beta


def b64_params(seed=1, nmodels=64):
    """(U, eps_d, eps, V, beta) of each model of the batch workload."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nmodels):
        nb = int(rng.integers(3, 7))
        U = rng.uniform(1, 6)
        beta = rng.uniform(5, 50)
        eps = rng.uniform(-2, 2, nb)
        V = rng.uniform(0.1, 1.0, nb)
        out.append((U, -U / 2, eps, V, beta))
    return out


def model_inputs(U, eps_d, eps, V, device=0):
    """One impurity model through the drop-in API: block sizes, block
    Hamiltonians, and the Fock actions of c^+_dn and n_d = n_up + n_dn
    (right block, left block, targets, coefficients) per part."""
    HExpr, imp = anderson_expr(U, eps_d, eps, V)
    ii = P.MakeIndexClassification(HExpr)
    hs = P.MakeHilbertSpace(ii, HExpr)
    hs.compute()
    S = P.StatesClassification()
    S.compute(hs)
    H = P.Hamiltonian(S, device)
    H.prepare(HExpr, hs)
    dims = [S.getBlockSize(b) for b in range(S.getNumberOfBlocks())]
    blocks = [np.array(H.getPart(b).getMatrix()) for b in range(len(dims))]
    up, dn = ii.getIndex(imp, 0, P.up), ii.getIndex(imp, 0, P.down)
    cdag = P.CreationOperator(ii, hs, S, H, dn)
    cdag.prepare(hs)
    nd = {}
    for i in (up, dn):
        n = P.QuadraticOperator(ii, hs, S, H, i, i)
        n.prepare(hs)
        for r, l, t, c in n.fockAction():
            t, c = np.asarray(t), np.asarray(c, dtype=float)
            acc = nd.setdefault(r, np.zeros(dims[r]))
            acc += np.where(t >= 0, c, 0.0)
    ndact = [(b, b, np.where(nd[b] != 0.0, np.arange(dims[b]), -1), nd[b]) for b in sorted(nd)]
    return dims, blocks, [(r, l, np.asarray(t), np.asarray(c)) for r, l, t, c in cdag.fockAction()], ndact


class BatchRun:
    """The batch workload on one libpgx context: the blocks of every model
    diagonalised by one eigensolve, per-model weights, one rotation of c^+_dn
    and of n_d over all models, then G_dn (nG fermionic frequencies) and
    chi_dd (nchi bosonic frequencies) of every model at its own beta."""

    def __init__(self, params, nG=1024, nchi=32, device=0):
        from .pgx import Engine
        self.params = params
        dims, blocks, cd_parts, nd_parts, first = [], [], [], [], [0]
        for U, epsd, eps, V, beta in params:
            d, bl, ca, na = model_inputs(U, epsd, eps, V, device)
            off = len(dims)
            dims += d
            blocks += bl
            cd_parts += [(r + off, l + off, t, c) for r, l, t, c in ca]
            nd_parts += [(r + off, l + off, t, c) for r, l, t, c in na]
            first.append(len(dims))
        self.dims, self.first = dims, first
        self.beta = np.array([p[4] for p in params])
        self.eng = Engine(device)
        self.eng.set_blocks(dims)
        self.eng.set_hamiltonian(blocks)
        self.eng.set_models(first, self.beta)
        self.h2d_bytes = sum(b.nbytes for b in blocks)
        self.cdag = self.eng.op_define(cd_parts)
        self.nd = self.eng.op_define(nd_parts)
        # G: outer = right block of c^+, inner = its left block; chi: diagonal blocks
        self.g_outer = np.array([r for r, l, _, _ in cd_parts], dtype=np.int32)
        self.g_inner = np.array([l for r, l, _, _ in cd_parts], dtype=np.int32)
        self.x_blocks = np.array([r for r, _, _, _ in nd_parts], dtype=np.int32)
        n = np.arange(nG)
        self.zG = 1j * np.pi * (2 * n[None, :] + 1) / self.beta[:, None]
        m = np.arange(nchi)
        self.zX = 1j * 2 * np.pi * m[None, :] / self.beta[:, None]
        self.nterms_G = int(sum(dims[o] * dims[i] for o, i in zip(self.g_outer, self.g_inner)))
        self.nterms_X = int(sum(dims[b] ** 2 for b in self.x_blocks))

    def step(self):
        e = self.eng
        e.eigh()
        e.weights_models()
        e.op_rotate(self.cdag)
        e.op_rotate(self.nd)
        if getattr(self, "_c", None) is not None:
            e.op_release(self._c)
        self._c = e.op_adjoint(self.cdag)
        G = e.gf_models(self._c, self.cdag, self.g_outer, self.g_inner, self.zG, coef_tol=0.0)
        X, _ = e.susc_models(self.nd, self.nd, self.x_blocks, self.x_blocks, self.zX, coef_tol=0.0)
        return G, X


class Chi3Run:
    """Three-point susceptibility chi3_PH(u0, u0, d0, d0) of a workload on one
    libpgx context with the Hamiltonian resident in HBM: eigensolve, weights,
    rotation of c^+ and c, chi3 on the duplets.  The parts are the ones the
    drop-in ThreePointSusceptibility::prepare selects."""

    def __init__(self, prob: Problem, channel=None, device=0):
        from .pgx import PGX_PH, Engine
        self.channel = PGX_PH if channel is None else channel
        self.prob = prob
        blocks, self.actions, _ = prob.engine_inputs()
        H, rho, ops = self._dropin_parts()
        self.eng = Engine(device)
        self.eng.set_blocks(prob.dims)
        self.eng.set_hamiltonian(blocks)
        self.cdag = {i: self.eng.op_define([(r, l, np.asarray(t), np.asarray(c)) for r, l, t, c in a])
                     for i, a in self.actions.items()}

    def _dropin_parts(self):
        pr = self.prob
        H = P.Hamiltonian(pr.S, pr.device)
        H.prepare(pr.HExpr, pr.hs)
        H.compute()
        rho = P.DensityMatrix(pr.S, H, pr.beta)
        rho.prepare()
        rho.compute()
        ops = P.FieldOperatorContainer(pr.ii, pr.hs, pr.S, H, {pr.u0, pr.d0})
        ops.prepareAll(pr.hs)
        ops.computeAll()
        u, d = pr.u0, pr.d0
        chi = P.ThreePointSusceptibility(P.Channel(self.channel), pr.S, H, ops.getCreationOperator(u),
                                         ops.getAnnihilationOperator(u), ops.getCreationOperator(d),
                                         ops.getAnnihilationOperator(d), rho)
        chi.prepare()
        self.part_blocks = chi.parts()
        return H, rho, ops

    def step(self, duplets):
        e = self.eng
        e.eigh()
        e.weights(self.prob.beta)
        u, d = self.prob.u0, self.prob.d0
        for i in (u, d):
            e.op_rotate(self.cdag[i])
        for op in getattr(self, "_adjoints", ()):
            e.op_release(op)
        c = {i: e.op_adjoint(self.cdag[i]) for i in (u, d)}
        self._adjoints = tuple(c.values())
        # operators CX1, C2, CX3, C4 = c+_u, c_u, c+_d, c_d -> (F1, F2, B1, B2) of the channel
        CX1, C2, CX3, C4 = self.cdag[u], c[u], self.cdag[d], c[d]
        F1, F2, B1, B2 = {0: (CX1, CX3, C2, C4), 1: (CX1, C2, CX3, C4), 2: (CX1, C4, CX3, C2)}[self.channel]
        parts = [((F2, F1) if sw else (F1, F2)) + (B1, B2, tuple(blk), bool(sw)) for blk, sw in self.part_blocks]
        self.parts = parts
        return e.chi3(self.channel, parts, duplets)


class EngineRun:
    """The G2 stage chain on one libpgx context with the Hamiltonian resident
    in HBM: eigensolve, weights, rotation of c^+ and c, G2 on the triples."""

    def __init__(self, prob: Problem, device=0, anchored=True, anchor_tol=1e-16, split=False, slices=6):
        from .pgx import PGX_G2_ANCHORED, PGX_G2_EXACT, PGX_G2_SPLIT_I8, Engine
        self.flags = PGX_G2_ANCHORED if anchored else PGX_G2_EXACT
        if split and anchored:
            self.flags |= PGX_G2_SPLIT_I8  # stacked products on the int8 tensor cores
        self.anchor_tol = anchor_tol if anchored else 0.0
        self.prob = prob
        blocks, self.actions, self.chains = prob.engine_inputs()
        self.eng = Engine(device)
        self.eng.set_blocks(prob.dims)
        self.eng.set_hamiltonian(blocks)
        self.eng.set_g2_split_slices(slices)
        self.h2d_bytes = sum(b.nbytes for b in blocks)
        self.cdag = {i: self.eng.op_define([(r, l, np.asarray(t), np.asarray(c)) for r, l, t, c in a])
                     for i, a in self.actions.items()}

    def prepare(self):
        """Eigensolve, weights, block truncation, rotation of c^+ and c; sets
        self.parts (the block chains of chi_(u0,d0,u0,d0) on this context)."""
        e = self.eng
        e.eigh()
        e.weights(self.prob.beta)
        if self.prob.dm_trunc:
            e.truncate_blocks(self.prob.dm_trunc)
        u, d = self.prob.u0, self.prob.d0
        for i in (u, d):
            e.op_rotate(self.cdag[i])
        for op in getattr(self, "_adjoints", ()):  # the previous step's c operators
            e.op_release(op)
        c = {i: e.op_adjoint(self.cdag[i]) for i in (u, d)}
        self._adjoints = tuple(c.values())
        slots = (c[u], c[d], self.cdag[u])  # C1, C2, CX3 of chi_(u0,d0,u0,d0)
        self.parts = [((slots[p[0]], slots[p[1]], slots[p[2]], self.cdag[d]), tuple(b), tuple(p), s)
                      for b, p, s in self.chains]
        return self.parts

    def g2(self, parts, triples, flags=None):
        """G2 of a list of block chains at the triples (one pgx_g2 call)."""
        return self.eng.g2(parts, triples, pole_res=1e-8, coef_tol=self.anchor_tol,
                           flags=self.flags if flags is None else flags)

    def step(self, triples):
        self.prepare()
        return self.g2(self.parts, triples)


def chain_cost(dims, anchors, nfreq):
    """Relative cost of one block chain's anchored G2 on an nfreq^3 cube:
    complex multiply-adds of its products over (z1, z3) pairs (those of at
    least 1e9 run about five times faster, on the int8 tensor cores) plus its
    contractions over the triples."""
    d1, d2, d3, d4 = dims
    r1, r2, r3, r4 = anchors
    n2 = float(nfreq) ** 2
    prods = [n2 * d3 * d4 * r2, n2 * r1 * d3 * d4, n2 * r3 * d1 * d2, n2 * d1 * d2 * r4]
    cost = sum(m / 5.0 if m >= 1e9 else m for m in prods)
    cost += float(nfreq) ** 3 * (r2 * (d3 + d4) + r3 * (d2 + d1) + r1 * (d4 + d3) + r4 * (d1 + d2)) / 2.0
    return cost
