"""CPU oracle, part 1: fermionic model layer (test infrastructure only).

This module is the checker's restatement of what pomerol obtains from its
third-party dependency libcommute (v1.0.0, fetched by the reference's
CMakeLists.txt:76-111 and not vendored): polynomial fermionic expressions,
the Fock-space action of their monomials, the index classification and the
two-phase invariant-subspace partition.  Only the tests, the smoke check and
the CPU baseline of bench.py import it; the product path never does.

Conventions restated here (reference call sites):
  * index tuples are (label: str, orbital: int, spin: int) with down=0, up=1
    (LatticePresets.hpp:31-35); the particle index of a tuple is its rank in
    sorted order (IndexClassification.hpp:58-66, 133-140);
  * mode i of the Fock space is bit i of the state number, modes ordered like
    the particle indices (libcommute builds the space from the sorted
    generators of H, HilbertSpace.hpp:113-119);
  * Jordan-Wigner sign of c_i / c^+_i on |s>: (-1)^(number of occupied modes
    below i).  Any consistent sign convention is related to another by a
    diagonal +-1 change of basis, so every correlator is unchanged;
  * partition: phase I = connected components of H's matrix graph, phase II
    = merges until every c_i and c^+_i maps a block into at most one block
    (HilbertSpace.hpp:144-169);
  * blocks are numbered by their smallest Fock state and list their states in
    ascending order (StatesClassification.hpp:110-118 pushes states in
    ascending order).
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

DOWN, UP = 0, 1


# --------------------------------------------------------------------------
# Expressions (libcommute::expression restated as a dict of monomials)
# --------------------------------------------------------------------------
class Expr:
    """Polynomial in fermionic operators: {monomial: coefficient}.

    A monomial is a tuple of generators (dagger: bool, index_tuple), written
    left to right in operator-product order.
    """

    def __init__(self, terms=None):
        self.terms = dict(terms or {})

    def copy(self):
        return Expr(self.terms)

    def __add__(self, other):
        r = self.copy()
        for m, c in other.terms.items():
            r.terms[m] = r.terms.get(m, 0) + c
        return r

    __radd__ = __add__

    def __iadd__(self, other):
        for m, c in other.terms.items():
            self.terms[m] = self.terms.get(m, 0) + c
        return self

    def __mul__(self, other):
        if isinstance(other, Expr):
            r = Expr()
            for m1, c1 in self.terms.items():
                for m2, c2 in other.terms.items():
                    m = m1 + m2
                    r.terms[m] = r.terms.get(m, 0) + c1 * c2
            return r
        return Expr({m: c * other for m, c in self.terms.items()})

    def __rmul__(self, s):
        return Expr({m: s * c for m, c in self.terms.items()})

    def __neg__(self):
        return self * -1.0

    def __sub__(self, other):
        return self + (-other)

    def dagger(self):
        return Expr({tuple((not d, ix) for d, ix in reversed(m)): np.conj(c)
                     for m, c in self.terms.items()})

    def plus_hc(self):
        """x + x^dagger (libcommute's `+ hc`, used by Hopping/Pairing)."""
        return self + self.dagger()

    def is_complex(self):
        return any(isinstance(c, complex) or np.iscomplexobj(c) and np.imag(c) != 0
                   for c in self.terms.values())

    def indices(self):
        out = set()
        for m in self.terms:
            for _, ix in m:
                out.add(ix)
        return out


def c(label, orb=0, spin=DOWN):
    return Expr({((False, (label, orb, spin)),): 1.0})


def c_dag(label, orb=0, spin=DOWN):
    return Expr({((True, (label, orb, spin)),): 1.0})


def n(label, orb=0, spin=DOWN):
    return c_dag(label, orb, spin) * c(label, orb, spin)


# Lattice presets (LatticePresets.cpp)
def Level(label, eps, norb=1):                      # LatticePresets.cpp:46-48, 56-63
    r = Expr()
    for o in range(norb):
        r += eps * n(label, o, UP) + eps * n(label, o, DOWN)
    return r


def Level1(label, eps, orb, spin):                  # LatticePresets.cpp:46-48
    return eps * n(label, orb, spin)


def Hopping(l1, l2, t, norb=1):                     # LatticePresets.cpp:75-83, 117-124
    r = Expr()
    for o in range(norb):
        for s in (UP, DOWN):
            r += HoppingS(l1, l2, t, o, o, s, s)
    return r


def HoppingS(l1, l2, t, o1, o2, s1, s2):            # LatticePresets.cpp:75-83
    return (t * c_dag(l1, o1, s1) * c(l2, o2, s2)).plus_hc()


def Magnetization(label, h, norb=1):                # LatticePresets.cpp:140-147
    r = Expr()
    for o in range(norb):
        r += Level1(label, h, o, UP) + Level1(label, -h, o, DOWN)
    return r


def Pairing(label, delta, norb=1):                  # LatticePresets.cpp (Pairing overloads)
    r = Expr()
    for o in range(norb):
        r += (delta * c_dag(label, o, UP) * c_dag(label, o, DOWN)).plus_hc()
    return r


def NupNdown(l1, l2, U, o1, o2, s1, s2):            # LatticePresets.cpp (NupNdown)
    return U * n(l1, o1, s1) * n(l2, o2, s2)


def Spinflip(label, J, o1, o2, s1, s2):
    return J * c_dag(label, o1, s1) * c_dag(label, o2, s2) * c(label, o2, s1) * c(label, o1, s2)


def PairHopping(label, J, o1, o2, s1, s2):
    return J * c_dag(label, o1, s1) * c_dag(label, o1, s2) * c(label, o2, s1) * c(label, o2, s2)


def CoulombS(label, U, eps, norb=1):                # LatticePresets.cpp:402-409
    r = Expr()
    for o in range(norb):
        r += Level1(label, eps, o, UP) + Level1(label, eps, o, DOWN) + NupNdown(label, label, U, o, o, UP, DOWN)
    return r


def CoulombP(label, U, Up, J, eps, norb=3):         # LatticePresets.cpp:423-448
    r = Expr()
    for o1 in range(norb):
        for s1 in (UP, DOWN):
            r += Level1(label, eps, o1, s1)
            for o2 in range(norb):
                if o1 != o2:
                    r += NupNdown(label, label, (Up - J) / 2.0, o1, o2, s1, s1)
            for s2 in (UP, DOWN):
                if s2 >= s1:
                    continue
                r += NupNdown(label, label, U, o1, o1, s1, s2)
                for o2 in range(norb):
                    if o1 != o2:
                        r += NupNdown(label, label, Up, o1, o2, s1, s2)
                        r += Spinflip(label, -J, o1, o2, s1, s2)
                        r += PairHopping(label, -J, o1, o2, s1, s2)
    return r


# --------------------------------------------------------------------------
# Index classification and Fock action
# --------------------------------------------------------------------------
class IndexInfo:
    """Sorted index tuples <-> particle indices (IndexClassification.hpp)."""

    def __init__(self, expr: Expr):
        self.tuples = sorted(expr.indices())
        self.index = {t: i for i, t in enumerate(self.tuples)}

    def getIndex(self, label, orb, spin):
        return self.index[(label, orb, spin)]

    def size(self):
        return len(self.tuples)


def apply_monomial(mono, info: IndexInfo, states: np.ndarray):
    """Apply a monomial to the Fock states `states` (vectorised).

    Returns (new_states, sign, valid).  Generators act right to left.
    """
    s = states.astype(np.int64).copy()
    sign = np.ones(len(s), dtype=np.float64)
    valid = np.ones(len(s), dtype=bool)
    for dag, ix in reversed(mono):
        bit = info.index[ix]
        mask = np.int64(1) << bit
        occ = (s & mask) != 0
        valid &= (~occ) if dag else occ
        below = s & (mask - 1)
        par = _popcount(below) & 1
        sign *= np.where(par == 1, -1.0, 1.0)
        s = s ^ mask
    return s, sign, valid


def _popcount(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64)
    return np.bitwise_count(x).astype(np.int64)


def build_matrix(expr: Expr, info: IndexInfo, dim: int) -> sp.csr_matrix:
    """Full-space sparse matrix of an expression: M[s', s] = <s'|expr|s>."""
    states = np.arange(dim, dtype=np.int64)
    rows, cols, vals = [], [], []
    cplx = expr.is_complex()
    for mono, coef in expr.terms.items():
        if coef == 0:
            continue
        if len(mono) == 0:
            rows.append(states); cols.append(states)
            vals.append(np.full(dim, coef, dtype=complex if cplx else float))
            continue
        t, sg, ok = apply_monomial(mono, info, states)
        rows.append(t[ok]); cols.append(states[ok])
        vals.append((coef * sg[ok]).astype(complex if cplx else float))
    if not rows:
        return sp.csr_matrix((dim, dim))
    r = np.concatenate(rows); cc = np.concatenate(cols); v = np.concatenate(vals)
    m = sp.coo_matrix((v, (r, cc)), shape=(dim, dim)).tocsr()
    m.sum_duplicates()
    m.eliminate_zeros()
    return m


# --------------------------------------------------------------------------
# Partition (HilbertSpace::compute, HilbertSpace.hpp:144-169)
# --------------------------------------------------------------------------
def partition(H: sp.csr_matrix, info: IndexInfo, dim: int):
    """Return block id per Fock state, blocks numbered by smallest state."""
    g = (H != 0).astype(np.int8)
    _, lab = connected_components(g + g.T, directed=False)
    parent = np.arange(lab.max() + 1)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    def union(a, b):
        ra, rb = find(a), find(b)
        if ra == rb:
            return False
        parent[max(ra, rb)] = min(ra, rb)
        return True

    states = np.arange(dim, dtype=np.int64)
    maps = []
    for i in range(info.size()):
        t, _, ok = apply_monomial(((True, info.tuples[i]),), info, states)
        maps.append((lab[states[ok]], lab[t[ok]]))
    while True:
        root = np.array([find(x) for x in range(len(parent))])
        merged = False
        for src_l, dst_l in maps:
            pairs = np.unique(np.stack([root[src_l], root[dst_l]], 1), axis=0)
            # c^+_i maps a block into one block (group by source), and c_i,
            # its reverse, too (group by target).
            for key, other in ((0, 1), (1, 0)):
                p = pairs[np.lexsort((pairs[:, other], pairs[:, key]))]
                same = p[1:, key] == p[:-1, key]
                for a, b in zip(p[:-1, other][same], p[1:, other][same]):
                    merged |= union(int(a), int(b))
        if not merged:
            break
    blk = np.array([find(x) for x in range(len(parent))])[lab]
    # renumber by smallest state
    _, first_state = np.unique(blk, return_index=True)
    order = np.argsort(first_state)
    ren = np.empty(blk.max() + 1, dtype=np.int64)
    ren[np.unique(blk)[order]] = np.arange(len(order))
    return ren[blk]


@dataclass
class Model:
    """Everything the ED stages need: blocks, H blocks, operator maps."""
    expr: Expr
    info: IndexInfo
    dim: int
    H: sp.csr_matrix
    block_of: np.ndarray
    blocks: list = field(default_factory=list)      # list of sorted state arrays
    inner: np.ndarray = None                         # inner index of each state
    complex: bool = False

    def block_sizes(self):
        return [len(b) for b in self.blocks]

    def h_block(self, b):
        st = self.blocks[b]
        return self.H[st][:, st].toarray()

    def monomial_parts(self, mono, coef=1.0):
        """Connections right->left of a monomial operator and, per right block,
        the inner target index (-1 if annihilated) and sign of each state
        (MonomialOperator.hpp:160-195 and MonomialOperatorPart.cpp:71-75)."""
        parts = {}
        for R, st in enumerate(self.blocks):
            t, sg, ok = apply_monomial(mono, self.info, st)
            if not ok.any():
                continue
            Ls = np.unique(self.block_of[t[ok]])
            assert len(Ls) == 1, "partition violates the one-block rule"
            L = int(Ls[0])
            tgt = np.where(ok, self.inner[np.where(ok, t, 0)], -1)
            parts[R] = (L, tgt.astype(np.int64), (sg * coef) * ok)
        return parts


def make_model(expr: Expr) -> Model:
    info = IndexInfo(expr)
    dim = 1 << info.size()
    H = build_matrix(expr, info, dim)
    blk = partition(H, info, dim)
    nb = blk.max() + 1
    order = np.argsort(blk, kind="stable")
    counts = np.bincount(blk, minlength=nb)
    blocks = np.split(order, np.cumsum(counts)[:-1])
    inner = np.empty(dim, dtype=np.int64)
    for b in blocks:
        inner[b] = np.arange(len(b))
    return Model(expr, info, dim, H, blk, [np.asarray(b) for b in blocks], inner, expr.is_complex())


# --------------------------------------------------------------------------
# Model presets used by the workloads (synthetic, seeded)
# --------------------------------------------------------------------------
def hubbard_atom(U, mu, label="A"):
    return CoulombS(label, U, -mu)


def plaquette(t=1.0, U=4.0, mu=2.0):
    """2x2 Hubbard plaquette: 4 sites A,B,C,D on a ring (nearest neighbours)."""
    sites = ["A", "B", "C", "D"]
    e = Expr()
    for s in sites:
        e += CoulombS(s, U, -mu)
    for a, b in zip(sites, sites[1:] + sites[:1]):
        e += Hopping(a, b, -t)
    return e


def hubbard_ring(L=8, t=1.0, U=4.0, mu=2.0):
    sites = [f"S{i}" for i in range(L)]
    e = Expr()
    for s in sites:
        e += CoulombS(s, U, -mu)
    for i in range(L):
        e += Hopping(sites[i], sites[(i + 1) % L], -t)
    return e


def anderson(U, eps_d, eps_bath, V_bath, imp="C"):
    e = CoulombS(imp, U, eps_d)
    for k, (ek, vk) in enumerate(zip(eps_bath, V_bath)):
        b = f"b{k}"
        e += Level(b, float(ek))
        e += Hopping(imp, b, float(vk))
    return e


def anderson_a5_params(seed=0, nb=5):
    """Anderson 1+5 workload: eps ~ U[-2,2], then V ~ U[0.2,0.8] (this draw order)."""
    rng = np.random.default_rng(seed)
    eps = rng.uniform(-2, 2, nb)
    V = rng.uniform(0.2, 0.8, nb)
    return 3.0, -1.5, eps, V, 20.0


def kanamori_k(U, J, eps, V, imp="d"):
    """Two-orbital Kanamori impurity (CoulombP with U' = U - 2J at half
    filling, eps_d = -(3U - 5J)/2) and two bath sites per orbital, each
    hybridised with its own orbital only: bath b{o}{k} has level eps[2o+k]
    and hopping V[2o+k] to orbital o, both spins."""
    e = CoulombP(imp, U, U - 2 * J, J, -(3 * U - 5 * J) / 2, 2)
    for o in range(2):
        for k in range(2):
            b = f"b{o}{k}"
            e += Level(b, float(eps[2 * o + k]))
            for s in (UP, DOWN):
                e += HoppingS(imp, b, float(V[2 * o + k]), o, 0, s, s)
    return e


def kanamori_k_params(seed=0):
    """Bath of the differentiation workload: eps ~ U[-2,2] (4), then
    V ~ U[0.2,0.8] (4); U=2.5, J=0.4, beta=30."""
    rng = np.random.default_rng(seed)
    eps = rng.uniform(-2, 2, 4)
    V = rng.uniform(0.2, 0.8, 4)
    return 2.5, 0.4, eps, V, 30.0
