"""The drop-in API (namespace Pomerol classes, via pomerol_b200._pomerol).

CPU tests: expression algebra, index classification and the Hilbert-space
partition agree with the oracle.  GPU tests: the reference's own test cases
(HamiltonianTest, GF1site, GF2site, GF4site, Anderson, GF1siteAnomalous,
Susceptibility, Vertex4, Anderson2PGF, 3PSusc1site, 3PSusc3site) written
against this API, at the reference tests' tolerances."""
import json
import os

import numpy as np
import pytest

from oracle import model as M

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


@pytest.fixture(scope="module")
def P():
    from pomerol_b200 import _pomerol
    return _pomerol


def cplx(a):
    return np.array([complex(x, y) for x, y in a])


def build(P, HExpr):
    ii = P.MakeIndexClassification(HExpr)
    hs = P.MakeHilbertSpace(ii, HExpr)
    hs.compute()
    S = P.StatesClassification()
    S.compute(hs)
    return ii, hs, S


def plaquette(P, L):
    k = KATS["gf4site"]
    e = P.RealExpr()
    for lab, U, eps in k["coulomb"]:
        e += L.CoulombS(lab, U, eps)
    for a, b, t in k["hopping"]:
        e += L.Hopping(a, b, t)
    return e


# ----------------------------------------------------------------- CPU
def test_index_classification_order(P):
    L = P.LatticePresets
    H = L.CoulombS("A", 1.0, -0.5) + L.CoulombS("B", 1.0, -0.5) + L.Hopping("A", "B", -1.0)
    ii = P.MakeIndexClassification(H)
    # sorted (label, orbital, spin) with down < up (GF2siteTest.cpp:63-66)
    assert [ii.getIndex(l, 0, s) for l, s in (("A", P.down), ("A", P.up), ("B", P.down), ("B", P.up))] == [0, 1, 2, 3]


@pytest.mark.parametrize("which", ["plaquette", "anderson2pgf", "kanamori", "pairing"])
def test_partition_matches_oracle(P, which):
    L = P.LatticePresets
    if which == "plaquette":
        e, eo = plaquette(P, L), None
        k = KATS["gf4site"]
        eo = M.Expr()
        for lab, U, eps in k["coulomb"]:
            eo += M.CoulombS(lab, U, eps)
        for a, b, t in k["hopping"]:
            eo += M.Hopping(a, b, t)
    elif which == "anderson2pgf":
        k = KATS["anderson2pgf"]
        e = L.CoulombS("C", k["U"], -k["mu"])
        eo = M.CoulombS("C", k["U"], -k["mu"])
        for i, (lv, hv) in enumerate(zip(k["levels"], k["hoppings"])):
            e += L.Level(f"b{i}", lv) + L.Hopping("C", f"b{i}", hv)
            eo += M.Level(f"b{i}", lv) + M.Hopping("C", f"b{i}", hv)
    elif which == "kanamori":
        e = L.CoulombP("d", 2.5, 1.7, 0.4, -3.0, 2) + L.Level("b", 0.3) + L.Hopping("d", "b", 0.5, 0, 0, P.up, P.up) \
            + L.Hopping("d", "b", 0.5, 0, 0, P.down, P.down)
        eo = M.CoulombP("d", 2.5, 1.7, 0.4, -3.0, 2) + M.Level("b", 0.3) + M.HoppingS("d", "b", 0.5, 0, 0, 1, 1) \
            + M.HoppingS("d", "b", 0.5, 0, 0, 0, 0)
    else:
        e = L.CoulombS("A", 1.0, -0.4) + L.Pairing("A", 0.1)
        eo = M.CoulombS("A", 1.0, -0.4) + M.Pairing("A", 0.1)
    ii, hs, S = build(P, e)
    m = M.make_model(eo)
    assert S.getNumberOfBlocks() == len(m.blocks)
    for b in range(len(m.blocks)):
        assert list(S.getFockStates(b)) == list(m.blocks[b])


# ----------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_hamiltonian_reference_case(P):
    L = P.LatticePresets
    HExpr = L.CoulombS("A", 1.0, -0.5) + L.CoulombS("B", 2.0, -1.0) + L.Hopping("A", "B", -1.0)
    ii, hs, S = build(P, HExpr)
    H = P.Hamiltonian(S)
    H.prepare(HExpr, hs)
    hmats = [H.getPart(b).getMatrix().copy() for b in range(S.getNumberOfBlocks())]
    H.compute()
    assert abs(H.getGroundEnergy() - KATS["hamiltonian"]["E0"]) < 1e-7
    for b in range(S.getNumberOfBlocks()):
        part = H.getPart(b)
        U = part.getMatrix()
        E = np.array(part.getEigenValues())
        assert np.abs(hmats[b] @ U - U * E[None, :]).max() < 1e-10
    # rotated c^+ versus transposed c (HamiltonianTest.cpp:96-133)
    ops = P.FieldOperatorContainer(ii, hs, S, H)
    ops.prepareAll(hs)
    ops.computeAll()
    i = ii.getIndex("B", 0, P.up)
    cd, c = ops.getCreationOperator(i), ops.getAnnihilationOperator(i)
    for R, Lb in cd.getBlockMapping().items():
        a = cd.getPartFromRightIndex(R).getMatrix()
        b = c.getPartFromRightIndex(Lb).getMatrix()
        assert np.abs(a - b.T).max() < 1e-12


def _setup(P, HExpr, beta):
    ii, hs, S = build(P, HExpr)
    H = P.Hamiltonian(S)
    H.prepare(HExpr, hs)
    H.compute()
    rho = P.DensityMatrix(S, H, beta)
    rho.prepare()
    rho.compute()
    ops = P.FieldOperatorContainer(ii, hs, S, H)
    ops.prepareAll(hs)
    ops.computeAll()
    return ii, hs, S, H, rho, ops


@pytest.mark.gpu
def test_gf1site_and_container(P):
    L = P.LatticePresets
    U, mu, beta = 1.0, 0.4, 10.0
    ii, hs, S, H, rho, ops = _setup(P, L.CoulombS("A", U, -mu), beta)
    dn = ii.getIndex("A", 0, P.down)
    GF = P.GreensFunction(S, H, ops.getAnnihilationOperator(dn), ops.getCreationOperator(dn), rho)
    GF.prepare()
    GF.compute()

    def ref(n):
        om = np.pi * (2 * n + 1) / beta
        w0, w1, w2 = 1.0, np.exp(beta * mu), np.exp(-beta * (-2 * mu + U))
        Z = w0 + 2 * w1 + w2
        return (w0 + w1) / Z / (1j * om + mu) + (w1 + w2) / Z / (1j * om + mu - U)
    for n in range(100):
        assert abs(GF(n) - ref(n)) < 1e-14
    G = P.GFContainer(ii, S, H, rho, ops)
    G.prepareAll([(0, 0), (0, 1), (1, 0), (1, 1)])
    G.computeAll()
    for n in range(-100, 100):
        assert abs(G(0, 0)(n) - ref(n)) < 1e-14 and abs(G(0, 1)(n)) < 1e-14
        assert abs(G(1, 0)(n)) < 1e-14 and abs(G(1, 1)(n) - ref(n)) < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["gf2site", "gf4site", "anderson"])
def test_gf_golden(P, case):
    L = P.LatticePresets
    k = KATS[case]
    if case == "gf2site":
        HExpr = L.CoulombS("A", k["U"], -k["mu"]) + L.CoulombS("B", k["U"], -k["mu"]) + L.Hopping("A", "B", k["t"])
        pairs = [("A", P.down, "G_A_down")]
    elif case == "gf4site":
        HExpr = plaquette(P, L)
        pairs = [("A", P.down, "G_A_down")]
    else:
        U = k["U"]
        HExpr = (L.CoulombS("C", U, -k["mu_over_U"] * U) + L.Magnetization("C", k["h"]) + L.Level("0", -k["epsilon"])
                 + L.Level("1", k["epsilon"]) + L.Hopping("C", "0", k["V"]) + L.Hopping("C", "1", k["V"]))
        pairs = [("C", P.up, "G_up"), ("C", P.down, "G_down")]
    ii, hs, S, H, rho, ops = _setup(P, HExpr, k["beta"])
    for lab, s, key in pairs:
        i = ii.getIndex(lab, 0, s)
        GF = P.GreensFunction(S, H, ops.getAnnihilationOperator(i), ops.getCreationOperator(i), rho)
        GF.prepare()
        GF.compute()
        v = np.array([GF(n) for n in range(10)])
        assert np.abs(v - cplx(k[key])).max() < k["tol"]


@pytest.mark.gpu
def test_gf1site_anomalous(P):
    L = P.LatticePresets
    U, mu, Delta, beta = 1.0, 0.4, 0.1, 10.0
    ii, hs, S, H, rho, ops = _setup(P, L.CoulombS("A", U, -mu) + L.Pairing("A", Delta), beta)
    e1, e2 = -mu, -2 * mu + U
    ep = np.sqrt(e2 * e2 + 4 * Delta * Delta)
    esc1, esc2 = 0.5 * (e2 - ep), 0.5 * (e2 + ep)
    a = -esc2 / np.sqrt(Delta ** 2 + esc2 ** 2)
    b = -esc1 / np.sqrt(Delta ** 2 + esc1 ** 2)
    w1, ws1, ws2 = np.exp(-beta * e1), np.exp(-beta * esc1), np.exp(-beta * esc2)
    Z = 2 * w1 + ws1 + ws2
    w1, ws1, ws2 = w1 / Z, ws1 / Z, ws2 / Z

    def G_ref(n):
        iw = 1j * np.pi * (2 * n + 1) / beta
        return ((w1 + ws1) * a * a / (iw - (e1 - esc1)) + (w1 + ws2) * (1 - a * a) / (iw - (e1 - esc2))
                + (ws1 + w1) * b * b / (iw - (esc1 - e1)) + (ws2 + w1) * (1 - b * b) / (iw - (esc2 - e1)))

    def F_ref(n):
        iw = 1j * np.pi * (2 * n + 1) / beta
        return (Delta / ep) * ((w1 + ws1) / (iw - (e1 - esc1)) - (w1 + ws2) / (iw - (e1 - esc2))
                               - (ws1 + w1) / (iw - (esc1 - e1)) + (ws2 + w1) / (iw - (esc2 - e1)))
    up, dn = ii.getIndex("A", 0, P.up), ii.getIndex("A", 0, P.down)
    G = P.GreensFunction(S, H, ops.getAnnihilationOperator(dn), ops.getCreationOperator(dn), rho)
    F = P.GreensFunction(S, H, ops.getAnnihilationOperator(up), ops.getAnnihilationOperator(dn), rho)
    for g in (G, F):
        g.prepare()
        g.compute()
    for n in range(100):
        assert abs(G(n) - G_ref(n)) < 1e-14 and abs(F(n) - F_ref(n)) < 1e-14
    Fc = P.GFContainer(ii, S, H, rho, ops, True)
    Fc.prepareAll([(0, 0), (0, 1), (1, 0), (1, 1)])
    Fc.computeAll()
    for n in range(-20, 20):
        assert abs(Fc(up, dn)(n) - F_ref(n)) < 1e-14 and abs(Fc(dn, up)(n) + F_ref(n)) < 1e-14
        assert abs(Fc(0, 0)(n)) < 1e-14


@pytest.mark.gpu
def test_susceptibility_reference_case(P):
    L = P.LatticePresets
    U, mu, h, beta = 1.0, 0.4, 0.01, 10.0
    ii, hs, S, H, rho, _ = _setup(P, L.CoulombS("A", U, -mu) + L.Magnetization("A", -h), beta)
    up, dn = ii.getIndex("A", 0, P.up), ii.getIndex("A", 0, P.down)
    sp = P.QuadraticOperator(ii, hs, S, H, up, dn)
    sm = P.QuadraticOperator(ii, hs, S, H, dn, up)
    nu = P.QuadraticOperator(ii, hs, S, H, up, up)
    nd = P.QuadraticOperator(ii, hs, S, H, dn, dn)
    nn = P.QuarticOperator(ii, hs, S, H, up, dn, dn, up)
    for o in (sp, sm, nu, nd, nn):
        o.prepare(hs)
        o.compute()
    wr = np.array([1.0, np.exp(-beta * (-mu - h)), np.exp(-beta * (-mu + h)), np.exp(-beta * (-2 * mu + U))])
    wr /= wr.sum()
    wu, wd, w2 = wr[1:]
    for o, ref in ((sp, 0), (sm, 0), (nu, wu + w2), (nd, wd + w2), (nn, w2)):
        ea = P.EnsembleAverage(o, rho)
        ea.compute()
        assert abs(ea() - ref) < 1e-14
    om = lambda n: 2 * np.pi * n / beta
    cases = [(sp, sm, lambda n: -(wu - wd) / (1j * om(n) - 2 * h)),
             (nu, nu, lambda n: (wu + w2) * (1 - wu - w2) * beta if n == 0 else 0),
             (nu, nd, lambda n: (w2 - (wu + w2) * (wd + w2)) * beta if n == 0 else 0)]
    for A, B, ref in cases:
        chi = P.Susceptibility(S, H, A, B, rho)
        chi.prepare()
        chi.compute()
        chi.subtractDisconnected()
        for n in range(20):
            assert abs(chi(n) - ref(n)) < 1e-14


@pytest.mark.gpu
def test_vertex4_reference_case(P):
    from tests.test_oracle_golden import _vertex4_refs
    L = P.LatticePresets
    U, beta, n_iw = 1.0, 40.0, 4
    ii, hs, S, H, rho, ops = _setup(P, L.CoulombS("A", U, -U / 2), beta)
    G = P.GFContainer(ii, S, H, rho, ops)
    G.prepareAll()
    G.computeAll()
    Chi = P.TwoParticleGFContainer(ii, S, H, rho, ops)
    Chi.PoleResolution = 1e-4
    Chi.CoefficientTolerance = 1e-12
    Chi.prepareAll()
    Chi.computeAll()
    up, dn = ii.getIndex("A", 0, P.up), ii.getIndex("A", 0, P.down)
    g_uuuu, g_udud, delta = _vertex4_refs(U, beta)
    Gu, Gd = G(up, up), G(dn, dn)
    cu = Chi(up, up, up, up)
    cud = Chi(up, dn, up, dn)
    for n1 in range(-n_iw, n_iw):
        for n2 in range(-n_iw, n_iw):
            for n3 in range(-n_iw, n_iw):
                n4 = n1 + n2 - n3
                ref = (g_uuuu(n1, n2, n3) * Gu(n1) * Gu(n2) * Gu(n3) * Gu(n4) + beta * Gu(n1) * Gu(n2) * delta(n1, n4)
                       - beta * Gu(n1) * Gu(n2) * delta(n1, n3))
                assert abs(cu(n1, n2, n3) - ref) < 1e-6
                ref = (g_udud(n1, n2, n3) * Gu(n1) * Gd(n2) * Gu(n3) * Gd(n4) - beta * Gu(n1) * Gd(n2) * delta(n1, n3))
                assert abs(cud(n1, n2, n3) - ref) < 1e-10
    # index-swap symmetry of the container: chi_{dudu}(n1,n2,n3) = chi_{udud}(n2,n1,n1+n2-n3)
    cdu = Chi(dn, up, dn, up)
    assert abs(cdu(1, -2, 0) - cud(-2, 1, -1)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("split,products", [(True, False), (False, False), (True, True)])
def test_anderson2pgf_reference_case(P, split, products):
    """Anderson2PGFTest's golden chi values through the container; products=True
    also runs the stacked products on the int8 tensor cores (SplitProducts)."""
    L = P.LatticePresets
    k = KATS["anderson2pgf"]
    HExpr = L.CoulombS("C", k["U"], -k["mu"])
    for i, (lv, hv) in enumerate(zip(k["levels"], k["hoppings"])):
        HExpr += L.Level(f"b{i}", lv) + L.Hopping("C", f"b{i}", hv)
    beta = k["beta"]
    ii = P.MakeIndexClassification(HExpr)
    hs = P.MakeHilbertSpace(ii, HExpr)
    hs.compute()
    S = P.StatesClassification()
    S.compute(hs)
    H = P.Hamiltonian(S)
    H.prepare(HExpr, hs)
    H.compute()
    rho = P.DensityMatrix(S, H, beta)
    rho.prepare()
    rho.compute()
    d0, u0 = ii.getIndex("C", 0, P.down), ii.getIndex("C", 0, P.up)
    ops = P.FieldOperatorContainer(ii, hs, S, H, {u0, d0})
    ops.prepareAll(hs)
    ops.computeAll()
    Chi4 = P.TwoParticleGFContainer(ii, S, H, rho, ops)
    Chi4.PoleResolution = k["pole_resolution"]
    Chi4.CoefficientTolerance = k["coefficient_tolerance"]
    Chi4.SplitProducts = products
    Chi4.prepareAll([(u0, u0, u0, u0), (u0, d0, u0, d0), (d0, d0, d0, d0)])
    Om, om = 1j * 2 * np.pi / beta, 1j * np.pi / beta
    freqs = [(om + Om, 1j * (2 * i + 1) * np.pi / beta, om) for i in range(10)]
    data = Chi4.computeAll(True, freqs, 0, split)
    ref = np.array(k["chi_uuuu"])
    assert np.abs(np.array(data[(u0, u0, u0, u0)]) - ref).max() < k["tol"]
    assert np.abs(np.array(data[(d0, d0, d0, d0)]) - ref).max() < k["tol"]
    # point evaluation through the element (the first section of the test)
    chi = Chi4(u0, u0, u0, u0).element()
    v = np.array([chi(om + Om, 1j * (2 * i + 1) * np.pi / beta, om) for i in range(10)])
    assert np.abs(v - ref).max() < k["tol"]


@pytest.mark.gpu
@pytest.mark.parametrize("J", [0.1, -0.1, 0.1j, -0.1j, 0.1 + 0.1j, 0.1 - 0.1j, -0.1 + 0.1j, -0.1 - 0.1j])
def test_anderson_complex_reference_case(P, J):
    """AndersonComplexTest.cpp:89-148 through the drop-in classes: complex
    Hermitian H from CoulombS + Hopping(C, C, J, 0, 0, up, down); all four
    G_{s1 s2}(n), n < 10, against the closed form at 1e-12."""
    from tests.test_gpu_parity import _anderson_complex_gf
    from oracle import model as M
    L = P.LatticePresets
    mu, U, beta = 1.2, 2.0, 10.0
    HExpr = P.add(L.CoulombS("C", U, -mu), L.Hopping("C", "C", complex(J), 0, 0, P.up, P.down))
    ii, hs, S, H, rho, ops = _setup(P, HExpr, beta)
    assert H.isComplex() == (complex(J).imag != 0)
    spin_of = {P.down: M.DOWN, P.up: M.UP}
    for s1 in (P.down, P.up):
        for s2 in (P.down, P.up):
            i1, i2 = ii.getIndex("C", 0, s1), ii.getIndex("C", 0, s2)
            GF = P.GreensFunction(S, H, ops.getAnnihilationOperator(i1), ops.getCreationOperator(i2), rho)
            GF.prepare()
            GF.compute()
            v = np.array([GF(n) for n in range(10)])
            ref = np.array([_anderson_complex_gf(J, spin_of[s1], spin_of[s2], n, mu, U, beta) for n in range(10)])
            assert np.abs(v - ref).max() < 1e-12


@pytest.mark.gpu
def test_vertex4_class_reference_case(P):
    """Vertex4Test.cpp:124-150 through the drop-in Vertex4: the connected
    vertex of the Hubbard atom, Gamma(n1,n2,n3) = g(n1,n2,n3) G(n1)G(n2)G(n3)G(n4),
    from Vertex4(chi_uuuu, G, G, G, G).compute(n_iw) at 1e-10; values outside
    the cached box come from the direct evaluation."""
    from tests.test_oracle_golden import _vertex4_refs
    L = P.LatticePresets
    U, beta, n_iw = 1.0, 40.0, 4
    ii, hs, S, H, rho, ops = _setup(P, L.CoulombS("A", U, -U / 2), beta)
    G = P.GFContainer(ii, S, H, rho, ops)
    G.prepareAll()
    G.computeAll()
    Chi = P.TwoParticleGFContainer(ii, S, H, rho, ops)
    Chi.PoleResolution = 1e-4
    Chi.CoefficientTolerance = 1e-12
    up = ii.getIndex("A", 0, P.up)
    Chi.prepareAll([(up, up, up, up)])
    Chi.computeAll()
    g_uuuu, _, _ = _vertex4_refs(U, beta)
    GF = G(up, up)
    chi = Chi(up, up, up, up).element()
    Gamma = P.Vertex4(chi, GF, GF, GF, GF)
    Gamma.compute(n_iw)
    assert Gamma.getNumberOfMatsubaras() == n_iw
    for n1 in range(-n_iw, n_iw):
        for n2 in range(-n_iw, n_iw):
            for n3 in range(-n_iw, n_iw):
                n4 = n1 + n2 - n3
                ref = g_uuuu(n1, n2, n3) * GF(n1) * GF(n2) * GF(n3) * GF(n4)
                assert abs(Gamma(n1, n2, n3) - ref) < 1e-10
    for n1, n2, n3 in ((5, -7, 2), (-6, 6, 0)):  # outside the box
        n4 = n1 + n2 - n3
        ref = g_uuuu(n1, n2, n3) * GF(n1) * GF(n2) * GF(n3) * GF(n4)
        assert abs(Gamma(n1, n2, n3) - ref) < 1e-10
        assert abs(Gamma.value(n1, n2, n3) - Gamma(n1, n2, n3)) < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("h_field", [0.0, 0.01])
def test_chi3_1site_reference_case(P, h_field):
    """3PSusc1siteTest.cpp:65-250 through the drop-in ThreePointSusceptibility:
    all channels and spin pairs of the Hubbard atom against the closed form
    at 1e-14 (relative to 1), and the PH / xPH crossing symmetry."""
    from tests.test_oracle_chi3 import AtomChi3
    L = P.LatticePresets
    U, mu, beta, n_iw = 1.0, 0.4, 10.0, 20
    ii, hs, S, H, rho, ops = _setup(P, L.CoulombS("A", U, -mu) + L.Magnetization("A", -h_field), beta)
    up, dn = ii.getIndex("A", 0, P.up), ii.getIndex("A", 0, P.down)
    g = AtomChi3(beta, U, mu, h_field)
    om = lambda n: np.pi * (2 * n + 1) / beta
    st = {up: 1, dn: 2}
    grid = [(a, b) for a in range(-n_iw, n_iw) for b in range(-n_iw, n_iw)]

    def chi3(ch, i1, i2, i3, i4):
        c = P.ThreePointSusceptibility(ch, S, H, ops.getCreationOperator(i1), ops.getAnnihilationOperator(i2),
                                       ops.getCreationOperator(i3), ops.getAnnihilationOperator(i4), rho)
        c.prepare()
        c.compute()
        return c

    for i1 in (up, dn):
        for i2 in (up, dn):
            other = dn if i1 == up else up
            c = chi3(P.PP, i1, i1, i2, i2)
            if i1 == i2:
                assert c.isVanishing()
            else:
                for a, b in grid:
                    ref = g(3, st[i2], 0, -om(a), -om(b)) + g(3, st[i1], 0, -om(b), -om(a))
                    assert abs(c(a, b) - ref) < 1e-14 * max(1.0, abs(ref))
            cph, cx = chi3(P.PH, i1, i1, i2, i2), chi3(P.xPH, i1, i1, i2, i2)
            for a, b in grid:
                if i1 == i2:
                    ref = g(st[i1], 0, st[i1], -om(a), om(b)) + g(3, st[other], 3, -om(a), om(b))
                    refx = -ref
                else:
                    s = st[i2]
                    ref = g(3, s, 3, -om(a), om(b)) - g(s, 3, s, om(a), -om(b))
                    refx = -g(st[i1], 0, st[i2], -om(a), om(b)) - g(st[i1], 3, st[i2], om(b), -om(a))
                assert abs(cph(a, b) - ref) < 1e-14 * max(1.0, abs(ref))
                assert abs(cx(a, b) - refx) < 1e-14 * max(1.0, abs(refx))
    ix = (up, dn)
    for a in ix:
        for b in ix:
            for c3 in ix:
                for d in ix:
                    ph, xph = chi3(P.PH, a, b, c3, d), chi3(P.xPH, a, d, c3, b)
                    for n1, n2 in grid[::7]:
                        assert abs(xph(n1, n2) + ph(n1, n2)) < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("channel", ["PP", "PH", "xPH"])
def test_chi3_3site_reference_case(P, channel):
    """3PSusc3siteTest.cpp:24-157: chi3 of the three-site Hubbard cluster at
    n1, n2 in {-1, 0, 1} against the golden values at 1e-10, through the
    class and through ThreePointSusceptibilityContainer.computeAll."""
    L = P.LatticePresets
    k = KATS["chi3_3site"]
    HExpr = P.RealExpr()
    for s in k["sites"]:
        HExpr += L.CoulombS(s, k["U"], -k["mu"])
    for a, b in (("A", "B"), ("B", "C"), ("C", "A")):
        HExpr += L.Hopping(a, b, -k["t"])
    beta = k["beta"]
    ii, hs, S, H, rho, ops = _setup(P, HExpr, beta)
    spin = {"up": P.up, "down": P.down}
    i1, i2, i3, i4 = [ii.getIndex(s, 0, spin[sp]) for s, sp in k[channel]["ops"]]
    ch = {"PP": P.PP, "PH": P.PH, "xPH": P.xPH}[channel]
    c = P.ThreePointSusceptibility(ch, S, H, ops.getCreationOperator(i1), ops.getAnnihilationOperator(i2),
                                   ops.getCreationOperator(i3), ops.getAnnihilationOperator(i4), rho)
    c.prepare()
    c.compute()
    ref = cplx(k[channel]["chi3"])
    got = np.array([c(a, b) for a in k["n"] for b in k["n"]])
    assert np.abs(got - ref).max() < k["tol"]
    cont = P.ThreePointSusceptibilityContainer(ch, ii, S, H, rho, ops)
    cont.prepareAll([(i1, i2, i3, i4)])
    freqs = [(1j * np.pi * (2 * a + 1) / beta, 1j * np.pi * (2 * b + 1) / beta) for a in k["n"] for b in k["n"]]
    res = cont.computeAll(False, freqs)
    # the element and its index-exchange aliases share one object; computeAll
    # visits the keys in order, so the first key of the group carries the
    # values and the later ones the empty vector of an already computed
    # element (ThreePointSusceptibilityContainer.cpp:30-40)
    group = sorted({(i1, i2, i3, i4), (i2, i1, i3, i4), (i1, i2, i4, i3), (i2, i1, i4, i3)})
    assert all(cont.isInContainer(*g) for g in group)
    assert np.abs(np.array(res[group[0]]) - ref).max() < k["tol"]
    assert all(len(res[g]) == 0 for g in group[1:])


@pytest.mark.gpu
def test_hamiltonian_reduce(P):
    """Hamiltonian::reduce (Hamiltonian.cpp:115-119, HamiltonianPart.cpp:151-172):
    every block keeps its eigenvalues up to E0 + Cutoff and the top-left
    corner of its eigenvector matrix of that size; a block left with none
    stays whole."""
    L = P.LatticePresets
    ii, hs, S, H, rho, ops = _setup(P, plaquette(P, L), 10.0)
    nb = S.getNumberOfBlocks()
    full_e = [list(H.getPart(b).getEigenValues()) for b in range(nb)]
    full_u = [np.array(H.getPart(b).getMatrix()) for b in range(nb)]
    E0, cut = H.getGroundEnergy(), 1.5
    H.reduce(cut)
    for b in range(nb):
        d = S.getBlockSize(b)
        keep = sum(1 for e in full_e[b] if e <= E0 + cut)
        e = list(H.getPart(b).getEigenValues())
        u = np.array(H.getPart(b).getMatrix())
        if keep == 0:
            assert e == full_e[b] and np.array_equal(u, full_u[b])
        else:
            assert e == full_e[b][:keep]
            assert np.array_equal(u.reshape(keep, keep), full_u[b].reshape(d, d)[:keep, :keep])
    assert any(len(H.getPart(b).getEigenValues()) < S.getBlockSize(b) for b in range(nb))
