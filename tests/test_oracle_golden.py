"""Pin the CPU oracle against the reference's own known-answer tests.

Golden vectors come from tests/golden/reference_kats.json (extracted from the
reference's test sources by tests/golden/make_golden.py); closed forms are the
formulas of GF1siteTest.cpp, SusceptibilityTest.cpp, AndersonComplexTest.cpp
and Vertex4Test.cpp restated.  Tolerances are the reference tests' own.
"""
import json
import os

import numpy as np
import pytest

from oracle import ed as EDm
from oracle import lehmann as L
from oracle import model as M

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


def cplx(a):
    return np.array([complex(x, y) for x, y in a])


def test_hamiltonian_ground_energy():
    e = M.CoulombS("A", 1.0, -0.5) + M.CoulombS("B", 2.0, -1.0) + M.Hopping("A", "B", -1.0)
    m = M.make_model(e)
    ed = EDm.ED(m, 10.0)
    k = KATS["hamiltonian"]
    assert abs(ed.E0 - k["E0"]) < k["tol"]
    for b in range(len(m.blocks)):
        h = m.h_block(b)
        assert np.abs(h @ ed.U[b] - ed.U[b] * ed.E[b][None, :]).max() < 1e-10


def test_gf1site_closed_form():
    U, mu, beta = 1.0, 0.4, 10.0
    m = M.make_model(M.CoulombS("A", U, -mu))
    ed = EDm.ED(m, beta)
    dn = m.info.getIndex("A", 0, 0)
    t = L.gf_terms(ed, ed.c(dn), ed.cdag(dn))
    n = np.arange(-100, 100)
    om = np.pi * (2 * n + 1) / beta
    w0, w1, w2 = 1.0, np.exp(beta * mu), np.exp(-beta * (-2 * mu + U))
    Z = w0 + 2 * w1 + w2
    ref = (w0 + w1) / Z / (1j * om + mu) + (w1 + w2) / Z / (1j * om + mu - U)
    assert np.abs(L.gf_eval(t, 1j * om) - ref).max() < 1e-14


@pytest.mark.parametrize("rule", [True, False])
def test_gf4site_golden(rule):
    k = KATS["gf4site"]
    e = M.Expr()
    for lab, U, eps in k["coulomb"]:
        e += M.CoulombS(lab, U, eps)
    for a, b, t in k["hopping"]:
        e += M.Hopping(a, b, t)
    m = M.make_model(e)
    ed = EDm.ED(m, k["beta"])
    dn = m.info.getIndex("A", 0, 0)
    t = L.gf_terms(ed, ed.c(dn), ed.cdag(dn), rule=rule)
    v = L.gf_eval(t, L.fermionic(np.arange(10), k["beta"]))
    assert np.abs(v - cplx(k["G_A_down"])).max() < k["tol"]


def test_gf2site_golden():
    k = KATS["gf2site"]
    e = M.CoulombS("A", k["U"], -k["mu"]) + M.CoulombS("B", k["U"], -k["mu"]) + M.Hopping("A", "B", k["t"])
    m = M.make_model(e)
    ed = EDm.ED(m, k["beta"])
    dn = m.info.getIndex("A", 0, 0)
    v = L.gf_eval(L.gf_terms(ed, ed.c(dn), ed.cdag(dn)), L.fermionic(np.arange(10), k["beta"]))
    assert np.abs(v - cplx(k["G_A_down"])).max() < k["tol"]


def test_anderson_golden():
    k = KATS["anderson"]
    U = k["U"]
    e = (M.CoulombS("C", U, -k["mu_over_U"] * U) + M.Magnetization("C", k["h"])
         + M.Level("0", -k["epsilon"]) + M.Level("1", k["epsilon"])
         + M.Hopping("C", "0", k["V"]) + M.Hopping("C", "1", k["V"]))
    m = M.make_model(e)
    ed = EDm.ED(m, k["beta"])
    z = L.fermionic(np.arange(10), k["beta"])
    for s, key in ((1, "G_up"), (0, "G_down")):
        i = m.info.getIndex("C", 0, s)
        v = L.gf_eval(L.gf_terms(ed, ed.c(i), ed.cdag(i)), z)
        assert np.abs(v - cplx(k[key])).max() < k["tol"]


@pytest.mark.parametrize("J", [0.1, -0.1, 0.1j, -0.1j, 0.1 + 0.1j, 0.1 - 0.1j, -0.1 + 0.1j, -0.1 - 0.1j])
def test_anderson_complex_closed_form(J):
    mu, U, beta = 1.2, 2.0, 10.0
    e = M.CoulombS("C", U, -mu) + M.HoppingS("C", "C", complex(J), 0, 0, M.UP, M.DOWN)
    m = M.make_model(e)
    ed = EDm.ED(m, beta)
    phi = np.angle(J)
    E = np.array([0, -mu - abs(J), -mu + abs(J), -2 * mu + U])
    w = np.exp(-beta * E)
    w /= w.sum()
    iw = 1j * np.pi * (2 * np.arange(10) + 1) / beta
    base = [0.5 * (w[1] + w[0]) / (iw - (E[1] - E[0])), 0.5 * (w[2] + w[0]) / (iw - (E[2] - E[0])),
            0.5 * (w[3] + w[1]) / (iw - (E[3] - E[1])), 0.5 * (w[3] + w[2]) / (iw - (E[3] - E[2]))]
    for s1 in (M.DOWN, M.UP):
        for s2 in (M.DOWN, M.UP):
            if s1 == s2:
                ref = sum(base)
            else:
                u = np.exp(1j * phi) if s1 == M.UP else np.exp(-1j * phi)
                ref = u * (-base[0] + base[1] + base[2] - base[3])
            i1, i2 = m.info.getIndex("C", 0, s1), m.info.getIndex("C", 0, s2)
            v = L.gf_eval(L.gf_terms(ed, ed.c(i1), ed.cdag(i2)), iw)
            assert np.abs(v - ref).max() < 1e-12


def test_susceptibility_closed_form():
    U, mu, h, beta = 1.0, 0.4, 0.01, 10.0
    m = M.make_model(M.CoulombS("A", U, -mu) + M.Magnetization("A", -h))
    ed = EDm.ED(m, beta)
    up, dn = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    sp, sm = ed.quadratic(up, dn), ed.quadratic(dn, up)
    nu, nd = ed.quadratic(up, up), ed.quadratic(dn, dn)
    nn = ed.quartic(up, dn, dn, up)
    wr = np.array([1.0, np.exp(-beta * (-mu - h)), np.exp(-beta * (-mu + h)), np.exp(-beta * (-2 * mu + U))])
    wr /= wr.sum()
    wu, wd, w2 = wr[1:]
    ea = lambda o: L.ensemble_average(ed, o)
    assert abs(ea(sp)) < 1e-14 and abs(ea(sm)) < 1e-14
    assert abs(ea(nu) - (wu + w2)) < 1e-14 and abs(ea(nd) - (wd + w2)) < 1e-14
    assert abs(ea(nn) - w2) < 1e-14
    n = np.arange(20)
    z = L.bosonic(n, beta)
    om = 2 * np.pi * n / beta
    v = L.susc_eval(L.susc_terms(ed, sp, sm), z, beta, ea(sp), ea(sm))
    assert np.abs(v - (-(wu - wd) / (1j * om - 2 * h))).max() < 1e-14
    v = L.susc_eval(L.susc_terms(ed, nu, nu), z, beta, ea(nu), ea(nu))
    assert np.abs(v - np.where(n == 0, (wu + w2) * (1 - wu - w2) * beta, 0)).max() < 1e-14
    v = L.susc_eval(L.susc_terms(ed, nu, nd), z, beta, ea(nu), ea(nd))
    assert np.abs(v - np.where(n == 0, (w2 - (wu + w2) * (wd + w2)) * beta, 0)).max() < 1e-14


def _vertex4_refs(U, beta):
    w = lambda n: np.pi * (2 * n + 1) / beta
    delta = lambda a, b: 1.0 if a == b else 0.0
    deltam = lambda a, b: 1.0 if a + b == -1 else 0.0

    def g_uuuu(n1, n2, n3):
        o1, o2 = w(n1), w(n2)
        return (-beta * (delta(n1, n3) - delta(n2, n3)) * (0.5 * U) ** 2
                * (1 + (0.5 * U / o1) ** 2) * (1 + (0.5 * U / o2) ** 2))

    def g_udud(n1, n2, n3):
        o1, o2, o3 = w(n1), w(n2), w(n3)
        o4 = o1 + o2 - o3
        ww = 1 / (1 + np.exp(beta * 0.5 * U))
        v = U - 0.125 * U ** 3 * (o1 ** 2 + o2 ** 2 + o3 ** 2 + o4 ** 2) / (o1 * o2 * o3 * o4)
        v += -0.1875 * U ** 5 / (o1 * o2 * o3 * o4)
        v += (-beta * (2 * deltam(n1, n2) + delta(n1, n3)) * ww * (0.5 * U) ** 2
              * (1 + (0.5 * U / o2) ** 2) * (1 + (0.5 * U / o3) ** 2))
        v += (beta * (2 * delta(n2, n3) + delta(n1, n3)) * (1 - ww) * (0.5 * U) ** 2
              * (1 + (0.5 * U / o1) ** 2) * (1 + (0.5 * U / o2) ** 2))
        return v
    return g_uuuu, g_udud, delta


@pytest.mark.parametrize("mode", ["exact", "direct"])
def test_vertex4_closed_form(mode):
    U, beta, n_iw = 1.0, 40.0, 4
    m = M.make_model(M.CoulombS("A", U, -U / 2))
    ed = EDm.ED(m, beta)
    up, dn = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    c = {i: ed.c(i) for i in (up, dn)}
    cd = {i: ed.cdag(i) for i in (up, dn)}
    gt = {i: L.gf_terms(ed, c[i], cd[i]) for i in (up, dn)}
    GF = lambda i, n: L.gf_eval(gt[i], L.fermionic(n, beta))[0]
    g_uuuu, g_udud, delta = _vertex4_refs(U, beta)
    trip = [(a, b, x) for a in range(-n_iw, n_iw) for b in range(-n_iw, n_iw) for x in range(-n_iw, n_iw)]
    fz = [tuple(L.fermionic(np.array(t), beta)) for t in trip]
    for (i, j, k, l), tol in (((up, up, up, up), 1e-6), ((up, dn, up, dn), 1e-10)):
        parts = L.g2_parts(ed, c[i], c[j], cd[k], cd[l])
        if mode == "exact":
            v = L.g2_exact(ed, parts, fz, res=1e-4)
        else:
            v = L.g2_direct(ed, parts, fz, res=1e-4, tol=1e-12, rule=True)
        for t, (n1, n2, n3) in enumerate(trip):
            n4 = n1 + n2 - n3
            if j == up:
                ref = (g_uuuu(n1, n2, n3) * GF(up, n1) * GF(up, n2) * GF(up, n3) * GF(up, n4)
                       + beta * GF(up, n1) * GF(up, n2) * delta(n1, n4)
                       - beta * GF(up, n1) * GF(up, n2) * delta(n1, n3))
            else:
                ref = (g_udud(n1, n2, n3) * GF(up, n1) * GF(dn, n2) * GF(up, n3) * GF(dn, n4)
                       - beta * GF(up, n1) * GF(dn, n2) * delta(n1, n3))
            assert abs(v[t] - ref) < tol, (n1, n2, n3)


def anderson2pgf_model():
    k = KATS["anderson2pgf"]
    e = M.CoulombS("C", k["U"], -k["mu"])
    for i, (lv, hv) in enumerate(zip(k["levels"], k["hoppings"])):
        e += M.Level(f"b{i}", lv) + M.Hopping("C", f"b{i}", hv)
    return k, e


def anderson2pgf_freqs(beta):
    Om, om = 1j * 2 * np.pi / beta, 1j * np.pi / beta
    return [(om + Om, 1j * (2 * i + 1) * np.pi / beta, om) for i in range(10)]


@pytest.mark.parametrize("mode", ["exact", "direct"])
def test_anderson2pgf_golden(mode):
    k, e = anderson2pgf_model()
    m = M.make_model(e)
    ed = EDm.ED(m, k["beta"])
    fz = anderson2pgf_freqs(k["beta"])
    for s in (M.UP, M.DOWN):
        i = m.info.getIndex("C", 0, s)
        parts = L.g2_parts(ed, ed.c(i), ed.c(i), ed.cdag(i), ed.cdag(i))
        if mode == "exact":
            v = L.g2_exact(ed, parts, fz, res=k["pole_resolution"])
        else:
            v = L.g2_direct(ed, parts, fz, res=k["pole_resolution"], tol=k["coefficient_tolerance"])
        assert np.abs(v - np.array(k["chi_uuuu"])).max() < k["tol"]


def test_vanishing_literal_uudd():
    """(u0,u0,d0,d0) changes (N_up, N_down) by (-2,+2): no block chain exists."""
    k, e = anderson2pgf_model()
    m = M.make_model(e)
    ed = EDm.ED(m, k["beta"])
    u, d = m.info.getIndex("C", 0, 1), m.info.getIndex("C", 0, 0)
    assert L.g2_parts(ed, ed.c(u), ed.c(u), ed.cdag(d), ed.cdag(d)) == []
