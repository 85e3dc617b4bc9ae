"""The three-point susceptibility oracle (oracle/chi3.py) pinned against the
reference's known answers: the closed form of the Hubbard atom
(3PSusc1siteTest.cpp:38-63, 106-250) and the three-site golden values
(3PSusc3siteTest.cpp:24-157)."""
import json
import os

import numpy as np
import pytest

from oracle import chi3 as X
from oracle import ed as EDm
from oracle import model as M

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


def cplx(a):
    return np.array([complex(x, y) for x, y in a])


class AtomChi3:
    """Closed form of the atom's 3-point function: states |0>, |up>, |dn>,
    |2> with energies 0, -mu - h, -mu + h, U - 2 mu (the atom's Hamiltonian
    is U n_up n_dn - mu n - h (n_up - n_dn))."""

    def __init__(self, beta, U, mu, h):
        self.beta = beta
        self.E = np.array([0.0, -mu - h, -mu + h, U - 2 * mu])
        r = np.exp(-beta * self.E)
        self.rho = r / r.sum()

    def __call__(self, i, j, k, w1, w2):
        E, rho = self.E, self.rho
        if abs(rho[k] - rho[i]) < 1e-14:
            d = 1.0 if abs(w1 + w2) < 1e-14 else 0.0
            return (1 / (1j * w2 + E[j] - E[k]) * (rho[i] + rho[j]) / (1j * w1 + E[i] - E[j])
                    + self.beta * d * rho[i] / (1j * w2 + E[j] - E[i]))
        return 1 / (1j * w2 + E[j] - E[k]) * ((rho[k] - rho[i]) / (1j * (w1 + w2) + E[i] - E[k])
                                               + (rho[i] + rho[j]) / (1j * w1 + E[i] - E[j]))


def _ops(ed, ixs):
    i1, i2, i3, i4 = ixs
    return ed.cdag(i1), ed.c(i2), ed.cdag(i3), ed.c(i4)


def _both(ed, channel, ixs, freqs):
    parts = X.chi3_parts(ed, channel, *_ops(ed, ixs))
    return parts, X.chi3_direct(ed, parts, channel, freqs), X.chi3_exact(ed, parts, channel, freqs)


@pytest.mark.parametrize("h", [0.0, 0.01])
def test_chi3_hubbard_atom_closed_form(h):
    U, mu, beta, n_iw = 1.0, 0.4, 10.0, 6
    m = M.make_model(M.CoulombS("A", U, -mu) + M.Magnetization("A", -h))
    ed = EDm.ED(m, beta)
    up, dn = m.info.getIndex("A", 0, M.UP), m.info.getIndex("A", 0, M.DOWN)
    g = AtomChi3(beta, U, mu, h)
    st = {up: 1, dn: 2}
    om = lambda n: np.pi * (2 * n + 1) / beta
    grid = [(a, b) for a in range(-n_iw, n_iw) for b in range(-n_iw, n_iw)]
    freqs = [(1j * om(a), 1j * om(b)) for a, b in grid]
    for i1 in (up, dn):
        for i2 in (up, dn):
            other = dn if i1 == up else up
            # particle-particle
            parts, d, e = _both(ed, X.PP, (i1, i1, i2, i2), freqs)
            if i1 == i2:
                assert not parts
            else:
                ref = np.array([g(3, st[i2], 0, -om(a), -om(b)) + g(3, st[i1], 0, -om(b), -om(a)) for a, b in grid])
                assert np.abs(d - ref).max() < 1e-14 and np.abs(e - ref).max() < 1e-13
            # particle-hole and crossed particle-hole
            if i1 == i2:
                ref = np.array([g(st[i1], 0, st[i1], -om(a), om(b)) + g(3, st[other], 3, -om(a), om(b))
                                for a, b in grid])
                refx = -ref
            else:
                s = st[i2]
                ref = np.array([g(3, s, 3, -om(a), om(b)) - g(s, 3, s, om(a), -om(b)) for a, b in grid])
                refx = np.array([-g(st[i1], 0, st[i2], -om(a), om(b)) - g(st[i1], 3, st[i2], om(b), -om(a))
                                 for a, b in grid])
            _, d, e = _both(ed, X.PH, (i1, i1, i2, i2), freqs)
            assert np.abs(d - ref).max() < 1e-13 and np.abs(e - ref).max() < 1e-13
            _, d, e = _both(ed, X.XPH, (i1, i1, i2, i2), freqs)
            assert np.abs(d - refx).max() < 1e-13 and np.abs(e - refx).max() < 1e-13


def test_chi3_crossing_symmetry():
    """chi3_xPH(1, 4, 3, 2) = -chi3_PH(1, 2, 3, 4) (3PSusc1siteTest.cpp:211-250)."""
    m = M.make_model(M.CoulombS("A", 1.0, -0.4) + M.Magnetization("A", -0.01))
    ed = EDm.ED(m, 10.0)
    ix = [m.info.getIndex("A", 0, M.UP), m.info.getIndex("A", 0, M.DOWN)]
    freqs = [(1j * np.pi * (2 * a + 1) / 10.0, 1j * np.pi * (2 * b + 1) / 10.0) for a in range(-3, 3)
             for b in range(-3, 3)]
    for a in ix:
        for b in ix:
            for c in ix:
                for d in ix:
                    _, ph, _ = _both(ed, X.PH, (a, b, c, d), freqs)
                    _, xph, _ = _both(ed, X.XPH, (a, d, c, b), freqs)
                    assert np.abs(xph + ph).max() < 1e-14


@pytest.mark.parametrize("channel", ["PP", "PH", "xPH"])
def test_chi3_three_site_golden(channel):
    k = KATS["chi3_3site"]
    e = M.Expr()
    for s in k["sites"]:
        e += M.CoulombS(s, k["U"], -k["mu"])
    for a, b in (("A", "B"), ("B", "C"), ("C", "A")):
        e += M.Hopping(a, b, -k["t"])
    m = M.make_model(e)
    ed = EDm.ED(m, k["beta"])
    spin = {"up": M.UP, "down": M.DOWN}
    ixs = [m.info.getIndex(s, 0, spin[sp]) for s, sp in k[channel]["ops"]]
    ch = {"PP": X.PP, "PH": X.PH, "xPH": X.XPH}[channel]
    freqs = [(1j * np.pi * (2 * a + 1) / k["beta"], 1j * np.pi * (2 * b + 1) / k["beta"]) for a in k["n"]
             for b in k["n"]]
    _, d, ex = _both(ed, ch, ixs, freqs)
    ref = cplx(k[channel]["chi3"])
    assert np.abs(d - ref).max() < k["tol"]
    assert np.abs(ex - ref).max() < k["tol"]
