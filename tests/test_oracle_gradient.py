"""The FP64 reference gradient (oracle/gradient.py) against central finite
differences of the exact Green's function: the pin of the checker that
pgx_gf_vjp is compared with."""
import copy

import numpy as np
import pytest

from oracle import ed as EDm
from oracle import gradient as GR
from oracle import lehmann as L
from oracle import model as M


def _expr(p):
    e = M.CoulombS("C", p["U"], -p["mu"]) + M.Magnetization("C", p["h"])
    for k, (ek, vk) in enumerate(zip(p["eps"], p["V"])):
        e += M.Level(f"b{k}", ek) + M.Hopping("C", f"b{k}", vk)
    return e


def _shift(p, th, d):
    q = copy.deepcopy(p)
    if len(th) == 1:
        q[th[0]] += d
    else:
        q[th[0]][th[1]] += d
    return q


@pytest.mark.parametrize("field,offdiag", [(0.0, False), (0.15, True)])
def test_reference_gradient_against_finite_differences(field, offdiag):
    beta, h = 8.0, 1e-5
    p0 = {"U": 2.0, "mu": 0.9, "h": field, "eps": [-0.6, 0.35], "V": [0.45, 0.3]}
    m = M.make_model(_expr(p0))
    keys = list(m.expr.terms)
    i = m.info.getIndex("C", 0, M.DOWN)
    j = m.info.getIndex("b0", 0, M.DOWN) if offdiag else i
    z = 1j * np.pi * (2 * np.arange(12) + 1) / beta
    ed = EDm.ED(m, beta)
    G = GR.gf_exact(m, beta, i, j, z, ed)
    ref = L.gf_eval(L.gf_terms(ed, EDm.adjoint(ed.cdag(i)), ed.cdag(j), rule=False), z)
    assert np.abs(G - ref).max() < 1e-14
    rng = np.random.default_rng(4)
    lam = rng.standard_normal(len(z)) + 1j * rng.standard_normal(len(z))
    dterm, dE = GR.gf_term_gradient(m, beta, i, j, z, lam)
    assert abs(sum(e.sum() for e in dE)) < 1e-12  # G depends on energy differences only
    for th in [("U",), ("mu",), ("h",), ("eps", 0), ("eps", 1), ("V", 0), ("V", 1)]:
        qp, qm = _shift(p0, th, h), _shift(p0, th, -h)
        dc = (GR.term_coefficients(_expr(qp), keys) - GR.term_coefficients(_expr(qm), keys)) / (2 * h)
        Lp = np.real(lam @ GR.gf_exact(M.make_model(_expr(qp)), beta, i, j, z))
        Lm = np.real(lam @ GR.gf_exact(M.make_model(_expr(qm)), beta, i, j, z))
        fd = (Lp - Lm) / (2 * h)
        assert abs(dc @ dterm - fd) <= 1e-7 * max(1.0, abs(fd)), th


def test_kanamori_model_shape():
    U, J, eps, V, beta = M.kanamori_k_params(0)
    m = M.make_model(M.kanamori_k(U, J, eps, V))
    assert m.dim == 4096 and m.info.size() == 12
    assert not m.complex
