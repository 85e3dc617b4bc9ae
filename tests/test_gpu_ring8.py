"""The Large configuration on the GPU: the 8-site Hubbard ring (dim 65536,
81 blocks up to 4900 states, beta = 5, truncateBlocks(1e-12)) through the C
ABI, against the oracle values committed in tests/golden/ring8_sample.json
(made by tests/golden/make_ring8.py with the numpy FP64 oracle).

  * G2 = chi_(u0,d0,u0,d0) at 64 triples of the 24^3 grid that include every
    resonant case (n1 + n2 = -1, n1 = n3, n2 = n3) and the grid's extreme
    frequencies, all 304 block chains: anchored sum with FP64 products, with
    the int8 split products (every product on the tensor cores), and with the
    anchor threshold of the benchmark, each within 1e-8 of max|G2| (the
    target of the Large configuration);
  * G_u0 on 256 fermionic and chi_zz on 48 bosonic frequencies at 1e-10.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import lehmann as L
from oracle import model as M

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "ring8_sample.json"


def _c(a):
    return np.array([complex(x, y) for x, y in a])


@pytest.fixture(scope="module")
def ring8():
    from tests.pgx_harness import GpuED
    doc = json.loads(GOLD.read_text())
    m = M.make_model(M.hubbard_ring())
    g = GpuED(m, 5.0)
    g.truncate(1e-12)
    yield g, m, doc
    g.eng.close()


def test_ring8_g_and_chi_zz(ring8):
    g, m, doc = ring8
    u, d = m.info.getIndex("S0", 0, 1), m.info.getIndex("S0", 0, 0)
    G = g.gf(g.c(u), g.cdag(u), L.fermionic(np.array(doc["g_u0_n"]), 5.0), coef_tol=0.0)
    ref = _c(doc["g_u0"])
    assert np.abs(G - ref).max() < 1e-10 * np.abs(ref).max()
    zb = L.bosonic(np.array(doc["chi_zz_m"]), 5.0)
    n = {i: g.quadratic(i, i) for i in (u, d)}
    chi = {(x, y): g.susc(n[x], n[y], zb, pole_res=1e-8, coef_tol=0.0)[0] for x in (u, d) for y in (u, d)}
    zz = 0.25 * (chi[(u, u)] - chi[(u, d)] - chi[(d, u)] + chi[(d, d)])
    ref = _c(doc["chi_zz"])
    assert np.abs(zz - ref).max() < 1e-10 * np.abs(ref).max()


@pytest.mark.parametrize("split,tol,slices,budget", [(False, 1e-16, 6, 0.0), (True, 1e-16, 6, 0.0), (True, 1e-13, 6, 0.0),
                                                     (True, 1e-13, 5, 0.0), (True, 1e-13, 5, 4.0)])
def test_ring8_g2_sample(ring8, split, tol, slices, budget):
    """Five base-254 digits per element leave about 250 times the product
    error of six; both stay far below 1e-8.  With the weight budget (the
    benchmark's setting: five digits, budget 4), products of anchor blocks
    whose largest Boltzmann weight is far below the dominant one run with
    fewer digits; the error stays within a few times that of five digits."""
    from pomerol_b200.pgx import PGX_G2_ANCHORED, PGX_G2_SPLIT_I8
    g, m, doc = ring8
    u, d = m.info.getIndex("S0", 0, 1), m.info.getIndex("S0", 0, 0)
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))
    assert len(parts) == doc["g2_parts"]
    fz = L.fermionic(np.array(doc["triples"]), 5.0)
    flags = PGX_G2_ANCHORED | (PGX_G2_SPLIT_I8 if split else 0)
    if split:
        g.eng.set_g2_split_threshold(0.0)  # every stacked and anchored product on the tensor cores
        g.eng.set_g2_split_slices(slices)
        g.eng.set_g2_split_weight_budget(budget)
    try:
        v = g.eng.g2(parts, fz, pole_res=1e-8, coef_tol=tol, flags=flags)
    finally:
        g.eng.set_g2_split_threshold(1e9)
        g.eng.set_g2_split_slices(6)
        g.eng.set_g2_split_weight_budget(4.0)
    ref = _c(doc["g2"])
    err = np.abs(v - ref).max() / np.abs(ref).max()
    print(f"ring8 G2 split={split} anchor_tol={tol:g} slices={slices} budget={budget:g}: max|diff|/max|G2| = {err:.2e}")
    assert err < 1e-8
    if not split:
        assert err < 1e-11  # FP64 products with the oracle's own anchor threshold


def test_ring8_count_dense_closed_form(ring8):
    """N_quad of the ring: every rotated element is non-zero at 1e-20, so the
    count takes the closed form (all quadruples minus those failing the weight
    filter); it must lie between the quadruples with a hot index1 or index3 and
    the total, and shrink when the weight threshold grows."""
    g, m, _ = ring8
    u, d = m.info.getIndex("S0", 0, 1), m.info.getIndex("S0", 0, 0)
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))
    n16 = g.eng.g2_count(parts, 1e-16, 1e-20)
    n12 = g.eng.g2_count(parts, 1e-12, 1e-20)
    dims = [len(b) for b in m.blocks]
    total = sum(int(np.prod([dims[b] for b in p[1]])) for p in parts)
    assert 0 < n12 < n16 <= total
