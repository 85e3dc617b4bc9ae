"""GPU parity through the C ABI (libpgx) against the CPU oracle and the
reference's known-answer tests.  Tolerances: eigen-residuals 1e-10 (as
HamiltonianTest.cpp:80-89), golden vectors at the reference tests' own
tolerances, and GPU-vs-oracle on the same inputs at 1e-10 relative (FP64)."""
import json
import os

import numpy as np
import pytest

from oracle import ed as EDm
from oracle import lehmann as L
from oracle import model as M

pytestmark = pytest.mark.gpu

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


@pytest.fixture(scope="module")
def harness():
    from tests.pgx_harness import GpuED
    return GpuED


def cplx(a):
    return np.array([complex(x, y) for x, y in a])


def plaquette_expr():
    k = KATS["gf4site"]
    e = M.Expr()
    for lab, U, eps in k["coulomb"]:
        e += M.CoulombS(lab, U, eps)
    for a, b, t in k["hopping"]:
        e += M.Hopping(a, b, t)
    return e


def test_eigh_residual_and_order(harness):
    m = M.make_model(plaquette_expr())
    g = harness(m, 10.0)
    for b in range(len(m.blocks)):
        h = m.h_block(b)
        E, U = g.E[b], g.U[b]
        assert np.all(np.diff(E) >= -1e-14)
        assert np.abs(h @ U - U * E[None, :]).max() < 1e-10
        assert np.abs(U.T @ U - np.eye(len(E))).max() < 1e-12
        assert np.abs(E - np.linalg.eigvalsh(h)).max() < 1e-11


def test_eigh_larger_blocks(harness):
    """Random symmetric blocks up to 300 with a degenerate spectrum."""
    rng = np.random.default_rng(7)
    dims = [1, 2, 3, 17, 64, 129, 300]
    blocks = []
    for d in dims:
        a = rng.standard_normal((d, d))
        h = (a + a.T) / 2
        if d == 129:   # exact degeneracies
            q, _ = np.linalg.qr(rng.standard_normal((d, d)))
            ev = np.repeat(np.arange(43.0), 3)
            h = (q * ev) @ q.T
        blocks.append(h)
    from pomerol_b200.pgx import Engine
    eng = Engine()
    eng.set_blocks(dims)
    eng.set_hamiltonian(blocks)
    eng.eigh()
    E, U = eng.eigensystem()
    for h, e, u in zip(blocks, E, U):
        scale = max(1.0, np.abs(e).max())
        assert np.abs(h @ u - u * e[None, :]).max() < 1e-10 * scale
        assert np.abs(u.T @ u - np.eye(len(e))).max() < 1e-11
        assert np.abs(e - np.linalg.eigvalsh(h)).max() < 1e-11 * scale


def test_eigh_every_householder_class():
    """One eigensolve whose blocks reach every Householder launch: thread-block
    clusters of 1, 2, 4 and 8 CTAs (the smallest that holds the block in
    distributed shared memory, up to 464 states), of 16 CTAs (465 to 513
    states) and the blocked large-block path (larger blocks).
    Spectra: random, tightly clustered (1e-9 spacings), two-level degenerate."""
    rng = np.random.default_rng(11)
    dims = [150, 200, 250, 256, 300, 401, 464, 465, 513, 514, 640]
    blocks = []
    for i, d in enumerate(dims):
        q, _ = np.linalg.qr(rng.standard_normal((d, d)))
        if i % 3 == 0:
            a = rng.standard_normal((d, d))
            h = (a + a.T) / 2
        elif i % 3 == 1:
            ev = np.r_[np.arange(d - 4) * 1e-9, [1.0, 2.0, 3.0, 4.0]]
            h = (q * ev) @ q.T
        else:
            ev = np.r_[np.zeros(d // 2), np.ones(d - d // 2)]
            h = (q * ev) @ q.T
        blocks.append((h + h.T) / 2)
    from pomerol_b200.pgx import Engine
    eng = Engine()
    eng.set_blocks(dims)
    eng.set_hamiltonian(blocks)
    eng.eigh()
    E, U = eng.eigensystem()
    for h, e, u in zip(blocks, E, U):
        scale = max(1.0, np.abs(e).max())
        assert np.all(np.diff(e) >= 0)
        assert np.abs(h @ u - u * e[None, :]).max() < 1e-10 * scale
        assert np.abs(u.T @ u - np.eye(len(e))).max() < 1e-11
        assert np.abs(e - np.linalg.eigvalsh(h)).max() < 1e-11 * scale


def test_eigh_large_blocks():
    """The blocked large-block path on blocks of 700, 1225 and 2100 states
    (random, tightly clustered and two-level degenerate spectra), next to
    small blocks on the cluster path, against LAPACK: residual, orthogonality
    and eigenvalues at 1e-10 / 1e-11 relative to the spectrum."""
    rng = np.random.default_rng(12)
    dims = [2100, 36, 1225, 700, 465]
    blocks = []
    for i, d in enumerate(dims):
        if i % 3 == 0:
            a = rng.standard_normal((d, d))
            h = (a + a.T) / 2
        else:
            q, _ = np.linalg.qr(rng.standard_normal((d, d)))
            ev = (np.r_[np.arange(d - 4) * 1e-9, [1.0, 2.0, 3.0, 4.0]] if i % 3 == 1
                  else np.r_[np.zeros(d // 2), np.ones(d - d // 2)])
            h = (q * ev) @ q.T
        blocks.append((h + h.T) / 2)
    from pomerol_b200.pgx import Engine
    eng = Engine()
    eng.set_blocks(dims)
    eng.set_hamiltonian(blocks)
    for _ in range(2):  # a second solve on the same context gives the same result
        eng.eigh()
        E, U = eng.eigensystem()
        for h, e, u in zip(blocks, E, U):
            scale = max(1.0, np.abs(e).max())
            assert np.all(np.diff(e) >= 0)
            assert np.abs(h @ u - u * e[None, :]).max() < 1e-10 * scale
            assert np.abs(u.T @ u - np.eye(len(e))).max() < 1e-11
            assert np.abs(e - np.linalg.eigvalsh(h)).max() < 1e-11 * scale


def test_hamiltonian_ground_energy(harness):
    e = M.CoulombS("A", 1.0, -0.5) + M.CoulombS("B", 2.0, -1.0) + M.Hopping("A", "B", -1.0)
    g = harness(M.make_model(e), 10.0)
    assert abs(min(x.min() for x in g.E) - KATS["hamiltonian"]["E0"]) < 1e-7


def test_weights_and_rotation_match_oracle(harness):
    m = M.make_model(plaquette_expr())
    g = harness(m, 10.0)
    ed = EDm.ED(m, 10.0)
    for b in range(len(m.blocks)):
        assert np.abs(g.w[b] - ed.w[b]).max() < 1e-13
    # rotation with the GPU's own eigenvectors (gauge fixed by the same U)
    ix = m.info.getIndex("A", 0, 0)
    op = g.cdag(ix)
    for k, (R, Lb) in enumerate(g.eng.op_info(op)):
        Lb2, tgt, sg = m.monomial_parts(((True, m.info.tuples[ix]),))[R]
        assert Lb2 == Lb
        G = np.zeros((len(m.blocks[Lb]), len(m.blocks[R])))
        ok = tgt >= 0
        np.add.at(G, tgt[ok], sg[ok, None] * g.U[R][ok, :])
        ref = g.U[Lb].T @ G
        assert np.abs(g.eng.op_read(op, k) - ref).max() < 1e-12
    c = g.c(ix)
    for k, (R, Lb) in enumerate(g.eng.op_info(c)):
        kk = [i for i, (r2, l2) in enumerate(g.eng.op_info(op)) if r2 == Lb][0]
        assert np.abs(g.eng.op_read(c, k) - g.eng.op_read(op, kk).T).max() == 0.0


def test_gf1site_closed_form(harness):
    U, mu, beta = 1.0, 0.4, 10.0
    m = M.make_model(M.CoulombS("A", U, -mu))
    g = harness(m, beta)
    dn = m.info.getIndex("A", 0, 0)
    n = np.arange(-100, 100)
    om = np.pi * (2 * n + 1) / beta
    w0, w1, w2 = 1.0, np.exp(beta * mu), np.exp(-beta * (-2 * mu + U))
    Z = w0 + 2 * w1 + w2
    ref = (w0 + w1) / Z / (1j * om + mu) + (w1 + w2) / Z / (1j * om + mu - U)
    v = g.gf(g.c(dn), g.cdag(dn), 1j * om)
    assert np.abs(v - ref).max() < 1e-14


def test_gf4site_golden(harness):
    k = KATS["gf4site"]
    m = M.make_model(plaquette_expr())
    g = harness(m, k["beta"])
    dn = m.info.getIndex("A", 0, 0)
    v = g.gf(g.c(dn), g.cdag(dn), L.fermionic(np.arange(10), k["beta"]))
    assert np.abs(v - cplx(k["G_A_down"])).max() < k["tol"]
    ed = EDm.ED(m, k["beta"])
    ref = L.gf_eval(L.gf_terms(ed, ed.c(dn), ed.cdag(dn), rule=False), L.fermionic(np.arange(256), k["beta"]))
    v = g.gf(g.c(dn), g.cdag(dn), L.fermionic(np.arange(256), k["beta"]), coef_tol=0.0)
    assert np.abs(v - ref).max() < 1e-12 * np.abs(ref).max()


def test_anderson_golden(harness):
    k = KATS["anderson"]
    U = k["U"]
    e = (M.CoulombS("C", U, -k["mu_over_U"] * U) + M.Magnetization("C", k["h"])
         + M.Level("0", -k["epsilon"]) + M.Level("1", k["epsilon"])
         + M.Hopping("C", "0", k["V"]) + M.Hopping("C", "1", k["V"]))
    m = M.make_model(e)
    g = harness(m, k["beta"])
    z = L.fermionic(np.arange(10), k["beta"])
    for s, key in ((1, "G_up"), (0, "G_down")):
        i = m.info.getIndex("C", 0, s)
        assert np.abs(g.gf(g.c(i), g.cdag(i), z) - cplx(k[key])).max() < k["tol"]


def test_susceptibility_closed_form(harness):
    U, mu, h, beta = 1.0, 0.4, 0.01, 10.0
    m = M.make_model(M.CoulombS("A", U, -mu) + M.Magnetization("A", -h))
    g = harness(m, beta)
    up, dn = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    sp, sm = g.quadratic(up, dn), g.quadratic(dn, up)
    nu, nd = g.quadratic(up, up), g.quadratic(dn, dn)
    wr = np.array([1.0, np.exp(-beta * (-mu - h)), np.exp(-beta * (-mu + h)), np.exp(-beta * (-2 * mu + U))])
    wr /= wr.sum()
    wu, wd, w2 = wr[1:]
    ea = g.eng.ensemble_average
    assert abs(ea(sp)) < 1e-14 and abs(ea(nu) - (wu + w2)) < 1e-14 and abs(ea(nd) - (wd + w2)) < 1e-14
    n = np.arange(20)
    z = L.bosonic(n, beta)
    om = 2 * np.pi * n / beta
    v, _ = g.susc(sp, sm, z)
    v = v - np.where(n == 0, ea(sp) * ea(sm) * beta, 0)
    assert np.abs(v - (-(wu - wd) / (1j * om - 2 * h))).max() < 1e-14
    v, _ = g.susc(nu, nu, z)
    v = v - np.where(n == 0, ea(nu) * ea(nu) * beta, 0)
    assert np.abs(v - np.where(n == 0, (wu + w2) * (1 - wu - w2) * beta, 0)).max() < 1e-14
    v, _ = g.susc(nu, nd, z)
    v = v - np.where(n == 0, ea(nu) * ea(nd) * beta, 0)
    assert np.abs(v - np.where(n == 0, (w2 - (wu + w2) * (wd + w2)) * beta, 0)).max() < 1e-14


def test_vertex4_closed_form(harness):
    from tests.test_oracle_golden import _vertex4_refs
    U, beta, n_iw = 1.0, 40.0, 4
    m = M.make_model(M.CoulombS("A", U, -U / 2))
    g = harness(m, beta)
    up, dn = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    GFv = {i: g.gf(g.c(i), g.cdag(i), L.fermionic(np.arange(-3 * n_iw, 3 * n_iw), beta)) for i in (up, dn)}
    GF = lambda i, n: GFv[i][n + 3 * n_iw]
    g_uuuu, g_udud, delta = _vertex4_refs(U, beta)
    trip = [(a, b, x) for a in range(-n_iw, n_iw) for b in range(-n_iw, n_iw) for x in range(-n_iw, n_iw)]
    fz = np.array([L.fermionic(np.array(t), beta) for t in trip])
    for (i, j, k, l), tol in (((up, up, up, up), 1e-6), ((up, dn, up, dn), 1e-10)):
        v, _ = g.g2(g.c(i), g.c(j), g.cdag(k), g.cdag(l), fz, pole_res=1e-4)
        for t, (n1, n2, n3) in enumerate(trip):
            n4 = n1 + n2 - n3
            if j == up:
                ref = (g_uuuu(n1, n2, n3) * GF(up, n1) * GF(up, n2) * GF(up, n3) * GF(up, n4)
                       + beta * GF(up, n1) * GF(up, n2) * delta(n1, n4) - beta * GF(up, n1) * GF(up, n2) * delta(n1, n3))
            else:
                ref = (g_udud(n1, n2, n3) * GF(up, n1) * GF(dn, n2) * GF(up, n3) * GF(dn, n4)
                       - beta * GF(up, n1) * GF(dn, n2) * delta(n1, n3))
            assert abs(v[t] - ref) < tol, (n1, n2, n3)


def test_anderson2pgf_golden(harness):
    from tests.test_oracle_golden import anderson2pgf_freqs, anderson2pgf_model
    k, e = anderson2pgf_model()
    m = M.make_model(e)
    g = harness(m, k["beta"])
    fz = np.array(anderson2pgf_freqs(k["beta"]))
    for s in (M.UP, M.DOWN):
        i = m.info.getIndex("C", 0, s)
        v, _ = g.g2(g.c(i), g.c(i), g.cdag(i), g.cdag(i), fz, pole_res=k["pole_resolution"])
        assert np.abs(v - np.array(k["chi_uuuu"])).max() < k["tol"]


def _anchored(g, parts, fz, tol=1e-16, pole_res=1e-8):
    from pomerol_b200.pgx import PGX_G2_ANCHORED
    return g.eng.g2(parts, fz, pole_res=pole_res, coef_tol=tol, flags=PGX_G2_ANCHORED)


def test_anchored_g2_vertex4_and_anderson2pgf(harness):
    """Weight-anchored sum reproduces the closed-form atom and the golden vector."""
    from tests.test_oracle_golden import anderson2pgf_freqs, anderson2pgf_model
    k, e = anderson2pgf_model()
    m = M.make_model(e)
    g = harness(m, k["beta"])
    fz = np.array(anderson2pgf_freqs(k["beta"]))
    i = m.info.getIndex("C", 0, M.UP)
    parts = g.g2_parts(g.c(i), g.c(i), g.cdag(i), g.cdag(i))
    v = _anchored(g, parts, fz, tol=1e-15, pole_res=k["pole_resolution"])
    assert np.abs(v - np.array(k["chi_uuuu"])).max() < k["tol"]
    exact = g.eng.g2(parts, fz, pole_res=k["pole_resolution"])
    assert np.abs(v - exact).max() < 1e-10 * np.abs(exact).max()


@pytest.mark.parametrize("beta", [2.0, 10.0])
def test_anchored_g2_plaquette_matches_exact_oracle(harness, beta):
    m = M.make_model(M.plaquette())
    g = harness(m, beta)
    ed = EDm.ED(m, beta)
    u, d = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    trip = [(a, b, x) for a in range(-4, 4) for b in range(-4, 4) for x in range(-4, 4)]
    fz = np.array([L.fermionic(np.array(t), beta) for t in trip])
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))
    v = _anchored(g, parts, fz)
    oparts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    sel = list(range(0, len(trip), 29))
    ref = L.g2_exact(ed, oparts, [tuple(fz[t]) for t in sel])
    assert np.abs(v[sel] - ref).max() < 1e-10 * np.abs(ref).max()
    # bosonic transfer 0 with equal energies exercises the delta branches
    assert np.abs(v - g.eng.g2(parts, fz)).max() < 1e-10 * np.abs(v).max()


@pytest.mark.parametrize("batch_bytes,chain_bytes", [(1, 1), (0, 1 << 20), (1 << 22, 300 << 10)])
def test_anchored_g2_tiles_match_untiled(harness, batch_bytes, chain_bytes):
    """Workspace limits small enough to batch one part at a time and to cut the
    (z1, z3) plane into tiles (1x1, and about 3x3 with ragged edges) give the
    untiled result up to the summation order, on an irregular triple list."""
    beta = 10.0
    m = M.make_model(M.plaquette())
    g = harness(m, beta)
    u, d = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    rng = np.random.default_rng(5)
    trip = [(a, b, x) for a in range(-5, 4) for b in range(-4, 4) for x in range(-3, 4)]
    trip = [trip[i] for i in sorted(rng.choice(len(trip), 300, replace=False))]
    fz = np.array([L.fermionic(np.array(t), beta) for t in trip])
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))
    v0 = _anchored(g, parts, fz)
    g.eng.set_g2_workspace(batch_bytes, chain_bytes)
    try:
        v1 = _anchored(g, parts, fz)
    finally:
        g.eng.set_g2_workspace(0, 0)
    assert np.abs(v1 - v0).max() < 1e-13 * np.abs(v0).max()


@pytest.mark.parametrize("pair", [False, True])
@pytest.mark.parametrize("M,N,K,nb", [(128, 64, 64, 1), (200, 150, 300, 2), (1000, 900, 2000, 3), (300, 140, 64, 1)])
def test_split_gemm_matches_fp64(M, N, K, nb, pair):
    """int8 tensor-core split product (balanced base-254 digits) against the
    FP64 product on seeded random complex matrices spread over four binary
    orders of magnitude, ragged tile edges included: six digits within 1e-12
    of max|C|, five within 1e-10 (and above six's error: the fifth digit pair
    diagonal is the last one kept), three between 1e-9 and 1e-4, which shows
    that every digit is used.  Both tile shapes: 128 x 256 on single CTAs,
    256 x 256 on CTA pairs (the exact int32 digit products and the same FP64
    summation order give the same result)."""
    from pomerol_b200.pgx import Engine
    eng = Engine()
    eng.set_split_cta_pair(pair)
    err6, _, _ = eng.split_gemm_check(M, N, K, nb, slices=6, seed=3)
    assert err6 < 1e-12
    err5, _, _ = eng.split_gemm_check(M, N, K, nb, slices=5, seed=3)
    assert err6 < err5 < 1e-10
    err3, _, _ = eng.split_gemm_check(M, N, K, nb, slices=3, seed=3)
    assert 1e-9 < err3 < 1e-4
    eng.set_split_cta_pair(not pair)
    assert eng.split_gemm_check(M, N, K, nb, slices=6, seed=3)[0] == err6


def test_anchored_g2_split_i8_anderson_a5(harness):
    """Anderson 1+5 (dim 4096, beta=20) on the 16^3 cube: the anchored G2 with
    every stacked and anchored product on the int8 tensor cores
    (PGX_G2_SPLIT_I8, threshold 0) against the FP64 anchored G2, within 1e-9
    of max|G2|."""
    from pomerol_b200.pgx import PGX_G2_ANCHORED, PGX_G2_SPLIT_I8
    U, epsd, eps, V, beta = M.anderson_a5_params(0)
    m = M.make_model(M.anderson(U, epsd, eps, V))
    g = harness(m, beta)
    u, d = m.info.getIndex("C", 0, 1), m.info.getIndex("C", 0, 0)
    n = np.arange(-8, 8)
    fz = L.fermionic(np.array([(a, b, x) for a in n for b in n for x in n]), beta)
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))
    v = _anchored(g, parts, fz)
    g.eng.set_g2_split_threshold(0.0)  # every stacked and anchored product on the tensor cores
    try:
        vs = g.eng.g2(parts, fz, pole_res=1e-8, coef_tol=1e-16, flags=PGX_G2_ANCHORED | PGX_G2_SPLIT_I8)
    finally:
        g.eng.set_g2_split_threshold(1e9)
    assert np.abs(vs - v).max() < 1e-9 * np.abs(v).max()


def test_anchored_g2_anderson_a5_subset(harness):
    """Anderson 1+5 (dim 4096, beta=20): anchored GPU sum vs the exact oracle
    on the largest block chains and a subset of the 16^3 cube."""
    U, epsd, eps, V, beta = M.anderson_a5_params(0)
    m = M.make_model(M.anderson(U, epsd, eps, V))
    g = harness(m, beta)
    ed = EDm.ED(m, beta)
    u, d = m.info.getIndex("C", 0, 1), m.info.getIndex("C", 0, 0)
    n = np.arange(-8, 8)
    trip = np.array([(a, b, x) for a in n for b in n for x in n])
    fz = L.fermionic(trip, beta)
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))
    v = _anchored(g, parts, fz)
    # dense GPU sum over every quadruple (exact mode) on the full cube
    vx = g.eng.g2(parts, fz)
    assert np.abs(v - vx).max() < 1e-9 * np.abs(vx).max()
    # exact oracle on a few triples, all chains: two ordinary ones, and two
    # resonant ones (n1 + n2 = -1 and n1 = n3; n2 = n3)
    oparts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    pick = [(-8, -8, -8), (7, 0, -3), (-1, 0, -1), (3, 5, 5)]
    sel = [int(np.flatnonzero((trip == np.array(t)).all(1))[0]) for t in pick]
    ref = L.g2_exact(ed, oparts, [tuple(fz[t]) for t in sel])
    assert np.abs(vx[sel] - ref).max() < 1e-9 * np.abs(ref).max()


def test_anchored_g2_anderson_a5_vs_anchored_oracle(harness):
    """Anderson 1+5 (dim 4096, beta=20), all 216 block chains, 64 triples
    (n1, n2, n3) in {-8, -1, 0, 7}^3, which hold every resonant case
    (n1 + n2 = -1, n1 = n3, n2 = n3) and the cube's extreme frequencies: the
    anchored GPU sum (FP64 products, and int8 split products) against the
    numpy anchored oracle at the same anchor threshold (1e-16): 1e-12 and
    1e-9 of max|G2|."""
    from oracle import g2_anchored as GA
    from pomerol_b200.pgx import PGX_G2_ANCHORED, PGX_G2_SPLIT_I8
    U, epsd, eps, V, beta = M.anderson_a5_params(0)
    m = M.make_model(M.anderson(U, epsd, eps, V))
    g = harness(m, beta)
    ed = EDm.ED(m, beta)
    u, d = m.info.getIndex("C", 0, 1), m.info.getIndex("C", 0, 0)
    S = (-8, -1, 0, 7)
    fz = L.fermionic(np.array([(a, b, x) for a in S for b in S for x in S]), beta)
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))
    oparts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    assert len(parts) == len(oparts) == 216
    ref = GA.g2_anchored(ed, oparts, fz, res=1e-8, anchor_tol=1e-16)
    v = _anchored(g, parts, fz)
    assert np.abs(v - ref).max() < 1e-12 * np.abs(ref).max()
    g.eng.set_g2_split_threshold(0.0)
    try:
        vs = g.eng.g2(parts, fz, pole_res=1e-8, coef_tol=1e-16, flags=PGX_G2_ANCHORED | PGX_G2_SPLIT_I8)
    finally:
        g.eng.set_g2_split_threshold(1e9)
    assert np.abs(vs - ref).max() < 1e-9 * np.abs(ref).max()


def test_g2_reference_rule_anderson_a5_small_chains(harness):
    """Anderson 1+5: the reference's own algorithm (oracle/g2_oracle.cpp,
    rule=1: sparse chase, weight filter, sub-term filters, TermList pole
    merging at PoleResolution 1e-8) on the 40 block chains with the fewest
    state quadruples, against the GPU sum of the same chains at 8 triples,
    resonant ones included.  These chains are cold (their G2 is about 5e-10),
    so the reference's absolute CoefficientTolerance (1e-16) filter drops a
    visible fraction of them: against the anchored sum at 1e-16 the stated
    tolerance is 1e-6 relative (the scale of the reference's own G2 test).
    With CoefficientTolerance 0 only the pole merge remains, and the exact
    GPU sum agrees to 1e-7 relative."""
    from oracle import g2c
    U, epsd, eps, V, beta = M.anderson_a5_params(0)
    m = M.make_model(M.anderson(U, epsd, eps, V))
    g = harness(m, beta)
    ed = EDm.ED(m, beta)
    u, d = m.info.getIndex("C", 0, 1), m.info.getIndex("C", 0, 0)
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))
    oparts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    size = [int(np.prod([len(ed.E[b]) for b in p["b"]])) for p in oparts]
    keep = [int(k) for k in np.argsort(size, kind="stable")[:40]]
    fz = L.fermionic(np.array([(-1, 0, -1), (3, -4, 2), (0, 0, 5), (-8, 7, 7), (5, 2, -6), (-3, 2, 4),
                               (1, 1, 1), (6, -7, -2)]), beta)
    sub, osub = [parts[k] for k in keep], [oparts[k] for k in keep]
    ref, nq, _ = g2c.evaluate(ed, osub, fz, pole_res=1e-8, coef_tol=1e-16, rule=True)
    assert nq > 0
    v = _anchored(g, sub, fz)
    assert np.abs(v - ref).max() < 1e-6 * np.abs(ref).max()
    ref0, _, _ = g2c.evaluate(ed, osub, fz, pole_res=1e-8, coef_tol=0.0, rule=True)
    vx = g.eng.g2(sub, fz)  # every quadruple, no filter
    assert np.abs(vx - ref0).max() < 1e-7 * np.abs(ref0).max()


@pytest.mark.parametrize("model", ["plaquette", "anderson3"])
@pytest.mark.parametrize("coef_tol,nz_tol", [(1e-16, 1e-20), (1e-16, 1e-12), (1e-4, 1e-20), (1e-3, 1e-12)])
def test_g2_count_matches_oracle(harness, model, coef_tol, nz_tol):
    """N_quad, the work unit of the G2 metric (pgx_g2_count: the closed form
    for chains without zero elements, the per-(i1, i3) kernel otherwise)
    against the oracle's enumeration of the reference's filter
    (TwoParticleGFPart.cpp:210-250) on the same rotated matrices and weights
    (read back from the device, since the count depends on the eigenbasis
    chosen inside degenerate subspaces): equal counts."""
    from types import SimpleNamespace

    from oracle import g2c
    if model == "plaquette":
        mdl, beta, site = M.make_model(M.plaquette()), 10.0, "A"
    else:
        U, epsd, eps, V, beta = M.anderson_a5_params(0)
        mdl, site = M.make_model(M.anderson(U, epsd, eps[:3], V[:3])), "C"
    g = harness(mdl, beta)
    u, d = mdl.info.getIndex(site, 0, 1), mdl.info.getIndex(site, 0, 0)
    parts = g.g2_parts(g.c(u), g.c(d), g.cdag(u), g.cdag(d))

    def mat(op, left):
        info = g.eng.op_info(op)
        k = next(i for i, (r, lb) in enumerate(info) if lb == left)
        return g.eng.op_read(op, k)

    oparts = [dict(b=b, O1=mat(ops[0], b[0]), O2=mat(ops[1], b[1]), O3=mat(ops[2], b[2]), CX4=mat(ops[3], b[3]),
                   perm=perm, sign=sign) for ops, b, perm, sign in parts]
    host = SimpleNamespace(E=g.E, w=g.w)
    n_gpu = g.eng.g2_count(parts, coef_tol, nz_tol)
    n_ref = g2c.count(host, oparts, coef_tol, nz_tol)
    assert n_gpu == n_ref > 0


def test_plaquette_g2_matches_oracle(harness):
    """Plaquette (t=1, U=4, mu=2, beta=10), chi_(u0,d0,u0,d0) on n in [-4,3]^3."""
    beta = 10.0
    m = M.make_model(M.plaquette())
    g = harness(m, beta)
    ed = EDm.ED(m, beta)
    u, d = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    trip = [(a, b, x) for a in range(-4, 4) for b in range(-4, 4) for x in range(-4, 4)]
    fz = np.array([L.fermionic(np.array(t), beta) for t in trip])
    v, parts = g.g2(g.c(u), g.c(d), g.cdag(u), g.cdag(d), fz)
    oparts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    assert len(parts) == len(oparts)
    sel = list(range(0, len(trip), 37))
    ref = L.g2_exact(ed, oparts, [tuple(fz[t]) for t in sel])
    assert np.abs(v[sel] - ref).max() < 1e-10 * np.abs(ref).max()


def test_device_reciprocal_error_bound():
    """The Newton-Raphson reciprocal of the Lehmann kernels against the
    correctly rounded 1/x: at most 2 ulp over 1e-40..1e40 (both the iterated
    range and the IEEE-division fallback outside [1e-30, 1e30])."""
    import ctypes
    from pomerol_b200 import pgx
    rng = np.random.default_rng(5)
    x = np.concatenate([10.0 ** rng.uniform(-40, 40, 200000), rng.uniform(0.5, 2.0, 50000),
                        np.array([1e-30 * (1 + 1e-15), 1e30 * (1 - 1e-15), 1.0, 3.0, 7.0])])
    out = np.empty_like(x)
    rc = pgx.load().pgx_recip_check(x.ctypes.data_as(ctypes.c_void_p), len(x), out.ctypes.data_as(ctypes.c_void_p))
    assert rc == pgx.PGX_OK
    ref = 1.0 / x
    ulp = np.abs(out - ref) / np.spacing(ref)
    assert ulp.max() <= 2.0


def _assembly_inputs(m):
    terms = [(tuple((dag, m.info.index[ix]) for dag, ix in mono), c) for mono, c in m.expr.terms.items()]
    fock = np.concatenate([np.asarray(b, dtype=np.uint64) for b in m.blocks])
    return terms, m.info.size(), fock, np.asarray(m.block_of), np.asarray(m.inner)


@pytest.mark.parametrize("name", ["plaquette", "anderson3", "complex_hopping"])
def test_device_hamiltonian_assembly(name):
    """pgx_assemble_hamiltonian against the oracle's block matrices
    (HamiltonianPart.cpp:56-76 semantics: <o|O_t|s> with Jordan-Wigner signs)."""
    from pomerol_b200.pgx import Engine
    if name == "plaquette":
        e = plaquette_expr()
    elif name == "anderson3":
        e = M.CoulombS("C", 2.0, -1.0) + M.Magnetization("C", 0.1)
        for k, (ek, vk) in enumerate([(-0.7, 0.4), (0.2, 0.3), (0.9, 0.5)]):
            e += M.Level(f"b{k}", ek) + M.Hopping("C", f"b{k}", vk)
    else:
        e = M.CoulombS("A", 1.0, -0.5) + M.CoulombS("B", 1.0, -0.5) + M.Hopping("A", "B", 0.3 + 0.4j)
    m = M.make_model(e)
    terms, nmodes, fock, sb, si = _assembly_inputs(m)
    eng = Engine()
    eng.set_blocks(m.block_sizes(), is_complex=m.complex)
    for _ in range(2):  # a second assembly on the same context starts from zero again
        eng.assemble_hamiltonian(terms, nmodes, fock, sb, si)
        got = eng.get_hamiltonian()
        for b in range(len(m.blocks)):
            ref = m.h_block(b)
            assert np.abs(got[b] - ref).max() <= 1e-14 * max(1.0, np.abs(ref).max())


def test_device_hamiltonian_assembly_rejects_bad_tables():
    from pomerol_b200.pgx import Engine, PgxError
    m = M.make_model(plaquette_expr())
    terms, nmodes, fock, sb, si = _assembly_inputs(m)
    eng = Engine()
    eng.set_blocks(m.block_sizes())
    bad = si.copy()
    bad[fock[0]] = (bad[fock[0]] + 1) % max(1, m.block_sizes()[sb[fock[0]]] + 1)
    with pytest.raises(PgxError):
        eng.assemble_hamiltonian(terms, nmodes, fock, sb, bad)
    with pytest.raises(PgxError):
        eng.assemble_hamiltonian([(((True, nmodes),), 1.0)], nmodes, fock, sb, si)


def test_host_side_failures_leave_the_context_usable():
    """Failures injected on the host, none of which reaches a kernel: a
    non-finite Hamiltonian entry (PGX_ERR_NUMERIC, nothing copied), a block
    of zero states (PGX_ERR_ARG), and a device allocation the GPU cannot
    satisfy (one block of 400000 states, 1.28 TB for its Hamiltonian alone:
    PGX_ERR_OOM, and no half-declared problem is left).  After each failure
    the same context diagonalises a small problem correctly."""
    from pomerol_b200.pgx import PGX_ERR_ARG, PGX_ERR_NUMERIC, PGX_ERR_OOM, PGX_ERR_STATE, Engine, PgxError
    rng = np.random.default_rng(11)
    a = rng.standard_normal((6, 6))
    h = (a + a.T) / 2
    eng = Engine()

    def solve_ok():
        eng.set_blocks([6])
        eng.set_hamiltonian([h])
        eng.eigh()
        (e,), _ = eng.eigensystem()
        assert np.abs(e - np.linalg.eigvalsh(h)).max() < 1e-12 * max(1.0, np.abs(e).max())

    for bad in (np.nan, np.inf):
        hb = h.copy()
        hb[2, 3] = hb[3, 2] = bad
        eng.set_blocks([6])
        with pytest.raises(PgxError) as ex:
            eng.set_hamiltonian([hb])
        assert ex.value.code == PGX_ERR_NUMERIC
        with pytest.raises(PgxError) as ex:
            eng.eigh()  # the refused upload left no Hamiltonian behind
        assert ex.value.code == PGX_ERR_STATE
        solve_ok()
    with pytest.raises(PgxError) as ex:
        eng.set_blocks([4, 0, 3])
    assert ex.value.code == PGX_ERR_ARG
    solve_ok()
    with pytest.raises(PgxError) as ex:
        eng.set_blocks([400000])
    assert ex.value.code == PGX_ERR_OOM
    with pytest.raises(PgxError) as ex:
        eng.set_hamiltonian([h])
    assert ex.value.code == PGX_ERR_STATE
    solve_ok()


def test_context_reused_across_problems_of_different_sizes():
    """pgx_set_blocks keeps a context's device buffers: a larger problem grows
    them, a smaller one reuses them; operator buffers of the previous problem
    are reused by the next one's operators."""
    from pomerol_b200.pgx import Engine
    rng = np.random.default_rng(3)
    eng = Engine()
    for dims in ([5, 40], [300, 7, 120], [3, 9]):
        blocks = []
        for d in dims:
            a = rng.standard_normal((d, d))
            blocks.append((a + a.T) / 2)
        eng.set_blocks(dims)
        eng.set_hamiltonian(blocks)
        eng.eigh()
        E, U = eng.eigensystem()
        for h, e, u in zip(blocks, E, U):
            scale = max(1.0, np.abs(e).max())
            assert np.abs(h @ u - u * e[None, :]).max() < 1e-10 * scale
            assert np.abs(e - np.linalg.eigvalsh(h)).max() < 1e-11 * scale
    from tests.pgx_harness import GpuED
    k = KATS["gf4site"]
    m = M.make_model(plaquette_expr())
    dn = m.info.getIndex("A", 0, 0)
    g = GpuED(m, k["beta"])
    for _ in range(3):  # the same context, problem set up again: operators reuse released buffers
        v = g.gf(g.c(dn), g.cdag(dn), L.fermionic(np.arange(10), k["beta"]))
        assert np.abs(v - cplx(k["G_A_down"])).max() < k["tol"]
        g.eng.set_blocks(m.block_sizes(), m.complex)
        g.eng.set_hamiltonian([m.h_block(b) for b in range(len(m.blocks))])
        g.eng.eigh()
        g.E, g.U = g.eng.eigensystem()
        g.w, g.Z = g.eng.weights(k["beta"])
        g._cdag, g._c = {}, {}


def test_released_operator_is_rejected_and_its_memory_reused(harness):
    from pomerol_b200.pgx import PgxError
    m = M.make_model(plaquette_expr())
    g = harness(m, 10.0)
    ix = m.info.getIndex("A", 0, 0)
    cd = g.cdag(ix)
    c1 = g.eng.op_adjoint(cd)
    ref = [g.eng.op_read(c1, k) for k in range(len(g.eng.op_info(c1)))]
    g.eng.op_release(c1)
    assert g.eng.op_info(c1) == []
    with pytest.raises(PgxError):
        g.eng.op_adjoint(c1)
    c2 = g.eng.op_adjoint(cd)  # takes the released buffers
    for k, r in enumerate(ref):
        assert np.array_equal(g.eng.op_read(c2, k), r)


def test_complex_hermitian_eigh():
    """Complex Hermitian blocks (real embedding of twice the size, complex
    eigenvectors formed from its pairs): random, exactly degenerate and
    near-degenerate spectra; residual, unitarity and eigenvalues."""
    from pomerol_b200.pgx import Engine
    rng = np.random.default_rng(21)
    dims = [1, 2, 5, 40, 120, 240]
    blocks = []
    for i, d in enumerate(dims):
        q, _ = np.linalg.qr(rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))
        if i == 3:
            ev = np.repeat(np.arange(d // 4 + 1, dtype=float), 4)[:d]
        elif i == 4:
            ev = np.r_[np.arange(d - 3) * 1e-9, [1.0, 2.0, 3.0]]
        else:
            a = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
            blocks.append((a + a.conj().T) / 2)
            continue
        h = (q * ev) @ q.conj().T
        blocks.append((h + h.conj().T) / 2)
    eng = Engine()
    eng.set_blocks(dims, is_complex=True)
    eng.set_hamiltonian(blocks)
    eng.eigh()
    E, U = eng.eigensystem()
    for h, e, u in zip(blocks, E, U):
        scale = max(1.0, np.abs(e).max())
        assert np.all(np.diff(e) >= 0)
        assert np.abs(h @ u - u * e[None, :]).max() < 1e-10 * scale
        assert np.abs(u.conj().T @ u - np.eye(len(e))).max() < 1e-11
        assert np.abs(e - np.linalg.eigvalsh(h)).max() < 1e-11 * scale


def _anderson_complex_gf(J, s1, s2, n, mu=1.2, U=2.0, beta=10.0):
    """Closed-form G_{s1 s2}(i w_n) of the atom CoulombS(U, -mu) with spin
    mixing J c+_up c_dn + h.c. (AndersonComplexTest.cpp:39-85): eigenstates
    0, (-mu -+ |J|), -2mu + U; the mixed components carry exp(+-i arg J)."""
    E = np.array([0.0, -mu - abs(J), -mu + abs(J), -2 * mu + U])
    w = np.exp(-beta * E)
    w /= w.sum()
    iw = 1j * np.pi * (2 * n + 1) / beta
    tr = [(1, 0, -1), (2, 0, 1), (3, 1, 1), (3, 2, -1)]  # (upper, lower, sign of the spin-mixed residue)
    res = 0
    for a, b, sg in tr:
        term = 0.5 * (w[a] + w[b]) / (iw - (E[a] - E[b]))
        if s1 == s2:
            res += term
        else:
            res += sg * np.exp(1j * np.angle(J) * (1 if s1 == M.UP else -1)) * term
    return res


@pytest.mark.parametrize("J", [0.1, -0.1, 0.1j, -0.1j, 0.1 + 0.1j, 0.1 - 0.1j, -0.1 + 0.1j, -0.1 - 0.1j])
def test_anderson_complex_closed_form(harness, J):
    """G of the bare Anderson atom with complex spin mixing (complex Hermitian
    H) against its closed form at 1e-12, as AndersonComplexTest.cpp:131-148."""
    mu, U, beta = 1.2, 2.0, 10.0
    m = M.make_model(M.CoulombS("C", U, -mu) + M.HoppingS("C", "C", J, 0, 0, M.UP, M.DOWN))
    assert m.complex == (complex(J).imag != 0)
    g = harness(m, beta)
    n = np.arange(10)
    z = 1j * np.pi * (2 * n + 1) / beta
    for s1 in (M.DOWN, M.UP):
        for s2 in (M.DOWN, M.UP):
            i1, i2 = m.info.getIndex("C", 0, s1), m.info.getIndex("C", 0, s2)
            v = g.gf(g.c(i1), g.cdag(i2), z)
            ref = np.array([_anderson_complex_gf(J, s1, s2, k) for k in n])
            assert np.abs(v - ref).max() < 1e-12


def _anderson_expr(p):
    """Anderson impurity C with bath sites b_k: U n_up n_dn - mu n + sum_k
    eps_k n_k + V_k (c+_C b_k + h.c.) (+ field h on C)."""
    e = M.CoulombS("C", p["U"], -p["mu"]) + M.Magnetization("C", p["h"])
    for k, (ek, vk) in enumerate(zip(p["eps"], p["V"])):
        e += M.Level(f"b{k}", ek) + M.Hopping("C", f"b{k}", vk)
    return e


def _term_coefs(p, keys):
    terms = M.make_model(_anderson_expr(p)).expr.terms
    assert set(terms) == set(keys)
    return np.array([complex(terms[k]).real for k in keys])


def _exact_gf(p, i, j, beta, z):
    """<c_i c+_j>(z) of the oracle's dense eigensolve (no term filtering)."""
    m = M.make_model(_anderson_expr(p))
    ed = EDm.ED(m, beta)
    return L.gf_eval(L.gf_terms(ed, EDm.adjoint(ed.cdag(i)), ed.cdag(j), rule=False), z)


@pytest.mark.parametrize("field,offdiag", [(0.0, False), (0.15, False), (0.15, True)])
def test_gf_vjp_against_finite_differences(field, offdiag):
    """pgx_gf_vjp: dL/dc_t of every assembled term, contracted with dc_t/dtheta
    for theta in (U, mu, eps_k, V_k, h), against central differences (step
    1e-5) of L(theta) evaluated with the oracle's exact G.  L = sum_n |G(z_n) -
    G_target(z_n)|^2 (lambda = 2 conj(G - G_target)) plus a random linear
    functional Re sum_n lambda'_n G(z_n); relative tolerance 1e-6."""
    from tests.pgx_harness import GpuED
    beta = 8.0
    p0 = {"U": 2.0, "mu": 0.9, "h": field, "eps": [-0.6, 0.35], "V": [0.45, 0.3]}
    m = M.make_model(_anderson_expr(p0))
    keys = list(m.expr.terms)
    terms, nmodes, fock, sb, si = _assembly_inputs(m)
    i = m.info.getIndex("C", 0, M.DOWN)
    j = m.info.getIndex("b0", 0, M.DOWN) if offdiag else i
    z = 1j * np.pi * (2 * np.arange(12) + 1) / beta
    g = GpuED(m, beta)
    g.eng.assemble_hamiltonian(terms, nmodes, fock, sb, si)
    g.eng.eigh()
    g.E, g.U = g.eng.eigensystem()
    g.w, g.Z = g.eng.weights(beta)
    op1, op2 = g.c(i), g.cdag(j)
    outer, inner = g.pair_parts(op1, op2)
    G = g.eng.gf(op1, op2, outer, inner, z, coef_tol=0.0)
    ref = _exact_gf(p0, i, j, beta, z)
    assert np.abs(G - ref).max() < 1e-12
    rng = np.random.default_rng(11)
    target = ref * (1 + 0.1 * rng.standard_normal(len(z))) + 0.01j
    lin = rng.standard_normal(len(z)) + 1j * rng.standard_normal(len(z))
    losses = {
        "squared": (lambda G: float(np.sum(np.abs(G - target) ** 2)), 2 * np.conj(G - target)),
        "linear": (lambda G: float(np.real(np.sum(lin * G))), lin),
    }
    h = 1e-5
    thetas = [("U",), ("mu",), ("h",), ("eps", 0), ("eps", 1), ("V", 0), ("V", 1)]

    def shifted(th, d):
        q = {k: (list(v) if isinstance(v, list) else v) for k, v in p0.items()}
        if len(th) == 1:
            q[th[0]] += d
        else:
            q[th[0]][th[1]] += d
        return q

    for name, (loss, lam) in losses.items():
        dterm, dE = g.eng.gf_vjp(op1, op2, outer, inner, z, lam)
        assert dterm.shape == (len(keys),) and dE.shape == (int(sum(m.block_sizes())),)
        assert abs(dE.sum()) < 1e-10 * max(1.0, np.abs(dE).max())  # G depends on energy differences only
        for th in thetas:
            if th == ("h",) and field == 0.0:
                continue
            qp, qm = shifted(th, h), shifted(th, -h)
            dc = (_term_coefs(qp, keys) - _term_coefs(qm, keys)) / (2 * h)
            got = float(dc @ dterm)
            fd = (loss(_exact_gf(qp, i, j, beta, z)) - loss(_exact_gf(qm, i, j, beta, z))) / (2 * h)
            assert abs(got - fd) <= 1e-6 * max(1.0, abs(fd)), (name, th, got, fd)


def _k_theta_coefs(keys, eps, V, U, J):
    from oracle import gradient as GR
    return GR.term_coefficients(M.kanamori_k(U, J, eps, V), keys)


def test_gf_vjp_kanamori_differentiation_workload():
    """Differentiation workload: two-orbital Kanamori impurity (U=2.5, J=0.4,
    U'=U-2J, half filling) with two bath sites per orbital (dim 4096),
    beta=30, L = sum_{n<512} |G_d0dn(i w_n) - G_target(i w_n)|^2, the target
    from the bath of seed 2.  The gradient of L with respect to the eight
    bath parameters and U, from pgx_gf_vjp through the torch.autograd wrapper
    of the test harness, against (1) the FP64 reference gradient of the oracle
    (1e-9 relative), (2) central differences (h=1e-6) of L evaluated with the
    GPU forward chain and (3) with the oracle's exact G (1e-6 relative)."""
    import torch
    from oracle import gradient as GR
    from tests.pgx_harness import GfTermChain, gf_of_terms
    U, J, eps, V, beta = M.kanamori_k_params(0)
    _, _, eps_t, V_t, _ = M.kanamori_k_params(2)
    m = M.make_model(M.kanamori_k(U, J, eps, V))
    keys = list(m.expr.terms)
    i = m.info.getIndex("d", 0, M.DOWN)
    z = 1j * np.pi * (2 * np.arange(512) + 1) / beta
    G_t = GR.gf_exact(M.make_model(M.kanamori_k(U, J, eps_t, V_t)), beta, i, i, z)
    theta0 = np.concatenate([eps, V, [U]])

    def coefs(th):
        return _k_theta_coefs(keys, th[0:4], th[4:8], th[8], J)

    # coefficients are linear in theta: the Jacobian from unit-sized differences is exact
    Jac = np.stack([(coefs(theta0 + 0.5 * e) - coefs(theta0 - 0.5 * e)) for e in np.eye(9)], axis=1)
    chain = GfTermChain(m, beta, i, i, z)
    Fn = gf_of_terms()
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    c0 = torch.from_numpy(coefs(theta0) - Jac @ theta0)
    G = Fn.apply(c0 + torch.from_numpy(Jac) @ theta, chain)
    loss = ((G - torch.from_numpy(G_t)).abs() ** 2).sum()
    loss.backward()
    grad = theta.grad.numpy()
    # (1) the FP64 reference gradient
    G_ref = GR.gf_exact(m, beta, i, i, z)
    assert np.abs(G.detach().numpy() - G_ref).max() < 1e-11
    dterm_ref, _ = GR.gf_term_gradient(m, beta, i, i, z, 2 * np.conj(G_ref - G_t))
    ref = Jac.T @ dterm_ref
    assert np.abs(grad - ref).max() <= 1e-9 * np.abs(ref).max(), (grad, ref)
    # timing of one gradient call (device time between events on the context's stream)
    lam = 2 * np.conj(G.detach().numpy() - G_t)
    chain.vjp(lam)
    chain.eng.profile_begin()
    chain.eng.timer_begin()
    chain.vjp(lam)
    ms = chain.eng.timer_end()
    prof = chain.eng.profile_end()
    print(f"\npgx_gf_vjp Kanamori dim 4096, 512 frequencies: {ms:.3f} ms device time")
    for k in prof:
        print(f"  {k['name']:<40s} {k['launches']:3d} launches {k['ms']:8.3f} ms")

    def loss_gpu(th):
        return float(np.sum(np.abs(chain.forward(coefs(th)) - G_t) ** 2))

    def loss_oracle(th):
        mm = M.make_model(M.kanamori_k(th[8], J, th[0:4], th[4:8]))
        return float(np.sum(np.abs(GR.gf_exact(mm, beta, i, i, z) - G_t) ** 2))

    h = 1e-6
    for k in range(9):
        e = np.eye(9)[k] * h
        fd = (loss_gpu(theta0 + e) - loss_gpu(theta0 - e)) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-6 * max(1.0, abs(fd)), (k, grad[k], fd)
    for k in (0, 5, 8):  # one bath energy, one hybridisation, U
        e = np.eye(9)[k] * h
        fd = (loss_oracle(theta0 + e) - loss_oracle(theta0 - e)) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-6 * max(1.0, abs(fd)), (k, grad[k], fd)


@pytest.mark.parametrize("channel", ["PP", "PH", "xPH"])
def test_chi3_three_site_golden(harness, channel):
    """pgx_chi3 on the reference's three-site cluster (3PSusc3siteTest.cpp:24-157):
    golden values at 1e-10 and the exact oracle at 1e-12."""
    from oracle import chi3 as X
    k = KATS["chi3_3site"]
    e = M.Expr()
    for s in k["sites"]:
        e += M.CoulombS(s, k["U"], -k["mu"])
    for a, b in (("A", "B"), ("B", "C"), ("C", "A")):
        e += M.Hopping(a, b, -k["t"])
    m = M.make_model(e)
    g = harness(m, k["beta"])
    spin = {"up": M.UP, "down": M.DOWN}
    ixs = [m.info.getIndex(s, 0, spin[sp]) for s, sp in k[channel]["ops"]]
    ch = {"PP": X.PP, "PH": X.PH, "xPH": X.XPH}[channel]
    freqs = [(L.fermionic(a, k["beta"]), L.fermionic(b, k["beta"])) for a in k["n"] for b in k["n"]]
    v, parts = g.chi3(ch, ixs, freqs)
    assert np.abs(v - cplx(k[channel]["chi3"])).max() < k["tol"]
    ed = EDm.ED(m, k["beta"])
    oparts = X.chi3_parts(ed, ch, ed.cdag(ixs[0]), ed.c(ixs[1]), ed.cdag(ixs[2]), ed.c(ixs[3]))
    assert len(parts) == len(oparts)
    assert np.abs(v - X.chi3_exact(ed, oparts, ch, freqs)).max() < 1e-12


@pytest.mark.parametrize("h", [0.0, 0.01])
def test_chi3_hubbard_atom_closed_form(harness, h):
    """All channels and spin combinations of the Hubbard atom against its
    closed form (3PSusc1siteTest.cpp:38-209), including the resonant
    beta delta at z1 = -xi z2, on a 12 x 12 grid."""
    from oracle import chi3 as X
    from tests.test_oracle_chi3 import AtomChi3
    U, mu, beta, n_iw = 1.0, 0.4, 10.0, 6
    m = M.make_model(M.CoulombS("A", U, -mu) + M.Magnetization("A", -h))
    g = harness(m, beta)
    up, dn = m.info.getIndex("A", 0, M.UP), m.info.getIndex("A", 0, M.DOWN)
    ga = AtomChi3(beta, U, mu, h)
    st = {up: 1, dn: 2}
    om = lambda n: np.pi * (2 * n + 1) / beta
    grid = [(a, b) for a in range(-n_iw, n_iw) for b in range(-n_iw, n_iw)]
    freqs = [(1j * om(a), 1j * om(b)) for a, b in grid]
    for i1 in (up, dn):
        for i2 in (up, dn):
            other = dn if i1 == up else up
            v, parts = g.chi3(X.PP, (i1, i1, i2, i2), freqs)
            if i1 == i2:
                assert not parts and np.all(v == 0)
            else:
                ref = np.array([ga(3, st[i2], 0, -om(a), -om(b)) + ga(3, st[i1], 0, -om(b), -om(a)) for a, b in grid])
                assert np.abs(v - ref).max() < 1e-13
            if i1 == i2:
                ref = np.array([ga(st[i1], 0, st[i1], -om(a), om(b)) + ga(3, st[other], 3, -om(a), om(b))
                                for a, b in grid])
                refx = -ref
            else:
                s = st[i2]
                ref = np.array([ga(3, s, 3, -om(a), om(b)) - ga(s, 3, s, om(a), -om(b)) for a, b in grid])
                refx = np.array([-ga(st[i1], 0, st[i2], -om(a), om(b)) - ga(st[i1], 3, st[i2], om(b), -om(a))
                                 for a, b in grid])
            v, _ = g.chi3(X.PH, (i1, i1, i2, i2), freqs)
            assert np.abs(v - ref).max() < 1e-13
            v, _ = g.chi3(X.XPH, (i1, i1, i2, i2), freqs)
            assert np.abs(v - refx).max() < 1e-13


@pytest.mark.parametrize("complex_h", [False, True])
def test_chi3_random_duplets_against_exact_oracle(harness, complex_h):
    """Anderson impurity with three bath sites (real, or with a complex
    hopping): every channel for several operator quadruples on a list of
    duplets that repeats values, contains the resonant z1 = -xi z2 pairs and
    off-axis complex frequencies, against the exact oracle (1e-11 relative)."""
    from oracle import chi3 as X
    beta = 6.0
    e = M.CoulombS("C", 2.2, -1.1) + M.Magnetization("C", 0.07)
    for k, (ek, vk) in enumerate([(-0.8, 0.5), (0.3, 0.35), (1.1, 0.6)]):
        e += M.Level(f"b{k}", ek) + M.Hopping("C", f"b{k}", vk)
    if complex_h:
        e += M.HoppingS("b0", "b1", 0.2 + 0.15j, 0, 0, M.UP, M.UP) + M.HoppingS("b0", "b1", 0.2 + 0.15j, 0, 0,
                                                                                  M.DOWN, M.DOWN)
    m = M.make_model(e)
    assert m.complex == complex_h
    g = harness(m, beta)
    ed = EDm.ED(m, beta)
    rng = np.random.default_rng(7)
    n = rng.integers(-5, 5, size=(40, 2))
    freqs = [(L.fermionic(a, beta), L.fermionic(b, beta)) for a, b in n]
    freqs += [(L.fermionic(a, beta), L.fermionic(-a - 1, beta)) for a in range(-3, 3)]   # z1 + z2 = 0
    freqs += [(L.fermionic(a, beta), L.fermionic(a, beta)) for a in range(-3, 3)]        # z1 - z2 = 0
    freqs += [(0.3 + 0.7j, -0.2 + 1.1j), (1.5 + 0.2j, 0.4 - 0.9j)]
    freqs += freqs[:5]
    up, dn = M.UP, M.DOWN
    c0 = lambda s: m.info.getIndex("C", 0, s)
    b0 = lambda s: m.info.getIndex("b0", 0, s)
    for ixs in [(c0(up), c0(up), c0(dn), c0(dn)), (c0(up), b0(up), c0(dn), b0(dn)), (c0(up), c0(dn), c0(dn), c0(up))]:
        for ch in (X.PP, X.PH, X.XPH):
            v, parts = g.chi3(ch, ixs, freqs)
            oparts = X.chi3_parts(ed, ch, ed.cdag(ixs[0]), ed.c(ixs[1]), ed.cdag(ixs[2]), ed.c(ixs[3]))
            assert len(parts) == len(oparts)
            ref = X.chi3_exact(ed, oparts, ch, freqs)
            assert np.abs(v - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max()), (ixs, ch)


def test_chi3_anderson5_workload_sample(harness):
    """chi3_PH(u0, u0, d0, d0) of the Anderson impurity with five bath sites
    (dim 4096, 72 parts, blocks up to 400) on the 16 x 16 fermionic square:
    three duplets, one of them resonant (z1 = z2), against the exact oracle
    (1e-10 relative), and the crossing symmetry chi3_xPH(1, 4, 3, 2) =
    -chi3_PH(1, 2, 3, 4) on the whole square (1e-12 relative)."""
    from oracle import chi3 as X
    U, epsd, eps, V, beta = M.anderson_a5_params(0)
    m = M.make_model(M.anderson(U, epsd, eps, V))
    g = harness(m, beta)
    u0, d0 = m.info.getIndex("C", 0, M.UP), m.info.getIndex("C", 0, M.DOWN)
    n = np.arange(-8, 8)
    freqs = [(L.fermionic(a, beta), L.fermionic(b, beta)) for a in n for b in n]
    v, parts = g.chi3(X.PH, (u0, u0, d0, d0), freqs)
    assert len(parts) == 72
    vx, _ = g.chi3(X.XPH, (u0, d0, d0, u0), freqs)
    assert np.abs(vx + v).max() <= 1e-12 * np.abs(v).max()
    ed = EDm.ED(m, beta)
    oparts = X.chi3_parts(ed, X.PH, ed.cdag(u0), ed.c(u0), ed.cdag(d0), ed.c(d0))
    sample = [freqs.index((L.fermionic(a, beta), L.fermionic(b, beta))) for a, b in ((1, 2), (-3, -3), (5, -8))]
    ref = X.chi3_exact(ed, oparts, X.PH, [freqs[q] for q in sample])
    assert np.abs(v[sample] - ref).max() <= 1e-10 * np.abs(ref).max()


def test_batch_of_models_against_oracle():
    """The batch workload's engine path (one context, blocks of every model
    in one eigensolve, per-model weights and frequencies) on all 64 models of
    the draw (3-6 bath sites, dims 256-16384, beta 5-50):
    G_dn on 64 fermionic and chi_dd on 8 bosonic frequencies of every model
    against the oracle's exact sums (1e-11 / 1e-10 relative); a second step
    on the same context reproduces the first up to the order of the
    evaluation's atomic accumulation (1e-13 relative)."""
    from pomerol_b200.workloads import BatchRun, b64_params
    params = b64_params()
    run = BatchRun(params, nG=64, nchi=8)
    G, X = run.step()
    G2, X2 = run.step()
    assert np.abs(G - G2).max() <= 1e-13 * np.abs(G).max() and np.abs(X - X2).max() <= 1e-13 * np.abs(X).max()
    for m, (U, epsd, eps, V, beta) in enumerate(params):
        mdl = M.make_model(M.anderson(U, epsd, eps, V))
        ed = EDm.ED(mdl, beta)
        up, dn = mdl.info.getIndex("C", 0, M.UP), mdl.info.getIndex("C", 0, M.DOWN)
        gref = L.gf_eval(L.gf_terms(ed, ed.c(dn), ed.cdag(dn), rule=False), run.zG[m])
        assert np.abs(G[m] - gref).max() <= 1e-11 * np.abs(gref).max(), m
        nu, ndn = ed.quadratic(up, up), ed.quadratic(dn, dn)
        nd = {}
        for R in set(nu) | set(ndn):
            Lb = (nu.get(R) or ndn.get(R))[0]
            mats = [o[R][1] for o in (nu, ndn) if R in o]
            nd[R] = (Lb, sum(mats))
        xref = L.susc_eval(L.susc_terms(ed, nd, nd, rule=False), run.zX[m], beta)
        assert np.abs(X[m] - xref).max() <= 1e-10 * np.abs(xref).max(), m


def test_eigensystem_checkpoint_reload(harness, tmp_path):
    """Eigendata checkpoint: the eigensystem saved from one context and
    loaded into a fresh one (pgx_set_eigensystem, no eigensolve) gives the
    same G as the solved context; a checkpoint of other blocks is refused."""
    from pomerol_b200.pgx import Engine, PgxError
    m = M.make_model(plaquette_expr())
    g = harness(m, 10.0)
    ix = m.info.getIndex("A", 0, M.DOWN)
    z = L.fermionic(np.arange(32), 10.0)
    ref = g.gf(g.c(ix), g.cdag(ix), z)
    path = str(tmp_path / "eig.npz")
    g.eng.save_eigensystem(path)
    from tests.pgx_harness import GpuED
    h = GpuED.__new__(GpuED)
    h.m, h.beta, h.eng = m, 10.0, Engine()
    h.eng.set_blocks(m.block_sizes(), m.complex)
    h.eng.load_eigensystem(path)
    h.E, h.U = h.eng.eigensystem()
    h.w, h.Z = h.eng.weights(10.0)
    h.retained = np.ones(len(m.blocks), dtype=bool)
    h._cdag, h._c = {}, {}
    v = h.gf(h.c(ix), h.cdag(ix), z)
    assert np.abs(v - ref).max() < 1e-15
    other = Engine()
    other.set_blocks([3, 5])
    with pytest.raises(ValueError):
        other.load_eigensystem(path)
    with pytest.raises(PgxError):
        other.set_eigensystem([np.array([2.0, 1.0, 0.0]), np.zeros(5)], [np.eye(3), np.eye(5)])


@pytest.mark.parametrize("same", [True, False])
def test_susc_vjp_against_finite_differences(same):
    """pgx_susc_vjp: the gradient of L = Re sum_m lambda_m chi_{n_i n_j}(i Omega_m)
    on 8 bosonic frequencies (Omega_0 = 0 carries the zero-pole terms) with
    respect to (U, mu, h, eps_k, V_k), against central differences (step
    1e-5) of the oracle's exact chi; relative tolerance 1e-6."""
    from tests.pgx_harness import GpuED
    beta = 8.0
    p0 = {"U": 2.0, "mu": 0.9, "h": 0.15, "eps": [-0.6, 0.35], "V": [0.45, 0.3]}
    m = M.make_model(_anderson_expr(p0))
    keys = list(m.expr.terms)
    terms, nmodes, fock, sb, si = _assembly_inputs(m)
    i = m.info.getIndex("C", 0, M.DOWN)
    j = i if same else m.info.getIndex("C", 0, M.UP)
    z = 2j * np.pi * np.arange(8) / beta
    g = GpuED(m, beta)
    g.eng.assemble_hamiltonian(terms, nmodes, fock, sb, si)
    g.eng.eigh()
    g.E, g.U = g.eng.eigensystem()
    g.w, g.Z = g.eng.weights(beta)
    A = g.quadratic(i, i)
    B = A if same else g.quadratic(j, j)
    outer, inner = g.pair_parts(A, B)

    def chi_oracle(p):
        mm = M.make_model(_anderson_expr(p))
        ed = EDm.ED(mm, beta)
        return L.susc_eval(L.susc_terms(ed, ed.quadratic(i, i), ed.quadratic(j, j), rule=False), z, beta)

    ref = chi_oracle(p0)
    X, _ = g.eng.susc(A, B, outer, inner, z, beta, pole_res=1e-8, coef_tol=0.0)
    assert np.abs(X - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
    rng = np.random.default_rng(21)
    lam = rng.standard_normal(len(z)) + 1j * rng.standard_normal(len(z))
    dterm, dE = g.eng.susc_vjp(A, B, outer, inner, z, lam, pole_res=1e-8)
    assert abs(dE.sum()) < 1e-10 * max(1.0, np.abs(dE).max())
    h = 1e-5
    for th in [("U",), ("mu",), ("h",), ("eps", 0), ("eps", 1), ("V", 0), ("V", 1)]:
        qp = {k: (list(v) if isinstance(v, list) else v) for k, v in p0.items()}
        qm = {k: (list(v) if isinstance(v, list) else v) for k, v in p0.items()}
        if len(th) == 1:
            qp[th[0]] += h
            qm[th[0]] -= h
        else:
            qp[th[0]][th[1]] += h
            qm[th[0]][th[1]] -= h
        dc = (_term_coefs(qp, keys) - _term_coefs(qm, keys)) / (2 * h)
        fd = (np.real(lam @ chi_oracle(qp)) - np.real(lam @ chi_oracle(qm))) / (2 * h)
        got = float(dc @ dterm)
        assert abs(got - fd) <= 1e-6 * max(1.0, abs(fd)), (th, got, fd)


def test_graph_capture_and_replay(harness):
    """pgx_graph_begin / end / replay: a captured [eigh, rotate c+] replayed on
    new block Hamiltonians gives the eigensystem and rotated operator of the
    direct calls (the same kernels in the same order: equal to 1e-15);
    entry points that cannot be captured are refused during the capture, and
    the graph refuses to replay once an operator was defined after it."""
    from pomerol_b200.pgx import PgxError
    m = M.make_model(plaquette_expr())
    g = harness(m, 10.0)
    ix = m.info.getIndex("A", 0, M.DOWN)
    op = g.cdag(ix)
    eng = g.eng
    eng.graph_begin()
    eng.eigh()
    with pytest.raises(PgxError):
        eng.weights(10.0)
    eng.op_rotate(op)
    gid = eng.graph_end()
    rng = np.random.default_rng(3)
    blocks2 = []
    for b in range(len(m.blocks)):
        h = m.h_block(b)
        blocks2.append(1.7 * h + 0.2 * np.eye(len(h)) + 1e-3 * (lambda a: a + a.T)(rng.standard_normal(h.shape)))
    eng.set_hamiltonian(blocks2)
    eng.graph_replay(gid)
    E1, U1 = eng.eigensystem()
    parts1 = [eng.op_read(op, k) for k in range(len(eng.op_info(op)))]
    for h, e in zip(blocks2, E1):
        assert np.abs(e - np.linalg.eigvalsh(h)).max() < 1e-12 * max(1.0, np.abs(e).max())
    eng.eigh()
    eng.op_rotate(op)
    E2, U2 = eng.eigensystem()
    parts2 = [eng.op_read(op, k) for k in range(len(eng.op_info(op)))]
    assert max(np.abs(a - b).max() for a, b in zip(E1, E2)) < 1e-15
    assert max(np.abs(a - b).max() for a, b in zip(U1, U2)) < 1e-15
    assert max(np.abs(a - b).max() for a, b in zip(parts1, parts2)) < 1e-15
    eng.graph_replay(gid)  # a second replay is fine
    g.cdag(m.info.getIndex("B", 0, M.UP))  # defines a new operator
    with pytest.raises(PgxError):
        eng.graph_replay(gid)
    eng.graph_destroy(gid)


def test_autotune_keeps_results(harness):
    """pgx_autotune_begin / end time the GEMM products of an eigensolve and a
    plaquette G2 in every tile class on this GPU; the G2 measured meanwhile
    and the tuned
    context's eigensystem and G2 agree with the untuned ones (different tile
    shapes change only the summation order: 1e-13)."""
    beta = 10.0
    m = M.make_model(M.plaquette())
    g = harness(m, beta)
    u, d = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    trip = [(a, b, x) for a in range(-2, 2) for b in range(-2, 2) for x in range(-2, 2)]
    fz = np.array([L.fermionic(np.array(t), beta) for t in trip])
    v0, _ = g.g2(g.c(u), g.c(d), g.cdag(u), g.cdag(d), fz)
    E0, U0 = g.eng.eigensystem()
    g.eng.autotune_begin()
    g.eng.eigh()
    g.w, g.Z = g.eng.weights(beta)
    g._cdag, g._c = {}, {}  # rotated again, under measurement
    vr, _ = g.g2(g.c(u), g.c(d), g.cdag(u), g.cdag(d), fz)
    changed = g.eng.autotune_end()
    assert np.abs(vr - v0).max() < 1e-13 * np.abs(v0).max()  # measuring leaves the real launches alone
    assert changed >= 0
    g.eng.eigh()
    E1, U1 = g.eng.eigensystem()
    assert max(np.abs(a - b).max() for a, b in zip(E0, E1)) < 1e-13
    g.E, g.U = E1, U1
    g.w, g.Z = g.eng.weights(beta)
    g._cdag, g._c = {}, {}
    v1, _ = g.g2(g.c(u), g.c(d), g.cdag(u), g.cdag(d), fz)
    assert np.abs(v1 - v0).max() < 1e-13 * np.abs(v0).max()
