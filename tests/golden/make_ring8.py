"""Generate tests/golden/ring8_sample.json: oracle values of the 8-site
Hubbard ring (the Large configuration) at a fixed sample, for the GPU parity
tests of that configuration.

Model: 8 sites with periodic boundaries, Hopping(t = -1) between i and
i + 1 mod 8, CoulombS(U = 4, eps = -mu = -2) on every site, beta = 5,
DensityMatrix::truncateBlocks(1e-12); dimension 65536 in 81 blocks.

Values (all from the numpy FP64 oracle in oracle/, nothing from the GPU):
  * G2 = chi_(u0,d0,u0,d0) (c_up c_dn c^+_up c^+_dn at site 0, the index
    order of pomerol's IndexCombination4) at the 64 fermionic triples
    (n1, n2, n3) in S^3 with S = {-12, -1, 0, 11}.  The set holds every
    resonant case of the sum: n1 + n2 = -1 (bosonic z1 + z2 = 0), n1 = n3 and
    n2 = n3, and the extreme frequencies of the 24^3 grid.  Every block chain
    of TwoParticleGF::prepare is summed by oracle.g2_anchored with anchor
    threshold 1e-16 (states of weight <= 1e-16 carry at most 4.9e-14 of the
    total weight, so the dropped part is below 1e-12 of max|G2|);
  * G_u0(i w_n) = <c_up0 c^+_up0> on n = 0..255 (exact, no filters);
  * chi_zz(i W_m) = (chi_nu,nu - chi_nu,nd - chi_nd,nu + chi_nd,nd) / 4 at
    site 0 on m = 0..47 (exact, no filters, disconnected part not removed;
    it cancels in this combination).

Run from the repository root (about half an hour on 8 cores):

    python tests/golden/make_ring8.py
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ed as EDm  # noqa: E402
from oracle import g2_anchored as GA  # noqa: E402
from oracle import lehmann as L  # noqa: E402
from oracle import model as M  # noqa: E402

OUT = Path(__file__).resolve().parent / "ring8_sample.json"
BETA, DM_TRUNC, ANCHOR_TOL, POLE_RES = 5.0, 1e-12, 1e-16, 1e-8
S = (-12, -1, 0, 11)
TRIPLES = [(a, b, c) for a in S for b in S for c in S]

_ED = None
_PARTS = None


def _part_value(k):
    from threadpoolctl import threadpool_limits
    with threadpool_limits(1):
        fz = [tuple(L.fermionic(np.array(t), BETA)) for t in TRIPLES]
        return k, GA.g2_part_anchored(_ED, _PARTS[k], fz, POLE_RES, ANCHOR_TOL)


def _chunked_eval(R, P, z, sign):
    """sum_t sign * R_t / (z - P_t) in chunks of terms (memory bound)."""
    out = np.zeros(len(z), dtype=complex)
    for i in range(0, len(R), 1 << 16):
        r, p = R[i:i + (1 << 16)], P[i:i + (1 << 16)]
        out += sign * (r[None, :] / (z[:, None] - p[None, :])).sum(1)
    return out


def main():
    global _ED, _PARTS
    t0 = time.time()
    m = M.make_model(M.hubbard_ring())
    ed = EDm.ED(m, BETA)
    ed.truncate_blocks(DM_TRUNC)
    u, d = m.info.getIndex("S0", 0, 1), m.info.getIndex("S0", 0, 0)
    print(f"ED: {time.time() - t0:.1f} s", flush=True)
    # G_u0 and chi_zz (exact term lists, evaluated in chunks)
    zf = L.fermionic(np.arange(256), BETA)
    R, P = L.gf_terms(ed, ed.c(u), ed.cdag(u), rule=False)
    G = _chunked_eval(R, P, zf, 1.0)
    zb = L.bosonic(np.arange(48), BETA)
    nn = {i: ed.quadratic(i, i) for i in (u, d)}
    chi = {}
    for x in (u, d):
        for y in (u, d):
            R, P, zero = L.susc_terms(ed, nn[x], nn[y], rule=False)
            v = _chunked_eval(R, P, zb, -1.0)
            v[0] += BETA * zero
            chi[(x, y)] = v
    zz = 0.25 * (chi[(u, u)] - chi[(u, d)] - chi[(d, u)] + chi[(d, d)])
    print(f"G, chi_zz: {time.time() - t0:.1f} s", flush=True)
    # G2 over every block chain, largest chains first, one process per core
    parts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    _ED, _PARTS = ed, parts
    cost = [np.prod([len(ed.E[b]) for b in p["b"]]) for p in parts]
    order = [int(k) for k in np.argsort(cost)[::-1]]
    g2 = np.zeros(len(TRIPLES), dtype=complex)
    done = 0
    with mp.get_context("fork").Pool(os.cpu_count()) as pool:
        for k, v in pool.imap_unordered(_part_value, order):
            g2 += v
            done += 1
            if done % 20 == 0:
                print(f"  {done}/{len(parts)} chains, {time.time() - t0:.0f} s", flush=True)
    print(f"G2: {time.time() - t0:.1f} s", flush=True)
    doc = {
        "model": "8-site Hubbard ring, PBC, t=1, U=4, mu=2, beta=5, truncateBlocks(1e-12)",
        "g2_component": "chi_(u0,d0,u0,d0): c_up c_dn c^+_up c^+_dn at site S0",
        "g2_parts": len(parts),
        "anchor_tol": ANCHOR_TOL,
        "pole_res": POLE_RES,
        "triples": TRIPLES,
        "g2": [[x.real, x.imag] for x in g2],
        "g_u0_n": list(range(256)),
        "g_u0": [[x.real, x.imag] for x in G],
        "chi_zz_m": list(range(48)),
        "chi_zz": [[x.real, x.imag] for x in zz],
        "generator": "tests/golden/make_ring8.py",
    }
    OUT.write_text(json.dumps(doc))
    print(f"wrote {OUT} ({time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
