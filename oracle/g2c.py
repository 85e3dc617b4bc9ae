"""ctypes face of the C++ oracle (oracle/g2_oracle.cpp): the reference's G2
enumeration + TermList + OpenMP frequency loop.  Test infrastructure only."""
import ctypes as C
from pathlib import Path

import numpy as np

_LIB = None
NZ_TOL = 1e-20   # non-zero threshold of rotated elements: the reference's sparseView(1e-8) keeps |x| > 1e-8 * 1e-12


def lib():
    global _LIB
    if _LIB is None:
        from . import build
        p = build.OUT
        if not p.exists():
            build.main()
        L = C.CDLL(str(p))
        P, I, D = C.c_void_p, C.c_int, C.c_double
        L.g2o_count.restype = C.c_longlong
        L.g2o_count.argtypes = [I, I, I, I] + [P] * 8 + [D, D]
        L.g2o_part.restype = C.c_longlong
        L.g2o_part.argtypes = [I, I, I, I] + [P] * 12 + [P, I, D, D, D, D, I, I, P, I, I, I, I, I, P, P, I]
        _LIB = L
    return _LIB


def _a(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def _part_arrays(ed, p):
    b = p["b"]
    mats = [_a(p["O1"]), _a(p["O2"]), _a(p["O3"]), _a(p["CX4"])]
    E = [_a(ed.E[x]) for x in b]
    w = [_a(ed.w[x]) for x in b]
    dims = [len(ed.E[x]) for x in b]
    return dims, mats, E, w


def count(ed, parts, coef_tol=1e-16, nz_tol=NZ_TOL):
    n = 0
    for p in parts:
        dims, mats, E, w = _part_arrays(ed, p)
        n += lib().g2o_count(*dims, *[m.ctypes.data for m in mats], *[x.ctypes.data for x in w], coef_tol, nz_tol)
    return n


def evaluate(ed, parts, freqs, pole_res=1e-8, coef_tol=1e-16, rule=True, nz_tol=NZ_TOL, rows=None, nthreads=0):
    """Sum over parts at triples `freqs` ((n,3) complex).  rows=(part_index,
    begin, end[, row_step[, col_step[, chase_step]]]) restricts to one part, a
    strided range of index1, every col_step-th index3 and every chase_step-th
    index2 and index4 (bounded sample).
    Returns (values, quadruples enumerated, [nr_terms, res_terms])."""
    z = np.ascontiguousarray(np.asarray(freqs, dtype=complex).reshape(-1, 3)).view(np.float64)
    out = np.zeros(2 * (len(z) // 6) if z.ndim == 1 else 2 * z.shape[0])
    out = np.zeros(2 * np.asarray(freqs).reshape(-1, 3).shape[0])
    nq = 0
    terms = np.zeros(2, dtype=np.int64)
    sel = range(len(parts)) if rows is None else [rows[0]]
    for k in sel:
        p = parts[k]
        dims, mats, E, w = _part_arrays(ed, p)
        r0, r1, rs = (0, dims[0], 1) if rows is None else (rows[1], rows[2], rows[3] if len(rows) > 3 else 1)
        cs = 1 if rows is None or len(rows) < 5 else rows[4]
        ks = 1 if rows is None or len(rows) < 6 else rows[5]
        perm = np.ascontiguousarray(p["perm"], dtype=np.int32)
        t = np.zeros(2, dtype=np.int64)
        nq += lib().g2o_part(*dims, *[m.ctypes.data for m in mats], *[x.ctypes.data for x in E],
                             *[x.ctypes.data for x in w], perm.ctypes.data, int(p["sign"]), ed.beta, pole_res,
                             coef_tol, nz_tol, int(rule), out.size // 2, z.ctypes.data, r0, r1, rs, cs, ks,
                             out.ctypes.data, t.ctypes.data, int(nthreads))
        terms += t
    return out.view(complex), nq, terms
