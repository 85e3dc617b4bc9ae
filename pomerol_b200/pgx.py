"""ctypes binding of libpgx's C ABI (include/pgx.h).

This is the Python face of the CUDA engine: plain numpy arrays in and out,
no torch types.  Loading fails loudly when the library is missing; there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libpgx.so"

PGX_OK, PGX_ERR_ARG, PGX_ERR_OOM, PGX_ERR_CUDA, PGX_ERR_TIMEOUT, PGX_ERR_NUMERIC, PGX_ERR_STATE, PGX_ERR_NODEV = range(8)
PGX_G2_EXACT, PGX_G2_REFERENCE_RULE, PGX_G2_ANCHORED, PGX_G2_SPLIT_I8 = 0, 1, 2, 4

EXPORTS = [
    "pgx_version", "pgx_create", "pgx_destroy", "pgx_last_error", "pgx_set_blocks", "pgx_set_hamiltonian",
    "pgx_eigh", "pgx_get_eigensystem", "pgx_ground_energy", "pgx_weights", "pgx_truncate_blocks",
    "pgx_op_define", "pgx_op_rotate", "pgx_op_adjoint", "pgx_op_info", "pgx_op_read", "pgx_gf", "pgx_susc",
    "pgx_ensemble_average", "pgx_g2", "pgx_g2_count", "pgx_g2_last_timing", "pgx_timer_begin", "pgx_timer_end",
    "pgx_launch_count", "pgx_eigh_noalloc", "pgx_profile_begin", "pgx_profile_end", "pgx_profile_kernel",
    "pgx_recip_check", "pgx_assemble_hamiltonian", "pgx_get_hamiltonian", "pgx_op_release",
    "pgx_gf_vjp", "pgx_susc_vjp", "pgx_chi3", "pgx_set_eigensystem", "pgx_autotune_begin", "pgx_autotune_end",
    "pgx_set_g2_workspace", "pgx_set_g2_split_threshold", "pgx_set_g2_split_slices", "pgx_set_g2_split_weight_budget", "pgx_set_split_cta_pair", "pgx_split_gemm_check", "pgx_graph_begin", "pgx_graph_end",
    "pgx_graph_replay", "pgx_graph_destroy", "pgx_set_models", "pgx_weights_models", "pgx_gf_models", "pgx_susc_models",
]


class PgxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pgx error {code}: {msg}")
        self.code = code


class G2Part(C.Structure):
    _fields_ = [("op", C.c_int32 * 4), ("block", C.c_int32 * 4), ("perm", C.c_int32 * 3), ("sign", C.c_int32)]


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"libpgx not built: {LIB_PATH} missing (run python -m pomerol_b200.build)")
        lib = C.CDLL(str(LIB_PATH))
        P, I32, D = C.c_void_p, C.c_int32, C.c_double
        lib.pgx_last_error.restype = C.c_char_p
        lib.pgx_last_error.argtypes = [P]
        lib.pgx_create.argtypes = [C.c_int, C.POINTER(P)]
        lib.pgx_destroy.argtypes = [P]
        lib.pgx_set_blocks.argtypes = [P, I32, P, I32]
        lib.pgx_set_hamiltonian.argtypes = [P, P]
        lib.pgx_eigh.argtypes = [P]
        lib.pgx_get_eigensystem.argtypes = [P, P, P]
        lib.pgx_ground_energy.argtypes = [P, P]
        lib.pgx_weights.argtypes = [P, D, P, P]
        lib.pgx_truncate_blocks.argtypes = [P, D, P]
        lib.pgx_op_define.argtypes = [P, I32, P, P, P, P, P]
        lib.pgx_op_rotate.argtypes = [P, I32]
        lib.pgx_op_adjoint.argtypes = [P, I32, P]
        lib.pgx_op_info.argtypes = [P, I32, P, P, P]
        lib.pgx_op_read.argtypes = [P, I32, I32, P]
        lib.pgx_gf.argtypes = [P, I32, I32, I32, P, P, I32, P, D, P]
        lib.pgx_susc.argtypes = [P, I32, I32, I32, P, P, I32, P, D, D, D, P, P]
        lib.pgx_ensemble_average.argtypes = [P, I32, P]
        lib.pgx_g2.argtypes = [P, I32, P, I32, P, D, D, I32, P]
        lib.pgx_g2_last_timing.argtypes = [P, P, P, P]
        lib.pgx_g2_count.argtypes = [P, I32, P, D, D, P]
        lib.pgx_timer_begin.argtypes = [P]
        lib.pgx_timer_end.argtypes = [P, P]
        lib.pgx_launch_count.restype = C.c_longlong
        lib.pgx_eigh_noalloc.argtypes = [P, I32, P, P, P]
        lib.pgx_profile_begin.argtypes = [P]
        lib.pgx_profile_end.argtypes = [P, P]
        lib.pgx_profile_kernel.argtypes = [P, I32, C.c_char_p, I32, P, P, P, P]
        lib.pgx_recip_check.argtypes = [P, I32, P]
        lib.pgx_assemble_hamiltonian.argtypes = [P, I32, P, P, I32, P, P, P]
        lib.pgx_get_hamiltonian.argtypes = [P, P]
        lib.pgx_op_release.argtypes = [P, I32]
        lib.pgx_gf_vjp.argtypes = [P, I32, I32, I32, P, P, I32, P, P, P, P]
        lib.pgx_susc_vjp.argtypes = [P, I32, I32, I32, P, P, I32, P, D, P, P, P]
        lib.pgx_chi3.argtypes = [P, I32, I32, P, I32, P, D, P]
        lib.pgx_set_eigensystem.argtypes = [P, P, P]
        lib.pgx_autotune_begin.argtypes = [P]
        lib.pgx_set_g2_workspace.argtypes = [P, C.c_int64, C.c_int64]
        lib.pgx_set_g2_split_threshold.argtypes = [P, C.c_double]
        lib.pgx_set_g2_split_slices.argtypes = [P, I32]
        lib.pgx_set_split_cta_pair.argtypes = [P, I32]
        lib.pgx_set_g2_split_weight_budget.argtypes = [P, D]
        lib.pgx_split_gemm_check.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                             P, P, P]
        lib.pgx_autotune_end.argtypes = [P, P]
        lib.pgx_graph_begin.argtypes = [P]
        lib.pgx_graph_end.argtypes = [P, P]
        lib.pgx_graph_replay.argtypes = [P, I32]
        lib.pgx_graph_destroy.argtypes = [P, I32]
        lib.pgx_set_models.argtypes = [P, I32, P, P]
        lib.pgx_weights_models.argtypes = [P, P, P, P]
        lib.pgx_gf_models.argtypes = [P, I32, I32, I32, P, P, I32, P, D, P]
        lib.pgx_susc_models.argtypes = [P, I32, I32, I32, P, P, I32, P, D, D, P, P]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Engine:
    """One libpgx context (one GPU, one stream, one ED problem)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.pgx_create(int(device), C.byref(h))
        if rc != PGX_OK:
            raise PgxError(rc, "pgx_create failed (no CUDA device?)")
        self.h = h
        self.dims = None
        self.is_complex = False

    def close(self):
        if getattr(self, "h", None):
            self.lib.pgx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != PGX_OK:
            raise PgxError(rc, self.lib.pgx_last_error(self.h).decode())

    # ---- blocks / eigensystem
    def set_blocks(self, dims, is_complex=False):
        self.dims = np.ascontiguousarray(dims, dtype=np.int32)
        self.is_complex = bool(is_complex)
        self._ck(self.lib.pgx_set_blocks(self.h, len(self.dims), _p(self.dims), int(is_complex)))
        self.eoff = np.concatenate([[0], np.cumsum(self.dims)]).astype(np.int64)
        self.moff = np.concatenate([[0], np.cumsum(self.dims.astype(np.int64) ** 2)]).astype(np.int64)

    def set_hamiltonian(self, blocks):
        packed = np.concatenate([np.ascontiguousarray(b, dtype=complex if self.is_complex else float).ravel()
                                 for b in blocks])
        if self.is_complex:
            packed = packed.view(np.float64)
        packed = np.ascontiguousarray(packed)
        self._ck(self.lib.pgx_set_hamiltonian(self.h, _p(packed)))

    def eigh(self):
        self._ck(self.lib.pgx_eigh(self.h))

    def eigensystem(self):
        E = np.empty(int(self.eoff[-1]))
        U = np.empty(int(self.moff[-1]) * (2 if self.is_complex else 1))
        self._ck(self.lib.pgx_get_eigensystem(self.h, _p(E), _p(U)))
        if self.is_complex:
            U = U.view(complex)
        Es = [E[self.eoff[b]:self.eoff[b + 1]] for b in range(len(self.dims))]
        Us = [U[self.moff[b]:self.moff[b + 1]].reshape(d, d) for b, d in enumerate(self.dims)]
        return Es, Us

    def weights(self, beta):
        w = np.empty(int(self.eoff[-1]))
        Z = np.zeros(1)
        self._ck(self.lib.pgx_weights(self.h, float(beta), _p(w), _p(Z)))
        return [w[self.eoff[b]:self.eoff[b + 1]] for b in range(len(self.dims))], float(Z[0])

    def truncate_blocks(self, tol):
        r = np.zeros(len(self.dims), dtype=np.int32)
        self._ck(self.lib.pgx_truncate_blocks(self.h, float(tol), _p(r)))
        return r.astype(bool)

    # ---- operators
    def op_define(self, parts):
        """parts: list of (right_block, left_block, target[int], coef[float])."""
        rb = np.array([p[0] for p in parts], dtype=np.int32)
        lb = np.array([p[1] for p in parts], dtype=np.int32)
        tg = np.ascontiguousarray(np.concatenate([np.asarray(p[2]) for p in parts]) if parts else np.zeros(0),
                                  dtype=np.int32)
        cf = np.ascontiguousarray(np.concatenate([np.asarray(p[3]) for p in parts]) if parts else np.zeros(0),
                                  dtype=np.float64)
        out = np.zeros(1, dtype=np.int32)
        self._ck(self.lib.pgx_op_define(self.h, len(parts), _p(rb), _p(lb), _p(tg), _p(cf), _p(out)))
        return int(out[0])

    def op_rotate(self, op):
        self._ck(self.lib.pgx_op_rotate(self.h, int(op)))

    def op_adjoint(self, op):
        out = np.zeros(1, dtype=np.int32)
        self._ck(self.lib.pgx_op_adjoint(self.h, int(op), _p(out)))
        return int(out[0])

    def op_info(self, op):
        n = np.zeros(1, dtype=np.int32)
        self._ck(self.lib.pgx_op_info(self.h, int(op), _p(n), None, None))
        r = np.zeros(max(int(n[0]), 1), dtype=np.int32)
        l = np.zeros(max(int(n[0]), 1), dtype=np.int32)
        self._ck(self.lib.pgx_op_info(self.h, int(op), _p(n), _p(r), _p(l)))
        return [(int(r[i]), int(l[i])) for i in range(int(n[0]))]

    def op_read(self, op, part):
        R, L = self.op_info(op)[part]
        out = np.empty(int(self.dims[L]) * int(self.dims[R]) * (2 if self.is_complex else 1))
        self._ck(self.lib.pgx_op_read(self.h, int(op), int(part), _p(out)))
        if self.is_complex:
            out = out.view(complex)
        return out.reshape(int(self.dims[L]), int(self.dims[R]))

    # ---- Lehmann sums
    def gf(self, op1, op2, outer, inner, z, coef_tol=1e-8):
        z = np.ascontiguousarray(np.asarray(z, dtype=complex))
        o = np.ascontiguousarray(outer, dtype=np.int32)
        i = np.ascontiguousarray(inner, dtype=np.int32)
        out = np.zeros(len(z), dtype=complex)
        self._ck(self.lib.pgx_gf(self.h, op1, op2, len(o), _p(o), _p(i), len(z), _p(z.view(np.float64)),
                                 float(coef_tol), _p(out.view(np.float64))))
        return out

    def susc(self, opA, opB, outer, inner, z, beta, pole_res=1e-8, coef_tol=1e-8):
        z = np.ascontiguousarray(np.asarray(z, dtype=complex))
        o = np.ascontiguousarray(outer, dtype=np.int32)
        i = np.ascontiguousarray(inner, dtype=np.int32)
        out = np.zeros(len(z), dtype=complex)
        zp = np.zeros(1, dtype=complex)
        self._ck(self.lib.pgx_susc(self.h, opA, opB, len(o), _p(o), _p(i), len(z), _p(z.view(np.float64)),
                                   float(pole_res), float(coef_tol), float(beta), _p(out.view(np.float64)),
                                   _p(zp.view(np.float64))))
        return out, complex(zp[0])

    def ensemble_average(self, op):
        out = np.zeros(1, dtype=complex)
        self._ck(self.lib.pgx_ensemble_average(self.h, int(op), _p(out.view(np.float64))))
        return complex(out[0])

    def g2(self, parts, triples, pole_res=1e-8, coef_tol=1e-16, flags=PGX_G2_EXACT):
        """parts: list of (ops[4], blocks[4], perm[3], sign); triples: (n,3) complex."""
        arr = (G2Part * max(len(parts), 1))()
        for k, (ops, blocks, perm, sign) in enumerate(parts):
            arr[k].op[:] = list(ops)
            arr[k].block[:] = list(blocks)
            arr[k].perm[:] = list(perm)
            arr[k].sign = int(sign)
        z = np.ascontiguousarray(np.asarray(triples, dtype=complex).reshape(-1, 3))
        out = np.zeros(len(z), dtype=complex)
        self._ck(self.lib.pgx_g2(self.h, len(parts), C.cast(arr, C.c_void_p), len(z), _p(z.view(np.float64)),
                                 float(pole_res), float(coef_tol), int(flags), _p(out.view(np.float64))))
        return out

    @staticmethod
    def _parts_array(parts):
        arr = (G2Part * max(len(parts), 1))()
        for k, (ops, blocks, perm, sign) in enumerate(parts):
            arr[k].op[:] = list(ops)
            arr[k].block[:] = list(blocks)
            arr[k].perm[:] = list(perm)
            arr[k].sign = int(sign)
        return arr

    def g2_count(self, parts, coef_tol=1e-16, nz_tol=1e-20):
        arr = self._parts_array(parts)
        out = np.zeros(1, dtype=np.int64)
        self._ck(self.lib.pgx_g2_count(self.h, len(parts), C.cast(arr, C.c_void_p), float(coef_tol), float(nz_tol),
                                       _p(out)))
        return int(out[0])

    def g2_timing(self):
        t = np.zeros(3)
        self._ck(self.lib.pgx_g2_last_timing(self.h, _p(t[0:1]), _p(t[1:2]), _p(t[2:3])))
        return {"total_ms": t[0], "gemm_ms": t[1], "gemm_flops": t[2]}


def launch_count() -> int:
    """Kernels launched by libpgx in this process."""
    return int(load().pgx_launch_count())


def _timer_begin(self):
    self._ck(self.lib.pgx_timer_begin(self.h))


def _timer_end(self):
    ms = np.zeros(1)
    self._ck(self.lib.pgx_timer_end(self.h, _p(ms)))
    return float(ms[0])


def _profile_begin(self):
    """Start recording per-kernel device times (CUDA event pairs on the
    context's stream) for the instrumented kernels."""
    self._ck(self.lib.pgx_profile_begin(self.h))


def _profile_end(self):
    """Stop recording; per kernel name: launches, total ms, algorithmic
    FLOPs and DRAM bytes summed over the launches (largest time first)."""
    n = np.zeros(1, dtype=np.int32)
    self._ck(self.lib.pgx_profile_end(self.h, _p(n)))
    out = []
    for i in range(int(n[0])):
        name = C.create_string_buffer(128)
        nl = np.zeros(1, dtype=np.int32)
        v = np.zeros(3)
        self._ck(self.lib.pgx_profile_kernel(self.h, i, name, 128, _p(nl), _p(v[0:1]), _p(v[1:2]), _p(v[2:3])))
        out.append({"name": name.value.decode(), "launches": int(nl[0]), "ms": float(v[0]),
                    "flops": float(v[1]), "bytes": float(v[2])})
    return out


PGX_TERM_OPS = 8


def _assemble_hamiltonian(self, terms, nmodes, fock, state_block, state_inner):
    """Device assembly of the block Hamiltonians: terms is a list of
    (ops, coef) with ops a sequence of (dagger, mode) pairs, left to right."""
    n = len(terms)
    ops = np.full((max(n, 1), PGX_TERM_OPS), -1, dtype=np.int32)
    coef = np.zeros((max(n, 1), 2))
    for t, (mono, c) in enumerate(terms):
        if len(mono) > PGX_TERM_OPS:
            raise ValueError("monomial longer than PGX_TERM_OPS operators")
        for k, (dag, mode) in enumerate(mono):
            ops[t, k] = 2 * int(mode) + (1 if dag else 0)
        coef[t] = (complex(c).real, complex(c).imag)
    fock = np.ascontiguousarray(fock, dtype=np.uint64)
    sb = np.ascontiguousarray(state_block, dtype=np.int32)
    si = np.ascontiguousarray(state_inner, dtype=np.int32)
    self._ck(self.lib.pgx_assemble_hamiltonian(self.h, n, _p(ops), _p(coef), int(nmodes), _p(fock), _p(sb), _p(si)))
    self._asm_nterms = n


def _get_hamiltonian(self):
    """The block Hamiltonians on the device, one dense array per block."""
    total = sum(d * d for d in self.dims)
    buf = np.zeros(total * (2 if self.is_complex else 1))
    self._ck(self.lib.pgx_get_hamiltonian(self.h, _p(buf)))
    out, o = [], 0
    for d in self.dims:
        if self.is_complex:
            m = buf[2 * o:2 * (o + d * d)].view(complex).reshape(d, d)
        else:
            m = buf[o:o + d * d].reshape(d, d)
        out.append(m.copy())
        o += d * d
    return out


def _gf_vjp(self, op1, op2, outer, inner, z, lam):
    """Reverse-mode derivative of gf(op1, op2, outer, inner, z): for a loss
    with dL = Re sum_n lam[n] dG(z_n), returns (dL/dc_t for every term of the
    last assemble_hamiltonian call, dL/dE_s for every state)."""
    z = np.ascontiguousarray(np.asarray(z, dtype=complex))
    lam = np.ascontiguousarray(np.asarray(lam, dtype=complex))
    if lam.shape != z.shape:
        raise ValueError("lam needs one entry per frequency")
    o = np.ascontiguousarray(outer, dtype=np.int32)
    i = np.ascontiguousarray(inner, dtype=np.int32)
    dterm = np.zeros(max(getattr(self, "_asm_nterms", 0), 1))
    dE = np.zeros(int(sum(self.dims)))
    self._ck(self.lib.pgx_gf_vjp(self.h, int(op1), int(op2), len(o), _p(o), _p(i), len(z), _p(z.view(np.float64)),
                                 _p(lam.view(np.float64)), _p(dterm), _p(dE)))
    return dterm[:getattr(self, "_asm_nterms", 0)], dE


PGX_PP, PGX_PH, PGX_XPH = 0, 1, 2


def _chi3(self, channel, parts, freqs, pole_res=1e-8):
    """Three-point susceptibility at (z1, z2) duplets.  parts: list of
    (f1, f2, b1, b2, (i, j, k, m), swapped) as ThreePointSusceptibility::prepare
    forms them (operators of the part, blocks <i|f1|j><j|f2|k><k|b1|m><m|b2|i>)."""
    desc = np.zeros((max(len(parts), 1), 9), dtype=np.int32)
    for q, (f1, f2, b1, b2, blk, sw) in enumerate(parts):
        desc[q] = [f1, f2, b1, b2, *blk, 1 if sw else 0]
    fz = np.ascontiguousarray(np.asarray(freqs, dtype=complex).reshape(-1, 2))
    out = np.zeros(len(fz), dtype=complex)
    self._ck(self.lib.pgx_chi3(self.h, int(channel), len(parts), _p(desc), len(fz), _p(fz.view(np.float64)),
                               float(pole_res), _p(out.view(np.float64))))
    return out


def _set_eigensystem(self, E, U):
    """Load an eigensystem (lists per block, as eigensystem() returns) in
    place of eigh()."""
    e = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64) for x in E]))
    dt = complex if self.is_complex else np.float64
    u = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=dt).ravel() for x in U]))
    if len(e) != int(sum(self.dims)) or len(u) != int(sum(d * d for d in self.dims)):
        raise ValueError("eigensystem does not match the blocks")
    self._ck(self.lib.pgx_set_eigensystem(self.h, _p(e), _p(u.view(np.float64))))


def _save_eigensystem(self, path):
    """Checkpoint the eigensystem and the block sizes to an .npz file."""
    E, U = self.eigensystem()
    np.savez(path, dims=np.asarray(self.dims), is_complex=self.is_complex, E=np.concatenate(E),
             U=np.concatenate([np.asarray(x).ravel() for x in U]))


def _load_eigensystem(self, path):
    """Reload an eigensystem saved by save_eigensystem into a context whose
    blocks are the same."""
    f = np.load(path)
    if list(f["dims"]) != list(self.dims) or bool(f["is_complex"]) != bool(self.is_complex):
        raise ValueError("the checkpoint's blocks differ from this context's")
    E, U, oe, ou = [], [], 0, 0
    for d in self.dims:
        E.append(f["E"][oe:oe + d])
        U.append(f["U"][ou:ou + d * d].reshape(d, d))
        oe += d
        ou += d * d
    self.set_eigensystem(E, U)


def _set_g2_workspace(self, batch_bytes=0, chain_bytes=0):
    """Workspace limits of the anchored G2 (0 keeps a default); a part whose
    workspace exceeds chain_bytes is evaluated in (z1, z3) tiles."""
    self._ck(self.lib.pgx_set_g2_workspace(self.h, int(batch_bytes), int(chain_bytes)))


def _set_g2_split_threshold(self, min_macs=1e9):
    """Products of at least min_macs complex multiply-adds use the int8
    tensor cores under PGX_G2_SPLIT_I8."""
    self._ck(self.lib.pgx_set_g2_split_threshold(self.h, float(min_macs)))


def _set_g2_split_slices(self, slices=6):
    """Balanced base-254 digits per operand element of the int8 split products."""
    self._ck(self.lib.pgx_set_g2_split_slices(self.h, int(slices)))


def _set_g2_split_weight_budget(self, budget=4.0):
    """Digits of each split product from its anchor block's largest weight;
    budget <= 0 gives every product the full digit count."""
    self._ck(self.lib.pgx_set_g2_split_weight_budget(self.h, float(budget)))


def _set_split_cta_pair(self, on=True):
    """256 x 256 split-product tiles on CTA pairs (True) or 128 x 256 tiles on
    single CTAs (False)."""
    self._ck(self.lib.pgx_set_split_cta_pair(self.h, int(bool(on))))


def _split_gemm_check(self, M, N, K, nb=1, slices=6, seed=1):
    """int8 split product vs FP64 on seeded random complex matrices:
    (max relative error, split ms, FP64 ms)."""
    r = np.zeros(3, dtype=np.float64)
    self._ck(self.lib.pgx_split_gemm_check(self.h, M, N, K, nb, slices, seed, _p(r[0:1]), _p(r[1:2]), _p(r[2:3])))
    return float(r[0]), float(r[1]), float(r[2])


def _autotune_begin(self):
    """Record the GEMM products of the following calls for autotune_end()."""
    self._ck(self.lib.pgx_autotune_begin(self.h))


def _autotune_end(self):
    """Time the recorded products in every tile class and keep the fastest per
    size bucket; returns the number of buckets that left the padding rule."""
    n = np.zeros(1, dtype=np.int32)
    self._ck(self.lib.pgx_autotune_end(self.h, _p(n)))
    return int(n[0])


def _graph_begin(self):
    """Start capturing eigh() / op_rotate() calls into a CUDA graph."""
    self._ck(self.lib.pgx_graph_begin(self.h))


def _graph_end(self):
    """Finish the capture; returns the graph id."""
    g = np.zeros(1, dtype=np.int32)
    self._ck(self.lib.pgx_graph_end(self.h, _p(g)))
    return int(g[0])


def _graph_replay(self, gid):
    self._ck(self.lib.pgx_graph_replay(self.h, int(gid)))


def _graph_destroy(self, gid):
    self._ck(self.lib.pgx_graph_destroy(self.h, int(gid)))


def _set_models(self, first_block, beta):
    """Independent models in this context: blocks first_block[m] ..
    first_block[m+1]-1 form model m at inverse temperature beta[m]."""
    f = np.ascontiguousarray(first_block, dtype=np.int32)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    self._ck(self.lib.pgx_set_models(self.h, len(b), _p(f), _p(b)))
    self.nmodels = len(b)


def _weights_models(self):
    """Per-model weights: (w per block as in weights(), E0[m], Z[m])."""
    w = np.empty(int(self.eoff[-1]))
    e0 = np.empty(self.nmodels)
    z = np.empty(self.nmodels)
    self._ck(self.lib.pgx_weights_models(self.h, _p(w), _p(e0), _p(z)))
    return [w[self.eoff[b]:self.eoff[b + 1]] for b in range(len(self.dims))], e0, z


def _pair_models(self, fn, op1, op2, outer, inner, z, *tol):
    z = np.ascontiguousarray(np.asarray(z, dtype=complex))
    if z.ndim != 2 or z.shape[0] != self.nmodels:
        raise ValueError("z must be nmodels x nz")
    o = np.ascontiguousarray(outer, dtype=np.int32)
    i = np.ascontiguousarray(inner, dtype=np.int32)
    out = np.zeros(z.shape, dtype=complex)
    return o, i, z, out


def _gf_models(self, op1, op2, outer, inner, z, coef_tol=1e-8):
    """G of every model at its own frequencies (z: nmodels x nz)."""
    o, i, z, out = _pair_models(self, None, op1, op2, outer, inner, z)
    self._ck(self.lib.pgx_gf_models(self.h, int(op1), int(op2), len(o), _p(o), _p(i), z.shape[1],
                                    _p(z.view(np.float64)), float(coef_tol), _p(out.view(np.float64))))
    return out


def _susc_models(self, opA, opB, outer, inner, z, pole_res=1e-8, coef_tol=1e-8):
    """chi of every model at its own frequencies (z: nmodels x nz); also the
    zero-pole sum of each model."""
    o, i, z, out = _pair_models(self, None, opA, opB, outer, inner, z)
    zero = np.zeros(self.nmodels, dtype=complex)
    self._ck(self.lib.pgx_susc_models(self.h, int(opA), int(opB), len(o), _p(o), _p(i), z.shape[1],
                                      _p(z.view(np.float64)), float(pole_res), float(coef_tol),
                                      _p(out.view(np.float64)), _p(zero.view(np.float64))))
    return out, zero


def _susc_vjp(self, opA, opB, outer, inner, z, lam, pole_res=1e-8):
    """Reverse-mode derivative of susc(opA, opB, outer, inner, z): as gf_vjp."""
    z = np.ascontiguousarray(np.asarray(z, dtype=complex))
    lam = np.ascontiguousarray(np.asarray(lam, dtype=complex))
    if lam.shape != z.shape:
        raise ValueError("lam needs one entry per frequency")
    o = np.ascontiguousarray(outer, dtype=np.int32)
    i = np.ascontiguousarray(inner, dtype=np.int32)
    dterm = np.zeros(max(getattr(self, "_asm_nterms", 0), 1))
    dE = np.zeros(int(sum(self.dims)))
    self._ck(self.lib.pgx_susc_vjp(self.h, int(opA), int(opB), len(o), _p(o), _p(i), len(z), _p(z.view(np.float64)),
                                   float(pole_res), _p(lam.view(np.float64)), _p(dterm), _p(dE)))
    return dterm[:getattr(self, "_asm_nterms", 0)], dE


def _op_release(self, op_id):
    """Give an operator's device memory back to the context for reuse."""
    self._ck(self.lib.pgx_op_release(self.h, int(op_id)))


Engine.op_release = _op_release
Engine.gf_vjp = _gf_vjp
Engine.susc_vjp = _susc_vjp
Engine.chi3 = _chi3
Engine.set_models = _set_models
Engine.graph_begin = _graph_begin
Engine.set_g2_workspace = _set_g2_workspace
Engine.split_gemm_check = _split_gemm_check
Engine.set_g2_split_threshold = _set_g2_split_threshold
Engine.set_g2_split_slices = _set_g2_split_slices
Engine.set_split_cta_pair = _set_split_cta_pair
Engine.set_g2_split_weight_budget = _set_g2_split_weight_budget
Engine.autotune_begin = _autotune_begin
Engine.autotune_end = _autotune_end
Engine.graph_end = _graph_end
Engine.graph_replay = _graph_replay
Engine.graph_destroy = _graph_destroy
Engine.set_eigensystem = _set_eigensystem
Engine.save_eigensystem = _save_eigensystem
Engine.load_eigensystem = _load_eigensystem
Engine.weights_models = _weights_models
Engine.gf_models = _gf_models
Engine.susc_models = _susc_models
Engine.assemble_hamiltonian = _assemble_hamiltonian
Engine.get_hamiltonian = _get_hamiltonian
Engine.timer_begin = _timer_begin
Engine.timer_end = _timer_end
Engine.profile_begin = _profile_begin
Engine.profile_end = _profile_end
