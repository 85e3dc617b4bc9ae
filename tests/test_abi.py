"""The C-ABI library loads and exports every entry point include/pgx.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "pgx.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|long long|const char\*)\s+(pgx_\w+)\s*\(", text, re.M)))


def test_header_lists_entry_points():
    syms = declared_symbols()
    assert "pgx_g2" in syms and "pgx_eigh" in syms and len(syms) >= 20


def test_library_exports_every_declared_symbol():
    from pomerol_b200 import pgx
    if not pgx.LIB_PATH.exists():
        pytest.fail("libpgx.so is not built (python -m pomerol_b200.build)")
    lib = ctypes.CDLL(str(pgx.LIB_PATH))
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert set(declared_symbols()) == set(pgx.EXPORTS)


def test_create_without_gpu_reports_status():
    import torch
    from pomerol_b200 import pgx
    lib = pgx.load()
    h = ctypes.c_void_p()
    rc = lib.pgx_create(0, ctypes.byref(h))
    if torch.cuda.is_available():
        assert rc == pgx.PGX_OK
        lib.pgx_destroy(h)
    else:
        assert rc in (pgx.PGX_ERR_NODEV, pgx.PGX_ERR_CUDA)
    assert lib.pgx_version() >= 10000
