"""pgx_eigh_noalloc: the eigensolve for callers that cannot let the library
allocate device memory (their memory belongs to an outer allocator such as an
application's caching pool or a fixed arena).

The test owns every device buffer (allocated here with torch, as such a
caller would from its own pool), calls the entry point through the C ABI
twice in a row on the same buffers, and checks the output against the
existing entry point (pgx_set_blocks / pgx_set_hamiltonian / pgx_eigh /
pgx_get_eigensystem) at the eigensolver tolerances of the other GPU tests.
It lives in its own file, collected last, and works alone or after the rest.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("n", [1, 7, 200, 256])
def test_eigh_noalloc_matches_pgx_eigh(n):
    import torch

    from pomerol_b200 import pgx

    lib = pgx.load()
    rng = np.random.default_rng(100 + n)
    a = rng.standard_normal((n, n))
    h = (a + a.T) / 2

    eng = pgx.Engine()
    eng.set_blocks([n])
    eng.set_hamiltonian([h])
    eng.eigh()
    (E0,), (U0,) = eng.eigensystem()
    eng.close()

    Hd = torch.from_numpy(h).to("cuda")
    Ed = torch.empty(n, dtype=torch.float64, device="cuda")
    Ud = torch.empty((n, n), dtype=torch.float64, device="cuda")
    scale = max(1.0, float(np.abs(E0).max()))
    for call in range(2):
        Ed.fill_(float("nan"))
        Ud.fill_(float("nan"))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = lib.pgx_eigh_noalloc(_ptr(Hd), n, _ptr(Ed), _ptr(Ud), None)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert rc == pgx.PGX_OK
        if call == 1:
            # the first call may load the library's kernels; from then on the
            # entry point leaves the device's free memory exactly as it was
            assert free1 == free0
        E1, U1 = Ed.cpu().numpy(), Ud.cpu().numpy()
        assert np.abs(E1 - E0).max() <= 1e-12 * scale
        # same eigenvectors up to sign: |U1^T U0| is the identity
        assert np.abs(np.abs(U1.T @ U0) - np.eye(n)).max() < 1e-10
        assert np.abs(h @ U1 - U1 * E1[None, :]).max() < 1e-10 * scale
        assert np.abs(U1.T @ U1 - np.eye(n)).max() < 1e-11


def test_eigh_noalloc_rejects_sizes_beyond_the_workspace():
    import torch

    from pomerol_b200 import pgx

    lib = pgx.load()
    n = 257
    Hd = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    Ed = torch.empty(n, dtype=torch.float64, device="cuda")
    Ud = torch.empty((n, n), dtype=torch.float64, device="cuda")
    assert lib.pgx_eigh_noalloc(_ptr(Hd), n, _ptr(Ed), _ptr(Ud), None) == pgx.PGX_ERR_ARG
    assert lib.pgx_eigh_noalloc(_ptr(Hd), 0, _ptr(Ed), _ptr(Ud), None) == pgx.PGX_ERR_ARG
