"""The balanced base-254 digit split of the int8 tensor-core products,
restated in numpy and checked on the CPU against its stated error bound.

Each row of A (each column of B) is scaled by 2^-e, e the exponent of its
largest |Re| or |Im|, and cut into S digits:
    127 x 2^-e = sum_s d_s 254^-s,   d_s integer in [-127, 127],
the leading digit rounded to the nearest integer, then each remainder (in
[-1/2, 1/2]) times 254 and rounded.  The product keeps the digit pairs
a + b < S, each exact in integers, weighted by 254^-(a+b) / 127^2.  The
element-wise error is below (S + 1) 254^-S K rowmax_i(A) colmax_j(B).
The GPU kernels (pomerol_b200/csrc/pgx_ozaki.cu) compute the same digits; the
GPU tests compare their products with FP64 ones.
"""
import numpy as np
import pytest


def _digits(x, S):
    """Digits of the rows of a real matrix x (n x K): (exponents e, digits
    of shape S x n x K)."""
    m = np.abs(x).max(axis=1)
    e = np.zeros(len(m), dtype=np.int64)
    nz = m > 0
    e[nz] = np.frexp(m[nz])[1]
    v = x * (127.0 * np.ldexp(1.0, -e))[:, None]
    ds = []
    for s in range(S):
        if s > 0:
            v = v * 254.0
        d = np.rint(v)
        v = v - d
        ds.append(d.astype(np.int64))
    return e, np.stack(ds)


def _split_product(A, B, S):
    """Real product A B through the digit split."""
    ea, da = _digits(A, S)
    eb, db = _digits(B.T, S)
    C = np.zeros((A.shape[0], B.shape[1]))
    for s in range(S):
        acc = np.zeros((A.shape[0], B.shape[1]), dtype=np.int64)
        for a in range(s + 1):
            acc += da[a] @ db[s - a].T  # exact integer products
        C += acc.astype(np.float64) * (254.0 ** -s / 127.0 ** 2)
    return C * np.ldexp(1.0, ea)[:, None] * np.ldexp(1.0, eb)[None, :]


def _matrix(rng, n, k):
    """Seeded values in [-1, 1) spread over four binary orders of magnitude."""
    return rng.uniform(-1.0, 1.0, (n, k)) * np.ldexp(1.0, -rng.integers(0, 4, (n, k)))


@pytest.mark.parametrize("S", [3, 4, 5, 6])
def test_digits_are_signed_bytes_and_reconstruct_the_row(S):
    rng = np.random.default_rng(S)
    x = _matrix(rng, 40, 300)
    x[3] = 0.0  # an all-zero row keeps zero digits
    e, d = _digits(x, S)
    assert d.min() >= -127 and d.max() <= 127
    rec = sum(d[s] * 254.0 ** -s for s in range(S)) / 127.0 * np.ldexp(1.0, e)[:, None]
    # the remainder after S digits is at most 254^-S of the row's scale 2^e
    # (plus the FP64 rounding of the scaling and of this reconstruction)
    scale = np.ldexp(1.0, e)[:, None]
    assert np.all(np.abs(rec - x) <= (254.0 ** -S + 8 * 2.0 ** -53) * scale)
    assert not d[:, 3].any()


@pytest.mark.parametrize("S", [3, 4, 5, 6])
def test_split_product_within_its_error_bound(S):
    rng = np.random.default_rng(10 + S)
    M, K, N = 37, 250, 29
    A, B = _matrix(rng, M, K), _matrix(rng, K, N)
    C = _split_product(A, B, S)
    ref = A @ B
    bound = (S + 1) * 254.0 ** -S * K * np.abs(A).max(axis=1)[:, None] * np.abs(B).max(axis=0)[None, :]
    assert np.all(np.abs(C - ref) <= bound + 1e-15 * np.abs(ref).max())
    # one digit fewer leaves about 254 times the error
    if S > 3:
        e_s = np.abs(C - ref).max()
        e_s1 = np.abs(_split_product(A, B, S - 1) - ref).max()
        assert 30.0 < e_s1 / max(e_s, 1e-300) < 3000.0


def test_complex_product_through_the_real_embedding():
    """Complex operands as one real product of twice the depth:
    A' = [Re A, Im A] and, per column of B, [Re B; -Im B] and [Im B; Re B]."""
    rng = np.random.default_rng(3)
    M, K, N, S = 21, 90, 17, 5
    A = _matrix(rng, M, K) + 1j * _matrix(rng, M, K)
    B = _matrix(rng, K, N) + 1j * _matrix(rng, K, N)
    Ar = np.hstack([A.real, A.imag])
    Br = np.zeros((2 * K, 2 * N))
    Br[:K, 0::2], Br[K:, 0::2] = B.real, -B.imag
    Br[:K, 1::2], Br[K:, 1::2] = B.imag, B.real
    Cr = _split_product(Ar, Br, S)
    C = Cr[:, 0::2] + 1j * Cr[:, 1::2]
    ref = A @ B
    assert np.abs(C - ref).max() < (S + 1) * 254.0 ** -S * 2 * K * np.abs(ref).max()
