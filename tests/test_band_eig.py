"""Host band eigensolver of the block Lanczos driver (tbgpu_band_eigenvalues,
in place of the reference's zhbevx RANGE='V') against numpy's dense Hermitian
solver; no GPU needed.  Bar: 1e-12 absolute on O(1) matrices, same count."""
import ctypes as C

import numpy as np
import pytest

from nemo3d_b200 import build as nb


@pytest.fixture(scope="module")
def lib():
    nb.build()
    L = C.CDLL(nb.LIB)
    L.tbgpu_band_eigenvalues.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_double,
                                         C.c_double, C.c_void_p, C.c_int]
    return L


def _band(rng, n, kd, real=False):
    A = np.zeros((n, n), complex)
    for d in range(min(kd, n - 1) + 1):
        v = rng.normal(size=n - d) + (0 if (real or d == 0) else 1j * rng.normal(size=n - d))
        A += np.diag(v, -d)
    A = A + np.tril(A, -1).conj().T
    ab = np.zeros((n, kd + 1), complex)
    for j in range(n):
        for i in range(j, min(n, j + kd + 1)):
            ab[j, i - j] = A[i, j]
    return A, np.ascontiguousarray(ab)


@pytest.mark.parametrize("n,kd", [(1, 0), (2, 1), (12, 3), (40, 6), (300, 6), (97, 1),
                                  (64, 8), (50, 0), (8, 12)])
def test_band_window_eigenvalues(lib, n, kd):
    rng = np.random.default_rng(n * 31 + kd)
    A, ab = _band(rng, n, kd)  # kd may exceed n - 1: the extra diagonals are empty
    ev = np.linalg.eigvalsh(A)
    for vl, vu in [(ev.min() - 1, ev.max() + 1), (np.quantile(ev, 0.3), np.quantile(ev, 0.7))]:
        w = np.zeros(n)
        m = lib.tbgpu_band_eigenvalues(n, kd, ab.ctypes.data, vl, vu, 1e-13, w.ctypes.data, n)
        want = ev[(ev > vl) & (ev <= vu)]
        assert m == len(want)
        assert np.abs(w[:m] - want).max(initial=0.0) < 1e-12 * max(1.0, np.abs(ev).max())


def test_block_tridiagonal_with_degenerate_pairs(lib):
    # a Lanczos-like block tridiagonal matrix with exactly repeated eigenvalues
    rng = np.random.default_rng(7)
    p, m = 3, 20
    Q, _ = np.linalg.qr(rng.normal(size=(p * m, p * m)) + 1j * rng.normal(size=(p * m, p * m)))
    d = np.repeat(rng.normal(size=p * m // 2), 2)
    H = (Q * d) @ Q.conj().T
    # band-reduce by a block Lanczos run to get the band form
    V = np.zeros((p * m, p * m), complex)
    V[:, :p], _ = np.linalg.qr(rng.normal(size=(p * m, p)) + 0j)
    T = np.zeros((p * m, p * m), complex)
    for k in range(m):
        Vk = V[:, k * p:(k + 1) * p]
        W = H @ Vk
        T[k * p:(k + 1) * p, k * p:(k + 1) * p] = Vk.conj().T @ W
        W -= V[:, :(k + 1) * p] @ (V[:, :(k + 1) * p].conj().T @ W)
        W -= V[:, :(k + 1) * p] @ (V[:, :(k + 1) * p].conj().T @ W)
        if k + 1 < m:
            Qk, Bk = np.linalg.qr(W)
            V[:, (k + 1) * p:(k + 2) * p] = Qk
            T[(k + 1) * p:(k + 2) * p, k * p:(k + 1) * p] = Bk
            T[k * p:(k + 1) * p, (k + 1) * p:(k + 2) * p] = Bk.conj().T
    n = p * m
    ab = np.zeros((n, p + 1), complex)
    for j in range(n):
        for i in range(j, min(n, j + p + 1)):
            ab[j, i - j] = T[i, j]
    ev = np.linalg.eigvalsh(T)
    w = np.zeros(n)
    got = lib.tbgpu_band_eigenvalues(n, p, np.ascontiguousarray(ab).ctypes.data, -1e9, 1e9,
                                     1e-13, w.ctypes.data, n)
    assert got == n
    assert np.abs(w - ev).max() < 1e-11
