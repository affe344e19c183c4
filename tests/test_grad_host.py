"""Host-side algebra of the FTLM parameter gradient (no GPU): the tridiagonal eigen-solver and the
Duhamel weights K, checked against numpy and against central differences of
g(eps) = e_1^T exp(-bT (T + eps G)) e_1 computed by dense diagonalisation."""
import ctypes as C

import numpy as np
import pytest

from ftlm_extended_hubbard_b200 import _lib


def _P(a):
    return a.ctypes.data_as(C.c_void_p)


def _tridiag(n, rng):
    a = rng.standard_normal(n) * 3.0
    b = np.abs(rng.standard_normal(n - 1)) + 0.1
    return a, b


@pytest.mark.parametrize("n", [1, 2, 7, 40, 96])
def test_tridiag_eigvec_matches_numpy(n):
    rng = np.random.default_rng(n)
    a, b = _tridiag(n, rng)
    lam = np.zeros(n)
    Z = np.zeros((n, n))
    _lib.call("ftlm_gpu_tridiag_eigvec", _P(a), _P(b), n, _P(lam), _P(Z))
    T = np.diag(a) + np.diag(b, 1) + np.diag(b, -1)
    np.testing.assert_allclose(lam, np.linalg.eigvalsh(T), atol=1e-12 * max(1.0, np.abs(lam).max()))
    np.testing.assert_allclose(Z.T @ Z, np.eye(n), atol=1e-12)
    np.testing.assert_allclose(T @ Z, Z * lam, atol=1e-11 * max(1.0, np.abs(lam).max()))


def _g(T, bT, shift):
    w, V = np.linalg.eigh(T)
    return float(np.sum(V[0] ** 2 * np.exp(-bT * (w - shift))))


@pytest.mark.parametrize("n,bT", [(1, 2.0), (5, 0.3), (30, 2.0), (60, 8.0)])
def test_duhamel_weights_give_the_derivative(n, bT):
    rng = np.random.default_rng(100 + n)
    a, b = _tridiag(n, rng)
    K = np.zeros((n, n))
    g = C.c_double()
    lmin = C.c_double()
    _lib.call("ftlm_gpu_duhamel_weights", _P(a), _P(b), n, bT, _P(K), C.byref(g), C.byref(lmin))
    T = np.diag(a) + np.diag(b, 1) + np.diag(b, -1)
    assert abs(lmin.value - np.linalg.eigvalsh(T)[0]) < 1e-12 * max(1.0, abs(lmin.value))
    assert abs(g.value - _g(T, bT, lmin.value)) < 1e-12  # 0 < g <= 1: weights sum to one
    np.testing.assert_allclose(K, K.T, atol=0)
    for trial in range(3):
        G = rng.standard_normal((n, n))
        G = G + G.T
        h = 1e-5
        fd = (_g(T + h * G, bT, lmin.value) - _g(T - h * G, bT, lmin.value)) / (2 * h)
        an = -np.sum(G * K)
        assert abs(an - fd) <= 1e-7 * max(1.0, abs(fd)), (trial, an, fd)
