"""The FP64 Hermitian eigensolver behind MDL (dh_eigen.cu, through
digHoloB200EigenHermitian) against numpy's LAPACK eigh.

The power meter takes the squared singular values of the batch coefficient
matrix from the eigenvalues of its FP64 Gram matrix (digHolo's
svdSingularValues, digHolo.cpp:3021-3055, uses cgesvd on the matrix
itself).  Tolerances: every eigenvalue within 1e-12 * max|lambda| of
numpy's; the eigenvectors of the smallest and largest eigenvalue unit norm
with residual ||G u - lambda u|| <= 1e-10 * max|lambda|.  Sizes cover the
trivial ones (1, 2, 3), odd sizes, the 120 and 240 of one and two
polarisations of 120 modes, 256 (a 256-frame batch) and 930 (two
polarisations of 465 modes); full-rank and rank-deficient Gram matrices
(the rank-deficient ones have a zero eigenvalue of high multiplicity).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _solve(lib, G):
    n = G.shape[0]
    g = np.ascontiguousarray(G.T).astype(np.complex128)   # column-major
    W = np.zeros(n)
    V = np.zeros(4 * n)
    rc = lib.digHoloB200EigenHermitian(n, g.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                       W.ctypes.data_as(C.POINTER(C.c_double)),
                                       V.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    return W, V.view(np.complex128).reshape(2, n)


@pytest.mark.parametrize("n", [1, 2, 3, 17, 120, 240, 256, 930])
@pytest.mark.parametrize("rank_frac", [1.0, 0.3])
def test_eigen_vs_numpy(lib, n, rank_frac):
    rng = np.random.default_rng(7 * n + int(rank_frac * 10))
    r = max(1, int(n * rank_frac))
    X = (rng.standard_normal((n, r)) + 1j * rng.standard_normal((n, r))) * 0.05
    G = X @ X.conj().T
    W, V = _solve(lib, G)
    we = np.linalg.eigvalsh(G)
    top = np.max(np.abs(we))
    assert np.all(np.diff(W) >= -1e-12 * top)
    assert np.max(np.abs(W - we)) <= 1e-12 * top
    for u, lam in ((V[0], W[0]), (V[1], W[-1])):
        assert abs(np.linalg.norm(u) - 1.0) <= 1e-10
        assert np.linalg.norm(G @ u - lam * u) <= 1e-10 * top


def test_eigen_graded_spectrum(lib):
    """A spectrum spread over 12 decades (the MDL of a lossy transfer
    matrix): the smallest eigenvalues keep an absolute accuracy of 1e-12 * max."""
    rng = np.random.default_rng(11)
    n = 240
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    lam = np.logspace(-12, 0, n)
    G = (Q * lam) @ Q.conj().T
    G = 0.5 * (G + G.conj().T)
    W, V = _solve(lib, G)
    assert np.max(np.abs(W - np.linalg.eigvalsh(G))) <= 1e-12
    assert np.linalg.norm(G @ V[1] - W[-1] * V[1]) <= 1e-11


def test_eigen_rejects_oversize(lib):
    W = np.zeros(1)
    g = np.zeros(2)
    assert lib.digHoloB200EigenHermitian(4096, g.ctypes.data_as(C.POINTER(C.c_double)),
                                         W.ctypes.data_as(C.POINTER(C.c_double)), None) == 5
