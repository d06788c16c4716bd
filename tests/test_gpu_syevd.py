"""GPU tests of rpa_b200_syevd, the symmetric eigensolver behind the T2 and
MBPT3 paths (replacement of real_EVD / LAPACK dsyevd), against numpy.linalg.eigh.

Tolerances: eigenvalues to 1e-12 * max|lambda|; residual |A Z - Z diag(w)|
and orthogonality |Z^T Z - I| to 1e-12 (relative to max|lambda| for the residual).
Cases cover one leaf (n <= 32), ragged trees, full deflation (identity, diagonal),
tight clusters, graded spectra and rank-deficient Gram matrices like the T2 one.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(handle, A, tol=1e-12):
    w, Z = handle.syevd(A)
    ref = np.linalg.eigvalsh(A)
    nrm = max(float(np.abs(ref).max()), 1e-300)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w - ref).max() <= tol * nrm
    assert np.abs(A @ Z - Z * w[None, :]).max() <= tol * nrm
    assert np.abs(Z.T @ Z - np.eye(len(w))).max() <= tol


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 64, 100, 257, 1000])
def test_random_symmetric(handle, n):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, n))
    _check(handle, X + X.T)


def test_full_deflation(handle):
    rng = np.random.default_rng(1)
    _check(handle, np.eye(150))
    _check(handle, np.diag(rng.standard_normal(300)))


def test_clusters_and_graded_spectrum(handle):
    rng = np.random.default_rng(2)
    Q, _ = np.linalg.qr(rng.standard_normal((300, 300)))
    w = np.repeat([1.0, 2.0, 3.0], 100) + 1e-13 * rng.standard_normal(300)
    _check(handle, (Q * w) @ Q.T)
    w = np.logspace(-14, 2, 300)
    _check(handle, (Q * w) @ Q.T)


def test_rank_deficient_gram(handle):
    # the T2 range finder's Gram matrix: normalised columns, numerical rank < n
    rng = np.random.default_rng(3)
    Y = rng.standard_normal((700, 90)) @ rng.standard_normal((90, 400))
    Y /= np.linalg.norm(Y, axis=0)
    _check(handle, Y.T @ Y)


def test_device_arrays_and_leading_dimension(handle):
    import torch
    rng = np.random.default_rng(4)
    n = 130
    X = rng.standard_normal((n, n))
    A = X + X.T
    big = np.zeros((n + 7, n))
    big[:n] = A
    At = torch.from_numpy(np.ascontiguousarray(big.T)).cuda()  # column-major (n+7) x n = At.T
    w = torch.zeros(n, dtype=torch.float64, device="cuda")
    lib = handle.lib
    assert lib.rpa_b200_syevd(handle._h, n, At.data_ptr(), n + 7, w.data_ptr()) == 0
    Z = At.T.cpu().numpy()[:n]
    wn = w.cpu().numpy()
    assert np.abs(wn - np.linalg.eigvalsh(A)).max() < 1e-12 * np.abs(wn).max()
    assert np.abs(A @ Z - Z * wn[None, :]).max() < 1e-12 * np.abs(wn).max()
