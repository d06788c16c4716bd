"""CPU model of FP64-accurate products from int8 slices (an Ozaki-type splitting): the arithmetic a
tensor-core trailing update of the log-det's Cholesky would use on the int8 pipe.

Model: every row of A and every column of B is scaled by a power of two so that its largest entry
lies in [1/2, 1), then cut into s slices of 7 bits each (int8 values in [-127, 127], the first
slice from the leading bits, each next one from the remainder).  The slice products A_p B_q are
exact in int32 (k * 127^2 < 2^31), and the products with p + q <= s + 1 are reassembled in FP64:
s(s+1)/2 int8 products per FP64 product.  Each dropped term is below 2^(-7s) of the row and
column maxima.  No GPU is needed; nothing in the library uses this arithmetic yet.
"""
import numpy as np
import pytest


def slices(M, s, axis):
    """Integer slices (int64 arrays holding int8 values) and the power-of-two scale of each row
    (axis=1) or column (axis=0) of M."""
    amax = np.max(np.abs(M), axis=axis, keepdims=True)
    e = np.where(amax > 0, np.floor(np.log2(np.where(amax > 0, amax, 1.0))) + 1.0, 0.0)
    x = M * np.exp2(-e)  # |x| < 1, so every slice fits int8 (powers of two: exact)
    out = []
    for _ in range(s):
        x = x * 128.0
        q = np.trunc(x)
        assert np.max(np.abs(q)) <= 127
        out.append(q.astype(np.int64))
        x = x - q  # exact
    return out, e


def int8_matmul(A, B, s):
    """A @ B from s int8 slices of each operand, exact int products, FP64 reassembly."""
    sa, ea = slices(A, s, axis=1)
    sb, eb = slices(B, s, axis=0)
    C = np.zeros((A.shape[0], B.shape[1]))
    # smallest terms first
    for t in range(s + 1, 1, -1):
        acc = np.zeros_like(C)
        for p in range(1, t):
            q = t - p
            if q <= s:
                prod = sa[p - 1] @ sb[q - 1]
                assert np.max(np.abs(prod)) < 2 ** 31  # an int32 accumulator holds it
                acc += prod.astype(np.float64)
        C += acc * 2.0 ** (-7 * t)
    return C * np.exp2(ea) * np.exp2(eb)


def exact_matmul(A, B):
    return (A.astype(np.longdouble) @ B.astype(np.longdouble))


def graded_panel(m, k, seed):
    # a Cholesky panel: columns of decaying size, entries of mixed sign
    rng = np.random.default_rng(seed)
    return rng.standard_normal((m, k)) * np.exp(-np.arange(k) / (k / 4.0))[None, :]


# Measured on this panel (error relative to |P| |P^T|): FP64 GEMM 1.8e-15; slices s = 7: 4.3e-13,
# s = 8: 4.2e-15, s = 9: 1.3e-16.  Each slice adds 7 bits; the dropped cross terms (p + q = s + 2,
# s + 1 of them per k) cost about 6, so FP64 accuracy needs s = 8-9: 36-45 int8 products.
@pytest.mark.parametrize("s,factor", [(8, 4.0), (9, 1.0)])
def test_int8_slices_reach_fp64_gemm_accuracy(s, factor):
    P = graded_panel(192, 256, 1)
    ref = exact_matmul(P, P.T)
    bound = np.abs(P) @ np.abs(P.T)
    err_fp64 = float(np.max(np.abs(P @ P.T - ref) / bound))
    err_int8 = float(np.max(np.abs(int8_matmul(P, P.T, s) - ref) / bound))
    assert err_int8 < factor * max(err_fp64, 2.0 ** -53)


def test_cholesky_log_det_with_int8_trailing_updates():
    rng = np.random.default_rng(3)
    n, nb = 384, 64
    X = rng.standard_normal((n, 3 * n)) * np.exp(-np.arange(n) / 60.0)[:, None]
    M = np.eye(n) + 0.8 * (X @ X.T) / np.linalg.eigvalsh(X @ X.T).max()  # 1 + Pi with lambda_max = 0.8

    def logdet(update):
        A = M.copy()
        for j in range(0, n, nb):
            J = slice(j, j + nb)
            L = np.linalg.cholesky(A[J, J])
            A[J, J] = L
            if j + nb < n:
                T = slice(j + nb, n)
                A[T, J] = np.linalg.solve(L, A[T, J].T).T
                A[T, T] -= update(A[T, J], A[T, J].T)
        return 2.0 * np.sum(np.log(np.diag(A)))

    # relative log-det error with s slices in every trailing update: s = 4: 1.1e-10, 5: 1.0e-12,
    # 6: 1.0e-14, 7 and 8: 0 (1 + Pi with lambda <= 0.8 is well conditioned)
    ref = logdet(lambda P, Q: P @ Q)
    assert abs(logdet(lambda P, Q: int8_matmul(P, Q, 6)) - ref) < 1e-13 * abs(ref)
    assert abs(logdet(lambda P, Q: int8_matmul(P, Q, 8)) - ref) < 1e-14 * abs(ref)
    assert abs(ref - np.linalg.slogdet(M)[1]) < 1e-12 * abs(ref)
