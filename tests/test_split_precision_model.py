"""CPU model of the split-BF16 arithmetic the tensor-core kernels use, checked against the FP64
oracle: why three bf16 products with FP32 accumulation in short segments meet the precision
budget of the exchange contraction and of the ring contractions of the T2 range finder.

Model: X = hi + lo with hi = bf16(x), lo = bf16(x - hi); each 16-deep K block of a product is
exact (bf16 x bf16 products are exact in FP32 and the block is summed before rounding) and is
added to an FP32 accumulator with round-toward-zero, the tensor core's accumulation rounding;
accumulators are restarted every `seg` K columns and the segments are added in IEEE FP32.
No GPU is needed.
"""
import math

import numpy as np
import pytest

from oracle import rpa_oracle as O


def bf16(x):
    x = np.asarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def split(x):
    hi = bf16(x)
    lo = bf16(x.astype(np.float32) - hi)
    return hi.astype(np.float64), lo.astype(np.float64)


def rz_add(acc32, v64):
    s = acc32.astype(np.float64) + v64
    f = s.astype(np.float32)
    over = np.abs(f.astype(np.float64)) > np.abs(s)
    f[over] = np.nextafter(f[over], np.float32(0))
    return f


def split_matmul(A, B, seg=64):
    """A (m x k) B^T-style product A @ B with both operands split, tensor-core accumulation model."""
    ah, al = split(A)
    bh, bl = split(B)
    m, k = A.shape
    n = B.shape[1]
    total = np.zeros((m, n), dtype=np.float32)
    for s0 in range(0, k, seg):
        acc = np.zeros((m, n), dtype=np.float32)
        for c0 in range(s0, min(k, s0 + seg), 16):
            sl = slice(c0, min(c0 + 16, k))
            for x, y in ((ah, bh), (ah, bl), (al, bh)):
                acc = rz_add(acc, x[:, sl] @ y[sl, :])
        total = (total.astype(np.float64) + acc.astype(np.float64)).astype(np.float32)
    return total.astype(np.float64)


def test_bf16_pair_keeps_16_bits():
    x = np.random.default_rng(0).standard_normal(10000) * 10.0 ** np.random.default_rng(1).uniform(-6, 6, 10000)
    hi, lo = split(x)
    assert np.max(np.abs(x - hi - lo) / np.abs(x)) < 2.0 ** -16


def _t2_case(seed=1, nq=96, no=5, nv=32):
    s = O.make_system(nq, no, nv, seed, decay=nq / 5.0, lam0=0.6)
    x, w = O.grid_for(s, 10)
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    vals, vecs = O.diagonalize_pi(pi)
    nov = no * nv
    omega = np.random.default_rng(seed).uniform(size=(nov, min(3 * nq, nov))) - 0.5
    A, U, _ = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-4)
    return s, A, U


@pytest.mark.parametrize("seg,bound", [(64, 5e-6), (512, 5e-5)])
def test_split_exchange_contraction_model(seg, bound):
    # W_ij = R_i U_j^T with the model above; E_x as in rpa_CC_EcExchange1
    s, A, U = _t2_case()
    ref = O.exchange_sosex(np.ascontiguousarray(U.T), A, s.R, s.no, s.nv)
    Rr = s.R.reshape(s.nq, s.nv, s.no, order="F")
    Ur = U.T.reshape(len(A), s.nv, s.no, order="F")
    e = []
    for j in range(s.no):
        for i in range(j, s.no):
            wij = split_matmul(Rr[:, :, i], Ur[:, :, j].T, seg)
            wji = split_matmul(Rr[:, :, j], Ur[:, :, i].T, seg) if i != j else wij
            e.append((1.0 if i == j else 2.0) * -float(np.sum(wij * wji * A[None, :])))
    got = math.fsum(e)
    assert abs(got - ref) < bound * abs(ref)


def test_split_ring_contractions_keep_the_t2_subspace():
    # I(1) M = -(1/4 pi) Z^T (Z M) with both products in the split model: the Gram rank, the
    # number of kept amplitudes and A itself stay those of the FP64 range finder
    s, A64, U64 = _t2_case(seed=2)
    x, w = O.grid_for(s, 10)
    d = O.dai(s.eps_o, s.eps_v)
    Z = []
    for k in range(len(x)):
        c = d / (d * d + x[k] ** 2)
        L = np.linalg.cholesky(np.eye(s.nq) + 4.0 * (s.R * c) @ s.R.T)
        Z.append(math.sqrt(w[k]) * np.linalg.solve(L, s.R * (-4.0 * c)))
    Z = np.vstack(Z)

    def run(split_mode):
        nov = Z.shape[1]
        G = min(3 * s.nq, nov)
        om = np.random.default_rng(2).uniform(size=(nov, G)) - 0.5
        om /= np.linalg.norm(om, axis=0)

        def apply_I(M):
            if split_mode:
                return -1.0 / (4 * math.pi) * split_matmul(Z.T, split_matmul(Z, M))
            return -1.0 / (4 * math.pi) * (Z.T @ (Z @ M))

        iom = apply_I(om)
        iom /= np.linalg.norm(iom, axis=0)
        sv, sV = np.linalg.eigh(iom.T @ iom)
        nt = int(np.sum(sv > 1e-10))
        T = iom @ (sV[:, G - nt:] / np.sqrt(sv[G - nt:]))
        tit = T.T @ apply_I(T)
        a = np.linalg.eigvalsh(0.5 * (tit + tit.T))
        amp = 0.5 * a / (a + 1.0)
        return nt, amp[np.abs(amp) > 1e-4]

    nt64, a64 = run(False)
    nt16, a16 = run(True)
    assert nt16 == nt64 and len(a16) == len(a64)
    assert np.max(np.abs(a16 - a64)) < 2e-5 * np.max(np.abs(a64))
