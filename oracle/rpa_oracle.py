"""FP64 CPU oracle for the Cholesky-vector RPA hot path.

TEST INFRASTRUCTURE ONLY.  This module checks the library: it is imported by
``tests/``, by ``__graft_entry__.smoke()`` and by the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py``, and by nothing else.  The product
path (``beyond-rpa_b200/``) never imports, links or executes it.

It restates, in numpy/scipy (ILP64 OpenBLAS/LAPACK, the same BLAS/LAPACK
routines the Fortran reference calls through MKL), the math of
modrzejewski/beyond-rpa for this path.  Every function cites the reference
file:line it follows (paths relative to the reference project root).

Parity status: **parity unpinned by the reference's own tests.**  The
reference ships no test suite, golden vectors or output logs, and it cannot
be compiled here (Fortran 2008 + MKL + coarrays; no gfortran in the image).
The restatement is pinned instead by the reference's built-in identities:
  (i)   E_c(log-det of Pi) == E_c(T2 eigen-decomposition), rpa_T2_EigRPA
        (src/rpa/rpa_CC_Doubles.f90:987-1009);
  (ii)  the small-coupling limit R -> eps*R equals the direct-MP2 formula of
        rpa_PT_Order2 (src/rpa/rpa_PT_Terms.f90:66) up to the frequency
        quadrature error;
  (iii) log-det by QR (the reference's DGEQRF) == Cholesky == sum ln(1+lambda);
  (iv)  exactness of the frequency grid on 1/(D^2+u^2)
        (src/rpa/OptFreqQuad.f90:125-169);
  (v)   size consistency of many-body-expansion differences
        (src/rpa/rpa_driver.f90:381-433).
The checks live in tests/test_oracle.py and the fixtures in tests/golden/.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg
import scipy.linalg.lapack as lapack

PI = math.pi
# src/rpa/rpa_definitions.f90:109-110
RPA_MIN_NFREQS = 8
RPA_MAX_NFREQS = 64
# src/rpa/rpa_definitions.f90:295-296,301,305,356,428,480
TARGET_ERROR_FREQ = 1.0e-6
TARGET_REL_ERROR_FREQ = 1.0e-3
CORE_ORB_THRESH = -3.0
SMALL_EIGENVAL_CUTOFF_T2 = 1.0e-10
MAX_BATCH_DIM_T2 = 100
GUESS_NVECS_T2 = 3.0
T2_CUTOFF_THRESH = 1.0e-4
# src/rpa/rpa_THC.f90:464 (THC_BlockDim)
THC_BLOCK_DIM = 500
# src/rpa/rpa_definitions.f90: T2 cutoff types (RPA_T2_CUTOFF_*)
T2_CUTOFF_EIG = 0
T2_CUTOFF_EIG_DIV_MAXEIG = 1
T2_CUTOFF_EIG_DIV_NELECTRON = 2
T2_CUTOFF_SUM_REJECTED = 3


# --------------------------------------------------------------------------
# Orbital-energy bookkeeping
# --------------------------------------------------------------------------

def ncore(orb_energies, nocc, core_thresh=CORE_ORB_THRESH):
    """Frozen-core count. rpa_NCore, src/rpa/OrbDiffHist.f90:126-146."""
    n = 0
    for k in range(nocc):
        if orb_energies[k] < core_thresh:
            n += 1
        else:
            break
    return n


def dai(eps_o, eps_v):
    """D(a,i) = e_a - e_i in the reference's ai = a + NVirt*(i-1) order.

    rpa_CC_D, src/rpa/rpa_CC_Doubles.f90:348-366 (a is the fast index)."""
    eps_o = np.asarray(eps_o, np.float64)
    eps_v = np.asarray(eps_v, np.float64)
    return (eps_v[:, None] - eps_o[None, :]).reshape(-1, order="F")


def dai_max_thresh(orb_energies, nocc, nvirt, core_thresh=CORE_ORB_THRESH):
    """Largest active excitation energy e_a1 - e_i0 (0 when every occupied orbital is frozen).

    rpa_DaiMaxThresh, src/rpa/OrbDiffHist.f90:10-39 (one spin)."""
    e = np.asarray(orb_energies, np.float64)
    nc = ncore(e, nocc, core_thresh)
    return float(e[nocc + nvirt - 1] - e[nc]) if nc < nocc else 0.0


def grid_for_cluster(sets, limit_dai=True, n=None, core_thresh=CORE_ORB_THRESH):
    """One grid for the subsystems of a many-body expansion: sets = [(orb_energies, nocc, nvirt)]
    with sets[0] the whole complex; histograms capped at its largest excitation energy when
    limit_dai (rpa_PostSCF, src/rpa/rpa_driver.f90:118-175)."""
    thresh = dai_max_thresh(*sets[0], core_thresh) if limit_dai else np.inf
    vals, wts = [], []
    for e, no, nv in sets:
        v, w = dai_histogram(e, no, nv, core_thresh, thresh)
        vals.append(v)
        wts.append(w)
    dv, dw = np.array(vals).T, np.array(wts).T
    if n is not None:
        x, w, *_ = opt_quad_scaling(n, dv, dw)
        return x, w
    return optimize_freq_quad(dv, dw)


def dai_histogram(orb_energies, nocc, nvirt, core_thresh=CORE_ORB_THRESH,
                  dai_max_thresh=np.inf, nbins=100):
    """Histogram of orbital-energy differences used by the grid optimiser.

    rpa_DaiHistogram, src/rpa/OrbDiffHist.f90:42-123."""
    e = np.asarray(orb_energies, np.float64)
    nc = ncore(e, nocc, core_thresh)
    if nc >= nocc:
        vals = np.zeros(nbins)
        vals[0] = np.finfo(np.float64).max
        vals[-1] = 0.0
        return vals, -np.ones(nbins)
    i0, i1 = nc, nocc - 1
    a0, a1 = nocc, nocc + nvirt - 1
    dmin = e[a0] - e[i1]
    dmax = min(dai_max_thresh, e[a1] - e[i0])
    if not dmin > 0.0:
        raise ValueError("Found invalid orbital energy gap. Cannot decompose energy denominators.")
    width = (dmax - dmin) / nbins
    vals = dmin + np.arange(nbins) * width
    d = (e[a0:a1 + 1][None, :] - e[i0:i1 + 1][:, None]).ravel()
    d = d[d <= dai_max_thresh]
    # nint() is round-half-away-from-zero in Fortran; the bin index is clamped to [1, nbins] as
    # the reference does, in floating point (a zero width, i.e. one distinct difference, gives
    # 0/0: bin 1, where gfortran's nint of a NaN clamps to)
    with np.errstate(invalid="ignore", divide="ignore"):
        x = (d - (dmin + width / 2.0)) / width
    kf = 1.0 + np.where(x >= 0, np.floor(x + 0.5), -np.floor(-x + 0.5))
    k = np.where(np.isnan(kf) | (kf < 1.0), 1.0, np.minimum(kf, nbins)).astype(np.int64)
    count = np.bincount(k - 1, minlength=nbins).astype(np.float64)
    with np.errstate(invalid="ignore"):  # no difference under the cap: 0/0, as in the reference
        return vals, np.abs(count / count.sum())


# --------------------------------------------------------------------------
# Frequency quadrature (transformed Gauss-Legendre, "Casimir-Polder")
# --------------------------------------------------------------------------

def gauss_legendre(n, max_abs_error=1.0e-14):
    """All n Gauss-Legendre roots (ascending) and weights on (-1,1).

    Follows quad_GaussLegendre, src/rpa/quadratures.f90:418-509: Newton
    iteration on theta = arccos(x) with the three-term Legendre recurrence
    (LegendrePolynomial, quadratures.f90:309-328) and weights
    w = 2 / (dP_n/dtheta)^2.  The initial guesses here are the classical
    theta_k = pi (k - 1/4)/(n + 1/2) (the reference uses the Tricomi and
    Gatteschi asymptotic guesses of the same roots); the converged roots agree
    to the Newton tolerance."""
    k = np.arange(1, n + 1, dtype=np.float64)
    theta = PI * (k - 0.25) / (n + 0.5)

    def legendre(x):
        pb = np.zeros_like(x)
        pa = np.ones_like(x)
        for a in range(1, n + 1):
            pc = pb
            pb = pa
            pa = (2 * a - 1.0) / a * x * pb - (a - 1.0) / a * pc
        return pa, pb

    for _ in range(100):
        x = np.cos(theta)
        pa, pb = legendre(x)
        p_theta = n * (x * pa - pb) / np.sin(theta)
        new = theta - pa / p_theta
        done = np.all(np.abs(new - theta) < max_abs_error)
        theta = new
        if done:
            break
    x = np.cos(theta)
    pa, pb = legendre(x)
    p_theta = n * (x * pa - pb) / np.sin(theta)
    w = 2.0 / p_theta ** 2
    order = np.argsort(x)
    return x[order], w[order]


def casimir_polder(n, alpha=0.5):
    """Semi-infinite GL quadrature x = a(1+t)/(1-t), w = 2 a w_GL/(1-t)^2.

    quad_CasimirPolder, src/rpa/quadratures.f90:570-643 (points ascending)."""
    t, wgl = gauss_legendre(n)
    x = alpha * (1.0 + t) / (1.0 - t)
    w = 2.0 * wgl * alpha / (1.0 - t) ** 2
    return x, w


def freq_quad_error(freqs, weights, dai_values, dai_weights):
    """(MaxRelError, RMSD) of sum_k w_k/(d^2+u_k^2) vs pi/(2d).

    rpa_FreqQuadError, src/rpa/OptFreqQuad.f90:125-169.  dai_values and
    dai_weights are (NBins, NDaiSets)."""
    dv = np.atleast_2d(np.asarray(dai_values, np.float64).T).T
    dw = np.atleast_2d(np.asarray(dai_weights, np.float64).T).T
    rel = np.zeros(dv.shape[1])
    err2 = np.zeros(dv.shape[1])
    for s in range(dv.shape[1]):
        m = dw[:, s] > 0.0
        d = dv[m, s]
        exact = PI / (2.0 * d)
        approx = (weights[None, :] / (d[:, None] ** 2 + freqs[None, :] ** 2)).sum(axis=1)
        if d.size:
            rel[s] = np.max(np.abs((approx - exact) / exact))
            err2[s] = np.sum(dw[m, s] * (approx - exact) ** 2)
    return float(rel.max()), float(math.sqrt(err2.max()))


def opt_quad_scaling(n, dai_values, dai_weights, min_alpha=0.1, max_alpha=15.0, nscan=15000):
    """Scan of the scale alpha minimising the RMSD.

    rpa_OptQuadScaling, src/rpa/OptFreqQuad.f90:75-122 (first minimum wins,
    strict '<' comparison)."""
    x0, w0 = casimir_polder(n, 1.0)
    dv = np.atleast_2d(np.asarray(dai_values, np.float64).T).T
    dw = np.atleast_2d(np.asarray(dai_weights, np.float64).T).T
    alphas = min_alpha + (max_alpha - min_alpha) * np.arange(nscan) / (nscan - 1)
    best = (np.inf, 0.0, 0.0)
    err2 = np.zeros((nscan, dv.shape[1]))
    rel = np.zeros((nscan, dv.shape[1]))
    for s in range(dv.shape[1]):
        m = dw[:, s] > 0.0
        if not m.any():  # no bin with weight > 0 (e.g. every difference above the cap): no error
            continue
        d = dv[m, s]
        exact = PI / (2.0 * d)
        for c0 in range(0, nscan, 1000):
            a = alphas[c0:c0 + 1000]
            u = a[:, None] * x0[None, :]
            w = a[:, None] * w0[None, :]
            approx = np.einsum("ak,abk->ab", w, 1.0 / (d[None, :, None] ** 2 + u[:, None, :] ** 2))
            err2[c0:c0 + 1000, s] = ((approx - exact[None, :]) ** 2 * dw[m, s][None, :]).sum(axis=1)
            rel[c0:c0 + 1000, s] = np.abs((approx - exact[None, :]) / exact[None, :]).max(axis=1)
    rmsd = np.sqrt(err2.max(axis=1))
    maxrel = rel.max(axis=1)
    for k in range(nscan):
        if rmsd[k] < best[0]:
            best = (rmsd[k], maxrel[k], alphas[k])
    a = best[2]
    return a * x0, a * w0, a, best[1], best[0]


def optimize_freq_quad(dai_values, dai_weights, target_error=TARGET_ERROR_FREQ,
                       target_rel_error=TARGET_REL_ERROR_FREQ,
                       min_n=RPA_MIN_NFREQS, max_n=RPA_MAX_NFREQS):
    """Smallest n whose optimally scaled grid meets both targets.

    rpa_OptimizeFreqQuad, src/rpa/OptFreqQuad.f90:12-72."""
    for n in range(min_n, max_n + 1):
        x, w, a, rel, rmsd = opt_quad_scaling(n, dai_values, dai_weights)
        if rmsd < target_error and rel < target_rel_error:
            return x, w
    raise RuntimeError("Quadrature did not converge to specified accuracy")


# --------------------------------------------------------------------------
# Pi(u) build
# --------------------------------------------------------------------------

def chi_factor(d, freq):
    """Chi = D/(D^2 + u^2). rpa_THC_ChiRkai, src/rpa/rpa_THC.f90:360-370."""
    return d / (d * d + freq * freq)


def pi_matrices(R, eps_o, eps_v, freqs, alpha=4.0, block_dim=THC_BLOCK_DIM):
    """Pi(:,:,u) = alpha * sum_ai R(:,ai) Chi_u(ai) R(:,ai)^T, full square FP64.

    rpa_THC_PiU / rpa_THC_PiU_BlockAlgo, src/rpa/rpa_THC.f90:215-340:
    ai columns in blocks of THC_BlockDim, for every frequency
    W = Chi*R_blk (rpa_THC_ChiRkai) then DGEMM Pi += alpha R_blk W^T
    (real_abT_x, beta = 1).  alpha = 4 closed shell, 2 per spin open shell
    (rpa_THC.f90:258-268)."""
    R = np.asarray(R, np.float64)
    nq, nov = R.shape
    d = dai(eps_o, eps_v)
    assert d.size == nov
    K = len(freqs)
    pi = np.zeros((K, nq, nq))
    for t in range(0, nov, block_dim):
        blk = R[:, t:t + block_dim]
        db = d[t:t + block_dim]
        for u in range(K):
            W = blk * chi_factor(db, freqs[u])[None, :]
            pi[u] += alpha * (blk @ W.T)
    return pi


# --------------------------------------------------------------------------
# Energy: ln det(1+Pi) - Tr Pi, frequency quadrature
# --------------------------------------------------------------------------

def logdet_qr(A):
    """ln|det A| via DGEQRF and sum ln|R_kk| accumulated exactly.

    real_LogDet, src/linear-algebra/real_linalg.f90:793-825.  The reference
    accumulates log(|a_kk|) in REAL(16); here the logs are FP64 and their
    sum is exactly rounded (math.fsum), which agrees to well below 1e-14."""
    qr, tau, work, info = lapack.dgeqrf(np.array(A, np.float64, order="F"))
    if info != 0:
        raise RuntimeError(f"DGEQRF returned error code {info}")
    return math.fsum(np.log(np.abs(np.diag(qr))).tolist())


def logdet_cholesky(A):
    """2 sum ln L_kk (identity (iii) against logdet_qr)."""
    L = np.linalg.cholesky(A)
    return 2.0 * math.fsum(np.log(np.diag(L)).tolist())


def ec_rpa_analytic(pi, weights, logdet=logdet_qr):
    """E_c = 1/(2 pi) sum_u w_u [ln det(1+Pi_u) - Tr Pi_u] and the E(u) list.

    rpa_CC_EcRPA_Analytic, src/rpa/rpa_CC.f90:412-471 (traces and E(u) in
    REAL(16): exactly rounded sums here)."""
    K = pi.shape[0]
    eu = np.zeros(K)
    terms = []
    for u in range(K):
        W = pi[u]
        tr = math.fsum(np.diag(W).tolist())
        A = W + np.eye(W.shape[0])
        ld = logdet(A)
        eu[u] = ld - tr
        terms.append(eu[u] * weights[u] / (2.0 * PI))
    return math.fsum(terms), eu


def ec_rpa(R, eps_o, eps_v, freqs, weights, alpha=4.0):
    """Pi build + analytic energy (the fused path the boundary replaces)."""
    pi = pi_matrices(R, eps_o, eps_v, freqs, alpha)
    return ec_rpa_analytic(pi, weights)


def direct_mp2(R, eps_o, eps_v):
    """Direct (ring) MP2: 2 sum_{ai,bj} (ai|bj)^2 / (e_i + e_j - e_a - e_b).

    rpa_PT_Order2 direct term, src/rpa/rpa_PT_Terms.f90:66 (closed shell,
    spatial orbitals).  E_c(RPA) of eps*R tends to this times eps^4."""
    d = dai(eps_o, eps_v)
    V = R.T @ R
    return 2.0 * float(np.sum(V * V / (-(d[:, None] + d[None, :]))))


# --------------------------------------------------------------------------
# Pi eigen-decomposition, direct-ring T2, EigRPA
# --------------------------------------------------------------------------

def diagonalize_pi(pi):
    """Ascending eigenpairs of every Pi(u). rpa_CC_Diagonalize_PiU,
    src/rpa/rpa_CC.f90:1108-1129 (symmetric_eigenproblem)."""
    w, v = np.linalg.eigh(pi)
    return w, v


def _apply_I(M, R, d, freqs, fweights, pi_vals, pi_vecs, lam):
    """I(lambda) M = -sum_u w_u/(4 pi) Chi_u R^T Q_u diag(l/(1+l pi_u)) Q_u^T R Chi_u M.

    rpa_CC_IM_v5, src/rpa/rpa_CC_Doubles.f90:369-422, with
    Chi_u = -4 D/(D^2+u^2) (rpa_CC_Chi, 276-292)."""
    out = np.zeros_like(M)
    for u in range(len(freqs)):
        chi = -(4.0 * d) / (d * d + freqs[u] ** 2)
        Q = pi_vecs[u]
        RChiM = R @ (chi[:, None] * M)
        MTChiRTQ = RChiM.T @ Q
        MTChiRTQ *= (lam / (1.0 + lam * pi_vals[u]))[None, :]
        MTChiRTQWQT = MTChiRTQ @ Q.T
        out += (-fweights[u] / (4.0 * PI)) * (chi[:, None] * (R.T @ MTChiRTQWQT.T))
    return out


def _normalize_columns(M):
    """rpa_CC_NormalizeColumns, src/rpa/rpa_CC_Doubles.f90:80-91."""
    return M / np.linalg.norm(M, axis=0)[None, :]


def t2_direct_ring(R, eps_o, eps_v, freqs, fweights, pi_vals, pi_vecs, omega,
                   lam=1.0, small_cutoff=SMALL_EIGENVAL_CUTOFF_T2,
                   cutoff_thresh=T2_CUTOFF_THRESH, cutoff_type=T2_CUTOFF_EIG,
                   common_thresh=-1.0, nocc=None):
    """Direct-ring T2 = U diag(A) U^T by randomised range finding.

    rpa_THC_CC_T2, src/rpa/rpa_CC_Doubles.f90:645-984 (sharp cutoff branch):
      IOmega = normalize(I(l) normalize(Omega))           (747-763)
      S = IOmega^T IOmega, EVD, keep eigenvalues > 1e-10  (770-781)
      T = IOmega S_vecs / sqrt(S_vals)                     (786-795)
      TIT = T^T I T, EVD, A = a/(2(a+1))                   (797-808)
      cutoff |A| <= K, K = T2CutoffThresh (supersystem) or the common
      threshold of the supersystem (subsystems)            (855-945)
      U = T TIT_vecs(:, 1:NT)                              (973-975)
    omega holds the guess vectors (nov x G): the reference draws them from
    gfortran's random_number stream, which is not reproducible outside
    gfortran, so parity is at the level of the converged subspace.
    Returns (A, U, K)."""
    d = dai(eps_o, eps_v)
    G = omega.shape[1]
    IOmega = np.zeros_like(omega)
    for q0 in range(0, G, MAX_BATCH_DIM_T2):
        Om = _normalize_columns(omega[:, q0:q0 + MAX_BATCH_DIM_T2])
        IOmega[:, q0:q0 + MAX_BATCH_DIM_T2] = _normalize_columns(
            _apply_I(Om, R, d, freqs, fweights, pi_vals, pi_vecs, lam))
    S = IOmega.T @ IOmega
    s_vals, s_vecs = np.linalg.eigh(S)
    nt = 0
    for i in range(G - 1, -1, -1):
        if s_vals[i] > small_cutoff:
            nt += 1
        else:
            break
    W = s_vecs[:, G - nt:] / np.sqrt(s_vals[G - nt:])[None, :]
    T = IOmega @ W
    TIT = T.T @ _apply_I(T, R, d, freqs, fweights, pi_vals, pi_vecs, lam)
    TIT = 0.5 * (TIT + TIT.T)
    a, vecs = np.linalg.eigh(TIT)
    A = 0.5 * (a / (a + 1.0))
    if common_thresh < 0.0:
        if cutoff_type == T2_CUTOFF_EIG:
            K = cutoff_thresh
        elif cutoff_type == T2_CUTOFF_EIG_DIV_MAXEIG:
            K = cutoff_thresh * np.max(np.abs(A))
        elif cutoff_type == T2_CUTOFF_EIG_DIV_NELECTRON:
            K = cutoff_thresh / (nocc * 2)
        elif cutoff_type == T2_CUTOFF_SUM_REJECTED:
            K = 0.0
            for i in range(len(A) - 1):
                if abs(A[i + 1:].sum()) < cutoff_thresh:
                    K = abs(A[i + 1])
                    break
        else:
            raise ValueError("Invalid value of T2CutoffThresh")
    else:
        K = common_thresh
    keep = 0
    for i in range(len(A)):
        if abs(A[i]) > K:
            keep = i + 1
        else:
            break
    if keep == 0:
        raise RuntimeError("Invalid T2CutoffThresh: no eigenvectors left after cutoff")
    U = T @ vecs[:, :keep]
    return A[:keep].copy(), U, K


def t2_eig_rpa(U, A, R):
    """EigRPA(mu) = 2 A_mu ||R U_mu||^2.

    rpa_T2_EigRPA, src/rpa/rpa_CC_Doubles.f90:987-1009; the sum is stored as
    RPA_ENERGY_T2_DIRECT_RING (src/rpa/rpa_THC.f90:126)."""
    RU = R @ U
    return 2.0 * A * np.sum(RU * RU, axis=0)


def exchange_sosex(V, A, R, nocc, nvirt, alpha=1.0, s2_operator=False):
    """E_x = -alpha sum_{abij} (aj|bi) T_aibj.

    rpa_CC_Exchange_SOSEX + rpa_CC_EcExchange1,
    src/rpa/rpa_CC_Exchange.f90:36-116.  V is (NT, NVirt, NOcc) (the
    NVecsT2 x nov row layout of that routine), R is (NQ, NVirt, NOcc);
    B = A/(1-4A^2) when the S2 operator is requested."""
    nq = R.shape[0]
    nt = V.shape[0]
    Rr = R.reshape(nq, nvirt, nocc, order="F")
    Vr = V.reshape(nt, nvirt, nocc, order="F")
    B = A / (1.0 - 4.0 * A * A) if s2_operator else A
    e = []
    for j in range(nocc):
        for i in range(j, nocc):
            Wij = Rr[:, :, i] @ Vr[:, :, j].T
            if i != j:
                Wji = Rr[:, :, j] @ Vr[:, :, i].T
                e.append(-2.0 * float(np.sum(Wji * Wij * B[None, :])))
            else:
                e.append(-float(np.sum(Wij * Wij * B[None, :])))
    return alpha * math.fsum(e)


# --------------------------------------------------------------------------
# Adjoint (no reference counterpart): dE_c/dR, dE_c/de
# --------------------------------------------------------------------------

def ec_grad(R, eps_o, eps_v, freqs, weights, alpha=4.0):
    """Analytic gradient of E_c = 1/(2pi) sum_u w_u [ln det(1+Pi_u) - Tr Pi_u].

    The reference has no gradients; this is the FP64 reference gradient:
      dE/dR(:,ai) = 1/(2pi) sum_u w_u 2 alpha c_u(ai) M_u R(:,ai),
      M_u = (1+Pi_u)^-1 - 1;
      dE/dD(ai)  = 1/(2pi) sum_u w_u alpha R(:,ai)^T M_u R(:,ai) dc_u/dD,
      dc/dD = (u^2 - D^2)/(D^2+u^2)^2; dD(ai)/de_a = 1, dD(ai)/de_i = -1."""
    nq, nov = R.shape
    no, nv = len(eps_o), len(eps_v)
    d = dai(eps_o, eps_v)
    pi = pi_matrices(R, eps_o, eps_v, freqs, alpha)
    dR = np.zeros_like(R)
    dD = np.zeros(nov)
    for u in range(len(freqs)):
        c = chi_factor(d, freqs[u])
        M = np.linalg.inv(np.eye(nq) + pi[u]) - np.eye(nq)
        MR = M @ R
        f = weights[u] / (2.0 * PI)
        dR += f * 2.0 * alpha * c[None, :] * MR
        dcdD = (freqs[u] ** 2 - d * d) / (d * d + freqs[u] ** 2) ** 2
        dD += f * alpha * np.sum(R * MR, axis=0) * dcdD
    dD2 = dD.reshape(nv, no, order="F")
    return dR, -dD2.sum(axis=0), dD2.sum(axis=1)


# --------------------------------------------------------------------------
# Many-body-expansion differences
# --------------------------------------------------------------------------

def eint_2body(e_ab, e_a, e_b):
    """rpa_Eint2Body, src/rpa/rpa_driver.f90:381-386 (FP64, left to right)."""
    return (e_ab - e_a) - e_b


def eint_nadd3(e):
    """3-body nonadditive energy from the 7 subsystem energies
    [ABC, AB, AC, BC, A, B, C]. rpa_EintNadd, src/rpa/rpa_driver.f90:389-400: the group
    differences in FP64, their combination in REAL(16) (here: exact sum, rounded once)."""
    abc, ab, ac, bc, a, b, c = e
    eabc = ((abc - a) - b) - c
    eab, ebc, eac = (ab - a) - b, (bc - b) - c, (ac - a) - c
    return math.fsum([eabc, -eab, -ebc, -eac])


def mbe_energy(nbody, e):
    """Interaction / nonadditive energy from subsystem energies in the reference order
    (src/common/sys_definitions.f90:19-36, 0-based): total, A, B, C, AB, BC, AC, D, AD, BD, CD,
    ABC, ABD, ACD, BCD.  rpa_Eint2Body / rpa_EintNadd / rpa_EintNadd4Body,
    src/rpa/rpa_driver.f90:381-433."""
    if nbody == 2:
        return eint_2body(e[0], e[1], e[2])
    tot, A, B, C, AB, BC, AC = e[:7]
    if nbody == 3:
        return eint_nadd3([tot, AB, AC, BC, A, B, C])
    D, AD, BD, CD, ABC, ABD, ACD, BCD = e[7:15]
    eabcd = (((tot - A) - B) - C) - D
    eabc, eabd = ((ABC - A) - B) - C, ((ABD - A) - B) - D
    eacd, ebcd = ((ACD - A) - C) - D, ((BCD - B) - C) - D
    eab, ebc, eac = (AB - A) - B, (BC - B) - C, (AC - A) - C
    ead, ebd, ecd = (AD - A) - D, (BD - B) - D, (CD - C) - D
    return math.fsum([eabcd, -eab, -ebc, -eac, -ead, -ebd, -ecd,
                      -eabc, eab, ebc, eac, -eabd, eab, ead, ebd,
                      -eacd, eac, ead, ecd, -ebcd, ebc, ebd, ecd])


# --------------------------------------------------------------------------
# Seeded synthetic inputs with the shapes of the measured workloads
# --------------------------------------------------------------------------

@dataclass
class RPASystem:
    R: np.ndarray            # (NQ, nov) FP64, ai = a + nv*i
    eps_o: np.ndarray        # active occupied energies (no)
    eps_v: np.ndarray        # virtual energies (nv)
    freqs: np.ndarray = field(default=None)
    weights: np.ndarray = field(default=None)
    alpha: float = 4.0

    @property
    def nq(self):
        return self.R.shape[0]

    @property
    def no(self):
        return len(self.eps_o)

    @property
    def nv(self):
        return len(self.eps_v)


def lambda_max_pi0(R, d, alpha=4.0, iters=60, seed=0):
    """Largest eigenvalue of Pi(0) = alpha R diag(1/D) R^T by power iteration."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(R.shape[0])
    lam = 0.0
    for _ in range(iters):
        w = alpha * (R @ ((R.T @ v) / d))
        lam = float(np.linalg.norm(w))
        v = w / lam
    return lam


def make_system(nq, no, nv, seed, occ_range=(-1.3, -0.4), virt_range=(0.03, 4.0),
                decay=50.0, scale=1.0, lam0=None, ncore_orbs=0):
    """Seeded synthetic twin: occ e ~ U[occ_range], virt e log-uniform in
    virt_range, R ~ N(0,1)*scale*exp(-Q/decay); optionally rescaled so that
    lambda_max(Pi(0)) = lam0.  Extra core orbitals (e < -3 Eh) are generated
    and frozen by rpa_NCore when ncore_orbs > 0; only active ones are kept."""
    rng = np.random.default_rng(seed)
    eo = np.sort(rng.uniform(occ_range[0], occ_range[1], no))
    lo, hi = np.log(virt_range[0]), np.log(virt_range[1])
    ev = np.sort(np.exp(rng.uniform(lo, hi, nv)))
    if ncore_orbs:
        core = np.sort(rng.uniform(-21.0, -19.0, ncore_orbs))
        allocc = np.concatenate([core, eo])
        nc = ncore(np.concatenate([allocc, ev]), len(allocc))
        eo = allocc[nc:]
    R = rng.standard_normal((nq, no * nv)) * scale
    R *= np.exp(-np.arange(nq) / decay)[:, None]
    if lam0 is not None:
        lm = lambda_max_pi0(R, dai(eo, ev))
        R *= math.sqrt(lam0 / lm)
    return RPASystem(R=R, eps_o=eo, eps_v=ev)


def grid_for(sys_, n=None):
    """Frequency grid for a system: histogram -> optimised grid (n fixed or
    chosen by the convergence targets)."""
    e = np.concatenate([sys_.eps_o, sys_.eps_v])
    vals, wts = dai_histogram(e, sys_.no, sys_.nv)
    if n is None:
        return optimize_freq_quad(vals, wts)
    x, w, *_ = opt_quad_scaling(n, vals, wts)
    return x, w


# --------------------------------------------------------------------------
# Split-BF16 emulation (used to size the precision budget of the tensor-core path)
# --------------------------------------------------------------------------

def to_bf16(x):
    """Round float64 -> float32 -> bf16 (round to nearest even), as float64."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def exchange_mbpt3_1(U, A, R, eps_o, eps_v):
    """MBPT3 exchange: E_x = -Tr(X K), the default exchange of the CC path.

    rpa_CC_Exchange_MBPT3_1 + rpa_CC_Ukl + rpa_CC_Dkl + rpa_CC_TrXK,
    src/rpa/rpa_CC_Exchange.f90:177-336, with real_Lyapunov
    (src/linear-algebra/real_linalg.f90:125-171: Schur form + DTRSYL; here
    scipy.linalg.solve_sylvester, the same Bartels-Stewart method):
      Ukl = (R U)^T (R U),  Dkl = U^T diag(D) U,
      A_mn = A_m D_mn + D_mn A_n,  B_mn = D_mn + 2 U_mn + 4 U_mn A_n,
      solve B^T X + X B = A,
      TrXK = sum_{i>=j} (2 - delta_ij) sum_mn X_mn (W_ji^T W_ij)_mn,  W_ij = R_i U_j^T.
    U is (nov, NT) (the Uaim layout; the routine's Vkai is its transpose)."""
    no, nv = len(eps_o), len(eps_v)
    nq = R.shape[0]
    nt = U.shape[1]
    d = dai(eps_o, eps_v)
    RU = R @ U
    Ukl = RU.T @ RU
    Dkl = U.T @ (d[:, None] * U)
    Am = A[:, None] * Dkl + Dkl * A[None, :]
    Bm = Dkl + 2.0 * Ukl + 4.0 * Ukl * A[None, :]
    X = scipy.linalg.solve_sylvester(Bm.T, Bm, Am)
    Rr = R.reshape(nq, nv, no, order="F")
    Vr = U.T.reshape(nt, nv, no, order="F")
    acc = []
    for j in range(no):
        for i in range(j, no):
            Wij = Rr[:, :, i] @ Vr[:, :, j].T
            Wji = Rr[:, :, j] @ Vr[:, :, i].T if i != j else Wij
            W = Wji.T @ Wij
            acc.append((2.0 if i != j else 1.0) * float(np.sum(X * W)))
    return -math.fsum(acc), X


# Pi(u) basis types (src/rpa/rpa_definitions.f90:92-104) and the default trace target
# (TargetErrorRandom = sqrt(1e-5), src/rpa/rpa_definitions.f90:279).
RPA_BASIS_RANDOM = 1
RPA_BASIS_EIGEN = 2
RPA_BASIS_FULL_CHOLESKY = 3
TARGET_ERROR_RANDOM = math.sqrt(1.0e-5)


def piu_basis(pi1, target_error=TARGET_ERROR_RANDOM, basis_type=RPA_BASIS_EIGEN, guess=None):
    """Basis G of the effective dielectric matrix from Pi at the lowest frequency.

    rpa_G, src/rpa/rpa.f90:31-173:
      EIGEN:  columns of G = eigenvectors of Pi, eigenvalues descending; RWR -> diag(lambda)
      RANDOM: G = guess; two subspace iterations G <- qr(Pi G); RWR -> G^T Pi G
      FULL:   G = I
    NVecs = the smallest p (1-based) with sum_{q=p}^{N} RWR(q,q) < target_error, scanning q from
    N down and stopping at the first failure (NVecs = N when RWR(N,N) >= target_error), exactly as
    the reference's loop; the reported trace error is that sum.  The reference draws the random
    guess with its own generator, so `guess` (N x N) is an input here.
    Returns (G, nvecs, abs_error, exact_trace)."""
    n = pi1.shape[0]
    exact = math.fsum(np.diag(pi1).tolist())
    if basis_type == RPA_BASIS_FULL_CHOLESKY:
        return np.eye(n), n, 0.0, exact
    if basis_type == RPA_BASIS_EIGEN:
        w, V = np.linalg.eigh(-pi1)
        G = V
        rwr = -w
    elif basis_type == RPA_BASIS_RANDOM:
        G = np.array(guess, dtype=np.float64)
        for _ in range(2):
            G, _ = np.linalg.qr(pi1 @ G)
        rwr = np.diag(G.T @ pi1 @ G).copy()
    else:
        raise ValueError("invalid basis type")
    nvecs, acc = n, []
    for p in range(n - 1, -1, -1):
        nxt = math.fsum(acc + [rwr[p]])
        if nxt < target_error:
            acc.append(rwr[p])
            nvecs = p + 1
        else:
            break
    return G, nvecs, math.fsum(acc), exact


def thc_r(Zgk, Xga, Xgi):
    """Cholesky vectors from THC factors, R(k, ai) = sum_g Z(g,k) X_a(g,a) X_i(g,i),
    ai = a + NVirt*i.  rpa_THC_Rkab / rpa_THC_Rkai, src/rpa/rpa_THC.f90:374-426."""
    ng, nv = Xga.shape
    no = Xgi.shape[1]
    kr = (Xga[:, :, None] * Xgi[:, None, :]).reshape(ng, nv * no, order="F")
    return Zgk.T @ kr


def make_thc_factors(ngrid, nq, no, nv, seed, scale=0.3):
    """Seeded synthetic THC factors (Zgk, Xga, Xgi) and orbital energies."""
    rng = np.random.default_rng(seed)
    Z = rng.standard_normal((ngrid, nq)) * scale * np.exp(-np.arange(nq) / (nq / 3.0))[None, :]
    Xa = rng.standard_normal((ngrid, nv)) / math.sqrt(ngrid)
    Xi = rng.standard_normal((ngrid, no)) / math.sqrt(ngrid)
    eo = np.sort(rng.uniform(-1.3, -0.4, no))
    ev = np.sort(np.exp(rng.uniform(math.log(0.03), math.log(4.0), nv)))
    return Z, Xa, Xi, eo, ev


def jctc2024_corrections(Zgk, Xgi, Yga, U, A, Lik=None, cutoff_pno=1.0e-5, boys_screening=False,
                         cutoff_vabij=1.0e-6):
    """Particle-hole corrections to direct RPA on THC factors with pair-natural orbitals.

    rpa_JCTC2024_Corrections, src/rpa/rpa_JCTC2024.f90:24-257, with _Tabij (684-703),
    _MaxVabab (260-278), _PackTransfMatrices (281-320), _Gaibj_Gabij_v2 (323-548), _S1ab
    (551-572) and _phRPA_Gab_jik (575-681).  U is (nov x NT) (the Uaim layout), A (NT); Lik
    (NOcc x NOcc) the occupied localisation (None: canonical orbitals).  The PNOs of each pair
    i >= j come from the full SVD of T(ab;ij) = sum_mu U(a,i,mu) A_mu U(b,j,mu) with singular
    values > cutoff_pno (RPA_SVD_FULL; the randomized SVD of the reference reduces to it when
    NVirt fits its subspace).
    Returns (EcRPA_PNO, Ec1b, Ec2bcd, Ec2ghij); E(SOSEX cumulant) = Ec1b / 2,
    E(PH3) = Ec2bcd + Ec2ghij."""
    ng, nq = Zgk.shape
    no = Xgi.shape[1]
    nv = Yga.shape[1]
    nt = len(A)
    Ur = np.asarray(U, dtype=np.float64).reshape(nv, no, nt, order="F")
    if Lik is not None:
        Xgi = Xgi @ Lik
        Ur = np.einsum("aim,ik->akm", Ur, Lik)
    maxvabab = 0.0
    if boys_screening:
        zxx = Zgk.T @ (Yga ** 2)
        maxvabab = float(np.max(np.sum(zxx ** 2, axis=0)))
    # pair-natural orbitals: T_ij = U s V^T, TaxPNO = [U | s V]
    tax = {}
    for j in range(no):
        for i in range(j, no):
            T = Ur[:, i, :] @ (Ur[:, j, :] * A[None, :]).T
            u, s, vt = np.linalg.svd(T)
            n = int(np.sum(s > cutoff_pno))
            if n > 0:
                tax[(i, j)] = np.concatenate([u[:, :n], vt[:n].T * s[None, :n]], axis=1)

    def packed(k, i):  # TaxPNO of the pair {k, i} or None
        return tax.get((max(k, i), min(k, i)))

    ec_rpa = ec1b = ec2bcd = ec2ghij = 0.0
    c2b = c2c = -4.0 * 0.5
    c2d = 2.0
    c2g = c2h = -4.0
    c2i = c2j = 2.0
    for j in range(no):
        wga = Yga * Xgi[:, j][:, None]
        zyx_gbj = Zgk @ (Zgk.T @ wga)
        for i in range(j, no):
            weight = 2.0 if i != j else 1.0
            wg = Xgi[:, i] * Xgi[:, j]
            zxx_kij = Zgk.T @ wg
            if boys_screening:
                vijij = float(zxx_kij @ zxx_kij)
                contrib = math.sqrt(abs(maxvabab * vijij)) > cutoff_vabij
            else:
                contrib = True
            zxx_gij = Zgk @ zxx_kij if contrib else None
            yx_gai = Yga * Xgi[:, i][:, None]
            pq_ij = packed(i, j)
            if pq_ij is not None:
                nij = pq_ij.shape[1] // 2
                P, Q = pq_ij[:, :nij], pq_ij[:, nij:]
                s1b = float(np.sum((yx_gai @ Q) * (zyx_gbj @ P)))
                s1a = float(np.sum((yx_gai @ P) * (zyx_gbj @ Q)))
                ec1b -= 2.0 * weight * s1b
                ec_rpa += 2.0 * weight * s1a
            g_bcd = np.zeros((nv, nv))
            g_ghij = np.zeros((nv, nv))
            for k in range(no):
                pq_kj, pq_ki = packed(k, j), packed(k, i)
                if pq_kj is None or pq_ki is None:
                    continue
                nkj, nki = pq_kj.shape[1] // 2, pq_ki.shape[1] // 2
                kj = [pq_kj[:, :nkj], pq_kj[:, nkj:]]
                ki = [pq_ki[:, :nki], pq_ki[:, nki:]]
                Pki, Qki, Pik, Qik = (0, 1, 1, 0) if k >= i else (1, 0, 0, 1)
                Pkj, Qkj, Pjk, Qjk = (0, 1, 1, 0) if k >= j else (1, 0, 0, 1)
                S_jk_ki = kj[Qjk].T @ ki[Pki]
                S_jk_ik = kj[Qjk].T @ ki[Pik]
                S_kj_ki = kj[Qkj].T @ ki[Pki]
                S_kj_ik = kj[Qkj].T @ ki[Pik]
                QS_jk_ki = ki[Qki] @ S_jk_ki.T
                QS_jk_ik = ki[Qik] @ S_jk_ik.T
                QS_kj_ki = ki[Qki] @ S_kj_ki.T
                QS_kj_ik = ki[Qik] @ S_kj_ik.T
                QS = [None, None]
                if contrib:
                    if i != j:
                        QS[Pjk] = (2.0 * c2g) * QS_jk_ki + (c2i + c2j) * QS_jk_ik
                        QS[Pkj] = (2.0 * c2h) * QS_kj_ik + (c2i + c2j) * QS_kj_ki
                    else:
                        QS[Pjk] = c2g * QS_jk_ki + (c2i + c2j) * QS_jk_ik
                        QS[Pkj] = c2h * QS_kj_ik
                    g_ghij += kj[0] @ QS[0].T + kj[1] @ QS[1].T
                if i != j:
                    QS[Pkj] = (2.0 * c2d) * QS_kj_ik + (c2b + c2c) * QS_kj_ki
                    QS[Pjk] = (c2b + c2c) * QS_jk_ik
                    g_bcd += kj[0] @ QS[0].T + kj[1] @ QS[1].T
                else:
                    QS[Pkj] = c2d * QS_kj_ik + (c2b + c2c) * QS_kj_ki
                    g_bcd += kj[Pkj] @ QS[Pkj].T
            if contrib:
                ec2ghij += float(np.sum(Yga * ((Yga @ g_ghij) * zxx_gij[:, None])))
            ec2bcd += float(np.sum((zyx_gbj @ g_bcd) * yx_gai))
    return ec_rpa, ec1b, ec2bcd, ec2ghij
