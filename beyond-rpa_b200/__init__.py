"""beyond-rpa_b200: B200 (sm_100a) Cholesky-vector RPA hot path.

Thin ctypes binding of the C ABI in include/rpa_b200.h (librpa_b200.so, built
in-tree by build.py).  The binding only marshals arguments: every array is
passed to the library as a pointer (numpy arrays as host pointers, torch CUDA
tensors as device pointers) and all compute runs in the CUDA library.  There
is no CPU fallback: if the library or a B200 is missing, calls raise.

Python names follow the reference routines they stand in for:
  pi_u            rpa_THC_PiU (src/rpa/rpa_THC.f90:215-282)
  ec_from_pi      rpa_CC_EcRPA_Analytic (src/rpa/rpa_CC.f90:412-471)
  ec_rpa          rpa_THC_PiU + rpa_CC_EcRPA_Analytic as chained in
                  rpa_THC_MBPT3 (src/rpa/rpa_THC.f90:106-108)
"""
from __future__ import annotations

import ctypes
import math
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "librpa_b200.so"
HEADER = HERE.parent / "include" / "rpa_b200.h"

RPA_OK = 0
RPA_ERR_INVALID_ARG = 1
RPA_ERR_NOT_SPD = 2
RPA_ERR_NONFINITE = 3
RPA_ERR_OOM = 4
RPA_ERR_CUDA = 5
RPA_ERR_TIMEOUT = 6
RPA_ERR_NO_DEVICE = 7
RPA_ERR_NOT_CONVERGED = 8
RPA_ERR_TOO_LARGE = 9
RPA_ERR_INTERNAL = 10

PREC_FP64 = 0
PREC_SPLIT_BF16 = 1
_PREC = {"fp64": PREC_FP64, "split": PREC_SPLIT_BF16, "split_bf16": PREC_SPLIT_BF16,
         PREC_FP64: PREC_FP64, PREC_SPLIT_BF16: PREC_SPLIT_BF16}

_i64 = ctypes.c_int64
_dbl = ctypes.c_double
_vp = ctypes.c_void_p
_lib = None


class _Instance(ctypes.Structure):
    """struct rpa_instance of include/rpa_b200.h."""
    _fields_ = [("NQ", _i64), ("NOcc", _i64), ("NVirt", _i64), ("R", _vp), ("ldR", _i64),
                ("OccEnergies", _vp), ("VirtEnergies", _vp), ("NFreqs", _i64), ("Freqs", _vp),
                ("FreqWeights", _vp), ("alpha", _dbl)]


class RPAError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        msg = _status_string(status)
        super().__init__(f"{msg} (status {status})" + (f": {detail}" if detail else ""))


def _status_string(status: int) -> str:
    lib = load_library()
    return lib.rpa_b200_status_string(int(status)).decode()


def load_library(path: str | os.PathLike | None = None):
    """Load librpa_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: run `python beyond-rpa_b200/build.py` first")
    lib = ctypes.CDLL(str(p))
    lib.rpa_b200_create.argtypes = [ctypes.POINTER(_vp), _i64, _i64]
    lib.rpa_b200_destroy.argtypes = [_vp]
    lib.rpa_b200_status_string.argtypes = [ctypes.c_int]
    lib.rpa_b200_status_string.restype = ctypes.c_char_p
    lib.rpa_b200_last_error.argtypes = [_vp]
    lib.rpa_b200_last_error.restype = ctypes.c_char_p
    lib.rpa_b200_last_timings.argtypes = [_vp, _vp, _i64]
    lib.rpa_b200_last_launches.argtypes = [_vp]
    lib.rpa_b200_last_launches.restype = _i64
    lib.rpa_b200_set_stream.argtypes = [_vp, _vp]
    lib.rpa_b200_pi.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _dbl, _i64, _vp, _i64]
    lib.rpa_b200_ec_from_pi.argtypes = [_vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp]
    lib.rpa_b200_ec.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _dbl, _i64, _vp, _vp]
    lib.rpa_b200_freq_grid.argtypes = [_i64, _i64, _vp, _dbl, _dbl, _dbl, _i64, _vp, _vp, _vp]
    lib.rpa_b200_ec_from_pi_noalloc.argtypes = [_i64, _vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp]
    lib.rpa_b200_dring_t2.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _dbl, _i64, _i64,
                                      _vp, ctypes.c_uint64, _dbl, _dbl, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _vp]
    lib.rpa_b200_ec_batched.argtypes = [_vp, _i64, _vp, _i64, _vp, _vp]
    lib.rpa_b200_ec_grad.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _dbl, _i64, _vp,
                                     _vp, _i64, _vp, _vp]
    lib.rpa_b200_exchange_sosex.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _dbl, _i64, _i64,
                                            _vp]
    lib.rpa_b200_syevd.argtypes = [_vp, _i64, _vp, _i64, _vp]
    lib.rpa_b200_jctc2024.argtypes = [_vp, _i64, _i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _vp, _i64,
                                      _vp, _vp, _i64, _dbl, _i64, _dbl, _vp, _vp]
    lib.rpa_b200_thc_r.argtypes = [_vp, _i64, _i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64]
    lib.rpa_b200_ec_thc.argtypes = [_vp, _i64, _i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _i64,
                                    _vp, _vp, _dbl, _i64, _vp, _vp]
    lib.rpa_b200_piu_basis.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _dbl, _dbl, _i64, _i64, _dbl,
                                       _vp, _i64, ctypes.c_uint64, _vp, _i64, _vp, _vp, _vp]
    lib.rpa_b200_project_basis.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64]
    lib.rpa_b200_exchange_mbpt3.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _i64, _vp, _i64,
                                            _vp, _vp, _i64]
    lib.rpa_b200_mbe_energy.argtypes = [_i64, _vp, _vp]
    lib.rpa_b200_freq_grid_mbe.argtypes = [_i64, _vp, _vp, _vp, _dbl, _i64, _dbl, _dbl, _i64, _vp, _vp, _vp]
    lib.rpa_b200_tune_logdet.argtypes = [_vp, _i64, _i64, _vp, _vp, _vp]
    lib.rpa_b200_set_logdet_plan.argtypes = [_vp, _i64, _i64, _i64]
    lib.rpa_b200_get_logdet_plan.argtypes = [_vp, _i64, _vp, _vp]
    lib.rpa_b200_set_autotune.argtypes = [_vp, _i64]
    lib.rpa_b200_set_workspace_limit.argtypes = [_vp, _i64]
    lib.rpa_b200_workspace_bytes.argtypes = [_vp, _vp, _vp]
    lib.rpa_b200_selftest_wait_timeout.argtypes = [_vp, _dbl]
    if path is None:
        _lib = lib
    return lib


SUBSYSTEMS = ("total", "A", "B", "C", "AB", "BC", "AC", "D", "AD", "BD", "CD", "ABC", "ABD", "ACD", "BCD")


def mbe_energy(energies, nbody):
    """Interaction (nbody 2) or nonadditive (3, 4) energy of a many-body expansion from the
    subsystem energies, in the order of SUBSYSTEMS (rpa_b200_mbe_energy; host code, no GPU)."""
    lib = load_library()
    need = {2: 3, 3: 7, 4: 15}.get(int(nbody))
    e = np.ascontiguousarray(energies, dtype=np.float64)
    if need is None or e.size < need:
        raise ValueError("nbody must be 2, 3 or 4 with 3, 7 or 15 subsystem energies")
    out = ctypes.c_double()
    st = lib.rpa_b200_mbe_energy(int(nbody), e.ctypes.data, ctypes.byref(out))
    if st != RPA_OK:
        raise RPAError(st, "rpa_b200_mbe_energy failed")
    return out.value


def freq_grid_mbe(sets, limit_dai=True, nfixed=0, core_thresh=-3.0, target_error=1e-6, target_rel_error=1e-3):
    """One grid for the subsystems of a many-body expansion (rpa_b200_freq_grid_mbe; host code):
    sets = [(orb_energies, nocc, nvirt), ...] with sets[0] the whole complex."""
    lib = load_library()
    arrs = [np.ascontiguousarray(e, dtype=np.float64) for e, _, _ in sets]
    no = np.array([int(n) for _, n, _ in sets], dtype=np.int64)
    nv = np.array([int(n) for _, _, n in sets], dtype=np.int64)
    for a, o, v in zip(arrs, no, nv):
        if a.size != o + v:
            raise ValueError("each orbital-energy set must hold NOcc + NVirt values")
    ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    x = np.zeros(64)
    w = np.zeros(64)
    n = ctypes.c_int64()
    st = lib.rpa_b200_freq_grid_mbe(len(arrs), no.ctypes.data, nv.ctypes.data, ctypes.cast(ptrs, _vp),
                                    float(core_thresh), 1 if limit_dai else 0, float(target_error),
                                    float(target_rel_error), int(nfixed), x.ctypes.data, w.ctypes.data,
                                    ctypes.byref(n))
    if st != RPA_OK:
        raise RPAError(st, "rpa_b200_freq_grid_mbe failed")
    return x[:n.value].copy(), w[:n.value].copy()


def freq_grid(orb_energies, nocc, nvirt, nfixed=0, core_thresh=-3.0, target_error=1e-6, target_rel_error=1e-3):
    """Frequency points and weights (rpa_b200_freq_grid; host code, no GPU needed)."""
    lib = load_library()
    e = np.ascontiguousarray(orb_energies, dtype=np.float64)
    if e.size != nocc + nvirt:
        raise ValueError("orb_energies must hold NOcc + NVirt values")
    x = np.zeros(64)
    w = np.zeros(64)
    n = ctypes.c_int64()
    st = lib.rpa_b200_freq_grid(int(nocc), int(nvirt), e.ctypes.data, float(core_thresh), float(target_error),
                                float(target_rel_error), int(nfixed), x.ctypes.data, w.ctypes.data,
                                ctypes.byref(n))
    if st != RPA_OK:
        raise RPAError(st, "rpa_b200_freq_grid")
    return x[: n.value].copy(), w[: n.value].copy()


def declared_functions() -> list[str]:
    """Function names declared by include/rpa_b200.h."""
    import re
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int64_t|int|const char\*)\s+(rpa_b200_\w+)\s*\(", text, re.M)))


# ----------------------------------------------------------------------------- marshalling

def _is_torch(x):
    return type(x).__module__.startswith("torch")


class _Arg:
    """Pointer + leading dimension of an array argument (keeps the owner alive)."""

    def __init__(self, ptr, ld=None, owner=None):
        self.ptr, self.ld, self.owner = ptr, ld, owner


def _vec(x):
    if _is_torch(x):
        if str(x.dtype) != "torch.float64" or not x.is_contiguous():
            raise ValueError("vector arguments must be contiguous float64")
        return _Arg(x.data_ptr(), owner=x)
    a = np.ascontiguousarray(x, dtype=np.float64)
    return _Arg(a.ctypes.data, owner=a)


def _colmajor(x, nrows):
    """(nrows x ncols) column-major view: returns pointer and leading dimension."""
    if _is_torch(x):
        import torch
        if x.dtype != torch.float64 or x.dim() != 2 or x.shape[0] != nrows:
            raise ValueError("expected a float64 (NQ, nov) tensor")
        if x.stride(0) != 1:
            raise ValueError("R must be column-major: stride(0) == 1 (use R_t.T of a contiguous (nov, NQ) tensor)")
        return _Arg(x.data_ptr(), ld=max(x.stride(1), nrows), owner=x)
    a = np.asarray(x, dtype=np.float64)
    if a.ndim != 2 or a.shape[0] != nrows:
        raise ValueError("expected an (NQ, nov) array")
    if not a.flags.f_contiguous:
        a = np.asfortranarray(a)
    return _Arg(a.ctypes.data, ld=nrows, owner=a)


class Handle:
    """A librpa_b200 handle bound to one GPU (rpa_b200_create / rpa_b200_destroy)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = _vp()
        st = self.lib.rpa_b200_create(ctypes.byref(h), int(device), 0)
        if st != RPA_OK:
            raise RPAError(st, "rpa_b200_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.rpa_b200_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != RPA_OK:
            raise RPAError(st, self.lib.rpa_b200_last_error(self._h).decode())

    def timings(self):
        """Phase times (ms) of the last call, CUDA events on the call's stream."""
        out = (ctypes.c_double * 6)()
        self._check(self.lib.rpa_b200_last_timings(self._h, ctypes.cast(out, _vp), 6))
        return {"staging_ms": out[0], "pi_ms": out[1], "logdet_ms": out[2], "other_ms": out[3],
                "contraction_ms": out[4], "split_ms": out[5]}

    def launches(self):
        """Kernels launched by the library during the last call."""
        return int(self.lib.rpa_b200_last_launches(self._h))

    def set_stream(self, stream=None):
        """Run calls on a cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self.lib.rpa_b200_set_stream(self._h, stream))

    # ------------------------------------------------------------------ log-det tile plans
    LOGDET_CANDIDATES = ((128, 64), (256, 64), (512, 64), (128, 128), (256, 128), (512, 128))

    def tune_logdet(self, nq, nmat):
        """Time every log-det tile plan (outer block, CTA tile) on `nmat` seeded SPD matrices of
        order `nq`; keep the fastest for nq's bucket.  Returns ((nb2, tile), {candidate: ms})."""
        nb2, tile = ctypes.c_int64(), ctypes.c_int64()
        ms = (ctypes.c_double * 6)()
        self._check(self.lib.rpa_b200_tune_logdet(self._h, int(nq), int(nmat), ctypes.byref(nb2), ctypes.byref(tile),
                                                  ctypes.cast(ms, _vp)))
        return (nb2.value, tile.value), dict(zip(self.LOGDET_CANDIDATES, list(ms)))

    def set_logdet_plan(self, nq, nb2, tile):
        """Store the log-det tile plan for nq's bucket of 256 orders."""
        self._check(self.lib.rpa_b200_set_logdet_plan(self._h, int(nq), int(nb2), int(tile)))

    def logdet_plan(self, nq):
        """(nb2, tile) used for matrices of order nq."""
        nb2, tile = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.rpa_b200_get_logdet_plan(self._h, int(nq), ctypes.byref(nb2), ctypes.byref(tile)))
        return nb2.value, tile.value

    def set_autotune(self, on=True):
        """Tune unseen order buckets inside ec_batched (on by default)."""
        self._check(self.lib.rpa_b200_set_autotune(self._h, 1 if on else 0))

    def set_workspace_limit(self, nbytes=0):
        """Cap the handle's device workspace at nbytes (0: no cap); over-cap calls raise RPA_ERR_OOM."""
        self._check(self.lib.rpa_b200_set_workspace_limit(self._h, int(nbytes)))

    def workspace_bytes(self):
        """(bytes the workspace holds now, cap or 0)."""
        used, limit = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.rpa_b200_workspace_bytes(self._h, ctypes.byref(used), ctypes.byref(limit)))
        return used.value, limit.value

    def selftest_wait_timeout(self, limit_ms=20.0):
        """Run the bounded-wait self-test; returns its status (RPA_ERR_TIMEOUT when detection works)."""
        return int(self.lib.rpa_b200_selftest_wait_timeout(self._h, float(limit_ms)))

    # ------------------------------------------------------------------ Pi(u)
    def pi_u(self, R, eps_o, eps_v, freqs, alpha=4.0, prec="split", out=None):
        """PiU(:,:,u) for every frequency; returns (K, NQ, NQ) (numpy unless `out` is given)."""
        nq = int(R.shape[0])
        no, nv, K = len(eps_o), len(eps_v), len(freqs)
        r = _colmajor(R, nq)
        eo, ev, fr = _vec(eps_o), _vec(eps_v), _vec(freqs)
        if out is None:
            out = np.empty((K, nq, nq), dtype=np.float64)
        optr = out.data_ptr() if _is_torch(out) else out.ctypes.data
        self._check(self.lib.rpa_b200_pi(self._h, nq, no, nv, r.ptr, r.ld, eo.ptr, ev.ptr, K, fr.ptr,
                                         float(alpha), _PREC[prec], optr, nq))
        return out

    # ------------------------------------------------------------------ energies
    def ec_from_pi(self, pi, weights):
        """E_c and E(u) from (K, NQ, NQ) Pi(u) matrices (lower triangles read)."""
        K, nq = int(pi.shape[0]), int(pi.shape[1])
        if _is_torch(pi):
            p = _Arg(pi.contiguous().data_ptr(), owner=pi.contiguous())
        else:
            a = np.ascontiguousarray(pi, dtype=np.float64)
            p = _Arg(a.ctypes.data, owner=a)
        w = _vec(weights)
        ec = ctypes.c_double()
        eu = np.zeros(K)
        self._check(self.lib.rpa_b200_ec_from_pi(self._h, nq, K, p.ptr, nq, w.ptr, ctypes.byref(ec),
                                                 eu.ctypes.data))
        return ec.value, eu

    def ec_grad(self, R, eps_o, eps_v, freqs, weights, alpha=4.0, prec="split", out=None):
        """E_c and its adjoint (rpa_b200_ec_grad): returns (Ec, dR, dOcc, dVirt).

        dR has R's (NQ, nov) column-major layout; with torch inputs pass `out` = (dR, dOcc, dVirt) tensors."""
        nq = int(R.shape[0])
        no, nv, K = len(eps_o), len(eps_v), len(freqs)
        r = _colmajor(R, nq)
        eo, ev, fr, w = _vec(eps_o), _vec(eps_v), _vec(freqs), _vec(weights)
        if out is None:
            dR = np.zeros((nq, no * nv), order="F")
            dO = np.zeros(no)
            dV = np.zeros(nv)
            p_dR, ld_dR, p_dO, p_dV = dR.ctypes.data, nq, dO.ctypes.data, dV.ctypes.data
        else:
            dR, dO, dV = out
            a = _colmajor(dR, nq)
            p_dR, ld_dR = a.ptr, a.ld
            p_dO, p_dV = _vec(dO).ptr, _vec(dV).ptr
        ec = ctypes.c_double()
        self._check(self.lib.rpa_b200_ec_grad(self._h, nq, no, nv, r.ptr, r.ld, eo.ptr, ev.ptr, K, fr.ptr, w.ptr,
                                              float(alpha), _PREC[prec], ctypes.byref(ec), p_dR, ld_dR, p_dO, p_dV))
        return ec.value, dR, dO, dV

    def mbe_energies(self, subsystems, nbody, prec="split", limit_dai=True, nfixed=0, core_thresh=-3.0,
                     basis=None, basis_target_error=math.sqrt(1e-5)):
        """Many-body-expansion driver (the energy part of rpa_PostSCF, src/rpa/rpa_driver.f90:25-433):
        one frequency grid shared by all subsystems (freq_grid_mbe), every subsystem's E_c in one
        batched call, then the interaction (nbody 2) or nonadditive (3, 4) energy (mbe_energy).

        subsystems: (R, eps_occ, eps_virt) per subsystem in the order of SUBSYSTEMS (3, 7 or 15 of
        them), R over the active occupied orbitals (those with eps >= core_thresh), eps_occ all
        occupied energies ascending.
        basis: None uses each R as given.  "eigen" or "random" compresses the Pi basis once, for the
        whole system (subsystems[0]) at the lowest frequency of the shared grid (piu_basis), and
        projects every subsystem onto it, R' = G^T R (project_basis), as the reference shares
        THC_ZgkPiU between all subsystems for size consistency (src/rpa/rpa.f90:2305-2322); all R
        must then have the same NQ rows (the cluster's Cholesky basis).
        Returns (E_c per subsystem, interaction energy, freqs, weights)."""
        ec, eint, x, w, _ = self._mbe_rpa(subsystems, nbody, prec, limit_dai, nfixed, core_thresh, basis,
                                          basis_target_error)
        return ec, eint, x, w

    def _mbe_rpa(self, subsystems, nbody, prec, limit_dai, nfixed, core_thresh, basis, basis_target_error):
        need = {2: 3, 3: 7, 4: 15}.get(int(nbody))
        if need is None or len(subsystems) != need:
            raise ValueError("nbody 2, 3 or 4 needs 3, 7 or 15 subsystems")
        sets = [(np.concatenate([np.asarray(eo, np.float64), np.asarray(ev, np.float64)]), len(eo), len(ev))
                for _, eo, ev in subsystems]
        x, w = freq_grid_mbe(sets, limit_dai=limit_dai, nfixed=nfixed, core_thresh=core_thresh)
        active = []
        for R, eo, ev in subsystems:
            eo = np.asarray(eo, np.float64)
            active.append((R, eo[eo >= core_thresh], np.asarray(ev, np.float64)))
        G = None
        if basis is not None:
            nq = int(active[0][0].shape[0])
            if any(int(R.shape[0]) != nq for R, _, _ in active):
                raise ValueError("a shared Pi basis needs every subsystem's R over the same NQ Cholesky vectors")
            R0, eo0, ev0 = active[0]
            G, _, _ = self.piu_basis(R0, eo0, ev0, float(x[0]), target_error=basis_target_error, basis=basis)
            active = [(self.project_basis(G, R), eo, ev) for R, eo, ev in active]
        ec, _ = self.ec_batched([(R, eo, ev, x, w) for R, eo, ev in active], prec=prec)
        return ec, mbe_energy(ec, nbody), x, w, (active, G)

    def mbe_beyond_rpa(self, subsystems, nbody, prec="split", limit_dai=True, nfixed=0, core_thresh=-3.0,
                       basis=None, basis_target_error=math.sqrt(1e-5), cutoff_thresh=1e-4, cutoff_type=0,
                       n_guess=None, seed=0):
        """Many-body expansion of RPA plus the SOSEX exchange energy (the beyond-RPA subsystem loop of
        rpa_PostSCF, src/rpa/rpa_driver.f90:83-91, 175-240): the shared grid and (optionally) the shared
        Pi basis of mbe_energies, then for every subsystem the direct-ring T2 amplitudes and the SOSEX
        energy.  The T2 eigenvalue cutoff threshold is fixed once by the whole system (dring_t2 with
        common_thresh < 0) and reused by every subsystem, as the reference shares
        T2CutoffCommonThresh for size-consistent interaction energies.  n_guess: guess vectors of the
        range finder (None: the reference's ceil(3 NQ), capped at NOcc NVirt).  The range finder drops
        Gram directions below its linear-dependency cutoff, so even with a shared threshold the
        exchange energies of non-interacting fragments add up only to the accuracy of the retained
        subspace (in the reference as here), while the RPA energies add up to rounding.
        Returns a dict: freqs, weights, ec and eint (RPA), ex and ex_int (SOSEX), eig_rpa (the T2
        eigenvalue energies), nt (amplitude counts) and common_thresh."""
        ec, eint, x, w, (active, _) = self._mbe_rpa(subsystems, nbody, prec, limit_dai, nfixed, core_thresh, basis,
                                                    basis_target_error)
        common = -1.0
        ex, eig, nts = [], [], []
        for R, eo, ev in active:
            t2 = self.dring_t2(R, eo, ev, x, w, prec=prec, seed=seed, n_guess=n_guess, cutoff_thresh=cutoff_thresh,
                               cutoff_type=cutoff_type, common_thresh=common)
            common = t2["common_thresh"]
            nts.append(t2["NT"])
            eig.append(float(np.sum(t2["EigRPA"])))
            ex.append(self.exchange_sosex(R, len(eo), len(ev), t2["U"], t2["A"], prec=prec))
        ex = np.array(ex)
        return {"freqs": x, "weights": w, "ec": ec, "eint": eint, "ex": ex, "ex_int": mbe_energy(ex, nbody),
                "eig_rpa": np.array(eig), "nt": nts, "common_thresh": common}

    def ec_batched(self, systems, prec="split"):
        """Energies of many systems in one call (rpa_b200_ec_batched).

        systems: sequence of (R, eps_o, eps_v, freqs, weights[, alpha]).  Returns (Ec array, list of E(u))."""
        n = len(systems)
        arr = (_Instance * n)()
        keep = []
        for i, sysx in enumerate(systems):
            R, eo, ev, fr, w = sysx[:5]
            alpha = sysx[5] if len(sysx) > 5 else 4.0
            nq = int(R.shape[0])
            r = _colmajor(R, nq)
            a_eo, a_ev, a_fr, a_w = _vec(eo), _vec(ev), _vec(fr), _vec(w)
            keep += [r, a_eo, a_ev, a_fr, a_w]
            arr[i] = _Instance(nq, len(eo), len(ev), r.ptr, r.ld, a_eo.ptr, a_ev.ptr, len(fr), a_fr.ptr, a_w.ptr,
                               float(alpha))
        ec = np.zeros(n)
        eu = np.zeros(sum(len(sysx[3]) for sysx in systems))
        self._check(self.lib.rpa_b200_ec_batched(self._h, n, ctypes.cast(arr, _vp), _PREC[prec], ec.ctypes.data,
                                                 eu.ctypes.data))
        out, o = [], 0
        for sysx in systems:
            out.append(eu[o:o + len(sysx[3])].copy())
            o += len(sysx[3])
        return ec, out

    # ------------------------------------------------------------------ beyond RPA
    def dring_t2(self, R, eps_o, eps_v, freqs, weights, alpha=4.0, prec="fp64", guess=None, n_guess=None, seed=0,
                 small_cutoff=1e-10, cutoff_thresh=1e-4, cutoff_type=0, common_thresh=-1.0, max_vecs=None,
                 u_out=None):
        """Direct-ring T2 = U diag(A) U^T (rpa_b200_dring_t2).  guess: (nov, G) guess vectors or None.
        u_out: optional column-major (nov, cap) device tensor that receives U (then returned as a view).

        Returns dict(A, U (nov x NT), EigRPA, NT, common_thresh, Ec)."""
        nq = int(R.shape[0])
        no, nv, K = len(eps_o), len(eps_v), len(freqs)
        nov = no * nv
        r = _colmajor(R, nq)
        eo, ev, fr, w = _vec(eps_o), _vec(eps_v), _vec(freqs), _vec(weights)
        if guess is not None:
            gm = _colmajor(guess, nov)
            G = int(guess.shape[1])
            gptr = gm.ptr
        else:
            gm = None
            G = int(n_guess if n_guess is not None else min(int(np.ceil(3.0 * nq)), nov))
            gptr = None
        if u_out is not None:
            uo = _colmajor(u_out, nov)
            cap = int(u_out.shape[1])
            U, uptr, ldu = u_out, uo.ptr, uo.ld
        else:
            cap = int(max_vecs or G)
            U = np.zeros((nov, cap), order="F")
            uptr, ldu = U.ctypes.data, nov
        A = np.zeros(cap)
        eig = np.zeros(cap)
        nt = ctypes.c_int64()
        ct = ctypes.c_double(common_thresh)
        ec = ctypes.c_double()
        self._check(self.lib.rpa_b200_dring_t2(self._h, nq, no, nv, r.ptr, r.ld, eo.ptr, ev.ptr, K, fr.ptr, w.ptr,
                                               float(alpha), _PREC[prec], G, gptr, int(seed), float(small_cutoff),
                                               float(cutoff_thresh), int(cutoff_type), ctypes.byref(ct), cap,
                                               A.ctypes.data, uptr, ldu, ctypes.byref(nt),
                                               eig.ctypes.data, ctypes.byref(ec)))
        n = nt.value
        Uo = U[:, :n] if u_out is not None else np.asfortranarray(U[:, :n])
        return {"A": A[:n].copy(), "U": Uo, "EigRPA": eig[:n].copy(), "NT": n,
                "common_thresh": ct.value, "Ec": ec.value}

    def exchange_sosex(self, R, nocc, nvirt, U, A, alpha=1.0, s2_operator=False, prec="fp64"):
        """SOSEX exchange energy -alpha sum (aj|bi) T_aibj (rpa_b200_exchange_sosex); prec "split"
        runs the pair contraction as split-BF16 on the tensor cores."""
        nq = int(R.shape[0])
        nov = nocc * nvirt
        r = _colmajor(R, nq)
        u = _colmajor(U, nov)
        a = _vec(A)
        ex = ctypes.c_double()
        self._check(self.lib.rpa_b200_exchange_sosex(self._h, nq, nocc, nvirt, r.ptr, r.ld, int(U.shape[1]), u.ptr,
                                                     u.ld, a.ptr, float(alpha), int(bool(s2_operator)), _PREC[prec],
                                                     ctypes.byref(ex)))
        return ex.value

    def syevd(self, A):
        """Eigenvalues (ascending) and eigenvectors of the symmetric matrix A (rpa_b200_syevd)."""
        n = int(A.shape[0])
        Z = np.array(A, dtype=np.float64, order="F", copy=True)
        w = np.zeros(n)
        self._check(self.lib.rpa_b200_syevd(self._h, n, Z.ctypes.data, n, w.ctypes.data))
        return w, Z

    def piu_basis(self, R, eps_o, eps_v, lowest_freq, target_error=math.sqrt(1e-5), basis="eigen", prec="fp64",
                  guess=None, seed=0, alpha=4.0):
        """Compressed Pi basis (rpa_b200_piu_basis): returns (G (NQ x NVecs), trace_error, exact_trace)."""
        nq = int(R.shape[0])
        no, nv = len(eps_o), len(eps_v)
        r = _colmajor(R, nq)
        eo, ev = _vec(eps_o), _vec(eps_v)
        bt = {"random": 1, "eigen": 2, "full": 3}[basis]
        G = np.zeros((nq, nq), order="F")
        gm = _colmajor(guess, nq) if guess is not None else None
        nvec = ctypes.c_int64()
        terr = ctypes.c_double()
        tex = ctypes.c_double()
        self._check(self.lib.rpa_b200_piu_basis(self._h, nq, no, nv, r.ptr, r.ld, eo.ptr, ev.ptr, float(lowest_freq),
                                                float(alpha), _PREC[prec], bt, float(target_error),
                                                gm.ptr if gm else None, gm.ld if gm else nq, int(seed),
                                                G.ctypes.data, nq, ctypes.byref(nvec), ctypes.byref(terr),
                                                ctypes.byref(tex)))
        return np.asfortranarray(G[:, :nvec.value]), terr.value, tex.value

    def project_basis(self, G, R):
        """R' = G^T R (rpa_b200_project_basis), numpy in, numpy out."""
        nq, nvec = int(G.shape[0]), int(G.shape[1])
        nov = int(R.shape[1])
        g = _colmajor(G, nq)
        r = _colmajor(R, nq)
        out = np.zeros((nvec, nov), order="F")
        self._check(self.lib.rpa_b200_project_basis(self._h, nq, nvec, nov, g.ptr, g.ld, r.ptr, r.ld,
                                                    out.ctypes.data, nvec))
        return out

    def thc_r(self, Zgk, Xga, Xgi, out=None):
        """Cholesky vectors from THC factors (rpa_b200_thc_r): R (NQ x NOcc*NVirt); numpy, or `out`
        (a column-major device tensor) when given."""
        ng = int(Zgk.shape[0])
        nq, nv, no = int(Zgk.shape[1]), int(Xga.shape[1]), int(Xgi.shape[1])
        z, xa, xi = _colmajor(Zgk, ng), _colmajor(Xga, ng), _colmajor(Xgi, ng)
        if out is not None:
            o = _colmajor(out, nq)
            R, rptr, ldr = out, o.ptr, o.ld
        else:
            R = np.zeros((nq, no * nv), order="F")
            rptr, ldr = R.ctypes.data, nq
        self._check(self.lib.rpa_b200_thc_r(self._h, ng, nq, no, nv, z.ptr, z.ld, xa.ptr, xa.ld, xi.ptr, xi.ld,
                                            rptr, ldr))
        return R

    def ec_thc(self, Zgk, Xga, Xgi, eps_o, eps_v, freqs, weights, alpha=4.0, prec="split"):
        """RPA energy from THC factors (rpa_b200_ec_thc): (E_c, E(u))."""
        ng = int(Zgk.shape[0])
        nq, nv, no = int(Zgk.shape[1]), int(Xga.shape[1]), int(Xgi.shape[1])
        z, xa, xi = _colmajor(Zgk, ng), _colmajor(Xga, ng), _colmajor(Xgi, ng)
        eo, ev, fr, w = _vec(eps_o), _vec(eps_v), _vec(freqs), _vec(weights)
        K = len(freqs)
        ec = ctypes.c_double()
        eu = np.zeros(K)
        self._check(self.lib.rpa_b200_ec_thc(self._h, ng, nq, no, nv, z.ptr, z.ld, xa.ptr, xa.ld, xi.ptr, xi.ld,
                                             eo.ptr, ev.ptr, K, fr.ptr, w.ptr, float(alpha), _PREC[prec],
                                             ctypes.byref(ec), eu.ctypes.data))
        return ec.value, eu

    def jctc2024(self, Zgk, Xgi, Yga, U, A, Lik=None, cutoff_pno=1e-5, boys_screening=False,
                 cutoff_vabij=1e-6):
        """Particle-hole corrections (rpa_b200_jctc2024): ((EcRPA_PNO, Ec1b, Ec2bcd, Ec2ghij),
        (max NVirtPNO, sum NVirtPNO, pairs without PNOs))."""
        ng = int(Zgk.shape[0])
        nq, no, nv = int(Zgk.shape[1]), int(Xgi.shape[1]), int(Yga.shape[1])
        z, xi, ya = _colmajor(Zgk, ng), _colmajor(Xgi, ng), _colmajor(Yga, ng)
        u = _colmajor(U, no * nv)
        a = _vec(A)
        lk = _colmajor(Lik, no) if Lik is not None else None
        en = np.zeros(4)
        st = np.zeros(3, dtype=np.int64)
        self._check(self.lib.rpa_b200_jctc2024(self._h, ng, nq, no, nv, z.ptr, z.ld, xi.ptr, xi.ld, ya.ptr, ya.ld,
                                               int(U.shape[1]), u.ptr, u.ld, a.ptr, lk.ptr if lk else None,
                                               lk.ld if lk else no, float(cutoff_pno), int(bool(boys_screening)),
                                               float(cutoff_vabij), en.ctypes.data, st.ctypes.data))
        return tuple(en), tuple(int(x) for x in st)

    def exchange_mbpt3(self, R, eps_o, eps_v, U, A, return_x=False, prec="fp64"):
        """MBPT3 exchange energy -Tr(X K) (rpa_b200_exchange_mbpt3); with return_x also the
        Lyapunov solution X; prec "split" runs the Tr(XK) pair contraction as split-BF16."""
        nq = int(R.shape[0])
        no, nv = len(eps_o), len(eps_v)
        nov = no * nv
        nt = int(U.shape[1])
        r = _colmajor(R, nq)
        u = _colmajor(U, nov)
        a, eo, ev = _vec(A), _vec(eps_o), _vec(eps_v)
        ex = ctypes.c_double()
        X = np.zeros((nt, nt), order="F") if return_x else None
        self._check(self.lib.rpa_b200_exchange_mbpt3(self._h, nq, no, nv, r.ptr, r.ld, eo.ptr, ev.ptr, nt, u.ptr, u.ld,
                                                     a.ptr, _PREC[prec], ctypes.byref(ex),
                                                     X.ctypes.data if return_x else None, nt))
        return (ex.value, X) if return_x else ex.value

    def ec_rpa(self, R, eps_o, eps_v, freqs, weights, alpha=4.0, prec="split"):
        """Fused Pi build + energy: returns (E_c, E(u))."""
        nq = int(R.shape[0])
        no, nv, K = len(eps_o), len(eps_v), len(freqs)
        r = _colmajor(R, nq)
        eo, ev, fr, w = _vec(eps_o), _vec(eps_v), _vec(freqs), _vec(weights)
        ec = ctypes.c_double()
        eu = np.zeros(K)
        self._check(self.lib.rpa_b200_ec(self._h, nq, no, nv, r.ptr, r.ld, eo.ptr, ev.ptr, K, fr.ptr, w.ptr,
                                         float(alpha), _PREC[prec], ctypes.byref(ec), eu.ctypes.data))
        return ec.value, eu


def build(force: bool = False):
    """Compile librpa_b200.so in-tree (nvcc, sm_100a)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_rpa_b200_build", HERE / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)
