/*
 * librpa_b200 -- C ABI of the B200 (sm_100a) Cholesky-vector RPA hot path.
 *
 * Conventions (chosen to match the Fortran reference, modrzejewski/beyond-rpa,
 * compiled with -fdefault-integer-8 / -i8):
 *   - every dimension and flag is int64_t (Fortran default INTEGER = 8 bytes);
 *   - every matrix is column-major with an explicit leading dimension;
 *   - Cholesky vectors R(Q, ai) with ai = a + NVirt*(i-1) (a fastest), i.e.
 *     the Rkai(NCholesky, NVirt*NOcc) arrays of src/rpa/rpa_THC.f90:362 and
 *     src/rpa/rpa_core_MO.f90:395;
 *   - array arguments may point to host memory (pageable or pinned), to
 *     managed memory, or to device memory of the handle's GPU; the library
 *     detects which (cudaPointerGetAttributes) and stages host data itself.
 *     Device memory of another GPU is refused with RPA_ERR_INVALID_ARG before
 *     any launch (kernels read device arguments in place): copy such data to
 *     the handle's GPU (or to the host) first;
 *   - scalar outputs (energies) are host pointers;
 *   - every call is synchronous on return and returns an rpa_status.
 * Errors: the Fortran reference stops with `error stop` after msg(...,
 * MSG_ERROR); this ABI returns a non-zero status instead, and the Fortran
 * shim maps it back to msg + error stop.
 * A handle must not be shared by two host threads at the same time.
 * Limits (checked before any GPU work):
 *   - 1 <= NQ <= 2^20 and 1 <= NFreqs <= 64 (RPA_ERR_INVALID_ARG otherwise);
 *   - NOcc * NVirt <= 2^31 - 1 (RPA_ERR_TOO_LARGE);
 *   - at most 64 frequencies per instance in rpa_b200_ec_batched (the
 *     reference's limit), at most 2^24 instances (and frequency groups of 16)
 *     per call (RPA_ERR_INVALID_ARG);
 *   - N <= 46340 in rpa_b200_syevd and NQ <= 46340 in rpa_b200_piu_basis (an
 *     N x N FP64 matrix indexed in 32-bit); GEMM dimensions of the T2, exchange,
 *     THC and JCTC paths <= 2^31 - 1 (RPA_ERR_TOO_LARGE);
 *   - rpa_b200_ec_from_pi_noalloc: the fixed scratch described at its
 *     declaration (RPA_ERR_TOO_LARGE);
 *   - device memory: RPA_ERR_OOM when a workspace cannot be allocated.
 */
#ifndef RPA_B200_H
#define RPA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
/* The library is built with hidden default visibility: exactly the entry points declared here
 * are exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum rpa_status {
  RPA_OK = 0,
  RPA_ERR_INVALID_ARG = 1,  /* bad dimension, NULL pointer, unsupported mode   */
  RPA_ERR_NOT_SPD = 2,      /* 1+Pi(u) not positive definite (Cholesky pivot) */
  RPA_ERR_NONFINITE = 3,    /* NaN/Inf in an input or result                 */
  RPA_ERR_OOM = 4,          /* device or host allocation failed               */
  RPA_ERR_CUDA = 5,         /* CUDA runtime / driver error                    */
  RPA_ERR_TIMEOUT = 6,      /* a bounded device-side wait expired             */
  RPA_ERR_NO_DEVICE = 7,    /* no sm_100 GPU visible                          */
  RPA_ERR_NOT_CONVERGED = 8, /* quadrature / eigen-solver did not converge    */
  RPA_ERR_TOO_LARGE = 9,    /* problem exceeds a size limit of the entry point
                                (e.g. the fixed scratch of
                                rpa_b200_ec_from_pi_noalloc)                   */
  RPA_ERR_INTERNAL = 10     /* unexpected host-side failure; no entry point
                                lets a C++ exception escape                    */
} rpa_status;

/* Precision of the Pi(u) contraction. */
#define RPA_PREC_FP64 0      /* plain FP64 (FP64 tensor-core DMMA)                 */
#define RPA_PREC_SPLIT_BF16 1 /* X = hi + lo (bf16), 3 tcgen05 products, FP32 acc,
                                 exact FP64 diagonal                               */

typedef struct rpa_b200_handle rpa_b200_handle;

/* Create / destroy a handle bound to one GPU (`device` = CUDA ordinal).
 * The handle owns a stream, a grow-only device workspace and the TMA
 * descriptors.  flags: reserved, pass 0.                                    */
int rpa_b200_create(rpa_b200_handle** handle, int64_t device, int64_t flags);
int rpa_b200_destroy(rpa_b200_handle* handle);
const char* rpa_b200_status_string(int status);
/* Human-readable detail of the last failing call on this handle. */
const char* rpa_b200_last_error(const rpa_b200_handle* handle);
/* Time (ms, CUDA events on the handle's stream) of the last call:
 * out[0] = staging (H2D copies, input screening), out[1] = Pi build,
 * out[2] = log-det (Cholesky + sums), out[3] = the rest (result copies),
 * out[4] = the Pi contraction kernel alone, out[5] = the scale/split pass. */
int rpa_b200_last_timings(const rpa_b200_handle* handle, double* out, int64_t n);
/* Number of kernels this library launched during the last call.           */
int64_t rpa_b200_last_launches(const rpa_b200_handle* handle);
/* Run subsequent calls on `stream` (a cudaStream_t of the handle's device;
 * NULL restores the handle's own stream).  Calls still synchronise the
 * stream before returning.                                                 */
int rpa_b200_set_stream(rpa_b200_handle* handle, void* stream);

/*
 * Tile plans of the FP64 log-det (the blocked Cholesky of 1 + Pi(u)), kept per
 * bucket of 256 matrix orders on the handle.  A plan is the outer block Nb2
 * (columns per trailing update: 128, 256 or 512) and the CTA tile edge of its
 * FP64 SYRK updates (64 or 128).  No reference counterpart: the reference
 * calls DGEQRF (src/linear-algebra/real_linalg.f90:815), whose blocking MKL
 * picks internally.
 *   rpa_b200_tune_logdet: time the six candidates on NMat seeded positive
 *     definite matrices of order NQ (handle workspace NMat*NQ*NQ doubles), keep
 *     the fastest for NQ's bucket, return it in *Nb2, *Tile; Ms (6 doubles or
 *     NULL) receives each candidate's time in the order (128,64) (256,64)
 *     (512,64) (128,128) (256,128) (512,128).
 *   rpa_b200_set_logdet_plan: store a plan (e.g. one a previous run tuned).
 *   rpa_b200_get_logdet_plan: the plan used for order NQ (256/64 if none).
 *   rpa_b200_set_autotune: 1 (default; 0 if RPA_B200_AUTOTUNE=0 at create)
 *     lets rpa_b200_ec_batched tune each bucket it meets for the first time,
 *     on the call's own Pi buffers (up to 128 matrices per bucket); 0 uses
 *     the stored or default plans only.
 */
int rpa_b200_tune_logdet(rpa_b200_handle* handle, int64_t NQ, int64_t NMat, int64_t* Nb2, int64_t* Tile,
                         double* Ms);
int rpa_b200_set_logdet_plan(rpa_b200_handle* handle, int64_t NQ, int64_t Nb2, int64_t Tile);
int rpa_b200_get_logdet_plan(const rpa_b200_handle* handle, int64_t NQ, int64_t* Nb2, int64_t* Tile);
int rpa_b200_set_autotune(rpa_b200_handle* handle, int64_t on);

/*
 * Device-memory cap of a handle.  No reference counterpart (the reference
 * allocates host arrays as it goes).  The handle's workspace grows on demand;
 * rpa_b200_set_workspace_limit caps it at Bytes (0 = no cap, the default).  An
 * allocation that would pass the cap fails as a failed cudaMalloc does: the
 * call returns RPA_ERR_OOM and the handle stays usable (raise the cap, or use
 * smaller problems).  Lowering the cap frees nothing already held.
 * rpa_b200_workspace_bytes reports the bytes held now and the cap (either
 * pointer may be NULL).
 */
int rpa_b200_set_workspace_limit(rpa_b200_handle* handle, int64_t Bytes);
int rpa_b200_workspace_bytes(const rpa_b200_handle* handle, int64_t* Used, int64_t* Limit);

/*
 * Failure-detection self-test.  No reference counterpart.  Every spin-wait
 * in this library's kernels is bounded: when its limit (4 s) passes, the
 * waiting thread records an error code on the device, the kernel returns, and
 * the call reports RPA_ERR_TIMEOUT with the CUDA context still usable.  This
 * entry point runs that same bounded wait on a barrier that nothing ever
 * arrives on, with the limit LimitMs (0 < LimitMs <= 4000), and reports the
 * result through the same path: it returns RPA_ERR_TIMEOUT when detection
 * works.  Nothing asynchronous is in flight while it waits, and the next call
 * on the handle starts clean.
 */
int rpa_b200_selftest_wait_timeout(rpa_b200_handle* handle, double LimitMs);

/*
 * Pi(u) matrices:  PiU(:,:,u) = alpha * sum_ai R(:,ai) Chi_u(ai) R(:,ai)^T,
 * Chi_u(ai) = D(ai) / (D(ai)^2 + u^2), D(ai) = VirtEnergies(a) - OccEnergies(i).
 * Replaces rpa_THC_PiU / rpa_THC_PiU_BlockAlgo / rpa_THC_ChiRkai
 * (src/rpa/rpa_THC.f90:215-371) and rpa_GPiUG_MO (src/rpa/rpa_core_MO.f90:347-406).
 * alpha = 4 closed shell, 2 per spin for open shell (rpa_THC.f90:258-268).
 * PiU: NQ x NQ x NFreqs, leading dimension ldPi >= NQ, full symmetric square
 * on return (as the reference's DGEMM produces).
 */
int rpa_b200_pi(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                double alpha, int64_t prec, double* PiU, int64_t ldPi);

/*
 * RPA correlation energy from given Pi(u) matrices:
 *   Ec = 1/(2 pi) sum_u w_u [ln det(1 + Pi(u)) - Tr Pi(u)],
 * log-det by FP64 Cholesky, traces and sums in double-double.
 * Replaces rpa_CC_EcRPA_Analytic (src/rpa/rpa_CC.f90:412-471) with
 * real_LogDet (src/linear-algebra/real_linalg.f90:776-825) and the energy loop
 * of rpa_FreqIntegral_MO (src/rpa/rpa.f90:1338-1380).
 * Only the lower triangle of each PiU(:,:,u) is read.  Eu (NFreqs, may be
 * NULL) receives E(u) = ln det(1+Pi(u)) - Tr Pi(u).
 */
int rpa_b200_ec_from_pi(rpa_b200_handle* h, int64_t NQ, int64_t NFreqs, const double* PiU, int64_t ldPi,
                        const double* FreqWeights, double* Ec, double* Eu);

/*
 * Fused Pi build + energy (Pi never leaves the GPU): the chain
 * rpa_THC_PiU -> rpa_CC_EcRPA_Analytic of rpa_THC_MBPT3
 * (src/rpa/rpa_THC.f90:106-108) and rpa_CC_PiU -> rpa_CC_EcRPA_Analytic of
 * rpa_CC_Energy_2 (src/rpa/rpa_CC.f90:781-785).
 */
int rpa_b200_ec(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                const double* FreqWeights, double alpha, int64_t prec, double* Ec, double* Eu);

/*
 * Imaginary-frequency quadrature (host code, no GPU needed): transformed
 * Gauss-Legendre points u_k = a(1+t_k)/(1-t_k), weights 2 a w_k/(1-t_k)^2,
 * with a scanned over [0.1, 15] (15000 points) to minimise the RMSD of
 * sum_k w_k/(D^2+u_k^2) against pi/(2D) over a 100-bin histogram of the
 * active D(ai).  Replaces rpa_OptimizeFreqQuad / rpa_OptQuadScaling /
 * rpa_FreqQuadError (src/rpa/OptFreqQuad.f90:12-169), quad_CasimirPolder
 * (src/rpa/quadratures.f90:570-643), rpa_DaiHistogram and rpa_NCore
 * (src/rpa/OrbDiffHist.f90:42-146).
 * OrbEnergies: NOcc occupied then NVirt virtual energies, each ascending;
 * occupied orbitals below CoreOrbThresh (reference default -3 Eh) are frozen.
 * NFixed > 0: exactly NFixed points; NFixed = 0: the smallest n in [8, 64]
 * with RMSD < TargetError and max relative error < TargetRelError
 * (reference defaults 1e-6 and 1e-3).  Freqs / FreqWeights need room for 64.
 */
int rpa_b200_freq_grid(int64_t NOcc, int64_t NVirt, const double* OrbEnergies, double CoreOrbThresh,
                       double TargetError, double TargetRelError, int64_t NFixed, double* Freqs,
                       double* FreqWeights, int64_t* NFreqs);

/*
 * One frequency grid shared by the subsystems of a many-body expansion (so that
 * their energies differ consistently): NSets orbital-energy sets (one per
 * subsystem and spin; set s has NOcc[s] occupied then NVirt[s] virtual
 * energies at OrbEnergies[s]), set 0 being the whole complex.  A Delta
 * histogram per set; LimitDai != 0 caps every histogram at the largest active
 * excitation energy of set 0 (GridLimitDai: excitations on ghost atoms of a
 * monomer must not stretch its histogram); the optimiser's RMSD and relative
 * error are the worst over the sets.  A set whose occupied orbitals are all
 * frozen takes no part.  Replaces the grid construction of rpa_PostSCF
 * (src/rpa/rpa_driver.f90:118-175) with rpa_DaiMaxThresh / rpa_DaiHistogram
 * (src/rpa/OrbDiffHist.f90:10-123) and the multi-set rpa_FreqQuadError
 * (src/rpa/OptFreqQuad.f90:125-169).  Other arguments as rpa_b200_freq_grid.
 */
int rpa_b200_freq_grid_mbe(int64_t NSets, const int64_t* NOcc, const int64_t* NVirt,
                           const double* const* OrbEnergies, double CoreOrbThresh, int64_t LimitDai,
                           double TargetError, double TargetRelError, int64_t NFixed, double* Freqs,
                           double* FreqWeights, int64_t* NFreqs);

/*
 * Interaction (NBody = 2) and nonadditive (NBody = 3, 4) energies of a many-body
 * expansion from the subsystem energies E, in the reference's subsystem order
 * (src/common/sys_definitions.f90:19-36), 0-based: E[0] whole system, E[1..3]
 * monomers A, B, C, E[4..6] dimers AB, BC, AC, E[7] monomer D, E[8..10] dimers
 * AD, BD, CD, E[11..14] trimers ABC, ABD, ACD, BCD; NBody = 2, 3, 4 reads
 * E[0..2], E[0..6], E[0..14].  Replaces rpa_Eint2Body, rpa_EintNadd and
 * rpa_EintNadd4Body (src/rpa/rpa_driver.f90:381-433): the group differences in
 * FP64 as there, their combination in double-double (the reference's REAL(16)).
 * Host-only; no handle.
 */
int rpa_b200_mbe_energy(int64_t NBody, const double* E, double* Eint);

/*
 * Adjoint of the RPA energy: dE_c/dR (NQ x nov, leading dimension lddR),
 * dE_c/dOccEnergies (NOcc) and dE_c/dVirtEnergies (NVirt); Ec (may be NULL)
 * the energy itself.  No counterpart in the reference (it has no gradients):
 *   dE/dR(:,ai) = sum_u w_u/(2 pi) 2 alpha c_u(ai) ((1+Pi_u)^{-1} - 1) R(:,ai),
 *   dE/dD(ai)   = sum_u w_u/(2 pi) alpha R(:,ai)^T ((1+Pi_u)^{-1} - 1) R(:,ai) dc_u/dD,
 * c_u = D/(D^2+u^2).  Pi(u) is recomputed (prec as in rpa_b200_ec) and
 * factorised; (1+Pi_u)^{-1} R comes from two batched triangular solves in FP64.
 * dR/dOcc/dVirt may be host or device pointers (dOcc/dVirt may be NULL).
 */
int rpa_b200_ec_grad(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                     const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                     const double* FreqWeights, double alpha, int64_t prec, double* Ec, double* dR, int64_t lddR,
                     double* dOcc, double* dVirt);

/* One system (a many-body-expansion fragment) of a batched call. */
typedef struct rpa_instance {
  int64_t NQ, NOcc, NVirt;
  const double* R; /* NQ x NOcc*NVirt, column-major, leading dimension ldR */
  int64_t ldR;
  const double* OccEnergies;
  const double* VirtEnergies;
  int64_t NFreqs; /* 1 .. 64 */
  const double* Freqs;
  const double* FreqWeights;
  double alpha;
} rpa_instance;

/*
 * RPA correlation energies of many independent systems of uneven size in one
 * call (the subsystem loop of rpa_PostSCF, src/rpa/rpa_driver.f90:175-240,
 * which the reference runs sequentially).  Instances are packed into
 * memory-bounded batches; per batch one multi-instance scale/split launch, one
 * persistent multi-instance tensor-core SYRK launch and one variable-order
 * batched Cholesky run as a single CUDA graph.  Ec[i] receives the energy of
 * instance i; Eu (may be NULL) the E(u) of all instances concatenated.  An
 * instance with more than 16 frequencies runs as consecutive groups of at
 * most 16 frequencies on the same R (E_c summed over its groups).
 */
int rpa_b200_ec_batched(rpa_b200_handle* h, int64_t ninst, const rpa_instance* inst, int64_t prec, double* Ec,
                        double* Eu);

/*
 * Direct-ring T2 amplitudes T2 = U diag(A) U^T (nov x nov) at coupling
 * strength 1, by the randomised range finder of the reference: guess vectors
 * Omega (nov x GuessNVecs; NULL -> uniform [-1/2,1/2) from `seed`), I*Omega,
 * Gram eigen-decomposition with the linear-dependency cutoff
 * SmallEigenvalsCutoff, Rayleigh-Ritz on T^T I T, A = a/(2(a+1)), and the
 * eigenvalue cutoff of type CutoffType (0 EIG, 1 EIG_DIV_MAXEIG,
 * 2 EIG_DIV_NELECTRON, 3 SUM_REJECTED) with threshold CutoffThresh; when
 * *CommonThresh < 0 (supersystem) the threshold used is returned in it,
 * otherwise *CommonThresh is used as the threshold (subsystems).
 * Replaces rpa_CC_Diagonalize_PiU (src/rpa/rpa_CC.f90:1108-1129) and
 * rpa_THC_CC_T2 / rpa_CC_T2_v5 / rpa_CC_IM_v5 / rpa_CC_MIM_v5 / rpa_T2_EigRPA
 * (src/rpa/rpa_CC_Doubles.f90:369-1009).  (1 + Pi(u))^{-1} is applied through
 * the Cholesky factors of the energy step instead of an eigen-decomposition of
 * Pi(u).  Outputs: A (NVecsT2, ascending = largest |A| first), U (nov x
 * NVecsT2, ldU >= nov; the Uaim layout), EigRPA(mu) = 2 A_mu |R U_mu|^2,
 * Ec (may be NULL) the RPA energy of the same Pi(u).  MaxNVecsT2 bounds the
 * capacity of A, U and EigRPA.
 */
int rpa_b200_dring_t2(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                      const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                      const double* FreqWeights, double alpha, int64_t prec, int64_t GuessNVecs, const double* Omega,
                      uint64_t seed, double SmallEigenvalsCutoff, double CutoffThresh, int64_t CutoffType,
                      double* CommonThresh, int64_t MaxNVecsT2, double* A, double* U, int64_t ldU,
                      int64_t* NVecsT2, double* EigRPA, double* Ec);

/*
 * Exchange (SOSEX) energy  Ex = -Alpha sum_{abij} (aj|bi) T_aibj with
 * T = U diag(B) U^T, B = A (S2Operator = 0) or A/(1 - 4A^2) (S2Operator = 1).
 * Replaces rpa_CC_Exchange_SOSEX + rpa_CC_EcExchange1
 * (src/rpa/rpa_CC_Exchange.f90:36-116).  U is (nov x NVecsT2) column-major
 * (ldU >= nov), i.e. the transpose of that routine's Vkai(NVecsT2, NVirt, NOcc).
 * Prec: RPA_PREC_FP64 (the pair GEMMs on FP64 DMMA) or RPA_PREC_SPLIT_BF16
 * (R and U split into bf16 hi/lo, three tcgen05 products per W tile, FP32
 * accumulation in 64-column segments, FP64 Hadamard sums).
 */
int rpa_b200_exchange_sosex(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R,
                            int64_t ldR, int64_t NVecsT2, const double* U, int64_t ldU, const double* A, double Alpha,
                            int64_t S2Operator, int64_t Prec, double* Ex);

/*
 * Cholesky vectors from THC factors: R(k, ai) = sum_g Zgk(g, k) Xga(g, a) Xgi(g, i),
 * ai = a + NVirt i, R (NQ x NOcc*NVirt, ldR >= NQ).  Zgk (NGrid x NQ), Xga (NGrid x
 * NVirt), Xgi (NGrid x NOcc) column-major.  Replaces rpa_THC_Rkab / rpa_THC_Rkai
 * (src/rpa/rpa_THC.f90:374-426): Khatri-Rao blocks and FP64 tensor-core GEMMs.
 */
int rpa_b200_thc_r(rpa_b200_handle* h, int64_t NGrid, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* Zgk,
                   int64_t ldZ, const double* Xga, int64_t ldXa, const double* Xgi, int64_t ldXi, double* R,
                   int64_t ldR);

/*
 * RPA energy from THC factors (rpa_THC_PiU with FullRkai, src/rpa/rpa_THC.f90:215-329,
 * followed by the energy of rpa_b200_ec): R is formed on the device and never leaves it.
 */
int rpa_b200_ec_thc(rpa_b200_handle* h, int64_t NGrid, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* Zgk,
                    int64_t ldZ, const double* Xga, int64_t ldXa, const double* Xgi, int64_t ldXi,
                    const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                    const double* FreqWeights, double alpha, int64_t prec, double* Ec, double* Eu);

/*
 * Particle-hole corrections to direct RPA on THC factors with pair-natural orbitals
 * (rpa_JCTC2024_Corrections and helpers, src/rpa/rpa_JCTC2024.f90:24-703; Cieslinski,
 * Tucholska, Modrzejewski, J. Chem. Theory Comput. 19, 6619 (2023)).  Zgk (NGrid x NQ),
 * Xgi (NGrid x NOcc), Yga (NGrid x NVirt): THC factors; U (NOcc*NVirt x NVecsT2, the Uaim
 * layout) and Am: the direct-ring T2 of rpa_b200_dring_t2; Lik (NOcc x NOcc, may be NULL):
 * the occupied localisation.  PNOs of each pair: singular vectors of T(ab;ij) with singular
 * values > CutoffThreshPNO.  BoysScreening = 1 skips the (ab|ij) contribution of pairs with
 * sqrt(max_a (aa|aa) (ij|ij)) <= CutoffThreshVabij.  Energies[4] = { EcRPA(PNO), Ec1b,
 * Ec2bcd, Ec2ghij }: E(SOSEX cumulant) = Ec1b / 2, E(PH3) = Ec2bcd + Ec2ghij.  PNOStats[3]
 * (may be NULL) = { max NVirtPNO, sum NVirtPNO, pairs without PNOs }.
 */
int rpa_b200_jctc2024(rpa_b200_handle* h, int64_t NGrid, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* Zgk,
                      int64_t ldZ, const double* Xgi, int64_t ldXi, const double* Yga, int64_t ldYa, int64_t NVecsT2,
                      const double* U, int64_t ldU, const double* Am, const double* Lik, int64_t ldL,
                      double CutoffThreshPNO, int64_t BoysScreening, double CutoffThreshVabij, double* Energies,
                      int64_t* PNOStats);

/* Basis types of the effective dielectric matrix (src/rpa/rpa_definitions.f90:92-104). */
#define RPA_BASIS_RANDOM 1
#define RPA_BASIS_EIGEN 2
#define RPA_BASIS_FULL_CHOLESKY 3

/*
 * Basis G of the effective dielectric matrix from Pi(LowestFreq) (one frequency of
 * rpa_b200_pi).  Replaces rpa_G (src/rpa/rpa.f90:31-173): BasisType
 * RPA_BASIS_EIGEN = eigenvectors of Pi by descending eigenvalue, RPA_BASIS_RANDOM
 * = two subspace iterations G <- qr(Pi G) from Guess (NQ x NQ, ldGuess; NULL:
 * uniform numbers from `seed`), RPA_BASIS_FULL_CHOLESKY = identity.  NVecs is
 * the smallest p with sum_{q>=p} RWR(q,q) < TargetError (RWR = diag of G^T Pi G),
 * scanning from the last column as the reference does; TraceError receives
 * that sum and ExactTrace Tr Pi (both may be NULL).  G (NQ x NVecs used, ldG >= NQ)
 * must hold NQ columns.  The random basis orthonormalises by shifted CholeskyQR3
 * and returns RPA_ERR_NOT_SPD when Pi G is numerically rank deficient (use the
 * eigenvector basis, the reference's default, for such Pi).
 */
int rpa_b200_piu_basis(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                       const double* OccEnergies, const double* VirtEnergies, double LowestFreq, double alpha,
                       int64_t prec, int64_t BasisType, double TargetError, const double* Guess, int64_t ldGuess,
                       uint64_t seed, double* G, int64_t ldG, int64_t* NVecs, double* TraceError,
                       double* ExactTrace);

/*
 * Rp = G^T R (NVecs x nov, ldRp >= NVecs): Cholesky vectors in the compressed basis,
 * the Cholesky-path counterpart of THC_ZgkPiU = Zgk G(:, 1:NVecsPiU)
 * (src/rpa/rpa.f90:2318-2320).  Energies and T2 then run with NQ = NVecs.
 */
int rpa_b200_project_basis(rpa_b200_handle* h, int64_t NQ, int64_t NVecs, int64_t nov, const double* G, int64_t ldG,
                           const double* R, int64_t ldR, double* Rp, int64_t ldRp);

/*
 * Symmetric eigen-decomposition A = Z diag(Eigenvals) Z^T, Eigenvals ascending,
 * A (N x N, column-major, ldA >= N; lower and upper triangles both read)
 * overwritten by the eigenvectors Z.  Replaces real_EVD with
 * ComputeEigenvecs = .true. (src/linear-algebra/real_linalg.f90:1501-1559,
 * LAPACK dsyevd): Householder tridiagonalisation, divide and conquer and
 * back-transformation, all on the GPU.  Used inside rpa_b200_dring_t2 and
 * rpa_b200_exchange_mbpt3.
 */
int rpa_b200_syevd(rpa_b200_handle* h, int64_t N, double* A, int64_t ldA, double* Eigenvals);

/*
 * MBPT3 exchange energy  Ex = -Tr(X K) = -sum_{abij} (aj|bi) (U X U^T)_aibj,
 * where X (NVecsT2 x NVecsT2) solves B^T X + X B = A with
 * A_mn = A_m D_mn + D_mn A_n, B_mn = D_mn + 2 U_mn + 4 U_mn A_n,
 * Ukl = (R U)^T (R U), Dkl = U^T diag(e_a - e_i) U.  Replaces
 * rpa_CC_Exchange_MBPT3_1 + rpa_CC_Ukl + rpa_CC_Dkl + rpa_CC_TrXK
 * (src/rpa/rpa_CC_Exchange.f90:177-336; the Lyapunov solve replaces
 * real_Lyapunov, src/linear-algebra/real_linalg.f90:125-171).  U and A are
 * the outputs of rpa_b200_dring_t2.  X (may be NULL, ldX >= NVecsT2) receives
 * the Lyapunov solution.  RPA_ERR_NOT_CONVERGED if the solve fails.  Prec
 * selects the Tr(XK) pair contraction as in rpa_b200_exchange_sosex (the
 * Lyapunov solve is FP64 in both).
 */
int rpa_b200_exchange_mbpt3(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R,
                            int64_t ldR, const double* OccEnergies, const double* VirtEnergies, int64_t NVecsT2,
                            const double* U, int64_t ldU, const double* A, int64_t Prec, double* Ex, double* X,
                            int64_t ldX);

/*
 * Allocation-free energy from given Pi(u) matrices.  No counterpart in the
 * reference: it exists for callers that cannot allocate GPU memory (a host
 * whose device memory belongs to a pool or arena it cannot grow, or code
 * running while the device-memory footprint must not change).  Same result
 * and arguments as rpa_b200_ec_from_pi, but no handle and no device
 * allocation: the working storage is one fixed array of
 * RPA_B200_NOALLOC_SCRATCH_BYTES (32 MiB) inside the library, which every GPU
 * that loads the library holds until process exit.
 *   - Limit: NFreqs*NQ*NQ + NFreqs*NQ + 4*NFreqs + 1 doubles must fit in the
 *     array (NQ = 512 with NFreqs <= 15; NQ = 400 with NFreqs <= 26);
 *     otherwise RPA_ERR_TOO_LARGE is returned before any GPU work.
 *   - PiU and FreqWeights may be host or device pointers; Ec/Eu are host.
 *   - stream: a cudaStream_t of `device`, or NULL for the default stream; the
 *     call synchronises it before returning.
 *   - All calls on a device share the array (contents persist between calls;
 *     the call clears what must start at zero).  Calls that overlap on the GPU
 *     race on it: serialise them.
 *   - The first call on a device looks the array's address up once
 *     (cudaGetSymbolAddress); make that first call before any stream capture.
 *     That first call is also when the device memory is committed: with CUDA's
 *     lazy module loading the 32 MiB array and the kernels this entry point
 *     uses are loaded onto the GPU at that moment, not when the library is
 *     loaded.  A caller whose device footprint is frozen later should make one
 *     call (any valid problem) before that point.
 *   - Only the lower triangle of each PiU(:,:,u) is read, as in
 *     rpa_b200_ec_from_pi.  Same limits on NQ (<= 2^20) and NFreqs (<= 64);
 *     device must be a CUDA ordinal below 64 (RPA_ERR_INVALID_ARG otherwise).
 */
#define RPA_B200_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int rpa_b200_ec_from_pi_noalloc(int64_t device, void* stream, int64_t NQ, int64_t NFreqs, const double* PiU,
                                int64_t ldPi, const double* FreqWeights, double* Ec, double* Eu);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* RPA_B200_H */
