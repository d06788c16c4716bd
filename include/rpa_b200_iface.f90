! Fortran interface to librpa_b200 (include/rpa_b200.h), for the reference's host code.
!
! The reference is Fortran 2008 compiled with 8-byte default integers
! (-fdefault-integer-8 / -i8), so every dimension is integer(c_int64_t) and every
! array is passed as a contiguous column-major dummy.  Add this file to the
! reference's sources (as src/rpa/rpa_b200_iface.f90) and link with -lrpa_b200.
! rpa_b200_check maps a non-zero status to the reference's msg(..., MSG_ERROR) +
! error stop.
module rpa_b200_iface
      use iso_c_binding
      implicit none

      integer(c_int), parameter :: RPA_OK = 0
      integer(c_int64_t), parameter :: RPA_PREC_FP64 = 0, RPA_PREC_SPLIT_BF16 = 1

      ! struct rpa_instance of include/rpa_b200.h (one system of rpa_b200_ec_batched)
      type, bind(C) :: rpa_instance
            integer(c_int64_t) :: NQ, NOcc, NVirt
            type(c_ptr) :: R                 ! c_loc(Rkai): NQ x NOcc*NVirt, leading dimension ldR
            integer(c_int64_t) :: ldR
            type(c_ptr) :: OccEnergies, VirtEnergies
            integer(c_int64_t) :: NFreqs     ! 1 .. 64
            type(c_ptr) :: Freqs, FreqWeights
            real(c_double) :: alpha
      end type rpa_instance

      interface
            integer(c_int) function rpa_b200_create(handle, device, flags) bind(C, name="rpa_b200_create")
                  import :: c_int, c_int64_t, c_ptr
                  type(c_ptr), intent(out) :: handle
                  integer(c_int64_t), value :: device, flags
            end function
            integer(c_int) function rpa_b200_destroy(handle) bind(C, name="rpa_b200_destroy")
                  import :: c_int, c_ptr
                  type(c_ptr), value :: handle
            end function
            type(c_ptr) function rpa_b200_last_error(handle) bind(C, name="rpa_b200_last_error")
                  import :: c_ptr
                  type(c_ptr), value :: handle
            end function
            integer(c_int) function rpa_b200_pi(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, &
                  NFreqs, Freqs, alpha, prec, PiU, ldPi) bind(C, name="rpa_b200_pi")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: h
                  integer(c_int64_t), value :: NQ, NOcc, NVirt, ldR, NFreqs, prec, ldPi
                  real(c_double), dimension(ldR, *), intent(in) :: R
                  real(c_double), dimension(*), intent(in) :: OccEnergies, VirtEnergies, Freqs
                  real(c_double), value :: alpha
                  real(c_double), dimension(ldPi, NQ, *), intent(out) :: PiU
            end function
            integer(c_int) function rpa_b200_ec_from_pi(h, NQ, NFreqs, PiU, ldPi, FreqWeights, Ec, Eu) &
                  bind(C, name="rpa_b200_ec_from_pi")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: h
                  integer(c_int64_t), value :: NQ, NFreqs, ldPi
                  real(c_double), dimension(ldPi, NQ, *), intent(in) :: PiU
                  real(c_double), dimension(*), intent(in) :: FreqWeights
                  real(c_double), intent(out) :: Ec
                  real(c_double), dimension(*), intent(out) :: Eu
            end function
            integer(c_int) function rpa_b200_ec(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, &
                  NFreqs, Freqs, FreqWeights, alpha, prec, Ec, Eu) bind(C, name="rpa_b200_ec")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: h
                  integer(c_int64_t), value :: NQ, NOcc, NVirt, ldR, NFreqs, prec
                  real(c_double), dimension(ldR, *), intent(in) :: R
                  real(c_double), dimension(*), intent(in) :: OccEnergies, VirtEnergies, Freqs, FreqWeights
                  real(c_double), value :: alpha
                  real(c_double), intent(out) :: Ec
                  real(c_double), dimension(*), intent(out) :: Eu
            end function
            integer(c_int) function rpa_b200_freq_grid(NOcc, NVirt, OrbEnergies, CoreOrbThresh, &
                  TargetError, TargetRelError, NFixed, Freqs, FreqWeights, NFreqs) &
                  bind(C, name="rpa_b200_freq_grid")
                  import :: c_int, c_int64_t, c_double
                  integer(c_int64_t), value :: NOcc, NVirt, NFixed
                  real(c_double), dimension(*), intent(in) :: OrbEnergies
                  real(c_double), value :: CoreOrbThresh, TargetError, TargetRelError
                  real(c_double), dimension(64), intent(out) :: Freqs, FreqWeights
                  integer(c_int64_t), intent(out) :: NFreqs
            end function

            ! ---- beyond-RPA path (T2, exchange, eigensolver, compressed Pi basis)
            integer(c_int) function rpa_b200_dring_t2(handle, NQ, NOcc, NVirt, R, ldR, OccEnergies, &
                  VirtEnergies, NFreqs, Freqs, FreqWeights, alpha, prec, GuessNVecs, Omega, seed, &
                  SmallEigenvalsCutoff, CutoffThresh, CutoffType, CommonThresh, MaxNVecsT2, A, U, ldU, &
                  NVecsT2, EigRPA, Ec) bind(C, name="rpa_b200_dring_t2")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle, Omega   ! Omega: c_null_ptr = generated guess vectors
                  integer(c_int64_t), value :: NQ, NOcc, NVirt, ldR, NFreqs, prec, GuessNVecs, seed, &
                        CutoffType, MaxNVecsT2, ldU
                  real(c_double), dimension(*), intent(in) :: R, OccEnergies, VirtEnergies, Freqs, FreqWeights
                  real(c_double), value :: alpha, SmallEigenvalsCutoff, CutoffThresh
                  real(c_double), intent(inout) :: CommonThresh   ! < 0: supersystem (set on return)
                  real(c_double), dimension(*), intent(out) :: A, U, EigRPA
                  integer(c_int64_t), intent(out) :: NVecsT2
                  real(c_double), intent(out) :: Ec
            end function

            integer(c_int) function rpa_b200_exchange_sosex(handle, NQ, NOcc, NVirt, R, ldR, NVecsT2, U, ldU, &
                  A, Alpha, S2Operator, Prec, Ex) bind(C, name="rpa_b200_exchange_sosex")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: NQ, NOcc, NVirt, ldR, NVecsT2, ldU, S2Operator
                  integer(c_int64_t), value :: Prec      ! 0: FP64, 1: split-BF16 pair contraction
                  real(c_double), dimension(*), intent(in) :: R, U, A
                  real(c_double), value :: Alpha
                  real(c_double), intent(out) :: Ex
            end function

            integer(c_int) function rpa_b200_exchange_mbpt3(handle, NQ, NOcc, NVirt, R, ldR, OccEnergies, &
                  VirtEnergies, NVecsT2, U, ldU, A, Prec, Ex, X, ldX) bind(C, name="rpa_b200_exchange_mbpt3")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle, X          ! X: c_null_ptr unless the Lyapunov solution is wanted
                  integer(c_int64_t), value :: NQ, NOcc, NVirt, ldR, NVecsT2, ldU, ldX, Prec
                  real(c_double), dimension(*), intent(in) :: R, OccEnergies, VirtEnergies, U, A
                  real(c_double), intent(out) :: Ex
            end function

            integer(c_int) function rpa_b200_thc_r(handle, NGrid, NQ, NOcc, NVirt, Zgk, ldZ, Xga, ldXa, Xgi, &
                  ldXi, R, ldR) bind(C, name="rpa_b200_thc_r")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: NGrid, NQ, NOcc, NVirt, ldZ, ldXa, ldXi, ldR
                  real(c_double), dimension(*), intent(in) :: Zgk, Xga, Xgi
                  real(c_double), dimension(ldR, *), intent(out) :: R
            end function

            integer(c_int) function rpa_b200_ec_thc(handle, NGrid, NQ, NOcc, NVirt, Zgk, ldZ, Xga, ldXa, Xgi, &
                  ldXi, OccEnergies, VirtEnergies, NFreqs, Freqs, FreqWeights, alpha, prec, Ec, Eu) &
                  bind(C, name="rpa_b200_ec_thc")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: NGrid, NQ, NOcc, NVirt, ldZ, ldXa, ldXi, NFreqs, prec
                  real(c_double), dimension(*), intent(in) :: Zgk, Xga, Xgi, OccEnergies, VirtEnergies, Freqs, &
                        FreqWeights
                  real(c_double), value :: alpha
                  real(c_double), intent(out) :: Ec
                  real(c_double), dimension(*), intent(out) :: Eu
            end function

            integer(c_int) function rpa_b200_jctc2024(handle, NGrid, NQ, NOcc, NVirt, Zgk, ldZ, Xgi, ldXi, &
                  Yga, ldYa, NVecsT2, U, ldU, Am, Lik, ldL, CutoffThreshPNO, BoysScreening, CutoffThreshVabij, &
                  Energies, PNOStats) bind(C, name="rpa_b200_jctc2024")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle, Lik        ! Lik: c_null_ptr = canonical orbitals
                  integer(c_int64_t), value :: NGrid, NQ, NOcc, NVirt, ldZ, ldXi, ldYa, NVecsT2, ldU, ldL, &
                        BoysScreening
                  real(c_double), dimension(*), intent(in) :: Zgk, Xgi, Yga, U, Am
                  real(c_double), value :: CutoffThreshPNO, CutoffThreshVabij
                  real(c_double), dimension(4), intent(out) :: Energies
                  integer(c_int64_t), dimension(3), intent(out) :: PNOStats
            end function

            integer(c_int) function rpa_b200_syevd(handle, N, A, ldA, Eigenvals) bind(C, name="rpa_b200_syevd")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: N, ldA
                  real(c_double), dimension(ldA, *), intent(inout) :: A
                  real(c_double), dimension(*), intent(out) :: Eigenvals
            end function

            integer(c_int) function rpa_b200_piu_basis(handle, NQ, NOcc, NVirt, R, ldR, OccEnergies, &
                  VirtEnergies, LowestFreq, alpha, prec, BasisType, TargetError, Guess, ldGuess, seed, G, ldG, &
                  NVecs, TraceError, ExactTrace) bind(C, name="rpa_b200_piu_basis")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle, Guess      ! Guess: c_null_ptr = generated (random basis only)
                  integer(c_int64_t), value :: NQ, NOcc, NVirt, ldR, prec, BasisType, ldGuess, seed, ldG
                  real(c_double), dimension(*), intent(in) :: R, OccEnergies, VirtEnergies
                  real(c_double), value :: LowestFreq, alpha, TargetError
                  real(c_double), dimension(ldG, *), intent(out) :: G
                  integer(c_int64_t), intent(out) :: NVecs
                  real(c_double), intent(out) :: TraceError, ExactTrace
            end function

            integer(c_int) function rpa_b200_project_basis(handle, NQ, NVecs, nov, G, ldG, R, ldR, Rp, ldRp) &
                  bind(C, name="rpa_b200_project_basis")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: NQ, NVecs, nov, ldG, ldR, ldRp
                  real(c_double), dimension(*), intent(in) :: G, R
                  real(c_double), dimension(ldRp, *), intent(out) :: Rp
            end function

            ! one frequency grid for all subsystems of an MBE cluster (set 1 = the whole complex)
            integer(c_int) function rpa_b200_freq_grid_mbe(NSets, NOcc, NVirt, OrbEnergies, CoreOrbThresh, &
                  LimitDai, TargetError, TargetRelError, NFixed, Freqs, FreqWeights, NFreqs) &
                  bind(C, name="rpa_b200_freq_grid_mbe")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  integer(c_int64_t), value :: NSets, LimitDai, NFixed
                  integer(c_int64_t), dimension(*), intent(in) :: NOcc, NVirt
                  type(c_ptr), dimension(*), intent(in) :: OrbEnergies   ! c_loc of each set's energies
                  real(c_double), value :: CoreOrbThresh, TargetError, TargetRelError
                  real(c_double), dimension(64), intent(out) :: Freqs, FreqWeights
                  integer(c_int64_t), intent(out) :: NFreqs
            end function

            ! interaction (NBody = 2) / nonadditive (3, 4) energies from subsystem energies in the
            ! sys_definitions order: replaces rpa_Eint2Body / rpa_EintNadd / rpa_EintNadd4Body
            integer(c_int) function rpa_b200_mbe_energy(NBody, E, Eint) bind(C, name="rpa_b200_mbe_energy")
                  import :: c_int, c_int64_t, c_double
                  integer(c_int64_t), value :: NBody
                  real(c_double), dimension(*), intent(in) :: E
                  real(c_double), intent(out) :: Eint
            end function

            ! FP64 log-det tile plans per bucket of 256 orders (Nb2 in 128/256/512, Tile in 64/128)
            integer(c_int) function rpa_b200_tune_logdet(handle, NQ, NMat, Nb2, Tile, Ms) &
                  bind(C, name="rpa_b200_tune_logdet")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: NQ, NMat
                  integer(c_int64_t), intent(out) :: Nb2, Tile
                  real(c_double), dimension(6), intent(out) :: Ms
            end function

            integer(c_int) function rpa_b200_set_logdet_plan(handle, NQ, Nb2, Tile) &
                  bind(C, name="rpa_b200_set_logdet_plan")
                  import :: c_int, c_int64_t, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: NQ, Nb2, Tile
            end function

            integer(c_int) function rpa_b200_get_logdet_plan(handle, NQ, Nb2, Tile) &
                  bind(C, name="rpa_b200_get_logdet_plan")
                  import :: c_int, c_int64_t, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: NQ
                  integer(c_int64_t), intent(out) :: Nb2, Tile
            end function

            integer(c_int) function rpa_b200_set_autotune(handle, on) bind(C, name="rpa_b200_set_autotune")
                  import :: c_int, c_int64_t, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: on
            end function

            ! Energies of many subsystems in one call (the subsystem loop of rpa_PostSCF);
            ! Eu: c_null_ptr or c_loc of sum(NFreqs) values, the E(u) of all instances in order
            integer(c_int) function rpa_b200_ec_batched(h, ninst, inst, prec, Ec, Eu) &
                  bind(C, name="rpa_b200_ec_batched")
                  import :: c_int, c_int64_t, c_double, c_ptr, rpa_instance
                  type(c_ptr), value :: h
                  integer(c_int64_t), value :: ninst, prec
                  type(rpa_instance), dimension(*), intent(in) :: inst
                  real(c_double), dimension(*), intent(out) :: Ec
                  type(c_ptr), value :: Eu
            end function

            ! Adjoint: dE_c/dR (NQ x nov, leading dimension lddR), dE_c/dOccEnergies, dE_c/dVirtEnergies;
            ! Ec, dOcc and dVirt may be c_null_ptr
            integer(c_int) function rpa_b200_ec_grad(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, &
                  NFreqs, Freqs, FreqWeights, alpha, prec, Ec, dR, lddR, dOcc, dVirt) bind(C, name="rpa_b200_ec_grad")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: h
                  integer(c_int64_t), value :: NQ, NOcc, NVirt, ldR, NFreqs, prec, lddR
                  real(c_double), dimension(ldR, *), intent(in) :: R
                  real(c_double), dimension(*), intent(in) :: OccEnergies, VirtEnergies, Freqs, FreqWeights
                  real(c_double), value :: alpha
                  type(c_ptr), value :: Ec, dOcc, dVirt
                  real(c_double), dimension(lddR, *), intent(out) :: dR
            end function

            ! Energy from given Pi(u) without a handle or any device allocation (32 MiB fixed scratch)
            integer(c_int) function rpa_b200_ec_from_pi_noalloc(device, stream, NQ, NFreqs, PiU, ldPi, &
                  FreqWeights, Ec, Eu) bind(C, name="rpa_b200_ec_from_pi_noalloc")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  integer(c_int64_t), value :: device, NQ, NFreqs, ldPi
                  type(c_ptr), value :: stream
                  real(c_double), dimension(ldPi, NQ, *), intent(in) :: PiU
                  real(c_double), dimension(*), intent(in) :: FreqWeights
                  real(c_double), intent(out) :: Ec
                  type(c_ptr), value :: Eu
            end function

            type(c_ptr) function rpa_b200_status_string(status) bind(C, name="rpa_b200_status_string")
                  import :: c_int, c_ptr
                  integer(c_int), value :: status
            end function

            ! out(1:min(n,6)) = staging, Pi build, log-det, other, tensor-core contraction, split pass (ms)
            integer(c_int) function rpa_b200_last_timings(handle, out, n) bind(C, name="rpa_b200_last_timings")
                  import :: c_int, c_int64_t, c_double, c_ptr
                  type(c_ptr), value :: handle
                  real(c_double), dimension(*), intent(out) :: out
                  integer(c_int64_t), value :: n
            end function

            integer(c_int64_t) function rpa_b200_last_launches(handle) bind(C, name="rpa_b200_last_launches")
                  import :: c_int64_t, c_ptr
                  type(c_ptr), value :: handle
            end function

            ! stream: a cudaStream_t of the handle's device, or c_null_ptr for the handle's own stream
            integer(c_int) function rpa_b200_set_stream(handle, stream) bind(C, name="rpa_b200_set_stream")
                  import :: c_int, c_ptr
                  type(c_ptr), value :: handle, stream
            end function
            ! ---- device-memory cap and failure-detection self-test (no reference counterparts)
            integer(c_int) function rpa_b200_set_workspace_limit(handle, Bytes) &
                  bind(C, name="rpa_b200_set_workspace_limit")
                  import :: c_int, c_int64_t, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), value :: Bytes        ! 0: no cap
            end function
            integer(c_int) function rpa_b200_workspace_bytes(handle, Used, Limit) &
                  bind(C, name="rpa_b200_workspace_bytes")
                  import :: c_int, c_int64_t, c_ptr
                  type(c_ptr), value :: handle
                  integer(c_int64_t), intent(out) :: Used, Limit
            end function
            integer(c_int) function rpa_b200_selftest_wait_timeout(handle, LimitMs) &
                  bind(C, name="rpa_b200_selftest_wait_timeout")
                  import :: c_int, c_double, c_ptr
                  type(c_ptr), value :: handle
                  real(c_double), value :: LimitMs          ! returns RPA_ERR_TIMEOUT when detection works
            end function
      end interface

contains

      subroutine rpa_b200_check(h, status)
            ! Map a non-zero status to the reference's error convention (msg + error stop).
            use display, only: msg, MSG_ERROR
            type(c_ptr), intent(in) :: h
            integer(c_int), intent(in) :: status
            character(kind=c_char), pointer :: s(:)
            integer :: n
            if (status /= RPA_OK) then
                  call c_f_pointer(rpa_b200_last_error(h), s, [512])
                  n = 0
                  do while (n < 512)
                        if (s(n+1) == c_null_char) exit
                        n = n + 1
                  end do
                  call msg("librpa_b200: " // transfer(s(1:n), repeat(" ", n)), MSG_ERROR)
                  error stop
            end if
      end subroutine rpa_b200_check
end module rpa_b200_iface
