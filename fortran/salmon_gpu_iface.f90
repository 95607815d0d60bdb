!
! salmon_gpu_iface.f90 -- ISO_C_BINDING interface to libsalmon_b200.so
! (include/salmon_gpu.h) for SALMON's ARTED code.
!
! A maintainer adds this module to src/ARTED/modules/ and calls the wrappers in
! place of the routines named beside them (paths relative to the SALMON tree).
! It is not compiled in this repository (no Fortran compiler here); the same
! entry points are exercised from C/Python with Fortran-ordered arrays by the
! tests.
!
module salmon_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: SGPU_PREC_C128 = 0, SGPU_PREC_C64 = 1

  type, bind(C) :: sgpu_desc
    integer(c_int32_t) :: NLx, NLy, NLz
    real(c_double)     :: Hx, Hy, Hz
    real(c_double)     :: aLx, aLy, aLz
    integer(c_int32_t) :: NK, NK_s, NK_e, NB, NBoccmax
    real(c_double)     :: lapx(0:4), lapy(0:4), lapz(0:4)
    real(c_double)     :: nabx(0:4), naby(0:4), nabz(0:4)
    integer(c_int32_t) :: NI, Nps, Nlma
    type(c_ptr)        :: Mps, Jxyz, Jxx, Jyy, Jzz, uV, iuV, a_tbl, occ
  end type

  type(c_ptr), save :: sgpu_h = c_null_ptr

  interface
    integer(c_int) function sgpu_create(desc, precision, h) bind(C, name="sgpu_create")
      import :: c_int, c_ptr, sgpu_desc
      type(sgpu_desc), intent(in)    :: desc
      integer(c_int), value          :: precision
      type(c_ptr), intent(out)       :: h
    end function
    integer(c_int) function sgpu_destroy(h) bind(C, name="sgpu_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    type(c_ptr) function sgpu_last_error() bind(C, name="sgpu_last_error")
      import :: c_ptr
    end function
    integer(c_int) function sgpu_set_state(h, zu) bind(C, name="sgpu_set_state")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: h
      complex(c_double_complex), intent(in) :: zu(*)
    end function
    integer(c_int) function sgpu_get_state(h, zu) bind(C, name="sgpu_get_state")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: h
      complex(c_double_complex), intent(out) :: zu(*)
    end function
    integer(c_int) function sgpu_set_vloc(h, vloc) bind(C, name="sgpu_set_vloc")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: vloc(*)
    end function
    integer(c_int) function sgpu_update_projector(h, kac) bind(C, name="sgpu_update_projector")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: kac(*)
    end function
    integer(c_int) function sgpu_hamiltonian(h, dt, flag_current) bind(C, name="sgpu_hamiltonian")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: dt
      integer(c_int), value :: flag_current
    end function
    integer(c_int) function sgpu_hpsi(h, ik, tpsi, htpsi, ttpsi) bind(C, name="sgpu_hpsi")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: h
      integer(c_int), value :: ik
      complex(c_double_complex), intent(in)  :: tpsi(*)
      complex(c_double_complex), intent(out) :: htpsi(*)
      type(c_ptr), value :: ttpsi            ! c_loc(ttpsi) or c_null_ptr
    end function
    integer(c_int) function sgpu_psi_rho(h, rho_l) bind(C, name="sgpu_psi_rho")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: rho_l(*)
    end function
    integer(c_int) function sgpu_current(h, kac, jav) bind(C, name="sgpu_current")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in)  :: kac(*)
      real(c_double), intent(out) :: jav(3)
    end function
    integer(c_int) function sgpu_energy_terms(h, kac, ekin, enl) bind(C, name="sgpu_energy_terms")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in)  :: kac(*)
      real(c_double), intent(out) :: ekin, enl
    end function
    ! ---- precision, device state, streams
    integer(c_int) function sgpu_set_precision(h, precision) bind(C, name="sgpu_set_precision")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: precision
    end function
    integer(c_int) function sgpu_synchronize(h) bind(C, name="sgpu_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    type(c_ptr) function sgpu_stream(h) bind(C, name="sgpu_stream")
      import :: c_ptr
      type(c_ptr), value :: h
    end function
    type(c_ptr) function sgpu_state_ptr(h) bind(C, name="sgpu_state_ptr")
      import :: c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function sgpu_set_state_dev(h, zu_dev) bind(C, name="sgpu_set_state_dev")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, zu_dev      ! device address (OpenACC host_data use_device)
    end function
    integer(c_int) function sgpu_hpsi_batch(h, ikb_s, ikb_e, tpsi, htpsi) bind(C, name="sgpu_hpsi_batch")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: ikb_s, ikb_e
      type(c_ptr), value :: tpsi, htpsi    ! device addresses in the handle's precision
    end function
    ! ---- self-consistent local potential (RT/dt_evolve.f90:190-207)
    integer(c_int) function sgpu_set_vpsl(h, vpsl) bind(C, name="sgpu_set_vpsl")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: vpsl(*)
    end function
    integer(c_int) function sgpu_update_vloc(h, rho, eh_exc) bind(C, name="sgpu_update_vloc")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      type(c_ptr), value :: rho            ! c_loc(rho) after the allreduce, or c_null_ptr
      type(c_ptr), value :: eh_exc         ! c_loc(e(2)) for (Eh, Exc), or c_null_ptr
    end function
    integer(c_int) function sgpu_get_vloc(h, vloc) bind(C, name="sgpu_get_vloc")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: vloc(*)
    end function
    ! ---- ground state (GS/*), FP64
    integer(c_int) function sgpu_gs_set_state(h, zu_gs) bind(C, name="sgpu_gs_set_state")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: h
      complex(c_double_complex), intent(in) :: zu_gs(*)
    end function
    integer(c_int) function sgpu_gs_get_state(h, zu_gs) bind(C, name="sgpu_gs_get_state")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: h
      complex(c_double_complex), intent(out) :: zu_gs(*)
    end function
    integer(c_int) function sgpu_gram_schmidt(h) bind(C, name="sgpu_gram_schmidt")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function sgpu_cg(h, ncg, esp_var, iters) bind(C, name="sgpu_cg")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: ncg
      type(c_ptr), value :: esp_var, iters ! c_loc(esp_var(NB,NK_s:NK_e)) / c_loc(iters) or c_null_ptr
    end function
    integer(c_int) function sgpu_set_cg_delta(h, delta_cg) bind(C, name="sgpu_set_cg_delta")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: delta_cg
    end function
    integer(c_int) function sgpu_cg_residuals(h, res) bind(C, name="sgpu_cg_residuals")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: res(*)
    end function
    integer(c_int) function sgpu_subspace_diag(h, esp) bind(C, name="sgpu_subspace_diag")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: esp(*)
    end function
    integer(c_int) function sgpu_gs_to_rt(h) bind(C, name="sgpu_gs_to_rt")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    ! ---- tuning and timing
    integer(c_int) function sgpu_set_param(h, param, val) bind(C, name="sgpu_set_param")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: param, val
    end function
    integer(c_int) function sgpu_get_param(h, param, val) bind(C, name="sgpu_get_param")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: param
      integer(c_int), intent(out) :: val
    end function
    integer(c_int) function sgpu_autotune(h, reps, nslab, split, ms_per_apply) bind(C, name="sgpu_autotune")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: reps
      integer(c_int), intent(out) :: nslab, split
      real(c_double), intent(out) :: ms_per_apply
    end function
    integer(c_int) function sgpu_time_kernel(h, kernel, reps, ms) bind(C, name="sgpu_time_kernel")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: kernel, reps
      real(c_double), intent(out) :: ms
    end function
    ! ---- several systems in one CUDA-graph replay
    ! occ: pass occ(1,NK_s) with ld_occ = NB; zu, occ and rho are device
    ! addresses (inside !$acc host_data use_device(zu_t, occ, rho))
    integer(c_int) function sgpu_psi_rho_static(precision, NL, nb, nk, zu, occ, ld_occ, rho, stream) &
        bind(C, name="sgpu_psi_rho_static")
      import :: c_int, c_ptr
      integer(c_int), value :: precision, NL, nb, nk, ld_occ
      type(c_ptr), value    :: zu, occ, rho, stream
    end function
    integer(c_int) function sgpu_vloc_history_reset(h) bind(C, name="sgpu_vloc_history_reset")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function sgpu_vloc_extrapolate(h) bind(C, name="sgpu_vloc_extrapolate")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function sgpu_check_desc(desc) bind(C, name="sgpu_check_desc")
      import :: c_int, sgpu_desc
      type(sgpu_desc), intent(in) :: desc
    end function
    ! device outputs for an allreduce on the device (psi_rho.f90:88, current.f90:286)
    integer(c_int) function sgpu_psi_rho_dev(h, rho_dev) bind(C, name="sgpu_psi_rho_dev")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, rho_dev
    end function
    integer(c_int) function sgpu_current_dev(h, kac, jav_dev) bind(C, name="sgpu_current_dev")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h, jav_dev
      real(c_double), intent(in) :: kac(*)
    end function
    integer(c_int) function sgpu_update_vloc_dev(h, rho_dev, eh_exc_dev) bind(C, name="sgpu_update_vloc_dev")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, rho_dev, eh_exc_dev
    end function
    integer(c_int) function sgpu_autotune_step(h, dt, reps, params, ms) bind(C, name="sgpu_autotune_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: dt
      integer(c_int), value :: reps
      integer(c_int), intent(out) :: params(6)
      real(c_double), intent(out) :: ms
    end function
    integer(c_int) function sgpu_batch_create(handles, n, b) bind(C, name="sgpu_batch_create")
      import :: c_int, c_ptr
      type(c_ptr), intent(in) :: handles(*)
      integer(c_int), value :: n
      type(c_ptr), intent(out) :: b
    end function
    integer(c_int) function sgpu_batch_step(b, dt, nsteps) bind(C, name="sgpu_batch_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: b
      real(c_double), intent(in) :: dt(*)
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function sgpu_batch_destroy(b) bind(C, name="sgpu_batch_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: b
    end function
  end interface

contains

  ! err_finalize on any non-zero status (ARTED/main.f90:21-33)
  subroutine sgpu_check(rc, what)
    integer(c_int), intent(in) :: rc
    character(*), intent(in)   :: what
    character(kind=c_char), pointer :: msg(:)
    character(len=512) :: text
    integer :: i
    if (rc == 0) return
    call c_f_pointer(sgpu_last_error(), msg, [512])
    text = ' '
    do i = 1, 512
      if (msg(i) == c_null_char) exit
      text(i:i) = msg(i)
    end do
    call err_finalize(what // ': ' // trim(text))
  end subroutine

  ! Call once after opt_vars_initialize_p2 and prep_ps_periodic
  ! (control/initialization.f90), before the RT loop.
  subroutine sgpu_init_from_globals(precision)
    use global_variables
    integer, intent(in) :: precision
    type(sgpu_desc), target :: d
    d%NLx = NLx; d%NLy = NLy; d%NLz = NLz
    d%Hx = Hx; d%Hy = Hy; d%Hz = Hz
    d%aLx = aLx; d%aLy = aLy; d%aLz = aLz
    d%NK = NK; d%NK_s = NK_s; d%NK_e = NK_e; d%NB = NB; d%NBoccmax = NBoccmax
    d%lapx = lapx(0:4); d%lapy = lapy(0:4); d%lapz = lapz(0:4)
    d%nabx = nabx(0:4); d%naby = naby(0:4); d%nabz = nabz(0:4)
    d%NI = NI; d%Nps = Nps; d%Nlma = Nlma
    d%Mps = c_loc(Mps); d%Jxyz = c_loc(Jxyz)
    d%Jxx = c_loc(Jxx); d%Jyy = c_loc(Jyy); d%Jzz = c_loc(Jzz)
    d%uV = c_loc(uV); d%iuV = c_loc(iuV); d%a_tbl = c_loc(a_tbl); d%occ = c_loc(occ)
    call sgpu_check(sgpu_create(d, int(precision, c_int), sgpu_h), 'sgpu_create')
    call sgpu_check(sgpu_set_state(sgpu_h, zu_t), 'sgpu_set_state')   ! !$acc enter data copyin(zu_t)
  end subroutine

  ! The ground-state sequence of one SCF iteration (control/ground_state.f90:135-139) on the
  ! device copy of zu_GS: Gram_Schmidt, diag_omp, Gram_Schmidt, CG_omp(Ncg), Gram_Schmidt.
  ! Load zu_GS once with sgpu_gs_set_state; esp and esp_var come back FP64.
  subroutine gpu_gs_iteration(ncg_in, esp_out, esp_var_out)
    use global_variables, only: NB, NK_s, NK_e
    integer, intent(in) :: ncg_in
    real(8), intent(out), target :: esp_out(NB, NK_s:NK_e), esp_var_out(NB, NK_s:NK_e)
    call sgpu_check(sgpu_gram_schmidt(sgpu_h), 'sgpu_gram_schmidt')
    call sgpu_check(sgpu_subspace_diag(sgpu_h, esp_out), 'sgpu_subspace_diag')
    call sgpu_check(sgpu_gram_schmidt(sgpu_h), 'sgpu_gram_schmidt')
    call sgpu_check(sgpu_cg(sgpu_h, int(ncg_in, c_int), c_loc(esp_var_out), c_null_ptr), 'sgpu_cg')
    call sgpu_check(sgpu_gram_schmidt(sgpu_h), 'sgpu_gram_schmidt')
  end subroutine

  ! Drop-in for psi_rho_RT + Hartree + Exc_Cor + Vloc = Vh + Vpsl + Vexc after the step
  ! (RT/dt_evolve.f90:190-207), on the device; rho after comm_summation is passed in.
  subroutine gpu_update_vloc(rho_in)
    real(8), intent(in), target :: rho_in(:)
    call sgpu_check(sgpu_update_vloc(sgpu_h, c_loc(rho_in), c_null_ptr), 'sgpu_update_vloc')
  end subroutine

  ! Drop-in for update_projector(kac) (common/projector.f90:29)
  subroutine gpu_update_projector(kac_in)
    use global_variables, only: NK
    real(8), intent(in) :: kac_in(NK,3)
    call sgpu_check(sgpu_update_projector(sgpu_h, kac_in), 'sgpu_update_projector')
  end subroutine

  ! Drop-in for hamiltonian(zu,flag_current) (RT/hamiltonian.f90:27); zu stays on the device
  subroutine gpu_hamiltonian(flag_current)
    use global_variables, only: dt, Vloc
    logical, intent(in) :: flag_current
    call sgpu_check(sgpu_set_vloc(sgpu_h, Vloc), 'sgpu_set_vloc')
    call sgpu_check(sgpu_hamiltonian(sgpu_h, dt, merge(1_c_int, 0_c_int, flag_current)), 'sgpu_hamiltonian')
  end subroutine

  ! Drop-in for psi_rho_RT(zu) (common/psi_rho.f90:40): rho_l, then the same comm_summation
  subroutine gpu_psi_rho_RT
    use global_variables, only: rho_l, rho, NL
    use salmon_parallel, only: nproc_group_tdks
    use salmon_communication, only: comm_summation
    call sgpu_check(sgpu_psi_rho(sgpu_h, rho_l), 'sgpu_psi_rho')
    call comm_summation(rho_l, rho, NL, nproc_group_tdks)
  end subroutine

  ! Drop-in for current_RT (RT/current.f90:65)
  subroutine gpu_current_RT
    use global_variables, only: kAc, jav
    use salmon_parallel, only: nproc_group_tdks
    use salmon_communication, only: comm_summation
    real(8) :: jav_l(3)
    call sgpu_check(sgpu_current(sgpu_h, kAc, jav_l), 'sgpu_current')
    call comm_summation(jav_l, jav, 3, nproc_group_tdks)
  end subroutine

  ! Drop-in for the `update self(zu_t)` points (control_sc.f90:215,395,414)
  subroutine gpu_sync_to_host
    use global_variables, only: zu_t
    call sgpu_check(sgpu_get_state(sgpu_h, zu_t), 'sgpu_get_state')
  end subroutine
end module salmon_gpu
