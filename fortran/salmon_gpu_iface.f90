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
