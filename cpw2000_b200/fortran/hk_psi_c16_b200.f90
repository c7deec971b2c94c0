!  hk_psi_c16 with the argument list of Src/hk_psi/reference/hk_psi_c16.f90:28-32,
!  forwarding to the B200 library through iso_c_binding.
!
!  Use it in place of Src/hk_psi/reference/hk_psi_c16.f90 when the Fortran side
!  should keep its own symbol (for example to add tracing); the library also
!  exports the gfortran-mangled hk_psi_c16_ directly, which needs no Fortran.
!  On a non-zero status it prints the library's message and stops, as the
!  reference does on its own errors.

subroutine hk_psi_c16(mtxd, neig, psi, hpsi, lnewanl,                    &
    ng, kgv,                                                             &
    ekpg, isort, vscr, kmscr,                                            &
    anlga, xnlkb, nanl,                                                  &
    mxddim, mxdbnd, mxdanl, mxdgve, mxdscr)

  use, intrinsic :: iso_c_binding, only : c_int, c_double, c_double_complex, c_ptr, c_char, c_null_char, &
                                          c_f_pointer
  implicit none

  integer, parameter          :: REAL64 = selected_real_kind(12)

  integer, intent(in)                ::  mxddim, mxdbnd, mxdanl, mxdgve, mxdscr
  integer, intent(in)                ::  mtxd, neig
  real(REAL64), intent(in)           ::  ekpg(mxddim)
  integer, intent(in)                ::  isort(mxddim)
  real(REAL64), intent(in)           ::  vscr(mxdscr)
  integer, intent(in)                ::  kmscr(7)
  integer, intent(in)                ::  ng
  integer, intent(in)                ::  kgv(3,mxdgve)
  integer, intent(in)                ::  nanl
  complex(REAL64), intent(in)        ::  anlga(mxddim,mxdanl)
  real(REAL64), intent(in)           ::  xnlkb(mxdanl)
  complex(REAL64), intent(in)        ::  psi(mxddim,mxdbnd)
  logical, intent(inout)             ::  lnewanl
  complex(REAL64), intent(out)       ::  hpsi(mxddim,mxdbnd)

  interface
    integer(c_int) function cpw_b200_hk_psi_c16(mtxd, neig, psi, hpsi, lnewanl, ng, kgv, ekpg, isort, &
        vscr, kmscr, anlga, xnlkb, nanl, mxddim, mxdbnd, mxdanl, mxdgve, mxdscr)                       &
        bind(C, name="cpw_b200_hk_psi_c16")
      import :: c_int, c_double, c_double_complex
      integer(c_int), intent(in) :: mtxd, neig, ng, nanl, mxddim, mxdbnd, mxdanl, mxdgve, mxdscr
      integer(c_int), intent(in) :: kgv(*), isort(*), kmscr(7)
      integer(c_int), intent(in) :: lnewanl
      real(c_double), intent(in) :: ekpg(*), vscr(*), xnlkb(*)
      complex(c_double_complex), intent(in) :: psi(*), anlga(*)
      complex(c_double_complex), intent(inout) :: hpsi(*)
    end function
    type(c_ptr) function cpw_b200_last_error() bind(C, name="cpw_b200_last_error")
      import :: c_ptr
    end function
  end interface

  integer(c_int) :: istat, lnew
  character(kind=c_char), pointer :: msg(:)
  integer :: i

  lnew = 0
  if(lnewanl) lnew = 1
  istat = cpw_b200_hk_psi_c16(mtxd, neig, psi, hpsi, lnew, ng, kgv, ekpg, isort,                 &
      vscr, kmscr, anlga, xnlkb, nanl, mxddim, mxdbnd, mxdanl, mxdgve, mxdscr)
!  lnewanl is never assigned: callers may pass a literal (Src/ALFA/berry_derivative.f90:229)

  if(istat /= 0) then
    call c_f_pointer(cpw_b200_last_error(), msg, [512])
    write(6,*)
    write(6,'("   STOPPED in hk_psi_c16 (B200 library), status ",i4)') istat
    do i = 1,512
      if(msg(i) == c_null_char) exit
      write(6,'(a)',advance='no') msg(i)
    enddo
    write(6,*)

    stop

  endif

  return

end subroutine hk_psi_c16
