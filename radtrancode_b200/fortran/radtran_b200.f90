! radtran_b200.f90 -- Fortran 2003 (ISO_C_BINDING) interface of the C ABI in
! include/radtran_b200.h, for the reference-side shims in this directory
! (cirsrtfg_wave_gpu.f, calc_phiret_gpu.f, newton_gpu.f).
!
! Not built here: no Fortran compiler is installed on this build host.  A
! maintainer compiles it with the reference's own flags, before the shims:
!     gfortran -c radtran_b200.f90
! and links libradtran_b200.so after the objects.
!
! Every derived type mirrors a C struct field for field (bind(C)); integers
! that the C functions take by value carry the `value` attribute.
module radtran_b200
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: RTB_OK = 0
  integer(c_int), parameter :: RTB_KTAB_BY_ID = -2

  ! rtb_atm: one cirsrtfg_wave call (the /LAYCOM/, /PATHCOM/, /LGRAD/ arrays
  ! by address, with their Fortran leading dimensions)
  type, bind(C) :: rtb_atm
     integer(c_int) :: nlayer, ngas, ncont, npath, npro, nv, nwave
     integer(c_int) :: ld_lay, ld_con, ld_v, ld_param
     type(c_ptr) :: press, temp, delh, pp, amount, cont, idgas, isogas, ktab
     type(c_ptr) :: nlayin, imod, layinc, scale, emtemp
     type(c_ptr) :: dte, dam, dco, dfp, xmap, vwave, xsec_ext
     integer(c_int) :: inormal, iray, itype, ispace, flagh2p, ilbl, inlte, iform
     real(c_float) :: tsurf, fwhm
     integer(c_int) :: nem
     type(c_ptr) :: vem, emissivity
     type(c_ptr) :: conv                          ! c_loc(an rtb_conv) or c_null_ptr
     type(c_ptr) :: hfp                           ! para-H2 fraction per layer (flagh2p = 1)
     real(c_float) :: radius1, radextra           ! km, iform = 3 (total flux of the planet)
     real(c_float) :: nlte_k1, nlte_A             ! calc_nlte_t, inlte = 1
     real(c_float) :: dist                        ! AU, cirsrtfg_wave's DIST (iform = 4)
     integer(c_int) :: ih2o, ich4, inh3, io3, iuvscat   ! /GASCONDEF/ switches of ngascon
  end type

  type, bind(C) :: rtb_conv
     integer(c_int) :: nconv
     type(c_ptr) :: vconv
     integer(c_int) :: nfwhm
     type(c_ptr) :: vfwhm, xfwhm
     integer(c_int) :: nfil
     type(c_ptr) :: vcen, nsub, vfil, fil
  end type

  interface
     integer(c_int) function rtb_create(device, ctx) bind(C, name="rtb_create")
       import
       integer(c_int), value :: device
       type(c_ptr) :: ctx
     end function
     type(c_ptr) function rtb_last_error(ctx) bind(C, name="rtb_last_error")
       import
       type(c_ptr), value :: ctx
     end function
     integer(c_int) function rtb_load_ktables(ctx, ntab, paths, idgas, isogas) bind(C, name="rtb_load_ktables")
       import
       type(c_ptr), value :: ctx
       integer(c_int), value :: ntab
       type(c_ptr) :: paths(*)                    ! NUL-terminated file names
       integer(c_int) :: idgas(*), isogas(*)
     end function
     integer(c_int) function rtb_load_cia(ctx, path, dnu) bind(C, name="rtb_load_cia")
       import
       type(c_ptr), value :: ctx
       character(kind=c_char) :: path(*)
       real(c_float), value :: dnu
     end function
     integer(c_int) function rtb_load_para_cia(ctx, path, dnu2, ipara) bind(C, name="rtb_load_para_cia")
       import
       type(c_ptr), value :: ctx
       character(kind=c_char) :: path(*)
       real(c_float), value :: dnu2
       integer(c_int), value :: ipara
     end function
     integer(c_int) function rtb_cirsrtfg_wave(ctx, atm, calcout, gradients, gradtsurf) &
          bind(C, name="rtb_cirsrtfg_wave")
       import
       type(c_ptr), value :: ctx
       type(rtb_atm) :: atm
       real(c_float) :: calcout(*), gradients(*), gradtsurf(*)
     end function
     integer(c_int) function rtb_calc_phiret_batch(ctx, nret, nx, ny, y, yn, sei, xn, xa, sai, phi, chisq) &
          bind(C, name="rtb_calc_phiret_batch")
       import
       type(c_ptr), value :: ctx
       integer(c_int), value :: nret, nx, ny
       real(c_float) :: y(*), yn(*), xn(*), xa(*), phi(*), chisq(*)
       real(c_double) :: sei(*), sai(*)
     end function
     integer(c_int) function rtb_calc_gain_matrix(ctx, nx, ny, ldx, ldy, kk, sxi, sei, dd, aa, nonpd) &
          bind(C, name="rtb_calc_gain_matrix")
       import
       type(c_ptr), value :: ctx
       integer(c_int), value :: nx, ny, ldx, ldy
       real(c_float) :: kk(*)
       real(c_double) :: sxi(*), sei(*), dd(*), aa(*)
       integer(c_int) :: nonpd
     end function
     integer(c_int) function rtb_calcnextxn(ctx, nx, ny, ldx, x0, xn, y, yn, dd, aa, x_out) &
          bind(C, name="rtb_calcnextxn")
       import
       type(c_ptr), value :: ctx
       integer(c_int), value :: nx, ny, ldx
       real(c_float) :: x0(*), xn(*), y(*), yn(*), x_out(*)
       real(c_double) :: dd(*), aa(*)
     end function
     integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
       import
       type(c_ptr), value :: s
     end function
  end interface

  type(c_ptr), save :: ctx = c_null_ptr

contains

  ! the context on device 0, created at the first call
  subroutine rtb_context_open()
    integer(c_int) :: st
    if (.not. c_associated(ctx)) then
       st = rtb_create(0_c_int, ctx)
       call rtb_check(st, 'rtb_create')
    end if
  end subroutine

  ! a non-zero status is the reference's STOP, with the library's message
  subroutine rtb_check(st, where)
    integer(c_int), intent(in) :: st
    character(*), intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    type(c_ptr) :: p
    integer :: n
    if (st == RTB_OK) return
    p = rtb_last_error(ctx)
    if (c_associated(p)) then
       n = int(c_strlen(p))
       call c_f_pointer(p, msg, [n])
       print *, where, ' (B200): status ', st, ': ', msg(1:n)
    else
       print *, where, ' (B200): status ', st
    end if
    stop
  end subroutine

  ! a blank-padded Fortran name as a NUL-terminated C string
  function c_name(name) result(s)
    character(*), intent(in) :: name
    character(kind=c_char, len=len_trim(name) + 1) :: s
    s = trim(name) // c_null_char
  end function
end module
