! specsim3d_gpu.f90 -- ISO_C_BINDING interface to libspecsim3d_gpu.so for the
! Fortran driver of SPECSIM3D (src/specsim3d.f90).
!
! The C declarations are in include/specsim3d_gpu.h.  Each interface below
! keeps the C argument order; arrays are passed by reference with the Fortran
! layout the library expects (res(nx,ny,nz,nreal) is C [nreal][nz][ny][nx]).
! Handles are type(c_ptr).  Every function returns 0 on success; the message of
! a failure comes from ss3d_message().
!
! Build (where a Fortran compiler exists):
!   gfortran -O3 -c specsim3d_gpu.f90
!   gfortran -O3 specsim3d_driver.f90 specsim3d_gpu.o -L../lib -lspecsim3d_gpu -Wl,-rpath,'$ORIGIN/../lib'
module specsim3d_gpu
  use, intrinsic :: iso_c_binding
  implicit none
  private

  integer(c_int), parameter, public :: SS3D_OK = 0, SS3D_EINVAL = 1, SS3D_ECUDA = 2, SS3D_ENOMEM = 3, &
                                       SS3D_ETOOLARGE = 4, SS3D_ENODATA = 5
  integer(c_int), parameter, public :: SS3D_FP64 = 0, SS3D_FP32 = 1
  integer(c_int), parameter, public :: SS3D_OUT_F32 = 0, SS3D_OUT_F64 = 1

  ! type(structure) of f90:95-100 without the derived rot/axes (computed inside)
  type, bind(c), public :: ss3d_struct
    integer(c_int) :: itype
    real(c_double) :: sill, ahmax, ahmin, avert, azimuth, dip, plunge
  end type

  type, bind(c), public :: ss3d_spec_stats
    integer(c_int) :: np(3)
    real(c_double) :: c0, maximag, maxreal, spos, sneg
  end type

  ! conditioning block of the parameter file, f90:740-750
  type, bind(c), public :: ss3d_cond_params
    integer(c_int) :: ixc, iyc, izc, ivc, iwc
    real(c_double) :: tmin, tmax
    integer(c_int) :: itrans
    real(c_double) :: skmean, zmin, zmax
    integer(c_int) :: ltail
    real(c_double) :: ltpar
    integer(c_int) :: utail
    real(c_double) :: utpar
    real(c_double) :: radius(3), angles(3)
    integer(c_int) :: ndmax
  end type

  type, bind(c), public :: ss3d_cond_stats
    integer(c_int) :: nd, nmerged, nout
    integer(c_int) :: nsb(3)
    integer(c_int64_t) :: nsum
    integer(c_int) :: nfail, nnone, nexact
    real(c_double) :: data_mean, data_var
  end type

  public :: ss3d_grid_size, ss3d_spectrum_create, ss3d_spectrum_free, ss3d_realize, ss3d_vario, &
            ss3d_condition, ss3d_set_stream, ss3d_message

  interface
    ! ipad rule, f90:1234-1253
    integer(c_int) function ss3d_grid_size(st, nst, d, n, ipad, np) bind(c, name="ss3d_grid_size")
      import :: c_int, c_double, ss3d_struct
      type(ss3d_struct), intent(in) :: st(*)
      integer(c_int), value :: nst
      real(c_double), intent(in) :: d(3)
      integer(c_int), intent(in) :: n(3)
      integer(c_int), value :: ipad
      integer(c_int), intent(out) :: np(3)
    end function

    ! covariance grid, forward FFT, S/N, amp (f90:1256-1292), resident on the GPU
    integer(c_int) function ss3d_spectrum_create(st, nst, nugget, d, n, ipad, sp, stats) &
        bind(c, name="ss3d_spectrum_create")
      import :: c_int, c_double, c_ptr, ss3d_struct, ss3d_spec_stats
      type(ss3d_struct), intent(in) :: st(*)
      integer(c_int), value :: nst
      real(c_double), value :: nugget
      real(c_double), intent(in) :: d(3)
      integer(c_int), intent(in) :: n(3)
      integer(c_int), value :: ipad
      type(c_ptr), intent(out) :: sp
      type(ss3d_spec_stats), intent(out) :: stats
    end function

    subroutine ss3d_spectrum_free(sp) bind(c, name="ss3d_spectrum_free")
      import :: c_ptr
      type(c_ptr), value :: sp
    end subroutine

    ! realizations r_first+1 .. r_first+nreal (f90:1302-1345); out is res(nx,ny,nz,nreal)
    ! of real(c_double) (out_dtype SS3D_OUT_F64) or real(c_float) (SS3D_OUT_F32);
    ! zstats(3,nreal): mean, variance, max|Im| per realization (f90:1343-1344)
    integer(c_int) function ss3d_realize(sp, iseed, r_first, nreal, igauss, precision, out, out_dtype, zstats) &
        bind(c, name="ss3d_realize")
      import :: c_int, c_int64_t, c_ptr, c_double
      type(c_ptr), value :: sp
      integer(c_int), value :: iseed
      integer(c_int64_t), value :: r_first
      integer(c_int), value :: nreal, igauss, precision
      type(c_ptr), value :: out
      integer(c_int), value :: out_dtype
      real(c_double), intent(out) :: zstats(*)
    end function

    ! experimental variograms (f90:394-480): gam(nlagmax, ndir, nreal), npairs(nlagmax, ndir)
    integer(c_int) function ss3d_vario(res, n, nreal, ndir, sx, sy, sz, nlag, gam, npairs) bind(c, name="ss3d_vario")
      import :: c_int, c_int64_t, c_double
      real(c_double), intent(in) :: res(*)
      integer(c_int), intent(in) :: n(3)
      integer(c_int), value :: nreal, ndir
      integer(c_int), intent(in) :: sx(*), sy(*), sz(*), nlag(*)
      real(c_double), intent(out) :: gam(*)
      integer(c_int64_t), intent(out) :: npairs(*)
    end function

    ! conditioning by kriging of the residual (f90:700-1081), res modified in place;
    ! rows(nvar, nrows) are the numeric rows of the GSLIB data file
    integer(c_int) function ss3d_condition(res, n, nreal, xmin, d, st, nst, nugget, cp, rows, nrows, nvar, &
                                           precision, cs, vrt, gtt, dxs, dys, dzs, dval, dg) &
        bind(c, name="ss3d_condition")
      import :: c_int, c_double, c_ptr, ss3d_struct, ss3d_cond_params, ss3d_cond_stats
      real(c_double), intent(inout) :: res(*)
      integer(c_int), intent(in) :: n(3)
      integer(c_int), value :: nreal
      real(c_double), intent(in) :: xmin(3), d(3)
      type(ss3d_struct), intent(in) :: st(*)
      integer(c_int), value :: nst
      real(c_double), value :: nugget
      type(ss3d_cond_params), intent(in) :: cp
      real(c_double), intent(in) :: rows(*)
      integer(c_int), value :: nrows, nvar, precision
      type(ss3d_cond_stats), intent(out) :: cs
      type(c_ptr), value :: vrt, gtt, dxs, dys, dzs, dval, dg
    end function

    integer(c_int) function ss3d_set_stream(stream) bind(c, name="ss3d_set_stream")
      import :: c_int, c_ptr
      type(c_ptr), value :: stream
    end function

    type(c_ptr) function ss3d_last_error_c() bind(c, name="ss3d_last_error")
      import :: c_ptr
    end function

    integer(c_size_t) function c_strlen(s) bind(c, name="strlen")
      import :: c_size_t, c_ptr
      type(c_ptr), value :: s
    end function
  end interface

contains

  ! message of the last failing call on this thread, as a Fortran string
  function ss3d_message() result(msg)
    character(len=:), allocatable :: msg
    type(c_ptr) :: p
    character(kind=c_char), pointer :: chars(:)
    integer :: i, nlen
    p = ss3d_last_error_c()
    nlen = int(c_strlen(p))
    call c_f_pointer(p, chars, [nlen])
    allocate(character(len=nlen) :: msg)
    do i = 1, nlen
      msg(i:i) = chars(i)
    end do
  end function

end module specsim3d_gpu
