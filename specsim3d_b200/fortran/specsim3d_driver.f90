! specsim3d_driver.f90 -- thin Fortran driver of the GPU library: the calling
! side of the ISO_C_BINDING module specsim3d_gpu (specsim3d_gpu.f90).
!
! It keeps the command line and parameter file of the reference program
! (src/specsim3d.f90:1111-1182) for the unconditional path:
!
!   specsim3d_driver file.par [--gauss] [--precision fp32] [--vario varfile]
!
!   [optional header lines up to one containing START OF PARAMETERS (<= 30)]
!   xmn ymn zmn
!   xsiz ysiz zsiz
!   nx ny nz
!   nugget nst
!   itype sill ahmax ahmin avert azimuth dip plunge      (nst lines)
!   iseed nreal ipad [igauss]
!   outbase
!
! and writes outbase.bin (raw float32 in the Fortran order res(nx,ny,nz,nreal),
! the reference's --bin output, f90:1357-1370) and, with --vario, the
! experimental variograms of every realization with their ensemble mean
! (columns dir, lag, npairs, gamma_mean).  All arithmetic runs in the library:
! spectrum (f90:1234-1292), realizations (f90:1302-1345), variograms
! (f90:394-480).  Conditioning, the other writers and the full stdout of the
! reference are left to the C++ drop-in (specsim3d_b200/bin/specsim3d).
!
! Build (where a Fortran compiler exists; none is installed in this image):
!   gfortran -O2 -c specsim3d_gpu.f90
!   gfortran -O2 specsim3d_driver.f90 specsim3d_gpu.o -L../lib -lspecsim3d_gpu -Wl,-rpath,'$ORIGIN/../lib'
program specsim3d_driver
  use, intrinsic :: iso_c_binding
  use specsim3d_gpu
  implicit none

  integer, parameter :: maxst = 10
  character(len=512) :: parfile, varfile, outbase, line
  character(len=64) :: arg
  logical :: want_vario, have_file
  integer :: narg, k, ios, ist, nst, ngauss_opt, precision
  integer(c_int) :: rc, ipad, igauss, iseed, nreal
  integer(c_int) :: n(3), np(3)
  real(c_double) :: origin(3), cell(3), nugget
  type(ss3d_struct) :: st(maxst)
  type(ss3d_spec_stats) :: sstats
  type(c_ptr) :: sp
  real(c_float), allocatable, target :: res32(:,:,:,:)
  real(c_double), allocatable, target :: res64(:,:,:,:)
  real(c_double), allocatable :: zst(:)

  ! ---- command line
  parfile = 'SPECSIM3D.PAR'
  varfile = ''
  want_vario = .false.
  ngauss_opt = 0
  precision = SS3D_FP64
  narg = command_argument_count()
  if (narg >= 1) call get_command_argument(1, parfile)
  k = 2
  do while (k <= narg)
    call get_command_argument(k, arg)
    if (trim(arg) == '--gauss') then
      ngauss_opt = 1
    else if (trim(arg) == '--precision') then
      k = k + 1
      if (k > narg) call fail('--precision needs fp32 or fp64')
      call get_command_argument(k, arg)
      if (trim(arg) == 'fp32') then
        precision = SS3D_FP32
      else if (trim(arg) /= 'fp64') then
        call fail('--precision needs fp32 or fp64')
      end if
    else if (trim(arg) == '--vario') then
      k = k + 1
      if (k > narg) call fail('--vario needs a variogram parameter file')
      call get_command_argument(k, varfile)
      want_vario = .true.
    else
      call fail('unknown option: '//trim(arg))
    end if
    k = k + 1
  end do

  ! ---- parameter file
  inquire(file=trim(parfile), exist=have_file)
  if (.not. have_file) call fail('Parameter file not found: '//trim(parfile))
  open(10, file=trim(parfile), status='old', action='read')
  call skip_header(10)
  read(10, *) origin
  read(10, *) cell
  read(10, *) n
  read(10, *) nugget, nst
  if (nst < 1 .or. nst > maxst) call fail('nstruct out of range')
  do ist = 1, nst
    read(10, *) st(ist)%itype, st(ist)%sill, st(ist)%ahmax, st(ist)%ahmin, st(ist)%avert, &
                st(ist)%azimuth, st(ist)%dip, st(ist)%plunge
    if (st(ist)%ahmax <= 0 .or. st(ist)%ahmin <= 0 .or. st(ist)%avert <= 0) call fail('ranges must be positive')
  end do
  read(10, '(a)') line
  igauss = ngauss_opt
  read(line, *, iostat=ios) iseed, nreal, ipad, k
  if (ios == 0) then
    if (k < 0 .or. k > 1) call fail('parameter file: igauss must be 0 or 1')
    if (k == 1) igauss = 1
  else
    read(line, *) iseed, nreal, ipad
  end if
  read(10, '(a)') outbase
  outbase = adjustl(outbase)
  close(10)

  ! ---- spectrum on the GPU (f90:1234-1292)
  rc = ss3d_grid_size(st, int(nst, c_int), cell, n, ipad, np)
  if (rc /= SS3D_OK) call fail(ss3d_message())
  rc = ss3d_spectrum_create(st, int(nst, c_int), nugget, cell, n, ipad, sp, sstats)
  if (rc /= SS3D_OK) call fail(ss3d_message())
  write(*, '(a,3i6)') ' periodic grid: ', sstats%np
  write(*, '(a,es15.7)') ' target variance C(0): ', sstats%c0
  write(*, '(a,es15.7)') ' sum of positive S:    ', sstats%spos

  ! ---- realizations (f90:1302-1345) and the .bin file (f90:1357-1370)
  allocate(zst(3 * nreal))
  allocate(res32(n(1), n(2), n(3), nreal))
  rc = ss3d_realize(sp, iseed, 0_c_int64_t, nreal, igauss, int(precision, c_int), c_loc(res32), SS3D_OUT_F32, zst)
  if (rc /= SS3D_OK) call fail(ss3d_message())
  do k = 1, nreal
    write(*, '(a,i6,a,2es15.7)') ' realization ', k, ': mean, variance ', zst(3 * k - 2), zst(3 * k - 1)
  end do
  open(11, file=trim(outbase)//'.bin', access='stream', form='unformatted', status='replace', action='write')
  write(11) res32
  close(11)

  ! ---- experimental variograms (f90:394-480) of the FP64 realizations
  if (want_vario) then
    allocate(res64(n(1), n(2), n(3), nreal))
    rc = ss3d_realize(sp, iseed, 0_c_int64_t, nreal, igauss, int(precision, c_int), c_loc(res64), SS3D_OUT_F64, zst)
    if (rc /= SS3D_OK) call fail(ss3d_message())
    call variograms(trim(varfile), trim(outbase)//'_vario_gpu.csv', res64, n, nreal)
  end if
  call ss3d_spectrum_free(sp)

contains

  subroutine fail(msg)
    character(len=*), intent(in) :: msg
    write(*, '(a)') ' '//trim(msg)
    stop 1
  end subroutine

  ! optional GSLIB header: lines up to one containing START OF PARAMETERS
  ! (any case), at most 30; without it the file is read from its first line
  subroutine skip_header(u)
    integer, intent(in) :: u
    character(len=512) :: h
    integer :: i, j, ios2
    do i = 1, 30
      read(u, '(a)', iostat=ios2) h
      if (ios2 /= 0) exit
      do j = 1, len_trim(h)
        if (h(j:j) >= 'a' .and. h(j:j) <= 'z') h(j:j) = achar(iachar(h(j:j)) - 32)
      end do
      if (index(h, 'START OF PARAMETERS') > 0) return
    end do
    rewind(u)
  end subroutine

  ! variogram file (f90:84-87): ndir iper / sx sy sz nlag per direction
  subroutine variograms(vfile, csvfile, res, nn, nr)
    character(len=*), intent(in) :: vfile, csvfile
    real(c_double), intent(in) :: res(*)
    integer(c_int), intent(in) :: nn(3), nr
    integer(c_int) :: ndir, iper, d, l, r, nlagmax, rc2
    integer(c_int), allocatable :: sx(:), sy(:), sz(:), nlag(:)
    real(c_double), allocatable :: gam(:,:,:)
    integer(c_int64_t), allocatable :: npairs(:,:)
    real(c_double) :: gm
    open(12, file=vfile, status='old', action='read')
    read(12, *) ndir, iper
    allocate(sx(ndir), sy(ndir), sz(ndir), nlag(ndir))
    do d = 1, ndir
      read(12, *) sx(d), sy(d), sz(d), nlag(d)
    end do
    close(12)
    nlagmax = maxval(nlag)
    allocate(gam(nlagmax, ndir, nr), npairs(nlagmax, ndir))
    rc2 = ss3d_vario(res, nn, nr, ndir, sx, sy, sz, nlag, gam, npairs)
    if (rc2 /= SS3D_OK) call fail(ss3d_message())
    open(13, file=csvfile, status='replace', action='write')
    write(13, '(a)') 'dir,lag,npairs,gamma_mean'
    do d = 1, ndir
      do l = 1, nlag(d)
        if (npairs(l, d) == 0) cycle
        gm = 0.0_c_double
        do r = 1, nr
          gm = gm + gam(l, d, r)
        end do
        gm = gm / real(nr, c_double)
        write(13, '(i0,",",i0,",",i0,",",es14.6)') d, l, npairs(l, d), gm
      end do
    end do
    close(13)
  end subroutine

end program specsim3d_driver
