! scarl.f90 -- Fortran 2003 ISO_C_BINDING interface to libscarl_b200 (the C ABI
! of include/scarl.h), for ScaRL-style Fortran hosts.  The argument order and
! array conventions follow the Fortran routines they replace: arrays are
! passed by reference in Fortran (column-major) order, scalars by value.
!
! Build:   gfortran -c scarl.f90
! Link:    ... -L<repo>/scarl_b200 -lscarl_b200 -lstdc++ -Wl,-rpath,<repo>/scarl_b200
module scarl_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: SCARL_OK = 0, SCARL_EINVAL = 1, SCARL_ENOMEM = 2, &
                               SCARL_EDEVICE = 3, SCARL_ETIMEOUT = 4, &
                               SCARL_EUNSUPPORTED = 5, SCARL_EIO = 6
  integer(c_int), parameter :: SCARL_FFT = 1, SCARL_FFT_MPI = 2
  integer(c_int), parameter :: SCARL_CM_GAUSSIAN = 1, SCARL_CM_VON_KARMAN = 2, &
                               SCARL_CM_EXPONENTIAL = 3
  integer(c_int), parameter :: SCARL_FOM_GAUSSIAN = 1, SCARL_FOM_LOGNORMAL = 2
  integer(c_int), parameter :: SCARL_F32 = 4, SCARL_F64 = 8
  ! OR'ed into SCARL_F32: pass 1's z DFT as split-BF16 tensor-core products
  integer(c_int), parameter :: SCARL_SPLIT_BF16 = 256
  integer(c_int), parameter :: SCARL_SPLIT_BF16_X = 512
  integer(c_int), parameter :: SCARL_GEN_DCT = 1, SCARL_GEN_SHINO = 2, SCARL_GEN_PADDED = 3
  integer(c_int), parameter :: SCARL_PAD_FULL = 0, SCARL_PAD_AUTO = 1, SCARL_PAD_LEARNED = 2, &
                               SCARL_PAD_SMOOTH = 3

  ! one deck entry (SRC_F/read_input.f90:257-299)
  type, bind(C) :: scarl_sample
    character(kind=c_char) :: name(256)
    real(c_double) :: xMinGlob(3), xMaxGlob(3), corrL(3), overlap(3)
    integer(c_int) :: pointsPerCorrL(3)
    integer(c_int) :: corrMod, margiFirst
    real(c_double) :: avg, std_dev
    integer(c_int) :: seedBase
    real(c_double) :: nu
  end type scarl_sample

  type, bind(C) :: scarl_layout
    integer(c_int) :: L(3), Np(3), Np_ovlp(3), topo_shape(3), nb_tiles
    real(c_double) :: xStep(3)
  end type scarl_layout

  type, bind(C) :: scarl_gen_opts
    integer(c_int) :: generator = SCARL_GEN_PADDED, dtype = SCARL_F64, nb_procs = 1
    integer(c_int) :: topo_shape(3) = 0, pad(3) = 0
    integer(c_int) :: pad_policy = SCARL_PAD_FULL
    real(c_double) :: pad_tol = 0d0
    integer(c_int) :: no_spectral_normalisation = 0, normalize_field = 0
    integer(c_int32_t) :: stream = 0
    integer(c_int) :: autotune = 0
    type(c_ptr) :: phiK = c_null_ptr
    integer(c_int) :: gen_meth = SCARL_FFT
    type(c_ptr) :: moments = c_null_ptr   ! c_loc of real(c_double) :: m(2), or c_null_ptr
  end type scarl_gen_opts

  interface
    integer(c_int) function scarl_ctx_create(device, budget_bytes, ctx) &
        bind(C, name="scarl_ctx_create")
      import :: c_int, c_size_t, c_ptr
      integer(c_int), value :: device
      integer(c_size_t), value :: budget_bytes
      type(c_ptr), intent(out) :: ctx
    end function

    integer(c_int) function scarl_ctx_destroy(ctx) bind(C, name="scarl_ctx_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    type(c_ptr) function scarl_last_error(ctx) bind(C, name="scarl_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function

    ! gen_std_gauss_FFT (SRC_F/fftw_ScaRL.f90:261): phiK / gammaK are c_loc of the
    ! (Np/2)^3 arrays or c_null_ptr
    integer(c_int) function scarl_gen_std_gauss_fft(ctx, data_real_3D, Np, xRange, corrL, &
        corrMod, seed, rank, phiK, gammaK) bind(C, name="scarl_gen_std_gauss_fft")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: data_real_3D(*)
      integer(c_int), intent(in) :: Np(3)
      real(c_double), intent(in) :: xRange(3), corrL(3)
      integer(c_int), value :: corrMod, seed, rank
      type(c_ptr), value :: phiK, gammaK
    end function

    ! gen_Std_Gauss_FFT_MPI (SRC_F/fftw_ScaRL.f90:424) on one GPU, Np = L
    integer(c_int) function scarl_gen_std_gauss_fft_mpi(ctx, data_real_3D, xRange, corrL, &
        corrMod, seed, rank, L, Np, phiK, gammaK) bind(C, name="scarl_gen_std_gauss_fft_mpi")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: data_real_3D(*)
      real(c_double), intent(in) :: xRange(3), corrL(3)
      integer(c_int), value :: corrMod, seed, rank
      integer(c_int), intent(in) :: L(3), Np(3)
      type(c_ptr), value :: phiK, gammaK
    end function

    ! gen_std_gauss_Shino_FFT (SRC_F/fftw_ScaRL.f90:157)
    integer(c_int) function scarl_gen_std_gauss_shino_fft(ctx, data_real_3D, Np, xRange, &
        corrL, pointsPerCorrL, corrMod, seed, rank) bind(C, name="scarl_gen_std_gauss_shino_fft")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: data_real_3D(*)
      integer(c_int), intent(in) :: Np(3), pointsPerCorrL(3)
      real(c_double), intent(in) :: xRange(3), corrL(3)
      integer(c_int), value :: corrMod, seed, rank
    end function

    integer(c_int) function scarl_sample_layout(s, gen_meth, nb_procs, topo_shape_in, lay) &
        bind(C, name="scarl_sample_layout")
      import :: c_int, c_ptr, scarl_sample, scarl_layout
      type(scarl_sample), intent(in) :: s
      integer(c_int), value :: gen_meth, nb_procs
      type(c_ptr), value :: topo_shape_in
      type(scarl_layout), intent(out) :: lay
    end function

    integer(c_int) function scarl_generate_sample(ctx, s, opts, global) &
        bind(C, name="scarl_generate_sample")
      import :: c_int, c_ptr, scarl_sample, scarl_gen_opts
      type(c_ptr), value :: ctx
      type(scarl_sample), intent(in) :: s
      type(scarl_gen_opts), intent(in) :: opts
      type(c_ptr), value :: global
    end function

    ! apply_UnityPartition_mtx (SRC_F/main_ScaRL.f90:1216)
    integer(c_int) function scarl_apply_unity_partition(ctx, field, Np, Np_ovlp, &
        partitionType, topo_pos, topo_shape) bind(C, name="scarl_apply_unity_partition")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: field(*)
      integer(c_int), intent(in) :: Np(3), Np_ovlp(3), topo_pos(3), topo_shape(3)
      integer(c_int), value :: partitionType
    end function

    ! multiVariateTransformation (SRC_F/main_ScaRL.f90:1355), dtype SCARL_F64
    integer(c_int) function scarl_multivariate_transformation(ctx, field, dtype, n, avg, &
        std_dev, margiFirst) bind(C, name="scarl_multivariate_transformation")
      import :: c_int, c_long_long, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: field(*)
      integer(c_int), value :: dtype, margiFirst
      integer(c_long_long), value :: n
      real(c_double), value :: avg, std_dev
    end function

    ! calculate_average_and_stdVar_MPI (SRC_F/Stat_ScaRL/statistics_RF.f90:18)
    integer(c_int) function scarl_moments(ctx, field, dtype, xNTotal, Nmc, evntAvg, &
        evntStdDev, globalAvg, globalStdDev) bind(C, name="scarl_moments")
      import :: c_int, c_long_long, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: field(*)
      integer(c_int), value :: dtype, Nmc
      integer(c_long_long), value :: xNTotal
      real(c_double), intent(out) :: evntAvg(*), evntStdDev(*), globalAvg, globalStdDev
    end function

    ! rebuild_Sk_FFT + rebuild_Sk (statistics_RF.f90:180-462)
    integer(c_int) function scarl_rebuild_sk(ctx, field, dtype, L, avg, stdDev, &
        tukey_literal, SkTot) bind(C, name="scarl_rebuild_sk")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: field(*)
      integer(c_int), value :: dtype, tukey_literal
      integer(c_int), intent(in) :: L(3)
      real(c_double), value :: avg, stdDev
      real(c_double), intent(out) :: SkTot(*)
    end function

    integer(c_int) function scarl_rebuild_corrL(SkTot, L, xStep, corrL_out) &
        bind(C, name="scarl_rebuild_corrL")
      import :: c_int, c_double
      real(c_double), intent(in) :: SkTot(*), xStep(3)
      integer(c_int), intent(in) :: L(3)
      real(c_double), intent(out) :: corrL_out(3)
    end function
  end interface

contains

  ! Drop-in for the reference call in create_fields (SRC_F/main_ScaRL.f90:512-515):
  !   call gen_std_gauss_FFT_gpu(k_mtx, Np, xRange, corrL, corrMod, seedStart, rank)
  ! on one lazily created context; stops with the library's message on error.
  subroutine gen_std_gauss_FFT_gpu(data_real_3D, Np, xRange, corrL, corrMod, seed, rank)
    real(c_double), dimension(:,:,:), intent(inout), target :: data_real_3D
    integer, dimension(3), intent(in) :: Np
    double precision, dimension(3), intent(in) :: xRange, corrL
    integer, intent(in) :: corrMod, seed, rank
    type(c_ptr), save :: ctx = c_null_ptr
    integer(c_int) :: rc
    if (.not. c_associated(ctx)) then
      rc = scarl_ctx_create(0_c_int, 0_c_size_t, ctx)
      if (rc /= SCARL_OK) stop "scarl_ctx_create failed"
    end if
    rc = scarl_gen_std_gauss_fft(ctx, data_real_3D, int(Np, c_int), xRange, corrL, &
                                 int(corrMod, c_int), int(seed, c_int), int(rank, c_int), &
                                 c_null_ptr, c_null_ptr)
    if (rc /= SCARL_OK) stop "scarl_gen_std_gauss_fft failed"
  end subroutine gen_std_gauss_FFT_gpu

end module scarl_gpu
