!    IMCOM_GPU_IFACE.F90 - ISO_C_BINDING interface of the B200 solve path
!
!    Binds the C-ABI declared in include/imcom_gpu.h so the reference's
!    Fortran driver (imcom.f90) and matrix module can call the GPU solve path
!    in their "build" branches.  Arrays are passed as the Fortran arrays the
!    module already allocates (column-major, leading dimension = rows); the
!    C side receives plain pointers.  Every function returns an integer
!    status (0 = success, < 0 bad argument, > 0 device or convergence
!    error); imcom_gpu_check turns a failure into the reference's
!    "IMCOM ERROR: ..." + STOP behaviour.
!
!    Link with -L<repo>/imcom_b200 -limcom_gpu.
!
MODULE imcom_gpu_iface

USE ISO_C_BINDING
implicit none

INTERFACE

  INTEGER(C_INT) FUNCTION imcom_gpu_create(device, ctx) BIND(C, NAME="imcom_gpu_create")
    IMPORT :: C_INT, C_PTR
    INTEGER(C_INT), VALUE :: device
    TYPE(C_PTR) :: ctx
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_destroy(ctx) BIND(C, NAME="imcom_gpu_destroy")
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: ctx
  END FUNCTION

  TYPE(C_PTR) FUNCTION imcom_gpu_last_error(ctx) BIND(C, NAME="imcom_gpu_last_error")
    IMPORT :: C_PTR
    TYPE(C_PTR), VALUE :: ctx
  END FUNCTION

  ! imcom_data module state: x_i, y_i, exp_i, X_a, Y_a, I_i, Ndiag
  INTEGER(C_INT) FUNCTION imcom_gpu_set_inputs(ctx, n, m, x_i, y_i, exp_i, X_a, Y_a, I_i, &
                                               Ndiag, psfxscale, psfyscale) &
                                               BIND(C, NAME="imcom_gpu_set_inputs")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: n, m
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: x_i, y_i, X_a, Y_a, I_i, Ndiag
    INTEGER(C_INT), DIMENSION(*), INTENT(IN) :: exp_i
    REAL(C_DOUBLE), VALUE :: psfxscale, psfyscale
  END FUNCTION

  ! G_unrot(n1psf, n2psf, nexppsf), rotangdeg(nexppsf), Gamma(n1psf, n2psf)
  INTEGER(C_INT) FUNCTION imcom_gpu_set_psfs(ctx, nps, nexppsf, psfconst, G_unrot, &
                                             rotangdeg, Gamma) BIND(C, NAME="imcom_gpu_set_psfs")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: nps, nexppsf, psfconst
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: G_unrot, rotangdeg, Gamma
  END FUNCTION

  ! imcom.f90:90-122 (rotation, r2c FFTs, imcom_calc_C)
  INTEGER(C_INT) FUNCTION imcom_gpu_psf_spectra(ctx, npoly, C_out, Gt_out, Gammat_out) &
                                                BIND(C, NAME="imcom_gpu_psf_spectra")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: npoly
    REAL(C_DOUBLE) :: C_out
    TYPE(C_PTR), VALUE :: Gt_out, Gammat_out   ! C_NULL_PTR or C_LOC(complex arrays)
  END FUNCTION

  ! imcom_get_A build branch (imcom_build_Alookup + imcom_lookup_A)
  INTEGER(C_INT) FUNCTION imcom_gpu_build_A(ctx, npoly, npad, A_out) &
                                            BIND(C, NAME="imcom_gpu_build_A")
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: npoly, npad
    TYPE(C_PTR), VALUE :: A_out                 ! C_LOC(A_aij) when saveA, else C_NULL_PTR
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_load_A(ctx, A) BIND(C, NAME="imcom_gpu_load_A")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: A
  END FUNCTION

  ! imcom_eigen_A (DSYEVR + reversal)
  INTEGER(C_INT) FUNCTION imcom_gpu_eigen_A(ctx, Q_out, L_out, cond_out) &
                                            BIND(C, NAME="imcom_gpu_eigen_A")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    TYPE(C_PTR), VALUE :: Q_out, L_out
    REAL(C_DOUBLE) :: cond_out
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_load_QL(ctx, Q, L) BIND(C, NAME="imcom_gpu_load_QL")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: Q, L
  END FUNCTION

  ! imcom_get_B build branch (imcom_build_Blookup + imcom_lookup_B)
  INTEGER(C_INT) FUNCTION imcom_gpu_build_B(ctx, npoly, npad, B_out) &
                                            BIND(C, NAME="imcom_gpu_build_B")
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: npoly, npad
    TYPE(C_PTR), VALUE :: B_out
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_load_B(ctx, B) BIND(C, NAME="imcom_gpu_load_B")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: B
  END FUNCTION

  ! imcom_build_P (DGEMM 'T','N')
  INTEGER(C_INT) FUNCTION imcom_gpu_build_P(ctx, P_out) BIND(C, NAME="imcom_gpu_build_P")
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: ctx
    TYPE(C_PTR), VALUE :: P_out
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_load_P(ctx, P) BIND(C, NAME="imcom_gpu_load_P")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: P
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_free_AB(ctx) BIND(C, NAME="imcom_gpu_free_AB")
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: ctx
  END FUNCTION

  ! imcom_bisect_kappa (USB -> UnotS)
  INTEGER(C_INT) FUNCTION imcom_gpu_bisect_kappa(ctx, UnotS, US_max, k_min, k_max, tol, &
                                                 maxnits, C_a, K_out, US_out, nevals_out) &
                                                 BIND(C, NAME="imcom_gpu_bisect_kappa")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: UnotS, maxnits
    REAL(C_DOUBLE), VALUE :: US_max, k_min, k_max, tol, C_a
    REAL(C_DOUBLE), DIMENSION(*) :: K_out, US_out
    TYPE(C_PTR), VALUE :: nevals_out
  END FUNCTION

  ! imcom_build_T
  INTEGER(C_INT) FUNCTION imcom_gpu_build_T(ctx, T_out) BIND(C, NAME="imcom_gpu_build_T")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*) :: T_out
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_load_T(ctx, T) BIND(C, NAME="imcom_gpu_load_T")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: T
  END FUNCTION

  ! imcom_build_image / imcom_build_S / imcom_build_U
  INTEGER(C_INT) FUNCTION imcom_gpu_build_image(ctx, H_out) BIND(C, NAME="imcom_gpu_build_image")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*) :: H_out
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_build_S(ctx, S_out) BIND(C, NAME="imcom_gpu_build_S")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*) :: S_out
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_build_U(ctx, C_a, U_out) BIND(C, NAME="imcom_gpu_build_U")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), VALUE :: C_a
    REAL(C_DOUBLE), DIMENSION(*) :: U_out
  END FUNCTION

  ! Options (no reference counterpart), e.g. option 3 = IMCOM_OPT_PRECISION,
  ! value 1 = IMCOM_PREC_SPLIT for the split-precision P and T; option 10 =
  ! IMCOM_OPT_SM_SHARE (SMs for this context's persistent grids when several
  ! contexts run side by side); option 11 = IMCOM_OPT_TAIL_CTAS (cluster that
  ! finishes the tridiagonalisation: 0 auto, 16, 8, -1 none)
  INTEGER(C_INT) FUNCTION imcom_gpu_set_option(ctx, option, value) &
                                               BIND(C, NAME="imcom_gpu_set_option")
    IMPORT :: C_INT, C_PTR, C_LONG_LONG
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: option
    INTEGER(C_LONG_LONG), VALUE :: value
  END FUNCTION

  ! imcom_bisect_kappa with the learned-kappa bracket (same K; weights set
  ! with imcom_gpu_mlp_set_weights)
  INTEGER(C_INT) FUNCTION imcom_gpu_bisect_kappa_learned(ctx, UnotS, US_max, k_min, k_max, &
                                                         tol, maxnits, C_a, K_out, US_out, &
                                                         nevals_out, fallback_out) &
                                                         BIND(C, NAME="imcom_gpu_bisect_kappa_learned")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: UnotS, maxnits
    REAL(C_DOUBLE), VALUE :: US_max, k_min, k_max, tol, C_a
    REAL(C_DOUBLE), DIMENSION(*) :: K_out, US_out
    TYPE(C_PTR), VALUE :: nevals_out, fallback_out
  END FUNCTION

  ! Report of the split-precision audit (8 values)
  INTEGER(C_INT) FUNCTION imcom_gpu_split_info(ctx, info8) BIND(C, NAME="imcom_gpu_split_info")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(8) :: info8
  END FUNCTION

  ! Eigendecomposition of `count` small symmetric positive semi-definite
  ! matrices (n <= 112) in one launch, one-sided Jacobi; ascending per matrix
  INTEGER(C_INT) FUNCTION imcom_gpu_eigh_jacobi_batched(ctx, n, count, A, Q, L, sweeps) &
                                                        BIND(C, NAME="imcom_gpu_eigh_jacobi_batched")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: n, count
    REAL(C_DOUBLE), DIMENSION(n, n, count) :: A, Q
    REAL(C_DOUBLE), DIMENSION(n, count) :: L
    INTEGER(C_INT), DIMENSION(count) :: sweeps
  END FUNCTION

  ! Wait for the context's queued work; returns the first asynchronous error
  INTEGER(C_INT) FUNCTION imcom_gpu_synchronize(ctx) BIND(C, NAME="imcom_gpu_synchronize")
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: ctx
  END FUNCTION

  ! Kappa map K_a from a previous solve (imcom_data.f90:104)
  INTEGER(C_INT) FUNCTION imcom_gpu_load_K(ctx, K) BIND(C, NAME="imcom_gpu_load_K")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: K
  END FUNCTION

  ! Learned-kappa MLP weights (12 -> 64 -> 64 -> 2, real(C_FLOAT) arrays,
  ! row-major [out][in]) and the feature normalisation (12 means, 12 stds)
  INTEGER(C_INT) FUNCTION imcom_gpu_mlp_set_weights(ctx, W1, b1, W2, b2, W3, b3, feat_mean, &
                                                    feat_std) &
                                                    BIND(C, NAME="imcom_gpu_mlp_set_weights")
    IMPORT :: C_INT, C_PTR, C_FLOAT
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_FLOAT), DIMENSION(*), INTENT(IN) :: W1, b1, W2, b2, W3, b3, feat_mean, feat_std
  END FUNCTION

  ! Per pixel (m each): 1 where the split audit recomputed the P column (or
  ! the T column) in FP64
  INTEGER(C_INT) FUNCTION imcom_gpu_split_pixels(ctx, fp64_P, fp64_T) &
                                                 BIND(C, NAME="imcom_gpu_split_pixels")
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), DIMENSION(*) :: fp64_P, fp64_T
  END FUNCTION

  ! GPU milliseconds of the last call of each stage (11 values, order as in
  ! include/imcom_gpu.h) and of the last A and B table builds (2 values)
  INTEGER(C_INT) FUNCTION imcom_gpu_stage_times(ctx, ms11) BIND(C, NAME="imcom_gpu_stage_times")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(11) :: ms11
  END FUNCTION

  INTEGER(C_INT) FUNCTION imcom_gpu_table_times(ctx, ms2) BIND(C, NAME="imcom_gpu_table_times")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    REAL(C_DOUBLE), DIMENSION(2) :: ms2
  END FUNCTION

  ! imcom_build_image for nstack image stacks sharing the resident T:
  ! I_stack(n, nstack) -> H(m, nstack), one FP64 GEMM (T read once)
  INTEGER(C_INT) FUNCTION imcom_gpu_build_images(ctx, nstack, I_stack, H) &
                                                 BIND(C, NAME="imcom_gpu_build_images")
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: ctx
    INTEGER(C_INT), VALUE :: nstack
    REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: I_stack
    REAL(C_DOUBLE), DIMENSION(*) :: H
  END FUNCTION

  ! FITS images without CFITSIO (host only, no context).  Paths are passed
  ! as trim(name)//C_NULL_CHAR.
  ! imcom_sizefits (imcom_io.f90:338-356)
  INTEGER(C_INT) FUNCTION imcom_fits_size(path, naxis1, naxis2, bitpix) &
                                          BIND(C, NAME="imcom_fits_size")
    IMPORT :: C_INT, C_CHAR
    CHARACTER(KIND=C_CHAR), DIMENSION(*), INTENT(IN) :: path
    INTEGER(C_INT) :: naxis1, naxis2, bitpix
  END FUNCTION

  ! imcom_readfits (imcom_io.f90:360-403): any BITPIX, BSCALE/BZERO applied,
  ! undefined pixels -666
  INTEGER(C_INT) FUNCTION imcom_fits_read(path, naxis1, naxis2, image) &
                                          BIND(C, NAME="imcom_fits_read")
    IMPORT :: C_INT, C_CHAR, C_DOUBLE
    CHARACTER(KIND=C_CHAR), DIMENSION(*), INTENT(IN) :: path
    INTEGER(C_INT), VALUE :: naxis1, naxis2
    REAL(C_DOUBLE), DIMENSION(naxis1, naxis2), INTENT(OUT) :: image
  END FUNCTION

  ! imcom_writefits (imcom_io.f90:407-457): BITPIX -64, replaces the file
  INTEGER(C_INT) FUNCTION imcom_fits_write(path, naxis1, naxis2, image) &
                                           BIND(C, NAME="imcom_fits_write")
    IMPORT :: C_INT, C_CHAR, C_DOUBLE
    CHARACTER(KIND=C_CHAR), DIMENSION(*), INTENT(IN) :: path
    INTEGER(C_INT), VALUE :: naxis1, naxis2
    REAL(C_DOUBLE), DIMENSION(naxis1, naxis2), INTENT(IN) :: image
  END FUNCTION

  ! imcom_writefitscube (imcom_io.f90:460-494)
  INTEGER(C_INT) FUNCTION imcom_fits_write_cube(path, naxis1, naxis2, naxis3, cube) &
                                                BIND(C, NAME="imcom_fits_write_cube")
    IMPORT :: C_INT, C_CHAR, C_DOUBLE
    CHARACTER(KIND=C_CHAR), DIMENSION(*), INTENT(IN) :: path
    INTEGER(C_INT), VALUE :: naxis1, naxis2, naxis3
    REAL(C_DOUBLE), DIMENSION(naxis1, naxis2, naxis3), INTENT(IN) :: cube
  END FUNCTION

  TYPE(C_PTR) FUNCTION imcom_fits_last_error() BIND(C, NAME="imcom_fits_last_error")
    IMPORT :: C_PTR
  END FUNCTION

END INTERFACE

TYPE(C_PTR), SAVE :: imcom_gpu_ctx = C_NULL_PTR

CONTAINS

SUBROUTINE imcom_gpu_check(status, what)
! Reference error behaviour (write + stop) for a failed C-ABI call.
implicit none
integer(C_INT), intent(IN) :: status
character(LEN=*), intent(IN) :: what
if (status.eq.0) return
call imcom_stop_with(status, what, imcom_gpu_last_error(imcom_gpu_ctx))
END SUBROUTINE imcom_gpu_check

SUBROUTINE imcom_fits_check(status, what)
! The same for the FITS functions, whose reason is kept per host thread.
implicit none
integer(C_INT), intent(IN) :: status
character(LEN=*), intent(IN) :: what
if (status.eq.0) return
call imcom_stop_with(status, what, imcom_fits_last_error())
END SUBROUTINE imcom_fits_check

SUBROUTINE imcom_stop_with(status, what, p)
implicit none
integer(C_INT), intent(IN) :: status
character(LEN=*), intent(IN) :: what
type(C_PTR), intent(IN) :: p
character(KIND=C_CHAR), dimension(:), pointer :: msg
integer :: i
interface
  integer(C_SIZE_T) function c_strlen(s) bind(C, name="strlen")
    import :: C_SIZE_T, C_PTR
    type(C_PTR), value :: s
  end function
end interface
call c_f_pointer(p, msg, [c_strlen(p)])
write(*, FMT='(A, I4)') "IMCOM ERROR: "//what//" failed with status ", status
write(*, FMT='(A)', ADVANCE='NO') "IMCOM ERROR: "
do i = 1, size(msg)
  write(*, FMT='(A)', ADVANCE='NO') msg(i)
end do
write(*, *)
stop
END SUBROUTINE imcom_stop_with

END MODULE imcom_gpu_iface
