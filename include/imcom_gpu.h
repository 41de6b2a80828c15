/*
 * imcom_gpu.h -- C-ABI of the B200 (sm_100a) IMCOM solve path.
 *
 * Drop-in boundary for the solve path of IMCOM (barnabytprowe/imcom,
 * Fortran 95).  The Fortran driver (imcom.f90) and I/O module (imcom_io.f90)
 * keep reading configs and FITS files; their "build" branches call these
 * functions through ISO_C_BINDING instead of the Fortran routines named on
 * each declaration.  The Fortran module state (imcom_data.f90:24-135) becomes
 * device buffers owned by an opaque context.
 *
 * Conventions
 *  - Every array is a plain host pointer to Fortran-ordered (column-major)
 *    storage with leading dimension = number of rows, exactly as the Fortran
 *    side allocates it.  double = real(KIND=8), int = default integer,
 *    complex arrays are interleaved (re, im) pairs = complex(KIND=8).
 *  - Indices passed in (exp_i) are 1-based, as in the reference.
 *  - Output pointers may be NULL: the result then stays on the device only
 *    (the reference's "None" filename / save=0 case) and the call returns
 *    without waiting for the GPU.  A call with a non-NULL host output waits
 *    for the GPU before it returns.
 *  - Return value: 0 on success; < 0 an invalid argument (-k = argument k,
 *    the LAPACK convention); > 0 a device, library or convergence error.
 *    imcom_gpu_last_error() gives the message.  Errors reached by the
 *    reference's `write + stop` paths come back as status codes so the
 *    Fortran shim can print "IMCOM ERROR: ..." and stop.
 *  - One context per host thread; calls on one context are serialised on its
 *    CUDA stream.
 */
#ifndef IMCOM_GPU_H
#define IMCOM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct imcom_ctx imcom_ctx;

/* Status codes (> 0). */
#define IMCOM_ERR_CUDA 1        /* CUDA runtime / kernel launch error        */
#define IMCOM_ERR_LIBRARY 2     /* cuFFT error                                */
#define IMCOM_ERR_STATE 3       /* a prerequisite stage has not run           */
#define IMCOM_ERR_NEVILLE 4     /* imcom_polint duplicate-abscissa trap       */
#define IMCOM_ERR_EIGEN 5       /* eigensolver did not converge (DSYEVR info) */
#define IMCOM_ERR_ALLOC 6       /* device allocation failed                   */
#define IMCOM_ERR_NOT_FINITE 7  /* non-finite input                           */
#define IMCOM_ERR_NOALLOC_SIZE 8 /* problem too large for imcom_gpu_build_P_noalloc */
#define IMCOM_ERR_SPLIT 9       /* split-precision product unavailable (K too large, pipeline wait ran out) */
#define IMCOM_ERR_FITS 10       /* FITS file missing, malformed or of another size */

/* Eigensolver selection for imcom_gpu_set_option(IMCOM_OPT_EIGENSOLVER). */
#define IMCOM_EIGH_DC 0         /* own tridiagonalisation + divide & conquer  */
#define IMCOM_EIGH_JACOBI 1     /* own one-sided Jacobi (n <= 112)            */
#define IMCOM_EIGH_LIBRARY 2    /* cuSOLVER syevd: comparison baseline only   */
#define IMCOM_EIGH_TWOSTAGE 3   /* own two-stage (dense -> band -> tridiagonal)
                                   reduction + divide & conquer               */

/* Options for imcom_gpu_set_option. */
#define IMCOM_OPT_EIGENSOLVER 1
#define IMCOM_OPT_EIGEN_MAXITER 2 /* iteration cap of the iterative solvers  */
/* Arithmetic of P = Q^T B and T = -1/2 Q P~ (the reference's DGEMM,
 * imcom_matrix.f90:699, and DGEMVs, imcom_matrix.f90:734). */
#define IMCOM_OPT_PRECISION 3
#define IMCOM_PREC_FP64 0       /* FP64 tensor cores (default)                 */
#define IMCOM_PREC_SPLIT 1      /* int8 digit slices on the tensor cores, exact
                                   int32 sums, per-pixel error audit and FP64
                                   recomputation of the pixels that fail it   */
#define IMCOM_OPT_SPLIT_SLICES_P 4 /* digit slices of the P product, 2..8 (7) */
#define IMCOM_OPT_SPLIT_SLICES_T 5 /* digit slices of the T product, 2..8 (6) */
#define IMCOM_OPT_SPLIT_TOL_US 6   /* audit bound on the relative U/S error of a
                                      kept pixel: 10^-value (7)                */
#define IMCOM_OPT_SPLIT_TOL_T 7    /* audit bound on the relative error of a
                                      kept T column: 10^-value (8)             */
/* Bisection kernel: 0 automatic (the autotuned choice for the problem
 * size), 1 columns streamed from L2 (any n), 2 columns resident in
 * registers and shared memory (n <= 4096).  Same results either way. */
#define IMCOM_OPT_BISECT_KERNEL 8
#define IMCOM_BISECT_AUTO 0
#define IMCOM_BISECT_STREAM 1
#define IMCOM_BISECT_RESIDENT 2
/* CTAs (of 4 pixel warps) per SM of the streaming bisection kernels: 1..64
 * that many; 0 (default) = automatic, as many as keep the P columns of the
 * pixels in flight within 80 MB, so that they stay in L2 across their U/S
 * evaluations instead of being read from HBM again at every evaluation. */
#define IMCOM_OPT_BISECT_CTAS_PER_SM 9
/* Number of SMs this context sizes its persistent and cooperative grids for
 * (the tridiagonalisation panel kernel, the resident bisection, split-K
 * GEMMs; with a share set, the FP64 GEMMs, the trailing updates and the
 * divide-and-conquer products also loop over their tiles on grids bounded by
 * it, so that contexts side by side keep off each other's SMs); 0 = the
 * whole device.  Contexts that solve independent patches at
 * the same time on one GPU each take a share.  Results agree to rounding
 * (the reduction order of the eigensolver follows the grid). */
#define IMCOM_OPT_SM_SHARE 10
/* Thread-block cluster that finishes the tridiagonalisation once the
 * trailing matrix fits its distributed shared memory: 0 = automatic (16 CTAs
 * where the device can place them, else 8), 8 or 16 = that many CTAs (8 if 16
 * cannot be placed), -1 = no cluster tail (panels to the end).  A 16-CTA
 * cluster must find 16 free SMs in one GPC, which contexts working side by
 * side can make wait; smaller clusters hold smaller tails.  Same results to
 * rounding either way. */
#define IMCOM_OPT_TAIL_CTAS 11
/* Kernel of imcom_gpu_build_images: 0 = the FP64 GEMM, 1 = a streaming
 * kernel for a few stacks (up to 8 stacks per pass over T, FP64 FMA, each
 * warp holding four columns of T against the stacks of its pass), 2 = the
 * streaming kernel up to IMCOM_STACKS_STREAM_MAX stacks and the GEMM above
 * (default).  Same sums to rounding. */
#define IMCOM_OPT_STACK_KERNEL 12
#define IMCOM_STACKS_GEMM 0
#define IMCOM_STACKS_STREAM 1
#define IMCOM_STACKS_AUTO 2      /* default: streaming up to IMCOM_STACKS_STREAM_MAX
                                   stacks, the GEMM above (measured crossover) */
#define IMCOM_STACKS_STREAM_MAX 32
/* Inverse 2-D FFT of the lookup tables (imcom_build_Alookup/Blookup): 0 =
 * embedding, cuFFT and shift as separate steps; 1 = the library's own
 * transform in two passes that skip the grid's zero lines and fuse the
 * embedding and the shift (sides L = npad nps whose prime factors are 2, 3, 5,
 * 7, 11 and 13, up to 8191, 6143 with a factor 3, 5119 with a 5, 3583 with a
 * 7, 5631 with an 11, 6655 with a 13; other sides keep cuFFT; nps = 576 with
 * npad = 3 takes a register path, three length-576 transforms per line);
 * 2 (default) = the own transform where it is faster than cuFFT (the
 * register path), cuFFT elsewhere.  Same tables to rounding. */
#define IMCOM_OPT_TABLE_FFT 13
#define IMCOM_TABLE_FFT_CUFFT 0
#define IMCOM_TABLE_FFT_OWN 1
#define IMCOM_TABLE_FFT_AUTO 2
/* Features of the learned-kappa bracket: 0 = every pixel scans all inputs
 * for its neighbours and bins P^2 by eigenmode band element by element;
 * 1 (default) = the neighbour features come from a per-pixel table built
 * once per set of inputs, and the band sums run over the bands' contiguous
 * ranges of eigenmodes (the band index is non-decreasing when L is in
 * descending order; otherwise the element-wise binning is kept).  Same
 * features to rounding, same kappa. */
#define IMCOM_OPT_KAPPA_FEATURES 14
/* Starting point of imcom_gpu_bisect_kappa_learned's Newton steps: 0
 * (default) = the network's prediction; 1 = no network, the middle of the
 * search range (the comparison that shows what the network saves).  Same
 * kappa either way. */
#define IMCOM_OPT_KAPPA_START 17
/* Iteration cap of the divide-and-conquer secular-equation solver (0 = the
 * default, 100; roots converge in at most about 10).  A root that reaches the
 * cap makes imcom_gpu_eigen_A return IMCOM_ERR_EIGEN, as DSYEVR's info > 0
 * stops the reference (imcom_matrix.f90:645-653). */
#define IMCOM_OPT_DC_MAXITER 15
/* Tests of the bounded device waits (0 = normal operation, the default).
 * Each bit makes one wait run out on a flag that nothing sets:
 *  IMCOM_STALL_SPLIT: the copy producer of the split GEMM (imcom_gpu_build_P
 *    with IMCOM_PREC_SPLIT) issues no copies, so the MMA issuer's first wait
 *    (bounded at 2 s) runs out; the kernel drains, frees its tensor memory
 *    and returns, and the next bisection returns IMCOM_ERR_SPLIT;
 *  IMCOM_STALL_TRIDIAG: the first grid barrier of the tridiagonalisation
 *    waits for one arrival more than the grid makes, so it gives up after
 *    IMCOM_OPT_EIGEN_MAXITER polls and imcom_gpu_eigen_A returns
 *    IMCOM_ERR_EIGEN (when the tridiagonalisation runs panels: n above the
 *    cluster tail's size, or IMCOM_OPT_TAIL_CTAS = -1).
 * The context stays usable: clear the option and the next call runs
 * normally. */
#define IMCOM_OPT_STALL_TEST 16
#define IMCOM_STALL_SPLIT 1
#define IMCOM_STALL_TRIDIAG 2

/* ---- context ---------------------------------------------------------- */

/* Create a context on CUDA device `device`.  No reference counterpart (the
 * reference keeps module globals, imcom_data.f90:18-216). */
int imcom_gpu_create(int device, imcom_ctx** ctx);
int imcom_gpu_destroy(imcom_ctx* ctx);
/* Last error message of this context ("" if none). */
const char* imcom_gpu_last_error(const imcom_ctx* ctx);
/* Wait for all queued work; returns the first asynchronous error. */
int imcom_gpu_synchronize(imcom_ctx* ctx);
int imcom_gpu_set_option(imcom_ctx* ctx, int option, long long value);

/* ---- inputs (module state) -------------------------------------------- */

/* Input and output geometry, image and noise vectors: the arrays built by
 * imcom_alloc_gims / imcom_build_xy / imcom_alloc_xy / imcom_build_XaYa /
 * imcom_build_Ndiag (imcom_io.f90:36-240, imcom_proc.f90:56-119,
 * imcom_matrix.f90:556-582).  x_i, y_i, I_i, Ndiag, exp_i: length n;
 * X_a, Y_a: length m.  I_i and Ndiag may be NULL (then H, S and S-mode
 * bisection are unavailable until set). */
int imcom_gpu_set_inputs(imcom_ctx* ctx, int n, int m, const double* x_i,
                         const double* y_i, const int* exp_i,
                         const double* X_a, const double* Y_a,
                         const double* I_i, const double* Ndiag,
                         double psfxscale, double psfyscale);

/* PSFs as padded and normalised by imcom_alloc_psfs (imcom_io.f90:244-335):
 * G_unrot (nps, nps, nexppsf), Gamma (nps, nps), rotangdeg (nexppsf).
 * psfconst is the value of imcom_test_psfconst (imcom_proc.f90:582-599). */
int imcom_gpu_set_psfs(imcom_ctx* ctx, int nps, int nexppsf, int psfconst,
                       const double* G_unrot, const double* rotangdeg,
                       const double* Gamma);

/* ---- solve path ------------------------------------------------------- */

/* Rotate each PSF (imcom_rotate_image, imcom_proc.f90:184-250, when
 * |angle| > 2 pi eps), Fourier transform it and Gamma with the reference's
 * Hermitian fill (imcom_ft_r2c, imcom_proc.f90:433-475; call site
 * imcom.f90:90-116), and compute C (imcom_calc_C, imcom_matrix.f90:546-552).
 * Gt_out (nps, nps, nexppsf) and Gammat_out (nps, nps) are complex and may
 * be NULL. */
int imcom_gpu_psf_spectra(imcom_ctx* ctx, int npoly, double* C_out,
                          double* Gt_out, double* Gammat_out);

/* Lookup tables for A (imcom_build_Alookup, imcom_matrix.f90:361-430) and
 * A assembly by 7th-order interpolation (imcom_lookup_A, :206-284).  This is
 * the build branch of imcom_get_A (:41-73).  A_out (n, n) may be NULL. */
int imcom_gpu_build_A(imcom_ctx* ctx, int npoly, int npad, double* A_out);
/* Cache-read branch of imcom_get_A (:49-68): A read from FITS by the caller. */
int imcom_gpu_load_A(imcom_ctx* ctx, const double* A);

/* Eigendecomposition of A in FP64, eigenvalues descending (imcom_eigen_A,
 * imcom_matrix.f90:586-678; build branch of imcom_get_QL, :155-202).
 * Q_out (n, n), L_out (n) may be NULL; cond_out receives max(L)/min(L). */
int imcom_gpu_eigen_A(imcom_ctx* ctx, double* Q_out, double* L_out,
                      double* cond_out);
/* Cache-read branch of imcom_get_QL (:164-198). */
int imcom_gpu_load_QL(imcom_ctx* ctx, const double* Q, const double* L);

/* Lookup tables for B (imcom_build_Blookup, :434-493) and B assembly
 * (imcom_lookup_B, :288-357): build branch of imcom_get_B (:77-109). */
int imcom_gpu_build_B(imcom_ctx* ctx, int npoly, int npad, double* B_out);
int imcom_gpu_load_B(imcom_ctx* ctx, const double* B);

/* P = Q^T B in FP64 (imcom_build_P, :682-712; build branch of imcom_get_P,
 * :113-151).  P2 = P*P is formed where it is used, bit-identical.  With
 * IMCOM_PREC_SPLIT the product runs on the int8 digit slices; the next
 * bisection audits every pixel and recomputes in FP64 the P columns of the
 * pixels whose kappa or U/S accuracy the split product cannot guarantee. */
int imcom_gpu_build_P(imcom_ctx* ctx, double* P_out);
int imcom_gpu_load_P(imcom_ctx* ctx, const double* P);

/* Release A and B (imcom.f90:159). */
int imcom_gpu_free_AB(imcom_ctx* ctx);

/* Per-pixel kappa bisection (imcom_bisect_kappa, imcom_bisect.f90:78-170,
 * with imcom_bisect_by_U :174-222 / imcom_bisect_by_S :226-267 and
 * imcom_U_from_kappa / imcom_S_from_kappa, imcom_matrix.f90:904-970).
 * UnotS != 0 solves U_a < US_max, else S_a < US_max.  K_out, US_out (m)
 * and nevals_out (m; evaluations per pixel) may be NULL. */
int imcom_gpu_bisect_kappa(imcom_ctx* ctx, int UnotS, double US_max,
                           double k_min, double k_max, double tol,
                           int maxnits, double C_a, double* K_out,
                           double* US_out, int* nevals_out);

/* Same contract and bit-identical K as imcom_gpu_bisect_kappa, with the
 * learned-kappa bracket: an MLP (imcom_gpu_mlp_set_weights) predicts
 * log10(kappa) and a bracket half-width per pixel; Newton steps in
 * log10(kappa) from that prediction, each one evaluation of U (or S) and its
 * derivative, and two probes find points on either side of the band where
 * the bisection stops; the bisection steps those points decide are skipped
 * and the rest are evaluated, so K_a and U_a (S_a) equal the plain
 * bisection's bit for bit.  fallback_out (m, may be NULL): 1 where no point
 * bounded the bisection.  No reference counterpart; replaces
 * imcom_bisect_kappa (imcom_bisect.f90:78-170). */
int imcom_gpu_bisect_kappa_learned(imcom_ctx* ctx, int UnotS, double US_max,
                                   double k_min, double k_max, double tol,
                                   int maxnits, double C_a, double* K_out,
                                   double* US_out, int* nevals_out,
                                   int* fallback_out);

/* T(:,a) = -1/2 Q (P(:,a) / (L + K_a)) (imcom_build_T,
 * imcom_matrix.f90:716-750).  Needs the bisection to have run (or
 * imcom_gpu_load_K).  T_out (n, m) may be NULL.  With IMCOM_PREC_SPLIT the
 * product runs on the int8 digit slices and the columns whose error bound
 * exceeds the T tolerance are recomputed in FP64. */
int imcom_gpu_build_T(imcom_ctx* ctx, double* T_out);
/* T-reuse path (imcom_bisect.f90:47-62): T read from FITS by the caller. */
int imcom_gpu_load_T(imcom_ctx* ctx, const double* T);
/* Kappa map from a previous solve (K_a, imcom_data.f90:104). */
int imcom_gpu_load_K(imcom_ctx* ctx, const double* K);

/* H = T^T I (imcom_build_image, imcom_matrix.f90:754-790). */
int imcom_gpu_build_image(imcom_ctx* ctx, double* H_out);
/* imcom_build_image for nstack image stacks observed with the geometry, mask
 * and PSFs of the resident T (built, or loaded from the cache with
 * imcom_gpu_load_T): column s of I_stack (n x nstack, leading dimension n) is
 * the I_i vector of stack s, column s of H_out (m x nstack, leading
 * dimension m) its H_a.  One FP64 GEMM H = T^T I, so T is read from HBM once
 * for all stacks.  Host arrays; H_out may be NULL (result kept on the
 * device). */
int imcom_gpu_build_images(imcom_ctx* ctx, int nstack, const double* I_stack, double* H_out);
/* The same on device arrays the caller owns (dI: n x nstack with leading
 * dimension ldi >= n; dH: m x nstack, ldh >= m), ordered on the library's
 * stream (imcom_gpu_get_stream) and not synchronised. */
int imcom_gpu_build_images_device(imcom_ctx* ctx, int nstack, const double* dI, long long ldi,
                                  double* dH, long long ldh);
/* S_a = sum_i T_ia^2 Ndiag_i (imcom_build_S, imcom_matrix.f90:839-877). */
int imcom_gpu_build_S(imcom_ctx* ctx, double* S_out);
/* U_a = U(K_a) (imcom_build_U, imcom_matrix.f90:795-835). */
int imcom_gpu_build_U(imcom_ctx* ctx, double C_a, double* U_out);

/* ---- learned kappa (no reference counterpart) -------------------------- */

/* Per-pixel features (12 per pixel, feature-major (12, m)): input-pixel
 * density near X_a, hit count, 8 log-moments of P2 weighted by L, and the
 * U/S target.  Needs P and L on the device. */
int imcom_gpu_kappa_features(imcom_ctx* ctx, int UnotS, double US_max,
                             double C_a, float* feat_out);
/* Install MLP weights (12 -> 64 -> 64 -> 2, fp32 host arrays, row-major
 * [out][in]) and the feature normalisation (mean/std, 12 each). */
int imcom_gpu_mlp_set_weights(imcom_ctx* ctx, const float* W1,
                              const float* b1, const float* W2,
                              const float* b2, const float* W3,
                              const float* b3, const float* feat_mean,
                              const float* feat_std);

/* Train the MLP on the GPU (Adam, bf16 activations, fp32 accumulation) on
 * normalised features (12 x nsamples, feature-major) and targets (log10
 * kappa, normalised).  params (5122 floats: W1 64x12 | b1 64 | W2 64x64 |
 * b2 64 | W3 2x64 | b3 2, row-major [out][in]) holds the initial values on
 * entry and the trained values on return; loss_out (epochs) may be NULL.
 * No reference counterpart. */
int imcom_gpu_mlp_train(imcom_ctx* ctx, int nsamples, const float* feat,
                        const float* target, int epochs, int batch, float lr,
                        unsigned seed, float* params, float* loss_out);
/* Summed training loss and its gradient (5122 floats) over nsamples samples
 * at the given parameters: the training kernel on one batch (for gradient
 * checks).  No reference counterpart. */
int imcom_gpu_mlp_gradient(imcom_ctx* ctx, int nsamples, const float* feat,
                           const float* target, const float* params,
                           float* grad_out, float* loss_out);

/* ---- split-precision products (no reference counterpart) --------------- */

/* Report of the split-precision path (IMCOM_OPT_PRECISION = IMCOM_PREC_SPLIT)
 * for the resident solve: info[0] digit slices of P, info[1] digit slices of
 * T, info[2] pixels whose P column was recomputed in FP64 by the audit of the
 * last bisection, info[3] pixels whose T column was recomputed in FP64 by
 * the last imcom_gpu_build_T, info[4] largest bound on the relative U (or S)
 * error among the pixels kept, info[5] largest bound on the relative T
 * column error caused by the split P among the pixels kept, info[6] the same
 * for the split T product, info[7] 1 if the resident P came from the split
 * product.  Bounds are six standard deviations of the error model: digit
 * rounding of each product term with standard deviation at most
 * 0.5 * 2^(1-8S) * sqrt(K) * scale_row * scale_col. */
int imcom_gpu_split_info(imcom_ctx* ctx, double* info8);
/* Per pixel (m each, may be NULL): 1 where the audit of the last bisection
 * recomputed the P column in FP64 (fp64_P), 1 where the last
 * imcom_gpu_build_T recomputed the T column in FP64 (fp64_T); zeros when no
 * split product was audited. */
int imcom_gpu_split_pixels(imcom_ctx* ctx, int* fp64_P, int* fp64_T);

/* ---- allocation-free projection ---------------------------------------- */

/* P = Q^T B (the product imcom_gpu_build_P forms) without allocating any
 * device memory, for callers that cannot call cudaMalloc or cudaFree: for
 * example a host application or framework that reserves the GPU's memory up
 * front in its own allocator, where allocating or freeing mid-run would
 * synchronise the device, fragment the reserved pool or fail outright.
 * No counterpart in the reference (which calls DGEMM, imcom_matrix.f90:699).
 *
 * dQ (n x n, leading dimension ldq), dB (n x m, ldb) and dP (n x m, ldp) are
 * DEVICE pointers owned by the caller, column-major; stream is a
 * cudaStream_t (NULL = the default stream).  The call only queues work: it
 * returns without waiting for the GPU.
 *
 * Scratch: the split-K partial sums live in a fixed 32 MiB device array that
 * every GPU loading the library holds until the process exits.  Limit:
 * 2 * round_up(n, 32) * m <= 4,194,304 (e.g. n = 2048 with m <= 1024) and
 * m <= 65,535; larger problems return IMCOM_ERR_NOALLOC_SIZE without touching
 * the GPU.  A CUDA error already pending on the calling thread (from the
 * caller's earlier work) is returned as IMCOM_ERR_CUDA before anything is
 * queued, and left pending.  The
 * first call on each device looks the array up and sets the kernel's
 * shared-memory limit, so make that first call before any stream capture.
 * All calls share the array: calls whose GPU work overlaps race.
 * Returns 0, -k for a bad argument k, IMCOM_ERR_NOALLOC_SIZE or
 * IMCOM_ERR_CUDA. */
int imcom_gpu_build_P_noalloc(const double* dQ, long long ldq, const double* dB,
                              long long ldb, double* dP, long long ldp, int n, int m,
                              void* stream);

/* ---- batched eigendecomposition of small systems ------------------------ */

/* Largest n of the one-sided Jacobi eigensolver (IMCOM_EIGH_JACOBI and the
 * batched call below): the matrix and its rotations fill one CTA's shared
 * memory. */
#define IMCOM_JACOBI_MAX_N 112

/* Eigendecomposition of `count` symmetric positive semi-definite n x n
 * matrices (n <= IMCOM_JACOBI_MAX_N), one thread block each, by one-sided
 * (Hestenes) Jacobi: the method IMCOM_EIGH_JACOBI applies to A, for many
 * small patches in one launch.  No reference counterpart: the reference
 * decomposes one A per run with DSYEVR (imcom_matrix.f90:617-643).
 * A: count matrices, column-major, contiguous (matrix b at A + b n^2);
 * Q: the eigenvectors in the same layout; L: count x n eigenvalues; both in
 * ascending order per matrix.  sweeps (may be NULL): Jacobi sweeps used per
 * matrix.  Host arrays; the call returns when Q and L are written.
 * Returns 0, -k for a bad argument k, IMCOM_ERR_EIGEN if a matrix does not
 * converge in 60 sweeps, IMCOM_ERR_CUDA / IMCOM_ERR_ALLOC. */
int imcom_gpu_eigh_jacobi_batched(imcom_ctx* ctx, int n, int count, const double* A,
                                  double* Q, double* L, int* sweeps);

/* ---- two-stage reduction (diagnostic) --------------------------------- */

/* First stage of the two-stage tridiagonalisation alone: the resident A
 * (built or loaded) reduced to a symmetric band matrix of bandwidth 32 by
 * blocked Householder transformations, returned as its 33 lower diagonals in
 * band storage, AB_out[d + c * ldb] = B(c + d, c) (ldb >= 33, n columns).
 * The band matrix has A's eigenvalues.  No reference counterpart (the
 * reference reduces A to tridiagonal form inside DSYEVR,
 * imcom_matrix.f90:617-643). */
int imcom_gpu_band_reduce(imcom_ctx* ctx, double* AB_out, int ldb);

/* ---- FITS files without CFITSIO (host only; no context, no GPU) -------- */

/* The primary image of a FITS file, for drivers that get their arrays from
 * this library and would otherwise link CFITSIO only to read and write them.
 * Paths are NUL-terminated; arrays are column-major (axis 1 fastest), as
 * FITS stores them.  Errors return IMCOM_ERR_FITS with the reason in
 * imcom_fits_last_error() (per host thread); bad arguments return -k. */
/* imcom_sizefits (imcom_io.f90:338-356): NAXIS1, NAXIS2 (1 for a
 * one-axis image) and BITPIX. */
int imcom_fits_size(const char* path, int* naxis1, int* naxis2, int* bitpix);
/* imcom_readfits (imcom_io.f90:360-403): the image as doubles.  Every BITPIX
 * is read, with BSCALE and BZERO applied; NaN pixels of floating-point
 * images and BLANK pixels of integer images become -666, the null value the
 * reference passes to CFITSIO.  The image must hold naxis1 x naxis2 values
 * (IMCOM_ERR_FITS otherwise, where the reference stops). */
int imcom_fits_read(const char* path, int naxis1, int naxis2, double* image);
/* imcom_writefits (imcom_io.f90:407-457): a BITPIX -64 image; an existing
 * file is replaced. */
int imcom_fits_write(const char* path, int naxis1, int naxis2, const double* image);
/* imcom_writefitscube (imcom_io.f90:460-494): the same with three axes. */
int imcom_fits_write_cube(const char* path, int naxis1, int naxis2, int naxis3,
                          const double* cube);
/* Reason for the last IMCOM_ERR_FITS of this host thread. */
const char* imcom_fits_last_error(void);

/* ---- device views (for callers that keep data on the GPU) -------------- */

/* Device pointer and leading dimension of an internal buffer:
 * which = 'A','Q','L','B','P','T','K','H','S','U', or 'W' for the T operand
 * P~ = P(:,a) / (L + K_a) (column-major, ld rows). */
int imcom_gpu_device_buffer(imcom_ctx* ctx, char which, void** dptr,
                            long long* ld);
/* Number of this library's own kernel launches since the process started
 * (library calls such as cuFFT are not counted). */
int imcom_gpu_launch_count(imcom_ctx* ctx, long long* count);
/* The context's CUDA stream (cudaStream_t), for callers that order their
 * own work or events against the library's. */
int imcom_gpu_get_stream(imcom_ctx* ctx, void** stream);
/* Milliseconds spent on the GPU by the last call of each stage (CUDA
 * events): [spectra, build_A, eigen_A, build_B, build_P, bisect, build_T,
 * epilogue, eigen tridiagonalisation, eigen divide and conquer, eigen
 * back-transformation] (11 values). */
int imcom_gpu_stage_times(imcom_ctx* ctx, double* ms11);
/* Milliseconds of the last lookup-table build (within build_A and build_B:
 * embedding, inverse FFT and shift) for the A tables and the B tables
 * (2 values; 0 where none has run). */
int imcom_gpu_table_times(imcom_ctx* ctx, double* ms2);

#ifdef __cplusplus
}
#endif
#endif /* IMCOM_GPU_H */
