// common.cuh -- shared definitions of the sm_100a IMCOM solve path.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/imcom_gpu.h"

namespace imcom {

// Device matrix: column-major, leading dimension ld >= rows (rounded up so
// that every column starts on a 256-byte boundary).
struct DMat {
  double* p = nullptr;
  long long rows = 0, cols = 0, ld = 0;
  size_t cap = 0;  // bytes allocated (kept when a smaller matrix reuses it)
  size_t bytes() const { return (size_t)ld * (size_t)cols * sizeof(double); }
};

inline long long pad_ld(long long rows) { return (rows + 31) / 32 * 32; }

enum Stage {
  ST_SPECTRA = 0, ST_A, ST_EIG, ST_B, ST_P, ST_BISECT, ST_T, ST_EPI,
  ST_EIG_TRD, ST_EIG_DC, ST_EIG_BT, ST_N
};

struct MlpWeights {
  float* w = nullptr;  // packed device weights (see kappa.cu)
  bool set = false;
};

struct EigWork;  // eigen.cu

// One operand of the split-precision product (ozaki.cu): S int8 digit
// slices of an FP64 matrix in tensor-core tile order, plus the power-of-two
// scale of every operand row.
struct SplitOp {
  int8_t* dig = nullptr;
  double* scale = nullptr;
  int* exps = nullptr;
  size_t dig_bytes = 0, scale_bytes = 0, exps_bytes = 0;
  long long rows = 0, K = 0, rb = 0, kb = 0;
  int S = 0, R = 0;
};

}  // namespace imcom

struct imcom_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int eig_mode = IMCOM_EIGH_DC;
  long long eig_maxiter = 0;
  int dc_maxiter = 0;     // IMCOM_OPT_DC_MAXITER (0: 100)
  int stall_test = 0;     // IMCOM_OPT_STALL_TEST bits

  // geometry
  int n = 0, m = 0;
  double psfx = 0, psfy = 0;
  double *x = nullptr, *y = nullptr, *X = nullptr, *Y = nullptr;
  double *I = nullptr, *Nd = nullptr;
  int* exp_i = nullptr;  // 1-based
  bool have_I = false, have_N = false;

  // PSFs
  int nps = 0, nexppsf = 0, psfconst = 0;
  double* G = nullptr;       // (nps, nps, E) real
  double* Gamma = nullptr;   // (nps, nps)
  double* rot = nullptr;     // host copy of angles (E)
  double2* Gt = nullptr;     // (nps, nps, E) complex
  double2* Gammat = nullptr; // (nps, nps)
  bool have_psf = false, have_spectra = false;
  double C_a = 0;

  // system
  imcom::DMat A, Q, B, P, T, Pt;  // Pt = P / (L + K_a), the T GEMM operand
  double* L = nullptr;
  double *K = nullptr, *US = nullptr, *H = nullptr, *S = nullptr, *U = nullptr;
  int* nev = nullptr;
  int* flags = nullptr;  // device status word(s)
  bool have_A = false, have_QL = false, have_B = false, have_P = false,
       have_K = false, have_T = false, have_Pt = false;
  int max_exp = 0;  // largest exp_i

  // tables and FFT scratch (kept between calls of the same size)
  double* tables = nullptr;
  size_t tables_bytes = 0;
  double2* fftbuf = nullptr;
  size_t fftbuf_bytes = 0;
  int table_fft = IMCOM_TABLE_FFT_AUTO;  // inverse FFT of the lookup tables
  double2* fft_tw = nullptr;              // exp(2 pi i t / L) of the own table FFT
  size_t fft_tw_bytes = 0;
  int fft_tw_L = 0;
  double2* r2c_tw = nullptr;              // exp(2 pi i t / nps) of the own PSF transform
  size_t r2c_tw_bytes = 0;
  int r2c_tw_L = 0;
  // work area bound to the shared cuFFT plans when this context runs them
  void* fft_work = nullptr;
  size_t fft_work_bytes = 0;

  int8_t* band = nullptr;   // eigenmode band indices of the learned-kappa features
  size_t band_bytes = 0;
  int kappa_feat = 1;       // IMCOM_OPT_KAPPA_FEATURES
  float2* nbr = nullptr;    // per pixel: neighbour count and exposures (valid for these inputs)
  size_t nbr_bytes = 0;
  bool nbr_valid = false;
  int* band_seg = nullptr;  // first eigenmode of bands 0..8, then a non-monotone flag
  size_t band_seg_bytes = 0;
  int* fb = nullptr;        // per-pixel fallback flags of the learned bisection
  size_t fb_bytes = 0;
  void* train_buf = nullptr;  // MLP training data and state
  size_t train_bytes = 0;
  void* gemm_ws = nullptr;  // split-K partial sums
  size_t gemm_ws_bytes = 0;

  // split-precision products (IMCOM_PREC_SPLIT)
  int prec = IMCOM_PREC_FP64;
  int bisect_kernel = IMCOM_BISECT_AUTO;
  int bisect_ctas = 0;  // CTAs per SM of the streaming pixel kernels (0: automatic)
  int sm_share = 0;     // SMs for persistent / cooperative grids (0: the whole device)
  int tail_ctas = 0;    // cluster of the tridiagonalisation tail (0 auto, -1 none, 8, 16)
  int stack_kernel = IMCOM_STACKS_AUTO;  // kernel of imcom_gpu_build_images
  void* jac_buf = nullptr;  // batched Jacobi: matrices, vectors, values, status
  size_t jac_bytes = 0;
  int split_SP = 7, split_ST = 6;        // digit slices of the P and T products
  double split_tol_us = 1e-7, split_tol_t = 1e-8;
  imcom::SplitOp sq_P, sq_T, sb_P, spt_T;  // Q columns, Q rows, B, P~
  bool sq_P_valid = false, sq_T_valid = false;
  double sq_T_norm = 0.0;  // 2-norm of the row scales of Q
  bool p_split = false;    // the resident P came from the split product
  bool p_audited = false, t_audited = false;  // sp_flag holds the audit's verdicts
  double* sp_margin = nullptr;  // per pixel: smallest distance of f to a decision threshold
  double* sp_est = nullptr;     // per pixel: U/S bound, T-from-P bound, T-product bound
  int* sp_flag = nullptr;
  int* sp_list = nullptr;
  size_t sp_margin_bytes = 0, sp_est_bytes = 0, sp_flag_bytes = 0, sp_list_bytes = 0;
  imcom::DMat fbX, fbY;  // gathered columns for the FP64 recomputation
  imcom::DMat stacks, stack_H;  // image stacks I (n x s) and H = T^T I (m x s)
  double split_info[8] = {};

  imcom::EigWork* eig = nullptr;
  imcom::MlpWeights mlp;
  float* feat = nullptr;
  float2* guess = nullptr;  // learned-kappa network outputs per pixel
  int kappa_nonet = 0;      // IMCOM_OPT_KAPPA_START: 1 = no network (Newton from mid-range)

  // capacity in bytes of every buffer grown by ensure_vec, keyed by the
  // address of the context field that holds its pointer
  std::unordered_map<void**, size_t> vec_cap;

  cudaEvent_t tab_ev[2][2] = {};  // around the last A (0) and B (1) table build
  bool tab_used[2] = {};
  cudaEvent_t ev0[imcom::ST_N] = {}, ev1[imcom::ST_N] = {};
  bool ev_used[imcom::ST_N] = {};
};

namespace imcom {

int set_err(imcom_ctx* c, int code, const char* fmt, ...);

#define IMC_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return ::imcom::set_err(ctx, IMCOM_ERR_CUDA, "%s: %s (%s:%d)", #call,   \
                              cudaGetErrorString(e_), __FILE__, __LINE__);    \
  } while (0)

extern unsigned long long g_launches;

#define IMC_LAUNCH()                                                          \
  do {                                                                        \
    __atomic_fetch_add(&::imcom::g_launches, 1ULL, __ATOMIC_RELAXED);         \
    cudaError_t e_ = cudaGetLastError();                                      \
    if (e_ != cudaSuccess)                                                    \
      return ::imcom::set_err(ctx, IMCOM_ERR_CUDA, "kernel launch: %s (%s:%d)",\
                              cudaGetErrorString(e_), __FILE__, __LINE__);    \
  } while (0)

#define IMC_CUFFT(call)                                                       \
  do {                                                                        \
    cufftResult r_ = (call);                                                  \
    if (r_ != CUFFT_SUCCESS)                                                  \
      return ::imcom::set_err(ctx, IMCOM_ERR_LIBRARY, "%s: cufft status %d",  \
                              #call, (int)r_);                                \
  } while (0)

#define IMC_TRY(expr)                                                         \
  do {                                                                        \
    int s_ = (expr);                                                          \
    if (s_ != 0) return s_;                                                   \
  } while (0)

// (Re)allocate a device matrix of the given shape; keeps the buffer when it
// is already large enough.  ensure_vec likewise keeps a vector whose buffer
// already holds `count` elements (the contents are not preserved on growth).
int ensure_mat(imcom_ctx* ctx, DMat& M, long long rows, long long cols);
// The lookup tables' inverse 2-D FFT in two pruned, fused passes
// (table_fft.cu); *done is false (and nothing is launched) for sides it does
// not take, which then go through cuFFT.
// The PSF spectra's forward real-to-complex transform of `count` n x n
// images (in) into half spectra ((n/2 + 1) x n each, k fastest), with H
// ((n/2 + 1) x n complex per image) as scratch (table_fft.cu); *done is false
// (and nothing is launched) for sides the own line transforms do not cover.
int psf_r2c_own(imcom_ctx* ctx, int n, int count, const double* in, double2* H, double2* half,
                bool* done);
// Whether table_fft_inverse takes its register path for these sides.
bool table_fft_fast(int nps, int L);
int table_fft_inverse(imcom_ctx* ctx, int nps, int L, int ntab, const int2* dpairs, double2* W,
                      double* tab, int isB, bool* done);
int ensure_buf(imcom_ctx* ctx, void** p, size_t& have, size_t need);
// Held around every device allocation and free, every cuFFT plan creation
// and every stream capture of the process.  cudaFree synchronises the device
// and cuFFT's planning allocates and frees; either one in a thread while
// another thread captures a graph can fail or invalidate the capture, so
// contexts on several host threads take turns at them.  Recursive: a capture
// may allocate.
std::recursive_mutex& alloc_mutex();
// `batch` contiguous 2-D side x side transforms on the context's stream
// through the process-wide plan cache: in place complex-to-complex
// (dir = CUFFT_FORWARD / CUFFT_INVERSE), or real side^2 -> side*(side/2+1)
// complex.  fft_attach/fft_free count the contexts sharing the plans.
int fft_z2z(imcom_ctx* ctx, int side, int batch, double2* data, int dir);
int fft_d2z(imcom_ctx* ctx, int side, int batch, const double* in, double2* out);
void fft_attach();
void fft_free(imcom_ctx* ctx);
template <class T>
int ensure_vec(imcom_ctx* ctx, T** p, size_t count);

int upload_mat(imcom_ctx* ctx, DMat& M, const double* host, long long rows,
               long long cols);
int download_mat(imcom_ctx* ctx, const DMat& M, double* host);

void stage_begin(imcom_ctx* ctx, Stage s);
void stage_end(imcom_ctx* ctx, Stage s);

// Number of SMs of the context's device (cached).
int sm_count(imcom_ctx* ctx);

// ---- kernels exported between translation units ----
// FP64 GEMM: C (M x N) = alpha * op(A) * op(B) + beta * C, column-major.
// transA: 'N' (A is M x K, ld lda) or 'T' (A is K x M).  transB: 'N' (B is
// K x N) or 'T' (B is N x K).
// C (M x M, lower triangle and the tiles crossing the diagonal) = alpha A B^T
// + beta C with A, B M x K column-major (the symmetric rank-2k update).
// C (M x 32) = A (M x K) B (K x 32), 'N', 'N' (a tile for 32 output columns).
int dgemm_nn_skinny32(imcom_ctx* ctx, long long M, long long K, const double* A, long long lda,
                      const double* B, long long ldb, double* C, long long ldc);
int dgemm_lower_nt(imcom_ctx* ctx, long long M, long long K, double alpha, const double* A,
                   long long lda, const double* B, long long ldb, double beta, double* C,
                   long long ldc);
int dgemm(imcom_ctx* ctx, char transA, char transB, long long M, long long N,
          long long K, double alpha, const double* A, long long lda,
          const double* B, long long ldb, double beta, double* C,
          long long ldc);

int eigen_dc(imcom_ctx* ctx, const DMat& A, DMat& W, double* w);

// Split-precision products (ozaki.cu).  split_operand slices the operand
// rows of X (cols: row r = column r of X; else row r of X) into S digits
// for row blocks of R (128: A operand, 64: B operand); split_gemm forms
// C = alpha * A B^T (C column-major, M = A rows, N = B rows).
int split_operand(imcom_ctx* ctx, const double* X, long long ld, long long rows, long long K,
                  bool cols, int S, int R, SplitOp& op);
int split_gemm(imcom_ctx* ctx, const SplitOp& a, const SplitOp& b, double alpha, double* C,
               long long ldc);
long long split_max_k(int S);
// The GEMM's bounded waits OR an error code into a device word; it is
// zeroed before a split stage and checked after the stage's last sync.
int split_reset_error(imcom_ctx* ctx);
int split_check_error(imcom_ctx* ctx);
void split_free(SplitOp& op);
void split_release(imcom_ctx* ctx);  // split.cu
int build_P_split(imcom_ctx* ctx);
int build_T_split(imcom_ctx* ctx);
int eigen_jacobi(imcom_ctx* ctx, const DMat& A, DMat& Q, double* L);
int eigen_library(imcom_ctx* ctx, const DMat& A, DMat& Q, double* L);
void eig_free(imcom_ctx* ctx);

}  // namespace imcom
