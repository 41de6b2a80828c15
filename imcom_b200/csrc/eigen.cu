// eigen.cu -- eigendecomposition of A (imcom_eigen_A, imcom_matrix.f90:586-678).
//
// The reference calls LAPACK DSYEVR('V', 'A', 'U') and reverses the result
// into descending eigenvalue order (:656-662), then reports
// condition = max(L) / min(L) (:664-671).  Four solvers sit behind one entry
// point (imcom_gpu_set_option(IMCOM_OPT_EIGENSOLVER)):
//   IMCOM_EIGH_DC       own FP64 blocked Householder tridiagonalisation +
//                       divide and conquer + back-transformation (eigen_dc.cu)
//   IMCOM_EIGH_JACOBI   own FP64 one-sided Jacobi for small systems, n <= 112
//                       (eigen_jacobi.cu)
//   IMCOM_EIGH_TWOSTAGE the same divide and conquer and back-transformation
//                       after a two-stage reduction, dense -> band -> tridiagonal
//                       (eigen_2s.cu)
//   IMCOM_EIGH_LIBRARY  cuSOLVER syevd, kept only as a comparison baseline.
// All of them return ascending eigenpairs in a work matrix; reverse_kernel
// writes them to Q and L in the reference's descending order.
#include <cusolverDn.h>

#include <cmath>
#include <vector>

#include "common.cuh"
#include "eigen.cuh"

namespace imcom {

namespace {

__global__ void reverse_kernel(const double* __restrict__ W, long long ldw,
                               const double* __restrict__ w, double* __restrict__ Q,
                               long long ldq, double* __restrict__ L, int n) {
  int j = blockIdx.y;  // destination column
  int src = n - 1 - j;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    Q[i + (size_t)j * ldq] = W[i + (size_t)src * ldw];
  if (blockIdx.x == 0 && threadIdx.x == 0) L[j] = w[src];
}

__global__ void copy_mat_kernel(const double* __restrict__ A, long long lda, double* __restrict__ B,
                                long long ldb, int rows, int cols) {
  int j = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x)
    B[i + (size_t)j * ldb] = A[i + (size_t)j * lda];
  (void)cols;
}

}  // namespace

int copy_mat(imcom_ctx* ctx, const double* A, long long lda, double* B, long long ldb, int rows,
             int cols) {
  if (rows <= 0 || cols <= 0) return 0;
  dim3 grd((rows + 255) / 256, cols);
  copy_mat_kernel<<<grd, 256, 0, ctx->stream>>>(A, lda, B, ldb, rows, cols);
  IMC_LAUNCH();
  return 0;
}

void eig_free(imcom_ctx* ctx) {
  if (!ctx->eig) return;
  EigWork* w = ctx->eig;
  std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
  if (w->W.p) cudaFree(w->W.p);
  if (w->w) cudaFree(w->w);
  if (w->Z.p) cudaFree(w->Z.p);
  if (w->V.p) cudaFree(w->V.p);
  if (w->U.p) cudaFree(w->U.p);
  if (w->buf) cudaFree(w->buf);
  if (w->solver) cusolverDnDestroy((cusolverDnHandle_t)w->solver);
  if (w->trd_exec) cudaGraphExecDestroy((cudaGraphExec_t)w->trd_exec);
  delete w;
  ctx->eig = nullptr;
}

EigWork* eig_work(imcom_ctx* ctx) {
  if (!ctx->eig) ctx->eig = new EigWork();
  return ctx->eig;
}

int eig_buf(imcom_ctx* ctx, size_t bytes) {
  EigWork* w = eig_work(ctx);
  return ensure_buf(ctx, &w->buf, w->buf_bytes, bytes);
}

int eigen_library(imcom_ctx* ctx, const DMat& A, DMat& W, double* w) {
  EigWork* ew = eig_work(ctx);
  int n = (int)A.rows;
  if (!ew->solver) {
    cusolverDnHandle_t h;
    if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS)
      return set_err(ctx, IMCOM_ERR_LIBRARY, "cusolverDnCreate failed");
    ew->solver = h;
  }
  cusolverDnHandle_t h = (cusolverDnHandle_t)ew->solver;
  cusolverDnSetStream(h, ctx->stream);
  IMC_TRY(copy_mat(ctx, A.p, A.ld, W.p, W.ld, n, n));
  int lwork = 0;
  if (cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, W.p,
                                  (int)W.ld, w, &lwork) != CUSOLVER_STATUS_SUCCESS)
    return set_err(ctx, IMCOM_ERR_LIBRARY, "cusolverDnDsyevd_bufferSize failed");
  IMC_TRY(eig_buf(ctx, (size_t)lwork * sizeof(double) + 256));
  double* work = (double*)ew->buf;
  int* info = ctx->flags + 8;
  if (cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, W.p, (int)W.ld, w,
                       work, lwork, info) != CUSOLVER_STATUS_SUCCESS)
    return set_err(ctx, IMCOM_ERR_LIBRARY, "cusolverDnDsyevd failed");
  int hinfo = 0;
  IMC_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (hinfo != 0)
    return set_err(ctx, IMCOM_ERR_EIGEN, "IMCOM ERROR: Internal error in eigensolver (info=%d)",
                   hinfo);
  return 0;
}

}  // namespace imcom

using namespace imcom;

extern "C" int imcom_gpu_eigen_A(imcom_ctx* ctx, double* Q_out, double* L_out, double* cond_out) {
  if (!ctx) return -1;
  if (!ctx->have_A) return set_err(ctx, IMCOM_ERR_STATE, "A has not been built or loaded");
  cudaSetDevice(ctx->device);
  int n = ctx->n;
  EigWork* ew = eig_work(ctx);
  stage_begin(ctx, ST_EIG);
  IMC_TRY(ensure_mat(ctx, ew->W, n, n));
  IMC_TRY(ensure_mat(ctx, ctx->Q, n, n));
  IMC_TRY(ensure_vec_keep(ctx, &ew->w, ew->w_cap, (size_t)n));
  int st;
  switch (ctx->eig_mode) {
    case IMCOM_EIGH_LIBRARY: st = eigen_library(ctx, ctx->A, ew->W, ew->w); break;
    case IMCOM_EIGH_JACOBI: st = eigen_jacobi(ctx, ctx->A, ew->W, ew->w); break;
    default: st = eigen_dc(ctx, ctx->A, ew->W, ew->w); break;
  }
  if (st) return st;
  // Reverse into descending order (imcom_matrix.f90:656-662).
  dim3 grd((n + 255) / 256, n);
  reverse_kernel<<<grd, 256, 0, ctx->stream>>>(ew->W.p, ew->W.ld, ew->w, ctx->Q.p, ctx->Q.ld,
                                                ctx->L, n);
  IMC_LAUNCH();
  stage_end(ctx, ST_EIG);
  ctx->have_QL = true;
  ctx->sq_P_valid = ctx->sq_T_valid = false;
  ctx->have_P = ctx->have_K = ctx->have_T = ctx->have_Pt = false;
  std::vector<double> hL(n);
  IMC_CUDA(cudaMemcpyAsync(hL.data(), ctx->L, n * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
  if (Q_out) IMC_TRY(download_mat(ctx, ctx->Q, Q_out));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  double lmax = hL[0], lmin = hL[0];
  for (int k = 1; k < n; ++k) {
    lmax = std::max(lmax, hL[k]);
    lmin = std::min(lmin, hL[k]);
  }
  if (L_out) std::copy(hL.begin(), hL.end(), L_out);
  if (cond_out) *cond_out = lmax / lmin;  // imcom_matrix.f90:664
  return 0;
}
