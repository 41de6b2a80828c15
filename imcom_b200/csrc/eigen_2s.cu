// eigen_2s.cu -- two-stage reduction of a symmetric matrix to tridiagonal
// form: dense -> band (bandwidth SB) by blocked Householder QR of panels and
// two-sided block updates on the FP64 DMMA GEMM, then band -> tridiagonal by
// bulge chasing.  Alternative to the one-stage dsytrd of eigen_dc.cu for the
// eigensolver that replaces DSYEVR in imcom_eigen_A (imcom_matrix.f90:617-643).
//
// Stage 1 (LAPACK dsytrd_sy2sb structure, lower): for the panel of columns
// k .. k+SB-1 the rows k+SB .. n-1 are factorised, P = Q R with
// Q = I - V T V^T; R goes into the band below the diagonal block, and the
// trailing matrix A22 = A(k+SB:, k+SB:) (full symmetric storage) becomes
// Q^T A22 Q through
//     W = A22 V T,  W <- W - 1/2 V (T^T (V^T W)),  A22 <- A22 - V W^T - W V^T.
// The panel QR runs in one thread-block cluster: each CTA holds a slice of
// the panel's rows in shared memory, and every column needs one cluster-wide
// exchange of its partial sums (the column's norm below the pivot, its dot
// products with the later columns, and the pivot row) through distributed
// shared memory.
#include <algorithm>
#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "common.cuh"
#include "eigen.cuh"

namespace imcom {

namespace {

constexpr int SB = 32;            // bandwidth of the first stage (panel width)
constexpr int SB_CTAS = 16;       // CTAs of the panel cluster (8 where 16 cannot be placed)
constexpr int SB_THREADS = 256;   // 32 columns x 8 row slices
constexpr int SB_SLICES = SB_THREADS / SB;

struct PanelArgs {
  double* A;       // full symmetric working matrix
  long long lda;
  double* V;       // reflectors: column k + j, rows k + SB ..; 1 at the pivot, 0 above
  long long ldv;
  double* tau;     // tau[k + j]
  int n, k, per;   // panel columns k .. k + SB - 1; rows per CTA
};

// Householder QR of the panel A(k+SB : n, k : k+SB) (LAPACK dgeqr2 with
// dlarfg's conventions) by a cluster of CTAs.  CTA q holds panel rows
// q*per .. q*per + per - 1 in shared memory (column-major, stride per).  For
// column j every CTA forms, over its rows, S_c = sum_{i > j} P(i,j) P(i,c)
// (c >= j; S_j is the squared norm below the pivot) and contributes the pivot
// row R_c = P(j, c) if it holds it; the 2 SB values of every CTA are stored
// into every CTA's shared memory (alternating buffers by column parity) and
// summed after one cluster barrier.  Then, in every CTA,
//   beta = -sign(alpha) sqrt(alpha^2 + S_j), tau = (beta - alpha) / beta,
//   v = [1; P(j+1:, j) / (alpha - beta)],  w_c = tau (R_c + S_c / (alpha - beta)),
// and the later columns are updated, P(:, c) -= v w_c.
__global__ void __launch_bounds__(SB_THREADS, 1) sb_panel_kernel(PanelArgs a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int q = (int)cl.block_rank(), nct = (int)cl.num_blocks();
  const int N = a.n - a.k - SB;  // panel rows
  const int per = a.per;
  const int rb = q * per, nr = max(0, min(per, N - rb));
  const int jmax = min(SB, N);
  extern __shared__ __align__(16) double psm[];
  double* P = psm;                                   // [SB][per]
  double* part = P + (size_t)SB * per;               // [2][SB_CTAS][2 SB] from every CTA
  double* red = part + 2 * SB_CTAS * 2 * SB;         // [SB_SLICES][2 SB]
  double* fin = red + SB_SLICES * 2 * SB;            // [2 SB] cluster totals
  const int c = threadIdx.x & (SB - 1), slice = threadIdx.x / SB;
  const size_t row0 = (size_t)a.k + SB + rb;
  for (int e = threadIdx.x; e < SB * nr; e += SB_THREADS) {
    const int cc = e / nr, i = e - cc * nr;
    P[(size_t)cc * per + i] = a.A[row0 + i + (size_t)(a.k + cc) * a.lda];
  }
  cl.sync();  // every CTA runs before any stores into its shared memory
  for (int j = 0; j < jmax; ++j) {
    double sdot = 0.0, rowv = 0.0;
    if (c >= j) {
      const double* pj = P + (size_t)j * per;
      const double* pc = P + (size_t)c * per;
      for (int i = slice; i < nr; i += SB_SLICES) {
        const int gi = rb + i;
        if (gi > j) sdot = fma(pj[i], pc[i], sdot);
        else if (gi == j) rowv = pc[i];
      }
    }
    red[slice * 2 * SB + c] = sdot;
    red[slice * 2 * SB + SB + c] = rowv;
    __syncthreads();
    double* mine = part + (size_t)(j & 1) * SB_CTAS * 2 * SB;
    if (threadIdx.x < 2 * SB) {
      double s = 0.0;
      for (int h = 0; h < SB_SLICES; ++h) s += red[h * 2 * SB + threadIdx.x];
      for (int r = 0; r < nct; ++r) cl.map_shared_rank(mine, r)[q * 2 * SB + threadIdx.x] = s;
    }
    cl.sync();
    if (threadIdx.x < 2 * SB) {
      double s = 0.0;
      for (int r = 0; r < nct; ++r) s += mine[r * 2 * SB + threadIdx.x];
      fin[threadIdx.x] = s;
    }
    __syncthreads();
    const double alpha = fin[SB + j], sig2 = fin[j];
    double t = 0.0, beta = alpha, scl = 0.0;
    if (sig2 != 0.0) {
      beta = -copysign(sqrt(alpha * alpha + sig2), alpha);
      t = (beta - alpha) / beta;
      scl = 1.0 / (alpha - beta);
    }
    if (c > j) {
      const double w = t * (fin[SB + c] + scl * fin[c]);
      const double* pj = P + (size_t)j * per;
      double* pc = P + (size_t)c * per;
      for (int i = slice; i < nr; i += SB_SLICES) {
        const int gi = rb + i;
        if (gi > j) pc[i] -= (pj[i] * scl) * w;
        else if (gi == j) pc[i] -= w;
      }
    }
    __syncthreads();
    if (c == j) {
      // column j: v below the pivot (kept in P until the write-back), beta on it
      double* pj = P + (size_t)j * per;
      for (int i = slice; i < nr; i += SB_SLICES) {
        const int gi = rb + i;
        if (gi > j) pj[i] *= scl;
        else if (gi == j) pj[i] = beta;
      }
    }
    if (q == 0 && threadIdx.x == 0) a.tau[a.k + j] = t;
    __syncthreads();
  }
  if (q == 0 && threadIdx.x < SB && threadIdx.x >= jmax) a.tau[a.k + threadIdx.x] = 0.0;
  // write back: R on and above the pivot into the band, zeros below; v into V
  for (int e = threadIdx.x; e < SB * nr; e += SB_THREADS) {
    const int cc = e / nr, i = e - cc * nr;
    const int gi = rb + i;
    const double p = P[(size_t)cc * per + i];
    const size_t col = (size_t)(a.k + cc);
    a.A[row0 + i + col * a.lda] = gi <= cc ? p : 0.0;
    a.V[row0 + i + col * a.ldv] = gi < cc ? 0.0 : (gi == cc ? 1.0 : p);
  }
}

inline size_t panel_smem(int per) {
  return ((size_t)SB * per + 2 * SB_CTAS * 2 * SB + SB_SLICES * 2 * SB + 2 * SB) * sizeof(double);
}

// T (upper triangular, ld SB) of the panel's block reflector from its Gram
// matrix G = V^T V (ld SB) and tau (LAPACK dlarft, forward, columnwise):
// T(j,j) = tau_j, T(0:j, j) = -tau_j T(0:j, 0:j) G(0:j, j).  One warp.
__global__ void sb_larft_kernel(const double* __restrict__ G, const double* __restrict__ tau,
                                double* __restrict__ T) {
  __shared__ double sT[SB][SB + 1];
  const int r = threadIdx.x;
  for (int cc = 0; cc < SB; ++cc) sT[r][cc] = 0.0;
  __syncwarp();
  for (int j = 0; j < SB; ++j) {
    const double tj = tau[j];
    double s = 0.0;
    if (r < j)
      for (int h = r; h < j; ++h) s += sT[r][h] * G[h + j * SB];
    __syncwarp();
    if (r < j) sT[r][j] = -tj * s;
    if (r == j) sT[j][j] = tj;
    __syncwarp();
  }
  for (int cc = 0; cc < SB; ++cc) T[r + cc * SB] = sT[r][cc];
}

// Band storage for the second stage: AB[d + c * ldb] = A(c + d, c) for
// d <= SB, zero for SB < d < ldb.
__global__ void band_extract_kernel(const double* __restrict__ A, long long lda, int n,
                                    double* __restrict__ AB, int ldb) {
  const int c = blockIdx.x;
  for (int d = threadIdx.x; d < ldb; d += blockDim.x)
    AB[d + (size_t)c * ldb] = (d <= SB && c + d < n) ? A[(c + d) + (size_t)c * lda] : 0.0;
}

}  // namespace

// X = [V(:, k:k+b) | W(:, 0:b)], Y = [W | V] (eigen_dc.cu)
__global__ void pack_update_kernel(const double* __restrict__ V, long long ldv,
                                   const double* __restrict__ W, long long ldw, int t0, int n,
                                   int b, double* __restrict__ X, double* __restrict__ Y,
                                   long long ldx);

// Cluster size for the panel kernel: 16 CTAs where the device can place them
// (non-portable size), else 8.
static int panel_cluster(imcom_ctx* ctx, int per, int* ctas) {
  const size_t smem = panel_smem(per);
  IMC_CUDA(cudaFuncSetAttribute(sb_panel_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
  // the device's ceiling, not this panel's need: the attribute is process-wide
  IMC_CUDA(cudaFuncSetAttribute(sb_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - 1024));
  for (int cs : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(SB_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, (void*)sb_panel_kernel, &cfg) == cudaSuccess &&
        nc >= 1) {
      *ctas = cs;
      return 0;
    }
  }
  cudaGetLastError();
  return set_err(ctx, IMCOM_ERR_CUDA, "the band reduction's panel cluster cannot be placed");
}

// Dense -> band: A (full symmetric, n x n, ld) is overwritten by the band
// matrix (bandwidth SB) below the diagonal and garbage elsewhere; the
// reflectors of panel p go to V (columns p SB ..), their tau to tau and the
// block reflectors' T factors (SB x SB each, column-major) to Tf.  AB
// receives the band in the storage of the second stage (ldb rows).
int sy2sb_gpu(imcom_ctx* ctx, DMat& Aw, DMat& V, double* tau, double* Tf, double* W,
              long long ldw, double* XY, double* AB, int ldb) {
  const int n = (int)Aw.rows;
  const long long ld = Aw.ld;
  IMC_CUDA(cudaMemsetAsync(V.p, 0, V.bytes(), ctx->stream));
  // cluster shape for the largest panel (rows per CTA fixed by it)
  int ctas = 16;
  const int Nmax = std::max(0, n - SB);
  int per = std::max(1, (Nmax + 15) / 16);
  {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    if (panel_smem(per) > (size_t)optin - 1024)
      return set_err(ctx, IMCOM_ERR_CUDA, "band reduction: panel of %d rows does not fit", Nmax);
  }
  IMC_TRY(panel_cluster(ctx, per, &ctas));
  if (ctas != 16) per = std::max(1, (Nmax + ctas - 1) / ctas);
  if (ctas != 16 && panel_smem(per) > 227 * 1024 - 1024)
    return set_err(ctx, IMCOM_ERR_CUDA, "band reduction: panel of %d rows does not fit", Nmax);
  double* G = Tf + (size_t)((n + SB - 1) / SB) * SB * SB;  // SB x SB Gram scratch
  double* M = G + SB * SB;                                   // SB x SB
  double* M2 = M + SB * SB;
  for (int k = 0; k + SB < n - 1; k += SB) {
    const int N = n - k - SB;
    const int pc = std::max(1, (N + ctas - 1) / ctas);
    PanelArgs pa{Aw.p, ld, V.p, V.ld, tau, n, k, pc};
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(SB_THREADS);
    cfg.dynamicSmemBytes = panel_smem(pc);
    cfg.stream = ctx->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    IMC_CUDA(cudaLaunchKernelEx(&cfg, sb_panel_kernel, pa));
    IMC_LAUNCH();
    const size_t r0 = (size_t)k + SB;
    const double* Vp = V.p + r0 + (size_t)k * V.ld;  // N x SB
    double* T = Tf + (size_t)(k / SB) * SB * SB;
    double* A22 = Aw.p + r0 + r0 * (size_t)ld;
    // T from G = V^T V
    IMC_TRY(dgemm(ctx, 'T', 'N', SB, SB, N, 1.0, Vp, V.ld, Vp, V.ld, 0.0, G, SB));
    sb_larft_kernel<<<1, SB, 0, ctx->stream>>>(G, tau + k, T);
    IMC_LAUNCH();
    // W = A22 V T (the first product into XY as scratch)
    double* X1 = XY;
    IMC_TRY(dgemm(ctx, 'N', 'N', N, SB, N, 1.0, A22, ld, Vp, V.ld, 0.0, X1, ldw));
    IMC_TRY(dgemm(ctx, 'N', 'N', N, SB, SB, 1.0, X1, ldw, T, SB, 0.0, W, ldw));
    // W -= 1/2 V (T^T (V^T W))
    IMC_TRY(dgemm(ctx, 'T', 'N', SB, SB, N, 1.0, Vp, V.ld, W, ldw, 0.0, M, SB));
    IMC_TRY(dgemm(ctx, 'T', 'N', SB, SB, SB, 1.0, T, SB, M, SB, 0.0, M2, SB));
    IMC_TRY(dgemm(ctx, 'N', 'N', N, SB, SB, -0.5, Vp, V.ld, M2, SB, 1.0, W, ldw));
    // A22 -= [V W] [W V]^T
    double* X = XY;
    double* Y = XY + (size_t)ldw * 2 * SB;
    dim3 grd((N + 255) / 256, SB);
    pack_update_kernel<<<grd, 256, 0, ctx->stream>>>(Vp - r0, V.ld, W - r0, ldw, (int)r0, n, SB,
                                                     X - r0, Y - r0, ldw);
    IMC_LAUNCH();
    IMC_TRY(dgemm(ctx, 'N', 'T', N, N, 2 * SB, -1.0, X, ldw, Y, ldw, 1.0, A22, ld));
  }
  band_extract_kernel<<<n, 128, 0, ctx->stream>>>(Aw.p, ld, n, AB, ldb);
  IMC_LAUNCH();
  return 0;
}

}  // namespace imcom

using namespace imcom;

// First stage alone, for tests: the band matrix of the resident A (loaded or
// built), SB + 1 diagonals in band storage AB_out[d + c * ldb], d <= SB.
extern "C" int imcom_gpu_band_reduce(imcom_ctx* ctx, double* AB_out, int ldb) {
  if (!ctx) return -1;
  if (!AB_out) return -2;
  if (ldb < SB + 1) return -3;
  if (!ctx->have_A) return set_err(ctx, IMCOM_ERR_STATE, "A has not been built or loaded");
  cudaSetDevice(ctx->device);
  const int n = ctx->n;
  EigWork* ew = eig_work(ctx);
  IMC_TRY(ensure_mat(ctx, ew->Z, n, n));
  IMC_TRY(ensure_mat(ctx, ew->V, n, n));
  IMC_TRY(copy_mat(ctx, ctx->A.p, ctx->A.ld, ew->Z.p, ew->Z.ld, n, n));
  const long long ldw = pad_ld(n);
  const int LDB = 2 * SB;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_tau = take((size_t)n * 8), o_T = take(((size_t)(n / SB + 1) * SB * SB + 3 * SB * SB) * 8);
  const size_t o_W = take((size_t)ldw * SB * 8), o_XY = take((size_t)ldw * 4 * SB * 8);
  const size_t o_AB = take((size_t)LDB * n * 8);
  IMC_TRY(eig_buf(ctx, off + 256));
  char* base = (char*)ew->buf;
  double* AB = (double*)(base + o_AB);
  IMC_TRY(sy2sb_gpu(ctx, ew->Z, ew->V, (double*)(base + o_tau), (double*)(base + o_T),
                    (double*)(base + o_W), ldw, (double*)(base + o_XY), AB, LDB));
  IMC_CUDA(cudaMemcpy2DAsync(AB_out, (size_t)ldb * 8, AB, (size_t)LDB * 8, (size_t)(SB + 1) * 8, n,
                             cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}
