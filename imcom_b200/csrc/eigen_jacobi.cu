// eigen_jacobi.cu -- one-sided (Hestenes) Jacobi eigensolver for small
// positive semi-definite systems, batched: one CTA per matrix, with the
// matrix and the accumulated rotations held in shared memory.
//
// The reference calls LAPACK DSYEVR (imcom_matrix.f90:617-643).  IMCOM's A is
// a Gram matrix of PSF overlaps (positive semi-definite) whose eigenvalues
// span many decades, and U and Sigma are set by the smallest of them; Jacobi
// methods compute those to high relative accuracy (Demmel & Veselic, "Jacobi's
// method is more accurate than QR", SIAM J. Matrix Anal. Appl. 13, 1992),
// which a tridiagonal reduction does not promise.
//
// Method (Hestenes 1958; the parallel ordering of Brent & Luk 1985):
//   G = A, V = I.  A sweep visits every column pair (p, q) once, in n'-1
//   rounds of n'/2 disjoint pairs (n' = n rounded up to even; the round-robin
//   "circle" ordering), one warp per pair:
//     alpha = g_p.g_p, beta = g_q.g_q, gamma = g_p.g_q;
//     if |gamma| > tol sqrt(alpha beta):
//       zeta = (beta - alpha) / (2 gamma), t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)),
//       c = 1 / sqrt(1 + t^2), s = c t;
//       (g_p, g_q) <- (c g_p - s g_q, s g_p + c g_q), the same for (v_p, v_q).
//   Sweeps repeat until one rotates nothing (at most max_sweeps; an error
//   status otherwise).  Then G = A V has orthogonal columns; for symmetric A
//   g_i = lambda_i v_i, and lambda_i = v_i.g_i keeps the sign.  The pairs are
//   returned in ascending order of lambda (the caller reverses them, as for
//   the other solvers).
//
// Limits: n <= JAC_MAX (G and V fill the shared memory); eigenvalue pairs
// +lambda, -lambda of an indefinite matrix are not separated (A is positive
// semi-definite here).
#include <cmath>
#include <vector>

#include "common.cuh"
#include "eigen.cuh"

namespace imcom {
namespace {

constexpr int JAC_THREADS = 512;
constexpr int JAC_MAX = IMCOM_JACOBI_MAX_N;
constexpr int JAC_MAX_SWEEPS = 60;

__device__ __forceinline__ double jwarp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Matrix b of the batch: A_b at A + b strideA (column-major, lda); output
// eigenvectors (ascending) at Q + b strideQ (ldq), eigenvalues at
// L + b strideL.  status[b] = sweeps used, or -1 if it did not converge.
__global__ void __launch_bounds__(JAC_THREADS, 1)
jacobi_kernel(const double* __restrict__ A, long long lda, long long strideA, int n,
              double* __restrict__ Q, long long ldq, long long strideQ,
              double* __restrict__ L, long long strideL, int* __restrict__ status) {
  extern __shared__ __align__(16) double jsm[];
  double* G = jsm;                   // n x n, column-major, ld n
  double* V = G + (size_t)n * n;     // n x n
  double* lam = V + (size_t)n * n;   // n
  __shared__ int rotated;
  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NW = JAC_THREADS / 32;
  const double* Ab = A + (size_t)b * strideA;
  for (int idx = tid; idx < n * n; idx += JAC_THREADS) {
    const int r = idx % n, c = idx / n;
    G[idx] = Ab[r + (long long)c * lda];
    V[idx] = (r == c) ? 1.0 : 0.0;
  }
  const int np = n + (n & 1);  // players of the round-robin (one idle when n is odd)
  const int m = np - 1;        // rotating players; player m is fixed
  const double tol = 2.0 * 1.1102230246251565e-16 * sqrt((double)n);
  int sweeps = 0;
  bool converged = (n <= 1);
  __syncthreads();
  while (!converged && sweeps < JAC_MAX_SWEEPS) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int s = 0; s < m; ++s) {
      // round s: (m, s) and ((s + k) mod m, (s - k) mod m), k = 1 .. np/2 - 1
      for (int k = wid; k < np / 2; k += NW) {
        int p, q;
        if (k == 0) {
          p = s;
          q = m;
        } else {
          p = (s + k) % m;
          q = (s - k + m) % m;
        }
        if (p > q) {
          const int t0 = p;
          p = q;
          q = t0;
        }
        if (q >= n) continue;  // the idle player
        double* gp = G + (size_t)p * n;
        double* gq = G + (size_t)q * n;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int r = lane; r < n; r += 32) {
          const double x = gp[r], y = gq[r];
          al = fma(x, x, al);
          be = fma(y, y, be);
          ga = fma(x, y, ga);
        }
        al = jwarp_sum(al);
        be = jwarp_sum(be);
        ga = jwarp_sum(ga);
        if (ga == 0.0 || !(fabs(ga) > tol * sqrt(al * be))) continue;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
        double* vp = V + (size_t)p * n;
        double* vq = V + (size_t)q * n;
        for (int r = lane; r < n; r += 32) {
          const double x = gp[r], y = gq[r];
          gp[r] = c * x - sn * y;
          gq[r] = sn * x + c * y;
          const double u = vp[r], w = vq[r];
          vp[r] = c * u - sn * w;
          vq[r] = sn * u + c * w;
        }
        if (lane == 0) rotated = 1;
      }
      __syncthreads();
    }
    ++sweeps;
    converged = (rotated == 0);
    __syncthreads();  // every thread has read `rotated` before the next sweep resets it
  }
  if (tid == 0) status[b] = converged ? sweeps : -1;
  // lambda_i = v_i . g_i
  for (int i = wid; i < n; i += NW) {
    double acc = 0.0;
    for (int r = lane; r < n; r += 32) acc = fma(V[(size_t)i * n + r], G[(size_t)i * n + r], acc);
    acc = jwarp_sum(acc);
    if (lane == 0) lam[i] = acc;
  }
  __syncthreads();
  // ascending order: the rank of lambda_i (ties by index) is its output slot
  double* Qb = Q + (size_t)b * strideQ;
  double* Lb = L + (size_t)b * strideL;
  for (int i = wid; i < n; i += NW) {
    const double li = lam[i];
    int rank = 0;
    for (int j = lane; j < n; j += 32) {
      const double lj = lam[j];
      rank += (lj < li || (lj == li && j < i)) ? 1 : 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rank += __shfl_xor_sync(0xffffffffu, rank, o);
    if (lane == 0) Lb[rank] = li;
    for (int r = lane; r < n; r += 32) Qb[r + (long long)rank * ldq] = V[(size_t)i * n + r];
  }
}

size_t jacobi_smem(int n) { return (2 * (size_t)n * n + n) * sizeof(double); }

int launch_jacobi(imcom_ctx* ctx, const double* A, long long lda, long long strideA, int n,
                  int count, double* Q, long long ldq, long long strideQ, double* L,
                  long long strideL, int* status) {
  if (n > JAC_MAX)
    return set_err(ctx, IMCOM_ERR_STATE,
                   "the Jacobi eigensolver takes n <= %d (shared memory); n = %d", JAC_MAX, n);
  const size_t smem = jacobi_smem(n);
  // the largest size's need: the attribute is process-wide (see usum.cuh)
  IMC_CUDA(cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)jacobi_smem(JAC_MAX)));
  jacobi_kernel<<<count, JAC_THREADS, smem, ctx->stream>>>(A, lda, strideA, n, Q, ldq, strideQ, L,
                                                           strideL, status);
  IMC_LAUNCH();
  return 0;
}

int check_jacobi(imcom_ctx* ctx, const int* status_dev, int count, int* sweeps_host) {
  std::vector<int> st((size_t)count);
  IMC_CUDA(cudaMemcpyAsync(st.data(), status_dev, (size_t)count * sizeof(int),
                           cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int b = 0; b < count; ++b) {
    if (sweeps_host) sweeps_host[b] = st[b];
    if (st[b] < 0)
      return set_err(ctx, IMCOM_ERR_EIGEN, "Jacobi eigensolver: matrix %d did not converge in %d "
                     "sweeps", b, JAC_MAX_SWEEPS);
  }
  return 0;
}

}  // namespace

int eigen_jacobi(imcom_ctx* ctx, const DMat& A, DMat& Q, double* L) {
  const int n = (int)A.rows;
  int* status = ctx->flags + 44;  // one slot: a single matrix
  IMC_TRY(launch_jacobi(ctx, A.p, A.ld, 0, n, 1, Q.p, Q.ld, 0, L, 0, status));
  return check_jacobi(ctx, status, 1, nullptr);
}

}  // namespace imcom

using namespace imcom;

// Batched eigendecomposition of `count` small symmetric positive semi-definite
// matrices (n <= IMCOM_JACOBI_MAX_N) on host arrays; see the header.
extern "C" int imcom_gpu_eigh_jacobi_batched(imcom_ctx* ctx, int n, int count, const double* A,
                                             double* Q, double* L, int* sweeps) {
  if (!ctx) return -1;
  if (n < 1 || n > JAC_MAX) return -2;
  if (count < 1) return -3;
  if (!A) return -4;
  if (!Q) return -5;
  if (!L) return -6;
  cudaSetDevice(ctx->device);
  const size_t nn = (size_t)n * n, mats = nn * (size_t)count;
  const size_t need = (2 * mats + (size_t)n * count) * sizeof(double) + (size_t)count * sizeof(int) +
                      256;
  IMC_TRY(ensure_buf(ctx, &ctx->jac_buf, ctx->jac_bytes, need));
  double* dA = (double*)ctx->jac_buf;
  double* dQ = dA + mats;
  double* dL = dQ + mats;
  int* dst = (int*)(dL + (size_t)n * count);
  IMC_CUDA(cudaMemcpyAsync(dA, A, mats * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  IMC_TRY(launch_jacobi(ctx, dA, n, (long long)nn, n, count, dQ, n, (long long)nn, dL, n, dst));
  IMC_CUDA(cudaMemcpyAsync(Q, dQ, mats * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(L, dL, (size_t)n * count * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
  return check_jacobi(ctx, dst, count, sweeps);
}
