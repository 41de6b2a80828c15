// split.cu -- the split-precision solve: P = Q^T B and T = -1/2 Q P~ on the
// int8 tensor-core product (ozaki.cu), with a per-pixel error audit that
// sends the pixels whose accuracy it cannot guarantee back to FP64.
//
// Error model.  The split product of S digit slices rounds every operand
// entry to half a unit of its last digit and drops the digit products of
// diagonals >= S.  The resulting error of an element of C = A B^T has
// standard deviation c_S * sqrt(K) * u_S * scale_A(row) * scale_B(col),
// u_S = 2^(-7-8(S-1)): c_S = 0.33, 0.37, 0.41 for S = 5, 6, 7 against an
// extended-precision product of random operands (maximum 1.7), 0.34 for
// S = 7 on the n = 4096 IMCOM system against FP64 DGEMM.  Below u_7 = 2^-55
// the FP64 result itself (and the FP64 path it is compared with) rounds at
// that level, so u_S is capped at u_7.  The audit uses c = 1 and bounds of
// Z = 6 standard deviations.
//
// P audit (after the bisection, per pixel a; E_a = Z c sqrt(n) u_SP tau_a,
// sigma_p the scale of mode p, tau_a the scale of pixel a):
//   * U(kappa) - U_max moves by at most
//       G_a = E_a / (2C) * sqrt(sum_p (sigma_p P_pa w_p)^2),
//     w_p = (L_p + 2 k_min) / (L_p + k_min)^2 >= (L_p + 2k)/(L_p + k)^2 for
//     every kappa >= k_min the bisection visits (imcom_U_from_kappa,
//     imcom_matrix.f90:904-922); S-mode uses the S weights Nd_p/(L_p+k_min)^2
//     and 1/2 instead of 1/(2C) (imcom_S_from_kappa, imcom_matrix.f90:955-970);
//   * every decision of the bisection (f < 0, |f| < tol, |f| < C eps and the
//     learned bracket tests) had a margin; the pixel is kept only if its
//     smallest margin exceeds G_a (then K_a and the evaluation count equal
//     those of the FP64 P) and G_a <= tol_us |U_a|;
//   * the T column error caused by P is at most
//       E_a sqrt(sum_p sigma_p^2 / (L_p + K_a)^2) / ||P~_a||   (relative),
//     kept if <= tol_t.
// T audit (per column a of the split T product): relative error at most
//   Z c sqrt(n) u_ST tau'_a ||sigma'||_2 / ||P~_a||, kept if <= tol_t, where
//   sigma' are the row scales of Q and tau'_a the scale of P~_a.
// Pixels that fail the P audit get their P column from the FP64 DGEMM and are
// bisected again; T columns that fail the T audit come from the FP64 DGEMM.
#include <cmath>

#include "common.cuh"
#include "solve.cuh"

namespace imcom {

namespace {

constexpr double SPLIT_C = 1.0;  // standard deviation per sqrt(K) u_S (measured <= 0.41)
constexpr double SPLIT_Z = 6.0;  // standard deviations in a bound

double split_unit(int S) { return std::ldexp(1.0, -7 - 8 * ((S < 7 ? S : 7) - 1)); }

__device__ __forceinline__ double wsum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct AuditArgs {
  const double* L;
  const double* P;
  long long ldp;
  const double* Nd;
  const double* K;
  const double* US;
  const double* margin;
  const double* sq;  // mode scales of the P product (columns of Q)
  const double* sb;  // pixel scales (columns of B)
  int n, m, UnotS;
  double C, k_min, E, tol_us, tol_t;
  int* flag;
  double* est;  // est[a] U/S bound (relative), est[m + a] T bound from P
};

__global__ void p_audit_kernel(AuditArgs g) {
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const bool U = g.UnotS != 0;
  for (int a = blockIdx.x * wpb + (threadIdx.x >> 5); a < g.m; a += gridDim.x * wpb) {
    const double* col = g.P + (size_t)a * g.ldp;
    const double k = g.K[a];
    double sG = 0.0, sT = 0.0, sP = 0.0;
    for (int p = lane; p < g.n; p += 32) {
      const double l = g.L[p], pp = col[p], sp = g.sq[p];
      const double lk = l + g.k_min;
      double w = U ? (l + 2.0 * g.k_min) / (lk * lk) : g.Nd[p] / (lk * lk);
      if (!(lk > 0.0)) w = INFINITY;
      const double t1 = sp * pp * w;
      sG += t1 * t1;
      const double lkk = l + k;
      const double r = sp / lkk, q = pp / lkk;
      sT += r * r;
      sP += q * q;
    }
    sG = wsum_d(sG);
    sT = wsum_d(sT);
    sP = wsum_d(sP);
    if (lane == 0) {
      const double Ea = g.E * g.sb[a];
      const double G = Ea * sqrt(sG) * (U ? 0.5 / g.C : 0.5);
      const double eT = Ea * sqrt(sT) / sqrt(sP);
      const double us = fabs(g.US[a]);
      const bool keep = (g.margin[a] > G) && (G <= g.tol_us * us) && (eT <= g.tol_t);
      g.flag[a] = keep ? 0 : 1;
      g.est[a] = keep ? G / us : 0.0;
      g.est[g.m + a] = keep ? eT : 0.0;
    }
  }
}

// Relative error bound of the split T product per column (warp per column).
__global__ void t_audit_kernel(const double* __restrict__ Pt, long long ldt,
                               const double* __restrict__ tau, const double* __restrict__ misc,
                               int n, int m, double E, double tol, int* __restrict__ flag,
                               double* __restrict__ est) {
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const double snorm = misc[0];
  for (int a = blockIdx.x * wpb + (threadIdx.x >> 5); a < m; a += gridDim.x * wpb) {
    const double* col = Pt + (size_t)a * ldt;
    double s = 0.0;
    for (int p = lane; p < n; p += 32) s += col[p] * col[p];
    s = wsum_d(s);
    if (lane == 0) {
      const double e = E * tau[a] * snorm / sqrt(s);
      const bool keep = e <= tol;
      flag[a] = keep ? 0 : 1;
      est[a] = keep ? e : 0.0;
    }
  }
}

// out[0] = sqrt(sum v^2) (one block)
__global__ void norm2_kernel(const double* __restrict__ v, long long n, double* out) {
  __shared__ double part[32];
  double s = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) s += v[i] * v[i];
  s = wsum_d(s);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
    s = wsum_d(s);
    if (threadIdx.x == 0) out[0] = sqrt(s);
  }
}

// out[0] = max v (one block)
__global__ void max_kernel(const double* __restrict__ v, long long n, double* out) {
  __shared__ double part[32];
  double s = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) s = fmax(s, v[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
    if (threadIdx.x == 0) out[0] = s;
  }
}

// Indices a with flag[a] != 0, in increasing order (one block of 1024).
__global__ void compact_kernel(const int* __restrict__ flag, int m, int* __restrict__ list,
                               int* __restrict__ count) {
  __shared__ int wcount[32];
  __shared__ int base, total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int start = 0; start < m; start += blockDim.x) {
    const int i = start + threadIdx.x;
    const bool f = i < m && flag[i] != 0;
    const unsigned b = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcount[warp] = __popc(b);
    __syncthreads();
    if (warp == 0) {
      const int v = lane < nw ? wcount[lane] : 0;
      int inc = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      if (lane < nw) wcount[lane] = inc - v;  // exclusive prefix
      if (lane == 31) total = inc;
    }
    __syncthreads();
    if (f) list[base + wcount[warp] + __popc(b & ((1u << lane) - 1u))] = i;
    __syncthreads();
    if (threadIdx.x == 0) base += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = base;
}

__global__ void gather_cols_kernel(const double* __restrict__ src, long long lds,
                                   const int* __restrict__ list, int n, double* __restrict__ dst,
                                   long long ldd) {
  const int j = blockIdx.y;
  const double* s = src + (size_t)list[j] * lds;
  double* d = dst + (size_t)j * ldd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = s[i];
}

__global__ void scatter_cols_kernel(const double* __restrict__ src, long long lds,
                                    const int* __restrict__ list, int n, double* __restrict__ dst,
                                    long long ldd) {
  const int j = blockIdx.y;
  const double* s = src + (size_t)j * lds;
  double* d = dst + (size_t)list[j] * ldd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = s[i];
}

// misc slots after the 3 m per-pixel estimates
constexpr int MISC_SNORM = 0, MISC_MAX_US = 1, MISC_MAX_TP = 2, MISC_MAX_TG = 3;

int ensure_split_buffers(imcom_ctx* ctx) {
  const size_t m = (size_t)ctx->m;
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->sp_margin, ctx->sp_margin_bytes, m * sizeof(double)));
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->sp_est, ctx->sp_est_bytes, (3 * m + 8) * sizeof(double)));
  // [0, m): pixels whose P column the bisection audit recomputed in FP64;
  // [m, 2m): columns of T recomputed in FP64
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->sp_flag, ctx->sp_flag_bytes, 2 * m * sizeof(int)));
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->sp_list, ctx->sp_list_bytes, m * sizeof(int)));
  return 0;
}

double* misc(imcom_ctx* ctx) { return ctx->sp_est + 3 * (size_t)ctx->m; }

// Compact the flagged pixels into sp_list; returns their number on the host.
int compact(imcom_ctx* ctx, const int* flag, int* nf) {
  int* dcount = ctx->flags + 20;
  compact_kernel<<<1, 1024, 0, ctx->stream>>>(flag, ctx->m, ctx->sp_list, dcount);
  IMC_LAUNCH();
  IMC_CUDA(cudaMemcpyAsync(nf, dcount, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

// dst(:, list) = op(Q) * src(:, list) in FP64 for the nf listed columns.
int fp64_columns(imcom_ctx* ctx, char transQ, double alpha, const DMat& src, DMat& dst, int nf) {
  const int n = ctx->n;
  IMC_TRY(ensure_mat(ctx, ctx->fbX, n, nf));
  IMC_TRY(ensure_mat(ctx, ctx->fbY, n, nf));
  dim3 grd((n + 255) / 256, nf);
  gather_cols_kernel<<<grd, 256, 0, ctx->stream>>>(src.p, src.ld, ctx->sp_list, n, ctx->fbX.p,
                                                   ctx->fbX.ld);
  IMC_LAUNCH();
  IMC_TRY(dgemm(ctx, transQ, 'N', n, nf, n, alpha, ctx->Q.p, ctx->Q.ld, ctx->fbX.p, ctx->fbX.ld,
                0.0, ctx->fbY.p, ctx->fbY.ld));
  scatter_cols_kernel<<<grd, 256, 0, ctx->stream>>>(ctx->fbY.p, ctx->fbY.ld, ctx->sp_list, n,
                                                    dst.p, dst.ld);
  IMC_LAUNCH();
  return 0;
}

}  // namespace

int build_P_split(imcom_ctx* ctx) {
  const int S = ctx->split_SP, n = ctx->n, m = ctx->m;
  if (n > split_max_k(S))
    return set_err(ctx, IMCOM_ERR_SPLIT,
                   "split P: n = %d exceeds the exact int32 range of %d slices (%lld)", n, S,
                   split_max_k(S));
  if (!ctx->sq_P_valid || ctx->sq_P.S != S) {
    // A operand rows = eigenmodes = columns of Q
    IMC_TRY(split_operand(ctx, ctx->Q.p, ctx->Q.ld, n, n, true, S, 128, ctx->sq_P));
    ctx->sq_P_valid = true;
  }
  IMC_TRY(split_reset_error(ctx));
  IMC_TRY(split_operand(ctx, ctx->B.p, ctx->B.ld, m, n, true, S, 128, ctx->sb_P));
  IMC_TRY(split_gemm(ctx, ctx->sq_P, ctx->sb_P, 1.0, ctx->P.p, ctx->P.ld));
  ctx->p_split = true;
  ctx->p_audited = ctx->t_audited = false;
  ctx->split_info[0] = S;
  ctx->split_info[2] = ctx->split_info[4] = ctx->split_info[5] = 0.0;
  ctx->split_info[7] = 1.0;
  return 0;
}

int split_margin_buffer(imcom_ctx* ctx, BisectArgs& a) {
  IMC_TRY(ensure_split_buffers(ctx));
  a.margin = ctx->sp_margin;
  return 0;
}

int split_audit(imcom_ctx* ctx, const BisectArgs& a) {
  const int n = ctx->n, m = ctx->m;
  AuditArgs g;
  g.L = ctx->L;
  g.P = ctx->P.p;
  g.ldp = ctx->P.ld;
  g.Nd = ctx->Nd;
  g.K = ctx->K;
  g.US = ctx->US;
  g.margin = ctx->sp_margin;
  g.sq = ctx->sq_P.scale;
  g.sb = ctx->sb_P.scale;
  g.n = n;
  g.m = m;
  g.UnotS = a.UnotS;
  g.C = a.C;
  g.k_min = a.k_min;
  g.E = SPLIT_Z * SPLIT_C * std::sqrt((double)n) * split_unit(ctx->sq_P.S);
  g.tol_us = ctx->split_tol_us;
  g.tol_t = ctx->split_tol_t;
  g.flag = ctx->sp_flag;
  g.est = ctx->sp_est;
  p_audit_kernel<<<(m + 7) / 8, 256, 0, ctx->stream>>>(g);
  IMC_LAUNCH();
  double* mc = misc(ctx);
  max_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->sp_est, m, mc + MISC_MAX_US);
  IMC_LAUNCH();
  max_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->sp_est + m, m, mc + MISC_MAX_TP);
  IMC_LAUNCH();
  int nf = 0;
  IMC_TRY(compact(ctx, ctx->sp_flag, &nf));
  if (nf > 0) {
    // FP64 P for the flagged pixels, then the plain bisection on them
    IMC_TRY(fp64_columns(ctx, 'T', 1.0, ctx->B, ctx->P, nf));
    BisectArgs b = a;
    b.margin = nullptr;
    b.list = ctx->sp_list;
    b.count = nf;
    IMC_TRY(launch_bisect(ctx, b));
  }
  double h[4];
  IMC_CUDA(cudaMemcpyAsync(h, mc, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_TRY(split_check_error(ctx));  // the P product's pipeline status
  ctx->p_audited = true;
  ctx->split_info[2] = nf;
  ctx->split_info[4] = h[MISC_MAX_US];
  ctx->split_info[5] = h[MISC_MAX_TP];
  return 0;
}

int build_T_split(imcom_ctx* ctx) {
  const int S = ctx->split_ST, n = ctx->n, m = ctx->m;
  if (n > split_max_k(S))
    return set_err(ctx, IMCOM_ERR_SPLIT,
                   "split T: n = %d exceeds the exact int32 range of %d slices (%lld)", n, S,
                   split_max_k(S));
  IMC_TRY(ensure_split_buffers(ctx));
  double* mc = misc(ctx);
  if (!ctx->sq_T_valid || ctx->sq_T.S != S) {
    // A operand rows = input pixels = rows of Q
    IMC_TRY(split_operand(ctx, ctx->Q.p, ctx->Q.ld, n, n, false, S, 128, ctx->sq_T));
    ctx->sq_T_valid = true;
  }
  norm2_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->sq_T.scale, n, mc + MISC_SNORM);
  IMC_LAUNCH();
  // a split P that no audit has checked yet (kappa loaded, not bisected)
  if (ctx->p_split && !ctx->p_audited) IMC_TRY(split_check_error(ctx));
  IMC_TRY(split_reset_error(ctx));
  IMC_TRY(split_operand(ctx, ctx->Pt.p, ctx->Pt.ld, m, n, true, S, 128, ctx->spt_T));
  IMC_TRY(split_gemm(ctx, ctx->sq_T, ctx->spt_T, -0.5, ctx->T.p, ctx->T.ld));
  const double E = SPLIT_Z * SPLIT_C * std::sqrt((double)n) * split_unit(S);
  double* est = ctx->sp_est + 2 * (size_t)m;
  int* tflag = ctx->sp_flag + m;
  t_audit_kernel<<<(m + 7) / 8, 256, 0, ctx->stream>>>(ctx->Pt.p, ctx->Pt.ld, ctx->spt_T.scale,
                                                        mc, n, m, E, ctx->split_tol_t, tflag,
                                                        est);
  IMC_LAUNCH();
  max_kernel<<<1, 1024, 0, ctx->stream>>>(est, m, mc + MISC_MAX_TG);
  IMC_LAUNCH();
  int nf = 0;
  IMC_TRY(compact(ctx, tflag, &nf));
  IMC_TRY(split_check_error(ctx));  // the T product's pipeline status
  if (nf > 0) IMC_TRY(fp64_columns(ctx, 'N', -0.5, ctx->Pt, ctx->T, nf));
  double h[4];
  IMC_CUDA(cudaMemcpyAsync(h, mc, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->t_audited = true;
  ctx->split_info[1] = S;
  ctx->split_info[3] = nf;
  ctx->split_info[6] = h[MISC_MAX_TG];
  return 0;
}

void split_release(imcom_ctx* ctx) {
  std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
  split_free(ctx->sq_P);
  split_free(ctx->sq_T);
  split_free(ctx->sb_P);
  split_free(ctx->spt_T);
  void* ptrs[] = {ctx->sp_margin, ctx->sp_est, ctx->sp_flag, ctx->sp_list, ctx->fbX.p,
                  ctx->fbY.p};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  ctx->sp_margin = ctx->sp_est = nullptr;
  ctx->sp_flag = ctx->sp_list = nullptr;
  ctx->fbX = DMat();
  ctx->fbY = DMat();
}

}  // namespace imcom

using namespace imcom;

extern "C" int imcom_gpu_split_pixels(imcom_ctx* ctx, int* fp64_P, int* fp64_T) {
  if (!ctx) return -1;
  const size_t m = (size_t)ctx->m;
  cudaSetDevice(ctx->device);
  if (fp64_P) {
    if (!ctx->p_audited) {
      for (size_t a = 0; a < m; ++a) fp64_P[a] = 0;
    } else {
      IMC_CUDA(cudaMemcpyAsync(fp64_P, ctx->sp_flag, m * sizeof(int), cudaMemcpyDeviceToHost,
                               ctx->stream));
    }
  }
  if (fp64_T) {
    if (!ctx->t_audited) {
      for (size_t a = 0; a < m; ++a) fp64_T[a] = 0;
    } else {
      IMC_CUDA(cudaMemcpyAsync(fp64_T, ctx->sp_flag + m, m * sizeof(int),
                               cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

extern "C" int imcom_gpu_split_info(imcom_ctx* ctx, double* info8) {
  if (!ctx) return -1;
  if (!info8) return -2;
  for (int i = 0; i < 8; ++i) info8[i] = ctx->split_info[i];
  info8[7] = ctx->p_split ? 1.0 : 0.0;
  return 0;
}
