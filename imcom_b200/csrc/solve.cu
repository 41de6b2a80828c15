// solve.cu -- P = Q^T B, per-pixel kappa bisection, T and the output maps.
//
//   imcom_gpu_build_P      imcom_build_P       imcom_matrix.f90:682-712
//   bisect_kernel          imcom_bisect_kappa  imcom_bisect.f90:78-170
//                          imcom_bisect_by_U   imcom_bisect.f90:174-222
//                          imcom_bisect_by_S   imcom_bisect.f90:226-267
//   imcom_gpu_build_T      imcom_build_T       imcom_matrix.f90:716-750
//   image_s_kernel         imcom_build_image   imcom_matrix.f90:754-790
//                          imcom_build_S       imcom_matrix.f90:839-877
//   eval_kernel            imcom_build_U       imcom_matrix.f90:795-835
//
// The bisection runs one warp per output pixel; the eigenvalues and the
// pixel's P column are staged in shared memory and every U/S evaluation is a
// warp-wide sum (usum.cuh).  Its epilogue also writes the T operand
// P~(:, a) = P(:, a) / (L + K_a) (the DGEMV argument of imcom_matrix.f90:734),
// so T = -1/2 Q P~ is a single FP64 GEMM.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "solve.cuh"
#include "usum.cuh"

namespace imcom {

namespace {

__global__ void __launch_bounds__(128, 7) bisect_kernel(BisectArgs a, PixelSmem plan) {
  extern __shared__ __align__(16) double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* lam = a.L;
  if (plan.lam_smem) {
    for (int p = threadIdx.x; p < a.n; p += blockDim.x) smem[p] = a.L[p];
    __syncthreads();
    lam = smem;
  }
  double* mycol = plan.col_smem ? smem + (size_t)a.n * (1 + warp) : nullptr;
  const int total = a.list ? a.count : a.m;
  for (int t = blockIdx.x * plan.warps + warp; t < total; t += gridDim.x * plan.warps) {
    const int pix = a.list ? a.list[t] : t;
    const double* col = a.P + (size_t)pix * a.ldp;
    if (mycol) {
      for (int p = lane; p < a.n; p += 32) mycol[p] = col[p];
      __syncwarp();
      col = mycol;
    }
    int nev;
    double k, us, mg;
    const StreamCol ev{lam, col, a.Nd, a.n, a.UnotS != 0, a.C};
    bisect_pixel(a, ev, lane, &nev, &k, &us, &mg);
    write_pixel(a, lam, a.P + (size_t)pix * a.ldp, pix, lane, nev, k, us, mg);
    __syncwarp();
  }
}

// Bisection with the pixel's column resident in its warp (n <= RES_MAX_N):
// one CTA per SM, pixels handed out by an atomic counter.
__global__ void __launch_bounds__(RES_WARPS_PLAIN * 32, 1) bisect_res_kernel(BisectArgs a,
                                                                            int* counter) {
  extern __shared__ __align__(16) double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int p = threadIdx.x; p < a.n; p += blockDim.x) smem[p] = a.L[p];
  __syncthreads();
  double* smw = smem + RES_MAX_N + (size_t)warp * RES_S * 32;
  ResCol rc;
  rc.lam = smem;
  rc.n = a.n;
  rc.jn = (a.n + 31) / 32;
  rc.U = a.UnotS != 0;
  rc.C = a.C;
  const int total = a.list ? a.count : a.m;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(counter, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= total) break;
    const int pix = a.list ? a.list[t] : t;
    const double* col = a.P + (size_t)pix * a.ldp;
    rc.load(col, a.Nd, lane, smw);
    __syncwarp();
    int nev;
    double k, us, mg;
    bisect_pixel(a, rc, lane, &nev, &k, &us, &mg);
    write_pixel(a, smem, col, pix, lane, nev, k, us, mg);
    __syncwarp();
  }
}

// U_a or S_a at the given K_a (one evaluation per pixel).
__global__ void eval_kernel(BisectArgs a, PixelSmem plan, double* __restrict__ out) {
  extern __shared__ __align__(16) double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* lam = a.L;
  if (plan.lam_smem) {
    for (int p = threadIdx.x; p < a.n; p += blockDim.x) smem[p] = a.L[p];
    __syncthreads();
    lam = smem;
  }
  for (int pix = blockIdx.x * plan.warps + warp; pix < a.m; pix += gridDim.x * plan.warps) {
    const double* col = a.P + (size_t)pix * a.ldp;
    double v = warp_us(a.UnotS != 0, lam, col, a.Nd, a.n, a.K[pix], a.C, lane);
    if (lane == 0) out[pix] = v;
  }
}

// H(:, s) = T^T I(:, s) for the stacks s0 .. s0+SG-1 of this grid row
// (blockIdx.y), streaming T once per pass.  Each warp holds STK_CPW columns
// of T; each lane takes the rows k = k0 + lane + 32 j of a chunk of STK_KC
// rows and keeps STK_CPW x SG partial sums in registers, so one T value
// (from HBM) serves SG stacks and one stack value (from shared memory)
// serves STK_CPW columns.  The chunk of the stacks is staged stack-major
// (Is[s][k]) so that a warp's 32 lanes read 32 consecutive doubles; rows past
// n and stacks past S are zero-filled and add nothing.  The next chunk's T
// values are loaded before the current chunk is summed.
constexpr int STK_WARPS = 4, STK_CPW = 4, STK_KC = 128, STK_J = STK_KC / 32;
constexpr int STK_COLS = STK_WARPS * STK_CPW;  // columns of T per CTA

template <int SG>
__global__ void __launch_bounds__(STK_WARPS * 32, 3)
stacks_kernel(const double* __restrict__ T, long long ldt, const double* __restrict__ I,
              long long ldi, double* __restrict__ H, long long ldh, int n, int m, int S) {
  __shared__ double Is[SG * STK_KC];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s0 = blockIdx.y * SG;
  const int sg = min(SG, S - s0);
  const long long a0 = ((long long)blockIdx.x * STK_WARPS + warp) * STK_CPW;
  const double* tcol[STK_CPW];
  bool cv[STK_CPW];
#pragma unroll
  for (int c = 0; c < STK_CPW; ++c) {
    cv[c] = a0 + c < m;
    tcol[c] = T + (cv[c] ? a0 + c : 0) * ldt;
  }
  double acc[STK_CPW][SG];
#pragma unroll
  for (int c = 0; c < STK_CPW; ++c)
#pragma unroll
    for (int s = 0; s < SG; ++s) acc[c][s] = 0.0;

  double tn[STK_J][STK_CPW];
  auto load_t = [&](int k0) {
#pragma unroll
    for (int j = 0; j < STK_J; ++j) {
      const int k = k0 + lane + 32 * j;
#pragma unroll
      for (int c = 0; c < STK_CPW; ++c) tn[j][c] = (cv[c] && k < n) ? __ldg(tcol[c] + k) : 0.0;
    }
  };
  load_t(0);
  for (int k0 = 0; k0 < n; k0 += STK_KC) {
    double tc[STK_J][STK_CPW];
#pragma unroll
    for (int j = 0; j < STK_J; ++j)
#pragma unroll
      for (int c = 0; c < STK_CPW; ++c) tc[j][c] = tn[j][c];
    if (k0 + STK_KC < n) load_t(k0 + STK_KC);
    __syncthreads();  // every warp is done with the previous chunk of Is
    for (int e = threadIdx.x; e < SG * STK_KC; e += blockDim.x) {
      const int s = e / STK_KC, kk = e - s * STK_KC;
      const int k = k0 + kk;
      Is[e] = (s < sg && k < n) ? I[k + (long long)(s0 + s) * ldi] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < STK_J; ++j) {
      const int kk = lane + 32 * j;
#pragma unroll
      for (int s = 0; s < SG; ++s) {
        const double iv = Is[s * STK_KC + kk];
#pragma unroll
        for (int c = 0; c < STK_CPW; ++c) acc[c][s] = fma(tc[j][c], iv, acc[c][s]);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < STK_CPW; ++c)
#pragma unroll
    for (int s = 0; s < SG; ++s) {
      double v = acc[c][s];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      // every lane holds the sum; one lane per (column, stack) writes it
      if (((c * SG + s) & 31) == lane && cv[c] && s < sg)
        H[(a0 + c) + (long long)(s0 + s) * ldh] = v;
    }
}

// H_a = sum_i T_ia I_i and S_a = sum_i T_ia (T_ia Ndiag_i), one warp per a.
__global__ void image_s_kernel(const double* __restrict__ T, long long ldt,
                               const double* __restrict__ I, const double* __restrict__ Nd,
                               int n, int m, double* __restrict__ H, double* __restrict__ S) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int a = blockIdx.x * wpb + warp; a < m; a += gridDim.x * wpb) {
    const double* col = T + (size_t)a * ldt;
    double h = 0.0, s = 0.0;
    for (int i = lane; i < n; i += 32) {
      double t = col[i];
      if (H) h += t * I[i];
      if (S) s = __dadd_rn(s, __dmul_rn(t, __dmul_rn(t, Nd[i])));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      h += __shfl_xor_sync(0xffffffffu, h, o);
      s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if (lane == 0) {
      if (H) H[a] = h;
      if (S) S[a] = s;
    }
  }
}

}  // namespace

int fill_bisect_args(imcom_ctx* ctx, BisectArgs& a, int UnotS, double US_max, double k_min,
                     double k_max, double tol, int maxnits, double C_a) {
  if (!ctx->have_P) return set_err(ctx, IMCOM_ERR_STATE, "P has not been built or loaded");
  if (!ctx->have_QL) return set_err(ctx, IMCOM_ERR_STATE, "L has not been built or loaded");
  if (!UnotS && !ctx->have_N)
    return set_err(ctx, IMCOM_ERR_STATE, "S-mode bisection needs Ndiag (imcom_gpu_set_inputs)");
  if (!(k_min > 0.0)) return -4;
  if (!(k_max > 0.0)) return -5;
  if (maxnits < 0) return -7;
  if (!(C_a > 0.0) || !std::isfinite(C_a)) return -8;
  a.L = ctx->L;
  a.P = ctx->P.p;
  a.ldp = ctx->P.ld;
  a.Nd = ctx->Nd;
  a.Pt = ctx->Pt.p;
  a.ldt = ctx->Pt.ld;
  a.K = ctx->K;
  a.US = ctx->US;
  a.nev = ctx->nev;
  a.margin = nullptr;
  a.list = nullptr;
  a.count = 0;
  a.n = ctx->n;
  a.m = ctx->m;
  a.UnotS = UnotS ? 1 : 0;
  a.US_max = US_max;
  a.k_min = k_min;
  a.k_max = k_max;
  a.tol = tol;
  a.C = C_a;
  a.eps = 1.1102230246251565e-16;  // DLAMCH('Espilon') (imcom_bisect.f90:187)
  a.lg_min = std::log10(k_min);
  a.lg_max = std::log10(k_max);
  a.maxnits = maxnits;
  return 0;
}

// Pixels in flight: every pixel's warp streams its P column at each U/S
// evaluation, so the columns of the pixels resident at once should fit in L2
// (an explicit IMCOM_OPT_BISECT_CTAS_PER_SM wins).
constexpr double kPixelL2Budget = 80.0 * 1024 * 1024;

int pixel_grid(imcom_ctx* ctx, const PixelSmem& plan, int m) {
  int blocks = (m + plan.warps - 1) / plan.warps;
  int per_sm = ctx->bisect_ctas;
  if (per_sm <= 0 && !plan.col_smem) {
    const double col = (double)ctx->n * sizeof(double) * plan.warps;  // one CTA's columns
    per_sm = std::max(1, (int)(kPixelL2Budget / (col * sm_count(ctx))));
  }
  if (per_sm > 0) blocks = std::min(blocks, per_sm * sm_count(ctx));
  return blocks;
}

int launch_bisect(imcom_ctx* ctx, const BisectArgs& a) {
  const int total = a.list ? a.count : a.m;
  if (total <= 0) return 0;
  if (use_resident(ctx->bisect_kernel, ctx->n)) {
    int* counter = ctx->flags + 24;
    IMC_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), ctx->stream));
    const size_t bytes = res_smem_bytes(RES_WARPS_PLAIN);
    IMC_CUDA(cudaFuncSetAttribute(bisect_res_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)bytes));
    const int grid = std::min(sm_count(ctx), (total + RES_WARPS_PLAIN - 1) / RES_WARPS_PLAIN);
    bisect_res_kernel<<<grid, RES_WARPS_PLAIN * 32, bytes, ctx->stream>>>(a, counter);
    IMC_LAUNCH();
    return 0;
  }
  PixelSmem plan = plan_pixel_smem(ctx->n);
  IMC_CUDA(cudaFuncSetAttribute(bisect_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kPixelSmemMax));
  bisect_kernel<<<pixel_grid(ctx, plan, total), plan.warps * 32, plan.bytes, ctx->stream>>>(a,
                                                                                          plan);
  IMC_LAUNCH();
  return 0;
}

int copy_pixel_outputs(imcom_ctx* ctx, double* K_out, double* US_out, int* nev_out) {
  int m = ctx->m;
  if (K_out)
    IMC_CUDA(cudaMemcpyAsync(K_out, ctx->K, m * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (US_out)
    IMC_CUDA(cudaMemcpyAsync(US_out, ctx->US, m * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream));
  if (nev_out)
    IMC_CUDA(cudaMemcpyAsync(nev_out, ctx->nev, m * sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->stream));
  if (K_out || US_out || nev_out) IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

}  // namespace imcom

using namespace imcom;

extern "C" int imcom_gpu_build_P(imcom_ctx* ctx, double* P_out) {
  if (!ctx) return -1;
  if (!ctx->have_QL) return set_err(ctx, IMCOM_ERR_STATE, "Q has not been built or loaded");
  if (!ctx->have_B) return set_err(ctx, IMCOM_ERR_STATE, "B has not been built or loaded");
  cudaSetDevice(ctx->device);
  stage_begin(ctx, ST_P);
  IMC_TRY(ensure_mat(ctx, ctx->P, ctx->n, ctx->m));
  if (ctx->prec == IMCOM_PREC_SPLIT) {
    IMC_TRY(build_P_split(ctx));
  } else {
    // P = Q^T B (DGEMM 'T', 'N', n, m, n)
    IMC_TRY(dgemm(ctx, 'T', 'N', ctx->n, ctx->m, ctx->n, 1.0, ctx->Q.p, ctx->Q.ld, ctx->B.p,
                  ctx->B.ld, 0.0, ctx->P.p, ctx->P.ld));
    ctx->p_split = false;
    ctx->p_audited = ctx->t_audited = false;
  }
  stage_end(ctx, ST_P);
  ctx->have_P = true;
  ctx->have_K = ctx->have_T = ctx->have_Pt = false;
  if (P_out) {
    IMC_TRY(download_mat(ctx, ctx->P, P_out));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->p_split) IMC_TRY(split_check_error(ctx));
  }
  return 0;
}

extern "C" int imcom_gpu_bisect_kappa(imcom_ctx* ctx, int UnotS, double US_max, double k_min,
                                      double k_max, double tol, int maxnits, double C_a,
                                      double* K_out, double* US_out, int* nevals_out) {
  if (!ctx) return -1;
  BisectArgs a;
  IMC_TRY(fill_bisect_args(ctx, a, UnotS, US_max, k_min, k_max, tol, maxnits, C_a));
  cudaSetDevice(ctx->device);
  stage_begin(ctx, ST_BISECT);
  IMC_TRY(ensure_mat(ctx, ctx->Pt, ctx->n, ctx->m));
  a.Pt = ctx->Pt.p;
  a.ldt = ctx->Pt.ld;
  if (ctx->p_split) IMC_TRY(split_margin_buffer(ctx, a));
  IMC_TRY(launch_bisect(ctx, a));
  if (ctx->p_split) IMC_TRY(split_audit(ctx, a));
  stage_end(ctx, ST_BISECT);
  ctx->have_K = true;
  ctx->have_Pt = true;
  ctx->have_T = false;
  return copy_pixel_outputs(ctx, K_out, US_out, nevals_out);
}

extern "C" int imcom_gpu_build_T(imcom_ctx* ctx, double* T_out) {
  if (!ctx) return -1;
  if (!ctx->have_K) return set_err(ctx, IMCOM_ERR_STATE, "kappa has not been solved or loaded");
  if (!ctx->have_QL || !ctx->have_P)
    return set_err(ctx, IMCOM_ERR_STATE, "Q, L and P are needed for T");
  cudaSetDevice(ctx->device);
  stage_begin(ctx, ST_T);
  if (!ctx->have_Pt) {
    IMC_TRY(make_Pt(ctx));
    ctx->have_Pt = true;
  }
  IMC_TRY(ensure_mat(ctx, ctx->T, ctx->n, ctx->m));
  if (ctx->prec == IMCOM_PREC_SPLIT) {
    IMC_TRY(build_T_split(ctx));
  } else {
    // T = -1/2 Q P~ with P~(:, a) = P(:, a) / (L + K_a) written by the bisection.
    IMC_TRY(dgemm(ctx, 'N', 'N', ctx->n, ctx->m, ctx->n, -0.5, ctx->Q.p, ctx->Q.ld, ctx->Pt.p,
                  ctx->Pt.ld, 0.0, ctx->T.p, ctx->T.ld));
    ctx->split_info[3] = 0.0;
    ctx->split_info[6] = 0.0;
    ctx->t_audited = false;
  }
  stage_end(ctx, ST_T);
  ctx->have_T = true;
  if (T_out) {
    IMC_TRY(download_mat(ctx, ctx->T, T_out));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}

// P~ from a loaded K (used when kappa came from imcom_gpu_load_K).
namespace imcom {
namespace {
__global__ void scale_cols_kernel(const double* __restrict__ P, long long ldp,
                                  const double* __restrict__ L, const double* __restrict__ K,
                                  double* __restrict__ Pt, long long ldt, int n, int m) {
  int a = blockIdx.y;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    Pt[p + (size_t)a * ldt] = __ddiv_rn(P[p + (size_t)a * ldp], __dadd_rn(L[p], K[a]));
}
}  // namespace

int make_Pt(imcom_ctx* ctx) {
  IMC_TRY(ensure_mat(ctx, ctx->Pt, ctx->n, ctx->m));
  dim3 grd((ctx->n + 255) / 256, ctx->m);
  scale_cols_kernel<<<grd, 256, 0, ctx->stream>>>(ctx->P.p, ctx->P.ld, ctx->L, ctx->K, ctx->Pt.p,
                                                  ctx->Pt.ld, ctx->n, ctx->m);
  IMC_LAUNCH();
  return 0;
}
}  // namespace imcom

extern "C" int imcom_gpu_build_image(imcom_ctx* ctx, double* H_out) {
  if (!ctx) return -1;
  if (!ctx->have_T) return set_err(ctx, IMCOM_ERR_STATE, "T has not been built or loaded");
  if (!ctx->have_I) return set_err(ctx, IMCOM_ERR_STATE, "I_i was not given to set_inputs");
  cudaSetDevice(ctx->device);
  stage_begin(ctx, ST_EPI);
  int blocks = (ctx->m + 7) / 8;
  image_s_kernel<<<blocks, 256, 0, ctx->stream>>>(ctx->T.p, ctx->T.ld, ctx->I, ctx->Nd, ctx->n,
                                                  ctx->m, ctx->H, nullptr);
  IMC_LAUNCH();
  stage_end(ctx, ST_EPI);
  if (H_out) {
    IMC_CUDA(cudaMemcpyAsync(H_out, ctx->H, ctx->m * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}

// H = T^T I for many image stacks that share T's geometry and mask (the
// production pattern of reusing one T, built or read from the cache, for
// every stack observed with the same dithers and PSFs).  Per stack it is
// imcom_build_image (imcom_matrix.f90:754-790); for all stacks together it is
// one FP64 GEMM (M = m, N = stacks, K = n) in which T crosses HBM once
// instead of once per stack.
template <int SG>
static int launch_stacks(imcom_ctx* ctx, int nstack, const double* dI, long long ldi, double* dH,
                         long long ldh) {
  const dim3 grid((unsigned)((ctx->m + STK_COLS - 1) / STK_COLS),
                  (unsigned)((nstack + SG - 1) / SG));
  stacks_kernel<SG><<<grid, STK_WARPS * 32, 0, ctx->stream>>>(ctx->T.p, ctx->T.ld, dI, ldi, dH,
                                                              ldh, ctx->n, ctx->m, nstack);
  IMC_LAUNCH();
  return 0;
}

static int build_images(imcom_ctx* ctx, int nstack, const double* dI, long long ldi,
                        double* dH, long long ldh) {
  stage_begin(ctx, ST_EPI);
  // the streaming kernel passes over T once per 8 stacks (~45 us each at
  // n = m = 4096), the GEMM's time is flat at ~215 us up to 64 stacks
  const bool stream = ctx->stack_kernel == IMCOM_STACKS_STREAM ||
                      (ctx->stack_kernel == IMCOM_STACKS_AUTO && nstack <= IMCOM_STACKS_STREAM_MAX);
  if (stream) {
    // passes of at most 8 stacks: 4 x 8 partial sums and two 4 x 4 blocks of
    // T values per lane fill the register budget of three CTAs per SM
    if ((nstack + 7) / 8 > 65535)
      return set_err(ctx, IMCOM_ERR_STATE, "%d stacks exceed one streaming launch", nstack);
    if (nstack == 1)
      IMC_TRY(launch_stacks<1>(ctx, nstack, dI, ldi, dH, ldh));
    else if (nstack == 2)
      IMC_TRY(launch_stacks<2>(ctx, nstack, dI, ldi, dH, ldh));
    else if (nstack <= 4)
      IMC_TRY(launch_stacks<4>(ctx, nstack, dI, ldi, dH, ldh));
    else
      IMC_TRY(launch_stacks<8>(ctx, nstack, dI, ldi, dH, ldh));
  } else {
    IMC_TRY(dgemm(ctx, 'T', 'N', ctx->m, nstack, ctx->n, 1.0, ctx->T.p, ctx->T.ld, dI, ldi, 0.0,
                  dH, ldh));
  }
  stage_end(ctx, ST_EPI);
  return 0;
}

extern "C" int imcom_gpu_build_images(imcom_ctx* ctx, int nstack, const double* I_stack,
                                      double* H_out) {
  if (!ctx) return -1;
  if (nstack < 0) return -2;
  if (!I_stack && nstack > 0) return -3;
  if (!ctx->have_T) return set_err(ctx, IMCOM_ERR_STATE, "T has not been built or loaded");
  if (nstack == 0) return 0;
  cudaSetDevice(ctx->device);
  IMC_TRY(upload_mat(ctx, ctx->stacks, I_stack, ctx->n, nstack));
  IMC_TRY(ensure_mat(ctx, ctx->stack_H, ctx->m, nstack));
  IMC_TRY(build_images(ctx, nstack, ctx->stacks.p, ctx->stacks.ld, ctx->stack_H.p,
                       ctx->stack_H.ld));
  if (H_out) IMC_TRY(download_mat(ctx, ctx->stack_H, H_out));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

extern "C" int imcom_gpu_build_images_device(imcom_ctx* ctx, int nstack, const double* dI,
                                             long long ldi, double* dH, long long ldh) {
  if (!ctx) return -1;
  if (nstack < 0) return -2;
  if (nstack > 0 && !dI) return -3;
  if (ldi < ctx->n || ldi < 1) return -4;
  if (nstack > 0 && !dH) return -5;
  if (ldh < ctx->m || ldh < 1) return -6;
  if (!ctx->have_T) return set_err(ctx, IMCOM_ERR_STATE, "T has not been built or loaded");
  if (nstack == 0) return 0;
  cudaSetDevice(ctx->device);
  return build_images(ctx, nstack, dI, ldi, dH, ldh);
}

extern "C" int imcom_gpu_build_S(imcom_ctx* ctx, double* S_out) {
  if (!ctx) return -1;
  if (!ctx->have_T) return set_err(ctx, IMCOM_ERR_STATE, "T has not been built or loaded");
  if (!ctx->have_N) return set_err(ctx, IMCOM_ERR_STATE, "Ndiag was not given to set_inputs");
  cudaSetDevice(ctx->device);
  int blocks = (ctx->m + 7) / 8;
  image_s_kernel<<<blocks, 256, 0, ctx->stream>>>(ctx->T.p, ctx->T.ld, ctx->I, ctx->Nd, ctx->n,
                                                  ctx->m, nullptr, ctx->S);
  IMC_LAUNCH();
  if (S_out) {
    IMC_CUDA(cudaMemcpyAsync(S_out, ctx->S, ctx->m * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}

extern "C" int imcom_gpu_build_U(imcom_ctx* ctx, double C_a, double* U_out) {
  if (!ctx) return -1;
  if (!ctx->have_K) return set_err(ctx, IMCOM_ERR_STATE, "kappa has not been solved or loaded");
  BisectArgs a;
  IMC_TRY(fill_bisect_args(ctx, a, 1, 0.0, 1.0, 1.0, 0.0, 0, C_a));
  cudaSetDevice(ctx->device);
  PixelSmem plan = plan_pixel_smem(ctx->n);
  plan.col_smem = false;
  plan.bytes = plan.lam_smem ? (size_t)ctx->n * sizeof(double) : 0;
  IMC_CUDA(cudaFuncSetAttribute(eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kPixelSmemMax));
  eval_kernel<<<pixel_grid(ctx, plan, ctx->m), plan.warps * 32, plan.bytes, ctx->stream>>>(
      a, plan, ctx->U);
  IMC_LAUNCH();
  if (U_out) {
    IMC_CUDA(cudaMemcpyAsync(U_out, ctx->U, ctx->m * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}
