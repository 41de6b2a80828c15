// kappa.cu -- learned kappa for the per-pixel bisection.
//
// The reference finds kappa per output pixel by log-space bisection
// (imcom_bisect_by_U / _by_S, imcom_bisect.f90:174-267).  Here a small MLP
// predicts log10(kappa) and a bracket half-width from 12 cheap per-pixel
// features; Newton steps in log10(kappa) from that start home in on the
// band where the bisection stops, two certificate evaluations cover the
// bisection's path there, and the reference's bisection sequence is then
// replayed with every decision the evaluated points settle taken for free.
// Because U(kappa) rises and S(kappa) falls monotonically in kappa, a point
// with f = U - U_max (or S - S_max) below -max(tol, C eps) settles every
// midpoint on its accept side and a point with f >= C eps every midpoint on
// its reject side (learned_pixel gives the details).  Only undecided
// midpoints are evaluated, with the plain bisection's evaluator, so K_a and
// U_a/S_a are bit-identical to the plain bisection.
//
// Features (feature-major, 12 x m, float):
//   0  inputs within a 2 x 2 px box around (X_a, Y_a)
//   1  distinct exposures among them
//   2-9  log10(sum_{p in band b} P2_p / (4 C lambda_b) + 1e-30), bands of
//        lambda / lambda_max by two decades (band 7: below 1e-14 or <= 0)
//   10 log10(US_max)
//   11 log10(lambda_max / C)
// MLP: 12 -> 64 (ReLU) -> 64 (ReLU) -> 2; weights and activations rounded to
// bf16, products accumulated in fp32.  Output 0 is log10(kappa), output 1 is
// log of the bracket half-width in decades (the host folds the target
// normalisation into the last layer).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "solve.cuh"
#include "usum.cuh"

namespace imcom {
namespace {

constexpr int NF = 12, NH = 64, NO = 2;
// packed parameters (floats): W1 | b1 | W2 | b2 | W3 | b3
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NF, OFF_W2 = OFF_B1 + NH,
              OFF_B2 = OFF_W2 + NH * NH, OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NO * NH,
              NPARAM = OFF_B3 + NO;
// device weight block: params (bf16-rounded weights) | feature mean | std
constexpr int OFF_MEAN = NPARAM, OFF_STD = NPARAM + NF, NWEIGHT = NPARAM + 2 * NF;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Band of every eigenmode: floor(-log10(L_p / L_max) / 2) clipped to 0..7
// (7 also for L_p <= 0); computed once per call instead of per pixel.
__global__ void band_index_kernel(const double* __restrict__ lam, int n,
                                  int8_t* __restrict__ band) {
  const double lmax = lam[0];  // eigenvalues are in descending order
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const double l = lam[p];
    const double r = (l > 0.0 && lmax > 0.0) ? l / lmax : 0.0;
    int b = (r > 0.0) ? (int)floor(-log10(r) * 0.5) : 7;
    band[p] = (int8_t)(b < 0 ? 0 : (b > 7 ? 7 : b));
  }
}

// Neighbour features of one pixel on one warp: the inputs within one pixel
// in x and y of (Xa, Ya), and the exposures they come from (as a bit mask).
__device__ __forceinline__ void neighbours(const double* __restrict__ x,
                                           const double* __restrict__ y,
                                           const int* __restrict__ expi, int n, double Xa,
                                           double Ya, int lane, double* cnt_out,
                                           unsigned* mask_out) {
  double cnt = 0.0;
  unsigned mask = 0u;
  for (int i = lane; i < n; i += 32) {
    double dx = x[i] - Xa, dy = y[i] - Ya;
    if (fabs(dx) < 1.0 && fabs(dy) < 1.0) {
      cnt += 1.0;
      mask |= 1u << ((expi[i] - 1) & 31);
    }
  }
  cnt = wsum(cnt);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mask |= __shfl_xor_sync(0xffffffffu, mask, o);
  *cnt_out = cnt;
  *mask_out = mask;
}

// The neighbour features of every pixel (one warp each), kept while the
// inputs stay the same: (count, number of exposures).
__global__ void neighbour_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                 const int* __restrict__ expi, int n,
                                 const double* __restrict__ X, const double* __restrict__ Y,
                                 int m, float2* __restrict__ nbr) {
  const int lane = threadIdx.x & 31;
  const int pix = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pix >= m) return;
  double cnt;
  unsigned mask;
  neighbours(x, y, expi, n, X[pix], Y[pix], lane, &cnt, &mask);
  if (lane == 0) nbr[pix] = make_float2((float)cnt, (float)__popc(mask));
}

// First eigenmode of each band: seg[k] = first p with bidx[p] >= k (k = 0..8,
// seg[8] = n), for a band index that is non-decreasing in p; seg[9] is set
// to 1 (it must be 0 before the launch) where it decreases somewhere.  With
// a non-decreasing index every seg[k] has exactly one writer.
__global__ void band_segments_kernel(const int8_t* __restrict__ bidx, int n,
                                     int* __restrict__ seg) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int b = bidx[p];
    const int prev = p > 0 ? bidx[p - 1] : -1;
    if (b < prev) {
      atomicOr(seg + 9, 1);
      continue;
    }
    for (int k = prev + 1; k <= b; ++k) seg[k] = p;
    if (p == n - 1)
      for (int k = b + 1; k <= 8; ++k) seg[k] = n;
  }
}

// Features of one pixel, every lane gets all 12.  nbr_pix (may be null):
// this pixel's entry of the neighbour table; seg (may be null): the band
// segments of band_segments_kernel, used when the band index was monotone.
__device__ void pixel_features(const double* __restrict__ x, const double* __restrict__ y,
                               const int* __restrict__ expi, int n, double Xa, double Ya,
                               const double* lam, const int8_t* __restrict__ bidx,
                               const double* col, double C, double US_max, int lane, float* f,
                               const float2* nbr_pix = nullptr, const int* seg = nullptr) {
  float cntf, nexpf;
  if (nbr_pix) {
    const float2 v = *nbr_pix;
    cntf = v.x;
    nexpf = v.y;
  } else {
    double cnt;
    unsigned mask;
    neighbours(x, y, expi, n, Xa, Ya, lane, &cnt, &mask);
    cntf = (float)cnt;
    nexpf = (float)__popc(mask);
  }
  const double lmax = lam[0];  // eigenvalues are in descending order
  double band[8];
#pragma unroll
  for (int b = 0; b < 8; ++b) band[b] = 0.0;
  if (seg && seg[9] == 0) {
    // the band index is non-decreasing: band b is the modes seg[b] .. seg[b+1]-1
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      double s = 0.0;
      for (int p = seg[b] + lane; p < seg[b + 1]; p += 32) s = fma(col[p], col[p], s);
      band[b] = s;
    }
  } else {
    for (int p = lane; p < n; p += 32) {
      const double pp = col[p];
      const int b = bidx[p];
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q == b) band[q] += pp * pp;
    }
  }
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const double s = wsum(band[b]);
    const double lc = lmax * pow(10.0, -(2.0 * b + 1.0));
    f[2 + b] = (float)log10(s / (4.0 * C * (lc > 0.0 ? lc : 1e-300)) + 1e-30);
  }
  f[0] = cntf;
  f[1] = nexpf;
  f[10] = (float)log10(fabs(US_max) + 1e-300);
  f[11] = (float)log10(fabs(lmax / C) + 1e-300);
}

// ---------------------------------------------------------------------------
// MLP inference on the tensor cores: one warp forms the outputs of 16 pixels
// with mma.sync m16n8k16 (bf16 operands, fp32 accumulation).  Layer 1 is
// [16 x 16] x [16 x 64] (12 features, zero-padded to K = 16), layer 2
// [16 x 64] x [64 x 64], layer 3 [16 x 64] x [64 x 8] (2 outputs, zero-padded
// columns).  The accumulator fragment of one layer is the operand fragment of
// the next (two 8-column tiles make one 16-wide K step), so activations stay
// in registers.  Rounding points as the training kernel and the numpy oracle:
// normalised features, weights and hidden activations in bf16, sums in fp32.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Shared-memory weights of the tensor-core forward: bf16 [out][in] rows
// (W1 padded to 16 inputs, W3 to 8 outputs), fp32 biases and normalisation.
struct MlpSmem {
  __nv_bfloat16 W1[NH][16];
  __nv_bfloat16 W2[NH][NH];
  __nv_bfloat16 W3[8][NH];
  float b1[NH], b2[NH], b3[NO], mean[NF], rstd[NF];
};

__device__ void load_mlp_smem(const float* __restrict__ W, MlpSmem& S) {
  for (int q = threadIdx.x; q < NH * 16; q += blockDim.x) {
    const int u = q / 16, k = q % 16;
    S.W1[u][k] = __float2bfloat16_rn(k < NF ? W[OFF_W1 + u * NF + k] : 0.0f);
  }
  for (int q = threadIdx.x; q < NH * NH; q += blockDim.x)
    S.W2[q / NH][q % NH] = __float2bfloat16_rn(W[OFF_W2 + q]);
  for (int q = threadIdx.x; q < 8 * NH; q += blockDim.x) {
    const int o = q / NH;
    S.W3[o][q % NH] = __float2bfloat16_rn(o < NO ? W[OFF_W3 + q] : 0.0f);
  }
  for (int q = threadIdx.x; q < NH; q += blockDim.x) {
    S.b1[q] = W[OFF_B1 + q];
    S.b2[q] = W[OFF_B2 + q];
  }
  if (threadIdx.x < NO) S.b3[threadIdx.x] = W[OFF_B3 + threadIdx.x];
  if (threadIdx.x < NF) {
    S.mean[threadIdx.x] = W[OFF_MEAN + threadIdx.x];
    S.rstd[threadIdx.x] = W[OFF_STD + threadIdx.x];
  }
}

__device__ __forceinline__ uint32_t smem_pair(const __nv_bfloat16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}

// Outputs (o0, o1) of pixels p0 .. p0+15 (feature-major feat, m pixels);
// written for pixels < m.
__device__ void mlp_forward_16(const MlpSmem& S, const float* __restrict__ feat, int m, int p0,
                               int lane, float2* __restrict__ out) {
  const int g = lane >> 2, t = lane & 3;
  auto x = [&](int row, int k) -> float {
    const int pix = p0 + row;
    if (k >= NF || pix >= m) return 0.0f;
    return (feat[(size_t)k * m + pix] - S.mean[k]) / S.rstd[k];
  };
  uint32_t a[4] = {pack_bf16(x(g, 2 * t), x(g, 2 * t + 1)),
                   pack_bf16(x(g + 8, 2 * t), x(g + 8, 2 * t + 1)),
                   pack_bf16(x(g, 2 * t + 8), x(g, 2 * t + 9)),
                   pack_bf16(x(g + 8, 2 * t + 8), x(g + 8, 2 * t + 9))};
  float h[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float bb0 = S.b1[8 * j + 2 * t], bb1 = S.b1[8 * j + 2 * t + 1];
    h[j][0] = bb0;
    h[j][1] = bb1;
    h[j][2] = bb0;
    h[j][3] = bb1;
    mma_bf16(h[j], a, smem_pair(&S.W1[8 * j + g][2 * t]), smem_pair(&S.W1[8 * j + g][2 * t + 8]));
  }
  // layer 2: the ReLU'd layer-1 tiles 2kt, 2kt+1 are the operand of K step kt
  uint32_t a2[4][4];
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const float* c0 = h[2 * kt];
    const float* c1 = h[2 * kt + 1];
    a2[kt][0] = pack_bf16(fmaxf(c0[0], 0.0f), fmaxf(c0[1], 0.0f));
    a2[kt][1] = pack_bf16(fmaxf(c0[2], 0.0f), fmaxf(c0[3], 0.0f));
    a2[kt][2] = pack_bf16(fmaxf(c1[0], 0.0f), fmaxf(c1[1], 0.0f));
    a2[kt][3] = pack_bf16(fmaxf(c1[2], 0.0f), fmaxf(c1[3], 0.0f));
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float bb0 = S.b2[8 * j + 2 * t], bb1 = S.b2[8 * j + 2 * t + 1];
    h[j][0] = bb0;
    h[j][1] = bb1;
    h[j][2] = bb0;
    h[j][3] = bb1;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
      mma_bf16(h[j], a2[kt], smem_pair(&S.W2[8 * j + g][16 * kt + 2 * t]),
               smem_pair(&S.W2[8 * j + g][16 * kt + 2 * t + 8]));
  }
  // layer 3
  float o[4] = {t == 0 ? S.b3[0] : 0.0f, t == 0 ? S.b3[1] : 0.0f, t == 0 ? S.b3[0] : 0.0f,
                t == 0 ? S.b3[1] : 0.0f};
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const float* c0 = h[2 * kt];
    const float* c1 = h[2 * kt + 1];
    const uint32_t a3[4] = {pack_bf16(fmaxf(c0[0], 0.0f), fmaxf(c0[1], 0.0f)),
                            pack_bf16(fmaxf(c0[2], 0.0f), fmaxf(c0[3], 0.0f)),
                            pack_bf16(fmaxf(c1[0], 0.0f), fmaxf(c1[1], 0.0f)),
                            pack_bf16(fmaxf(c1[2], 0.0f), fmaxf(c1[3], 0.0f))};
    mma_bf16(o, a3, smem_pair(&S.W3[g][16 * kt + 2 * t]), smem_pair(&S.W3[g][16 * kt + 2 * t + 8]));
  }
  // columns 0 and 1 (the two outputs) sit in the lanes with t = 0
  if (t == 0) {
    if (p0 + g < m) out[p0 + g] = make_float2(o[0], o[1]);
    if (p0 + g + 8 < m) out[p0 + g + 8] = make_float2(o[2], o[3]);
  }
}

constexpr int MLP_WARPS = 4;

__global__ void __launch_bounds__(MLP_WARPS * 32) mlp_infer_kernel(const float* __restrict__ W,
                                                                   const float* __restrict__ feat,
                                                                   int m,
                                                                   float2* __restrict__ out) {
  __shared__ __align__(16) MlpSmem S;
  load_mlp_smem(W, S);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int p0 = (blockIdx.x * MLP_WARPS + warp) * 16; p0 < m; p0 += gridDim.x * MLP_WARPS * 16)
    mlp_forward_16(S, feat, m, p0, lane, out);
}

// The 12 features of every pixel (one warp each), feature-major.
__global__ void features_kernel(BisectArgs a, const double* __restrict__ x,
                                const double* __restrict__ y, const int* __restrict__ expi,
                                const double* __restrict__ X, const double* __restrict__ Y,
                                const int8_t* __restrict__ bidx, const float2* __restrict__ nbr,
                                const int* __restrict__ seg, float* __restrict__ feat) {
  const int lane = threadIdx.x & 31;
  const int pix = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pix >= a.m) return;
  float f[NF];
  pixel_features(x, y, expi, a.n, X[pix], Y[pix], a.L, bidx, a.P + (size_t)pix * a.ldp, a.C,
                 a.US_max, lane, f, nbr ? nbr + pix : nullptr, seg);
  if (lane < NF) {
#pragma unroll
    for (int k = 0; k < NF; ++k)
      if (k == lane) feat[(size_t)k * a.m + pix] = f[k];
  }
}

struct LearnedExtra {
  const float2* guess;  // MLP outputs per pixel (log10 kappa, log half-width), or null
  int* fallback;
  double half_scale;  // bracket half-width = half_scale * exp(output 1), decades
  double min_half;    // smallest half-width, decades
  double margin;      // safety margin of the known-decision tests (units of U or S)
  int max_newton;     // Newton steps toward the root before the replay
};

// One pixel of the learned-kappa bisection.
//
// 1. Start from the network's log10(kappa) (the middle of the range when no
//    network is given).  When its bracket reaches the start of the range the
//    reference's first evaluation (kappa_min for U, kappa_max for S) comes
//    first, and the pixel is done if it returns there.
// 2. Newton steps in x = log10(kappa) toward f = -w/2 (w = max(tol, C eps)),
//    the middle of the band in which the bisection stops, each from one
//    evaluation of f and f' (the same U/S sum as the bisection, bit for bit,
//    with the derivative summed alongside), safeguarded to the interval the
//    evaluated points have bracketed.
// 3. Certificates: the bisection's sequence of midpoints is followed with f
//    predicted by the tangent at the last Newton point, and the last
//    midpoint predicted to be accepted and the last predicted to be rejected
//    before the one predicted to stop it are evaluated.
// Every evaluated point with f < -(max(tol, C eps) + margin) makes each
// bisection midpoint on its accept side a known accept that cannot trigger an
// exit; every point with f >= C eps + margin makes each midpoint on its
// reject side a known reject.  U(kappa) rises and S(kappa) falls
// monotonically, and the margin covers the rounding of the computed sums.
// 4. Replay of the reference's bisection sequence (imcom_bisect.f90:174-267):
//    known decisions cost nothing, the other midpoints are evaluated.  K_a,
//    U_a/S_a and the reported value are bit-identical to the plain bisection.
// The nw warps that share the evaluator run it in lock step (same values,
// same branches); warp wid 0 writes the scalars.
// guess: this pixel's network outputs, or null (start from the middle).
template <class Eval>
__device__ __forceinline__ void learned_pixel(const BisectArgs& a, const LearnedExtra& ex,
                                              const double* lam, const double* col,
                                              const Eval& ev, int pix, int lane, int wid,
                                              int nw, const float2* guess) {
  const bool U = a.UnotS != 0;
  const double rlo = a.lg_min, rhi = a.lg_max;  // the reference's search range
  double x0 = 0.5 * (rlo + rhi), hw = 0.5 * (rhi - rlo);
  if (guess) {
    const float2 o = *guess;
    if (isfinite(o.x) && isfinite(o.y)) {
      x0 = (double)o.x;
      hw = ex.half_scale * exp((double)fminf(fmaxf(o.y, -20.0f), 5.0f));
      hw = fmin(fmax(hw, ex.min_half), 4.0);
    }
  }
  int nev = 0;
  double k_root = 0.0, us = 0.0;
  const double ceps = __dmul_rn(a.C, a.eps);
  const double wband = fmax(a.tol, ceps);
  const double thr = wband + ex.margin;
  double mg = INFINITY;  // smallest decision margin over the evaluations
  double accb = U ? -INFINITY : INFINITY;  // known accept beyond this point
  double rejb = U ? INFINITY : -INFINITY;  // known reject beyond this point
  auto note = [&](double pt, double fp) {
    mg = fmin(mg, fmin(fabs(fp + thr), fabs(fp - (ceps + ex.margin))));
    if (fp < -thr) accb = U ? fmax(accb, pt) : fmin(accb, pt);
    else if (fp >= ceps + ex.margin) rejb = U ? fmin(rejb, pt) : fmax(rejb, pt);
  };
  const double k0 = U ? a.k_min : a.k_max;
  double f0 = 0.0;
  bool have_f0 = false;
  // 1. the range start first when the bracket reaches it
  if (U ? (x0 - hw <= rlo) : (x0 + hw >= rhi)) {
    us = ev(k0, lane);
    ++nev;
    f0 = __dsub_rn(us, a.US_max);
    have_f0 = true;
    mg = fmin(mg, fabs(f0));
  }
  if (have_f0 && !(f0 < 0.0)) {
    k_root = k0;
  } else {
    // 2. Newton toward the middle of the stopping band
    const double ftgt = -0.5 * wband;
    double x = fmin(fmax(x0, rlo + 1e-9 * (rhi - rlo)), rhi - 1e-9 * (rhi - rlo));
    double xc = x, fc = 0.0, gc = 0.0;
    bool conv = false;
    for (int it = 0; it < ex.max_newton; ++it) {
      double gd;
      const double fx = __dsub_rn(ev.eval_d(pow(10.0, x), lane, &gd), a.US_max);
      ++nev;
      note(x, fx);
      xc = x;
      fc = fx;
      gc = gd;
      if (fabs(fx - ftgt) <= 2.0 * wband) {
        conv = true;
        break;
      }
      // the interval of x the evaluated points leave for the target
      const double lo_x = U ? fmax(accb, rlo) : fmax(rejb, rlo);
      const double hi_x = U ? fmin(rejb, rhi) : fmin(accb, rhi);
      double xn = x - (fx - ftgt) / gd;
      if (!(gd != 0.0) || !(xn > lo_x && xn < hi_x)) xn = 0.5 * (lo_x + hi_x);
      if (!(xn > rlo && xn < rhi) || xn == x) break;
      x = xn;
    }
    // 3. certificates: follow the bisection's sequence with f predicted by
    // the tangent at the last Newton point, up to the midpoint predicted to
    // stop it; evaluate the last midpoint predicted to be accepted and the
    // last predicted to be rejected.  If they are (f < -thr, f >= C eps +
    // margin), every earlier decision of the replay is known.
    if (conv && gc != 0.0 && isfinite(gc)) {
      const double lo = U ? a.lg_min : a.lg_max, hi = U ? a.lg_max : a.lg_min;
      double root = lo, dx = __dsub_rn(hi, lo);
      double lastA = NAN, lastR = NAN;
      for (int i = 1; i <= a.maxnits; ++i) {
        dx = __dmul_rn(0.5, dx);
        const double mid = __dadd_rn(root, dx);
        if (U ? (mid <= accb) : (mid >= accb)) {
          root = mid;
          continue;
        }
        if (U ? (mid >= rejb) : (mid <= rejb)) continue;
        const double fp = fc + gc * (mid - xc);
        if (fp < 0.0) {
          if (fabs(fp) < a.tol) break;
          root = mid;
          lastA = mid;
        } else {
          if (fabs(fp) < ceps) break;
          lastR = mid;
        }
      }
      const double pts[2] = {lastA, lastR};
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double pt = pts[e];
        if (!(pt > rlo && pt < rhi)) continue;  // none (NaN) or outside the range
        const double fp = __dsub_rn(ev(pow(10.0, pt), lane), a.US_max);
        ++nev;
        note(pt, fp);
      }
    }
    const bool have_acc = U ? (accb > rlo) : (accb < rhi);
    const bool have_rej = U ? (rejb < rhi) : (rejb > rlo);
    if (lane == 0 && wid == 0 && ex.fallback) ex.fallback[pix] = (have_acc || have_rej) ? 0 : 1;
    // 4. replay.  The reference evaluates f0 at the start of the range first
    // and returns there if f0 >= 0; a known accept point inside the range
    // implies f0 < 0 by monotonicity, so f0 is then only needed if no later
    // step is accepted.
    if (!have_acc && !have_f0) {
      us = ev(k0, lane);
      ++nev;
      f0 = __dsub_rn(us, a.US_max);
      have_f0 = true;
      mg = fmin(mg, fabs(f0));
    }
    if (have_f0 && !(f0 < 0.0)) {
      k_root = k0;
    } else {
      const double lo = U ? a.lg_min : a.lg_max, hi = U ? a.lg_max : a.lg_min;
      double root = lo, dx = __dsub_rn(hi, lo);
      bool last_known = false, any_acc = false;
      for (int i = 1; i <= a.maxnits; ++i) {
        dx = __dmul_rn(0.5, dx);
        const double mid = __dadd_rn(root, dx);
        const bool known_acc = U ? (mid <= accb) : (mid >= accb);
        const bool known_rej = U ? (mid >= rejb) : (mid <= rejb);
        if (known_acc) {
          root = mid;
          any_acc = true;
          last_known = true;
          continue;
        }
        if (known_rej) continue;
        const double fmid = __dsub_rn(ev(pow(10.0, mid), lane), a.US_max);
        ++nev;
        mg = fmin(mg, decision_margin(fmid, a.tol, ceps));
        if (fmid < 0.0) {
          root = mid;
          any_acc = true;
          last_known = false;
          us = __dadd_rn(fmid, a.US_max);
          if (fabs(fmid) < a.tol) break;
        }
        if (fabs(fmid) < ceps) break;
      }
      if (!any_acc) {
        if (!have_f0) {
          us = ev(k0, lane);
          ++nev;
          mg = fmin(mg, fabs(__dsub_rn(us, a.US_max)));
        }
      } else if (last_known) {
        // value the reference holds at the last accepted midpoint
        const double fl = __dsub_rn(ev(pow(10.0, root), lane), a.US_max);
        ++nev;
        us = __dadd_rn(fl, a.US_max);
      }
      k_root = pow(10.0, root);
    }
  }
  if (lane == 0 && wid == 0 && ex.fallback && have_f0 && !(f0 < 0.0)) ex.fallback[pix] = 0;
  write_pixel(a, lam, col, pix, lane, nev, k_root, us, mg, wid, nw);
}

// The learned-kappa bisection: one CTA of four warps per pixel sharing each
// U/S evaluation (CtaCol), one pixel per CTA, so the block scheduler hands
// the next pixel to whichever CTA finishes first -- the evaluation counts
// vary from pixel to pixel (network start, Newton steps), and with about
// one resident warp per pixel a kernel of one-warp pixels lasts as long as
// its slowest pixels.
constexpr int LB_WARPS = 4;
static_assert(LB_WARPS == 4, "CtaCol splits the four partial sums of the one-warp evaluator");

__global__ void __launch_bounds__(LB_WARPS * 32, 7) learned_bisect_kernel(BisectArgs a,
                                                                          LearnedExtra ex) {
  __shared__ double red[2 * 2 * LB_WARPS * 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pix = blockIdx.x;
  if (pix >= a.m) return;
  const double* col = a.P + (size_t)pix * a.ldp;
  const CtaCol ev{a.L, col, a.Nd, a.n, a.UnotS != 0, a.C, red, warp, 0};
  learned_pixel(a, ex, a.L, col, ev, pix, lane, warp, LB_WARPS,
                ex.guess ? ex.guess + pix : nullptr);
}

// The same with the features and the network in the pixel's CTA (the table
// features, IMCOM_OPT_KAPPA_FEATURES = 1): the CTA sums the column's band
// masses in its first pass over the column -- which leaves the column in L2
// for the evaluations that follow --, warp 0 forms the 12 features and runs
// the tensor-core forward (mlp_forward_16, one valid row) on weights staged
// in shared memory, and the Newton steps start from its outputs.  This
// replaces a separate pass of the features kernel over all of P and two
// launches.
struct FusedTables {
  const float2* nbr;      // neighbour count and exposures per pixel
  const int8_t* bidx;     // band index per eigenmode
  const int* seg;         // band segments (seg[9] != 0: the index is not monotone)
  const float* weights;   // the network (device weight block)
};

__global__ void __launch_bounds__(LB_WARPS * 32, 7) learned_fused_kernel(BisectArgs a,
                                                                         LearnedExtra ex,
                                                                         FusedTables ft) {
  __shared__ double red[2 * 2 * LB_WARPS * 32];
  __shared__ __align__(16) MlpSmem S;
  __shared__ double sband[LB_WARPS][8];
  __shared__ float sfeat[16];
  __shared__ float2 sguess;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
  const int pix = blockIdx.x;
  if (pix >= a.m) return;
  const double* col = a.P + (size_t)pix * a.ldp;
  load_mlp_smem(ft.weights, S);
  double band[8];
#pragma unroll
  for (int b = 0; b < 8; ++b) band[b] = 0.0;
  if (ft.seg[9] == 0) {
#pragma unroll
    for (int b = 0; b < 8; ++b)
      for (int p = ft.seg[b] + tid; p < ft.seg[b + 1]; p += LB_WARPS * 32)
        band[b] = fma(col[p], col[p], band[b]);
  } else {
    for (int p = tid; p < a.n; p += LB_WARPS * 32) {
      const double pp = col[p];
      const int bb = ft.bidx[p];
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q == bb) band[q] += pp * pp;
    }
  }
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const double v = wsum(band[b]);
    if (lane == 0) sband[warp][b] = v;
  }
  __syncthreads();
  if (warp == 0) {
    const double lmax = a.L[0];  // eigenvalues are in descending order
    if (lane < 16) {
      float f = 0.0f;
      if (lane == 0) f = ft.nbr[pix].x;
      else if (lane == 1) f = ft.nbr[pix].y;
      else if (lane < 10) {
        const int b = lane - 2;
        double sb = 0.0;
#pragma unroll
        for (int w = 0; w < LB_WARPS; ++w) sb += sband[w][b];
        const double lc = lmax * pow(10.0, -(2.0 * b + 1.0));
        f = (float)log10(sb / (4.0 * a.C * (lc > 0.0 ? lc : 1e-300)) + 1e-30);
      } else if (lane == 10) {
        f = (float)log10(fabs(a.US_max) + 1e-300);
      } else if (lane == 11) {
        f = (float)log10(fabs(lmax / a.C) + 1e-300);
      }
      sfeat[lane] = f;
    }
    __syncwarp();
    mlp_forward_16(S, sfeat, 1, 0, lane, &sguess);
  }
  __syncthreads();
  const CtaCol ev{a.L, col, a.Nd, a.n, a.UnotS != 0, a.C, red, warp, 0};
  learned_pixel(a, ex, a.L, col, ev, pix, lane, warp, LB_WARPS, &sguess);
}

// ---------------------------------------------------------------------------
// Training: forward + backward for tiles of 32 samples per CTA, bf16
// activations, fp32 accumulation; per-CTA gradient partials are added to a
// global fp32 gradient with one atomic per parameter per CTA.
// Loss per sample: (o0 - t)^2 + 0.25 (o1 - log(|o0 - t| + 0.01))^2, the second
// term with the target held fixed (it fits the log of the first head's error).
// ---------------------------------------------------------------------------
constexpr int TB = 32;  // samples per CTA tile

__global__ void __launch_bounds__(256) mlp_grad_kernel(const float* __restrict__ params,
                                                       const float* __restrict__ feat, int nall,
                                                       const float* __restrict__ target,
                                                       const int* __restrict__ idx, int nb,
                                                       float* __restrict__ grad,
                                                       float* __restrict__ loss) {
  __shared__ float sW1[NH * NF], sW2[NH * NH], sW3[NO * NH], sb1[NH], sb2[NH], sb3[NO];
  __shared__ float X0[TB][NF + 1];
  // H1 and H2 hold the activations, then (in place) their gradients
  __shared__ float H1[TB][NH + 1], H2[TB][NH + 1];
  __shared__ float DO[TB][NO];
  __shared__ float sloss[256];
  const int tid = threadIdx.x;
  for (int q = tid; q < NH * NF; q += 256) sW1[q] = bf16r(params[OFF_W1 + q]);
  for (int q = tid; q < NH * NH; q += 256) sW2[q] = bf16r(params[OFF_W2 + q]);
  for (int q = tid; q < NO * NH; q += 256) sW3[q] = bf16r(params[OFF_W3 + q]);
  for (int q = tid; q < NH; q += 256) {
    sb1[q] = params[OFF_B1 + q];
    sb2[q] = params[OFF_B2 + q];
  }
  if (tid < NO) sb3[tid] = params[OFF_B3 + tid];
  const int s0 = blockIdx.x * TB;
  for (int q = tid; q < TB * NF; q += 256) {
    int r = q / NF, k = q % NF, s = s0 + r;
    float v = 0.0f;
    if (s < nb) {
      int g = idx ? idx[s] : s;
      v = bf16r(feat[(size_t)k * nall + g]);
    }
    X0[r][k] = v;
  }
  __syncthreads();
  // layer 1
  for (int q = tid; q < TB * NH; q += 256) {
    int r = q / NH, u = q % NH;
    float s = sb1[u];
#pragma unroll
    for (int k = 0; k < NF; ++k) s = fmaf(sW1[u * NF + k], X0[r][k], s);
    H1[r][u] = bf16r(fmaxf(s, 0.0f));
  }
  __syncthreads();
  // layer 2
  for (int q = tid; q < TB * NH; q += 256) {
    int r = q / NH, u = q % NH;
    float s = sb2[u];
    for (int v = 0; v < NH; ++v) s = fmaf(sW2[u * NH + v], H1[r][v], s);
    H2[r][u] = bf16r(fmaxf(s, 0.0f));
  }
  __syncthreads();
  // output, loss and d loss / d output
  float lsum = 0.0f;
  if (tid < TB) {
    int r = tid, s = s0 + r;
    float o[NO];
#pragma unroll
    for (int j = 0; j < NO; ++j) {
      float acc = sb3[j];
      for (int v = 0; v < NH; ++v) acc = fmaf(sW3[j * NH + v], H2[r][v], acc);
      o[j] = acc;
    }
    float d0 = 0.0f, d1 = 0.0f;
    if (s < nb) {
      int g = idx ? idx[s] : s;
      float e = o[0] - target[g];
      float lt = logf(fabsf(e) + 0.01f);
      float e1 = o[1] - lt;
      lsum = e * e + 0.25f * e1 * e1;
      d0 = 2.0f * e;
      d1 = 0.5f * e1;
    }
    DO[r][0] = d0;
    DO[r][1] = d1;
  }
  sloss[tid] = lsum;
  __syncthreads();
  // dW3, db3 (need H2 before it is overwritten)
  for (int q = tid; q < NO * NH; q += 256) {
    int j = q / NH, v = q % NH;
    float g = 0.0f;
    for (int r = 0; r < TB; ++r) g = fmaf(DO[r][j], H2[r][v], g);
    atomicAdd(&grad[OFF_W3 + q], g);
  }
  if (tid < NO) {
    float g = 0.0f;
    for (int r = 0; r < TB; ++r) g += DO[r][tid];
    atomicAdd(&grad[OFF_B3 + tid], g);
  }
  __syncthreads();
  // H2 <- d(pre-activation 2) = (W3^T dO) masked by ReLU, in place
  for (int q = tid; q < TB * NH; q += 256) {
    int r = q / NH, u = q % NH;
    float g = DO[r][0] * sW3[u] + DO[r][1] * sW3[NH + u];
    H2[r][u] = H2[r][u] > 0.0f ? g : 0.0f;
  }
  __syncthreads();
  // dW2 = dH2^T H1, db2 (need H1 before it is overwritten)
  for (int q = tid; q < NH * NH; q += 256) {
    int u = q / NH, v = q % NH;
    float g = 0.0f;
    for (int r = 0; r < TB; ++r) g = fmaf(H2[r][u], H1[r][v], g);
    atomicAdd(&grad[OFF_W2 + q], g);
  }
  for (int q = tid; q < NH; q += 256) {
    float g = 0.0f;
    for (int r = 0; r < TB; ++r) g += H2[r][q];
    atomicAdd(&grad[OFF_B2 + q], g);
  }
  __syncthreads();
  // H1 <- d(pre-activation 1) = (W2^T dH2) masked by ReLU, in place
  for (int q = tid; q < TB * NH; q += 256) {
    int r = q / NH, v = q % NH;
    float g = 0.0f;
    for (int u = 0; u < NH; ++u) g = fmaf(sW2[u * NH + v], H2[r][u], g);
    H1[r][v] = H1[r][v] > 0.0f ? g : 0.0f;
  }
  __syncthreads();
  // dW1 = dH1^T X0, db1
  for (int q = tid; q < NH * NF; q += 256) {
    int u = q / NF, k = q % NF;
    float g = 0.0f;
    for (int r = 0; r < TB; ++r) g = fmaf(H1[r][u], X0[r][k], g);
    atomicAdd(&grad[OFF_W1 + q], g);
  }
  for (int q = tid; q < NH; q += 256) {
    float g = 0.0f;
    for (int r = 0; r < TB; ++r) g += H1[r][q];
    atomicAdd(&grad[OFF_B1 + q], g);
  }
  for (int w = 128; w > 0; w >>= 1) {
    __syncthreads();
    if (tid < w) sloss[tid] += sloss[tid + w];
  }
  if (tid == 0) atomicAdd(loss, sloss[0]);
}

// Adam step on fp32 master parameters with the batch-mean gradient.
__global__ void adam_kernel(float* __restrict__ params, const float* __restrict__ grad,
                            float* __restrict__ m1, float* __restrict__ m2, float lr, float b1,
                            float b2, float c1, float c2, float inv_batch) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= NPARAM) return;
  float g = grad[q] * inv_batch;
  float a = b1 * m1[q] + (1.0f - b1) * g;
  float b = b2 * m2[q] + (1.0f - b2) * g * g;
  m1[q] = a;
  m2[q] = b;
  params[q] -= lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
}

}  // namespace

// Band index of every eigenmode, and with IMCOM_OPT_KAPPA_FEATURES = 1 the
// band segments and (once per set of inputs) the neighbour table.
int feature_tables(imcom_ctx* ctx, const float2** nbr, const int** seg) {
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->band, ctx->band_bytes, (size_t)ctx->n));
  band_index_kernel<<<(ctx->n + 255) / 256, 256, 0, ctx->stream>>>(ctx->L, ctx->n, ctx->band);
  IMC_LAUNCH();
  *nbr = nullptr;
  *seg = nullptr;
  if (!ctx->kappa_feat) return 0;
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->band_seg, ctx->band_seg_bytes, 10 * sizeof(int)));
  IMC_CUDA(cudaMemsetAsync(ctx->band_seg, 0, 10 * sizeof(int), ctx->stream));
  band_segments_kernel<<<(ctx->n + 255) / 256, 256, 0, ctx->stream>>>(ctx->band, ctx->n,
                                                                      ctx->band_seg);
  IMC_LAUNCH();
  if (!ctx->nbr_valid) {
    IMC_TRY(ensure_buf(ctx, (void**)&ctx->nbr, ctx->nbr_bytes, (size_t)ctx->m * sizeof(float2)));
    neighbour_kernel<<<(ctx->m + 7) / 8, 256, 0, ctx->stream>>>(ctx->x, ctx->y, ctx->exp_i,
                                                                ctx->n, ctx->X, ctx->Y, ctx->m,
                                                                ctx->nbr);
    IMC_LAUNCH();
    ctx->nbr_valid = true;
  }
  *nbr = ctx->nbr;
  *seg = ctx->band_seg;
  return 0;
}

// Features of every pixel into ctx->feat (12 x m, feature-major) and, with
// the network installed and selected, its outputs into ctx->guess.
int kappa_guess(imcom_ctx* ctx, const BisectArgs& a, bool network) {
  IMC_TRY(ensure_vec(ctx, &ctx->feat, (size_t)NF * ctx->m));
  IMC_TRY(ensure_vec(ctx, &ctx->guess, (size_t)ctx->m));
  const float2* nbr;
  const int* seg;
  IMC_TRY(feature_tables(ctx, &nbr, &seg));
  features_kernel<<<(ctx->m + 7) / 8, 256, 0, ctx->stream>>>(a, ctx->x, ctx->y, ctx->exp_i,
                                                             ctx->X, ctx->Y, ctx->band, nbr, seg,
                                                             ctx->feat);
  IMC_LAUNCH();
  if (network) {
    const int per_block = MLP_WARPS * 16;
    const int blocks = std::min((ctx->m + per_block - 1) / per_block, 4 * sm_count(ctx));
    mlp_infer_kernel<<<blocks, MLP_WARPS * 32, 0, ctx->stream>>>(ctx->mlp.w, ctx->feat, ctx->m,
                                                                ctx->guess);
    IMC_LAUNCH();
  }
  return 0;
}

int fill_learned(imcom_ctx* ctx, LearnedExtra& ex) {
  if (!ctx->mlp.set && !ctx->kappa_nonet)
    return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_mlp_set_weights has not run");
  ex.guess = nullptr;  // set by the caller once kappa_guess has sized ctx->guess
  ex.fallback = nullptr;
  ex.half_scale = 3.0;
  ex.min_half = 0.02;
  ex.margin = 1e-10;
  ex.max_newton = 8;
  return 0;
}

}  // namespace imcom

using namespace imcom;

extern "C" int imcom_gpu_kappa_features(imcom_ctx* ctx, int UnotS, double US_max, double C_a,
                                        float* feat_out) {
  if (!ctx) return -1;
  if (!feat_out) return -5;
  BisectArgs a;
  IMC_TRY(fill_bisect_args(ctx, a, UnotS, US_max, 1.0, 1.0, 0.0, 0, C_a));
  cudaSetDevice(ctx->device);
  IMC_TRY(kappa_guess(ctx, a, false));
  IMC_CUDA(cudaMemcpyAsync(feat_out, ctx->feat, (size_t)NF * ctx->m * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

extern "C" int imcom_gpu_mlp_set_weights(imcom_ctx* ctx, const float* W1, const float* b1,
                                         const float* W2, const float* b2, const float* W3,
                                         const float* b3, const float* mean, const float* stdv) {
  if (!ctx) return -1;
  const float* parts[8] = {W1, b1, W2, b2, W3, b3, mean, stdv};
  for (int q = 0; q < 8; ++q)
    if (!parts[q]) return -(q + 2);
  std::vector<float> h(NWEIGHT);
  auto put = [&](int off, const float* src, int cnt, bool round) {
    for (int q = 0; q < cnt; ++q) {
      float v = src[q];
      if (round) v = __bfloat162float(__float2bfloat16_rn(v));
      h[off + q] = v;
    }
  };
  put(OFF_W1, W1, NH * NF, true);
  put(OFF_B1, b1, NH, false);
  put(OFF_W2, W2, NH * NH, true);
  put(OFF_B2, b2, NH, false);
  put(OFF_W3, W3, NO * NH, true);
  put(OFF_B3, b3, NO, false);
  put(OFF_MEAN, mean, NF, false);
  put(OFF_STD, stdv, NF, false);
  for (int q = 0; q < NF; ++q)
    if (!(h[OFF_STD + q] > 0.0f)) return set_err(ctx, -9, "feature std must be positive");
  cudaSetDevice(ctx->device);
  if (!ctx->mlp.w) IMC_TRY(ensure_vec(ctx, &ctx->mlp.w, NWEIGHT));
  IMC_CUDA(cudaMemcpyAsync(ctx->mlp.w, h.data(), NWEIGHT * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->mlp.set = true;
  return 0;
}

extern "C" int imcom_gpu_bisect_kappa_learned(imcom_ctx* ctx, int UnotS, double US_max,
                                              double k_min, double k_max, double tol,
                                              int maxnits, double C_a, double* K_out,
                                              double* US_out, int* nevals_out,
                                              int* fallback_out) {
  if (!ctx) return -1;
  BisectArgs a;
  IMC_TRY(fill_bisect_args(ctx, a, UnotS, US_max, k_min, k_max, tol, maxnits, C_a));
  LearnedExtra ex;
  IMC_TRY(fill_learned(ctx, ex));
  cudaSetDevice(ctx->device);
  stage_begin(ctx, ST_BISECT);
  IMC_TRY(ensure_mat(ctx, ctx->Pt, ctx->n, ctx->m));
  a.Pt = ctx->Pt.p;
  a.ldt = ctx->Pt.ld;
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->fb, ctx->fb_bytes, (size_t)ctx->m * sizeof(int)));
  ex.fallback = ctx->fb;
  if (ctx->p_split) IMC_TRY(split_margin_buffer(ctx, a));
  const bool fused = !ctx->kappa_nonet && ctx->kappa_feat;
  if (!ctx->kappa_nonet && !fused) {
    IMC_TRY(kappa_guess(ctx, a, true));
    ex.guess = ctx->guess;  // after kappa_guess: it may have grown the buffer
  }
  if (fused) {
    const float2* nbr;
    const int* seg;
    IMC_TRY(feature_tables(ctx, &nbr, &seg));
    FusedTables ft{nbr, ctx->band, seg, ctx->mlp.w};
    learned_fused_kernel<<<ctx->m, LB_WARPS * 32, 0, ctx->stream>>>(a, ex, ft);
  } else {
    learned_bisect_kernel<<<ctx->m, LB_WARPS * 32, 0, ctx->stream>>>(a, ex);
  }
  IMC_LAUNCH();
  if (ctx->p_split) IMC_TRY(split_audit(ctx, a));
  stage_end(ctx, ST_BISECT);
  ctx->have_K = true;
  ctx->have_Pt = true;
  ctx->have_T = false;
  if (fallback_out)
    IMC_CUDA(cudaMemcpyAsync(fallback_out, ctx->fb, ctx->m * sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->stream));
  return copy_pixel_outputs(ctx, K_out, US_out, nevals_out);
}

// Gradient of the summed loss over `nsamples` samples at the given parameters
// (the training kernel on one batch; used by the tests' gradient check).
extern "C" int imcom_gpu_mlp_gradient(imcom_ctx* ctx, int nsamples, const float* feat,
                                      const float* target, const float* params, float* grad_out,
                                      float* loss_out) {
  if (!ctx) return -1;
  if (nsamples <= 0) return -2;
  if (!feat) return -3;
  if (!target) return -4;
  if (!params) return -5;
  if (!grad_out) return -6;
  cudaSetDevice(ctx->device);
  float *d = nullptr;
  size_t need = ((size_t)NF * nsamples + nsamples + 2 * NPARAM + 64) * sizeof(float);
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->train_buf, ctx->train_bytes, need));
  d = (float*)ctx->train_buf;
  float* dfeat = d;
  float* dtarget = dfeat + (size_t)NF * nsamples;
  float* dparams = dtarget + nsamples;
  float* dgrad = dparams + NPARAM;
  float* dloss = dgrad + NPARAM;
  IMC_CUDA(cudaMemcpyAsync(dfeat, feat, (size_t)NF * nsamples * sizeof(float),
                           cudaMemcpyHostToDevice, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(dtarget, target, nsamples * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(dparams, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
  IMC_CUDA(cudaMemsetAsync(dgrad, 0, (NPARAM + 1) * sizeof(float), ctx->stream));
  mlp_grad_kernel<<<(nsamples + TB - 1) / TB, 256, 0, ctx->stream>>>(
      dparams, dfeat, nsamples, dtarget, nullptr, nsamples, dgrad, dloss);
  IMC_LAUNCH();
  IMC_CUDA(cudaMemcpyAsync(grad_out, dgrad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost,
                           ctx->stream));
  float l = 0.0f;
  IMC_CUDA(cudaMemcpyAsync(&l, dloss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (loss_out) *loss_out = l;
  return 0;
}

// Adam training on normalised features/targets; params in/out (packed).
extern "C" int imcom_gpu_mlp_train(imcom_ctx* ctx, int nsamples, const float* feat,
                                   const float* target, int epochs, int batch, float lr,
                                   unsigned seed, float* params, float* loss_out) {
  if (!ctx) return -1;
  if (nsamples <= 0) return -2;
  if (!feat) return -3;
  if (!target) return -4;
  if (epochs <= 0) return -5;
  if (batch <= 0) return -6;
  if (!(lr > 0.0f)) return -7;
  if (!params) return -9;
  cudaSetDevice(ctx->device);
  size_t need = ((size_t)NF * nsamples + nsamples + 4 * NPARAM + 64) * sizeof(float) +
                (size_t)nsamples * sizeof(int);
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->train_buf, ctx->train_bytes, need));
  float* dfeat = (float*)ctx->train_buf;
  float* dtarget = dfeat + (size_t)NF * nsamples;
  float* dparams = dtarget + nsamples;
  float* dgrad = dparams + NPARAM;
  float* dm1 = dgrad + NPARAM + 1;
  float* dm2 = dm1 + NPARAM;
  int* didx = (int*)(dm2 + NPARAM + 16);
  IMC_CUDA(cudaMemcpyAsync(dfeat, feat, (size_t)NF * nsamples * sizeof(float),
                           cudaMemcpyHostToDevice, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(dtarget, target, nsamples * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(dparams, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
  IMC_CUDA(cudaMemsetAsync(dm1, 0, 2 * (NPARAM + 8) * sizeof(float), ctx->stream));
  // shuffled order per epoch (host xorshift, reproducible from the seed)
  std::vector<int> order(nsamples);
  unsigned s = seed ? seed : 1u;
  auto rnd = [&]() {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return s;
  };
  const float b1 = 0.9f, b2 = 0.999f;
  int step = 0;
  std::vector<float> eloss(epochs, 0.0f);
  float* dloss = dgrad + NPARAM;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int q = 0; q < nsamples; ++q) order[q] = q;
    for (int q = nsamples - 1; q > 0; --q) std::swap(order[q], order[rnd() % (q + 1)]);
    IMC_CUDA(cudaMemcpyAsync(didx, order.data(), nsamples * sizeof(int), cudaMemcpyHostToDevice,
                             ctx->stream));
    IMC_CUDA(cudaMemsetAsync(dloss, 0, sizeof(float), ctx->stream));
    for (int b0 = 0; b0 < nsamples; b0 += batch) {
      const int nb = std::min(batch, nsamples - b0);
      IMC_CUDA(cudaMemsetAsync(dgrad, 0, NPARAM * sizeof(float), ctx->stream));
      mlp_grad_kernel<<<(nb + TB - 1) / TB, 256, 0, ctx->stream>>>(
          dparams, dfeat, nsamples, dtarget, didx + b0, nb, dgrad, dloss);
      IMC_LAUNCH();
      ++step;
      const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
      adam_kernel<<<(NPARAM + 255) / 256, 256, 0, ctx->stream>>>(dparams, dgrad, dm1, dm2, lr, b1,
                                                                b2, c1, c2, 1.0f / nb);
      IMC_LAUNCH();
    }
    IMC_CUDA(cudaMemcpyAsync(&eloss[ep], dloss, sizeof(float), cudaMemcpyDeviceToHost,
                             ctx->stream));
  }
  IMC_CUDA(cudaMemcpyAsync(params, dparams, NPARAM * sizeof(float), cudaMemcpyDeviceToHost,
                           ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (loss_out)
    for (int ep = 0; ep < epochs; ++ep) loss_out[ep] = eloss[ep] / nsamples;
  return 0;
}
