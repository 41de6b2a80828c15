// usum.cuh -- per-output-pixel U(kappa) and S(kappa) on one warp.
//
// imcom_U_from_kappa (imcom_matrix.f90:904-922):
//   U = (C - 1/4 sum_p (L_p + 2k) P2_pa / ((L_p + k)(L_p + k))) / C
// imcom_S_from_kappa (imcom_matrix.f90:955-970):
//   S = 1/4 sum_p Ndiag_p P2_pa / ((L_p + k)(L_p + k))
// Each term's numerator and (L_p + k)^2 are formed with the reference's
// operations (explicit _rn intrinsics: no FMA contraction); the quotient is
// the numerator times a Newton-refined reciprocal of (L_p + k)^2, which
// shortens the per-term dependency chain of a correctly rounded division
// (the term may differ from num / den by one rounding).  The sum over p is a
// per-lane sum (four partial sums) followed by an xor-butterfly, which leaves
// the bit-identical total in every lane so control flow stays warp-uniform.
// Every U/S evaluator of the library uses these terms and this order, so the
// plain, learned and split-precision bisections take identical decisions.
#pragma once

namespace imcom {

// lam / col / nd may point to shared or global memory.  col holds P(:, a)
// (P2 = P * P is formed here, bit-identical to the reference's P2_ia).
// Each lane keeps four independent partial sums (modes p = lane + 32 j with
// j mod 4 selecting the sum) so that four divisions are in flight per lane;
// the partials are added as (s0 + s1) + (s2 + s3) before the butterfly.
// 1/a by two Newton-Raphson steps r <- r + r (1 - a r) from the PTX
// rcp.approx.ftz.f64 seed (measured relative error 2^-19.9 on B200; after
// two steps 4.2M random arguments over |a| in [1e-30, 1e30] gave the correctly
// rounded reciprocal).  Arguments here are (L_p + k)^2 >= (C eps)^2, never
// subnormal.
__device__ __forceinline__ double rcp_nr(double a) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
  double e = fma(-a, r, 1.0);
  r = fma(r, e, r);
  e = fma(-a, r, 1.0);
  return fma(r, e, r);
}

__device__ __forceinline__ double uterm(double l, double pp, double k, double k2) {
  const double p2 = __dmul_rn(pp, pp);
  const double t = __dadd_rn(l, k);
  return __dmul_rn(__dmul_rn(__dadd_rn(l, k2), p2), rcp_nr(__dmul_rn(t, t)));
}

__device__ __forceinline__ double sterm(double l, double pp, double nd, double k) {
  const double p2 = __dmul_rn(pp, pp);
  const double t = __dadd_rn(l, k);
  return __dmul_rn(__dmul_rn(nd, p2), rcp_nr(__dmul_rn(t, t)));
}

// The same terms with the kappa derivative's term added to *d: P2 / (L + k)^3
// (U mode) or Nd P2 / (L + k)^3 (S mode).  The returned term is the one
// uterm / sterm return, formed by the same operations.
__device__ __forceinline__ double uterm_d(double l, double pp, double k, double k2, double* d) {
  const double p2 = __dmul_rn(pp, pp);
  const double t = __dadd_rn(l, k);
  const double r = rcp_nr(__dmul_rn(t, t));
  *d = fma(p2 * r, t * r, *d);
  return __dmul_rn(__dmul_rn(__dadd_rn(l, k2), p2), r);
}

__device__ __forceinline__ double sterm_d(double l, double pp, double nd, double k, double* d) {
  const double p2 = __dmul_rn(pp, pp);
  const double t = __dadd_rn(l, k);
  const double r = rcp_nr(__dmul_rn(t, t));
  const double v = __dmul_rn(__dmul_rn(nd, p2), r);
  *d = fma(v, t * r, *d);
  return v;
}

__device__ __forceinline__ double warp_reduce_sum(double s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
}

// Modes p = lane + 32 j go to partial sum j mod 4, in increasing j; blocks
// of eight modes per lane keep eight column loads in flight.
// D = true also sums the derivative terms into *dsum (every lane gets the
// total) in four partials of their own, so they add no dependent chain; the
// derivative only steers the Newton steps, so its summation order is free.
// The U sum is formed by exactly the same operations either way.
template <bool D>
__device__ __forceinline__ double warp_usum_t(const double* lam, const double* col, int n,
                                              double k, int lane, double* dsum) {
  const double k2 = __dmul_rn(2.0, k);
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;  // derivative partials
#define UT(l_, c_, d_) (D ? uterm_d(l_, c_, k, k2, &d_) : uterm(l_, c_, k, k2))
  int p = lane;
  for (; p + 224 < n; p += 256) {
    double c[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      c[q] = col[p + 32 * q];
      l[q] = lam[p + 32 * q];
    }
    s0 = __dadd_rn(s0, UT(l[0], c[0], d0));
    s1 = __dadd_rn(s1, UT(l[1], c[1], d1));
    s2 = __dadd_rn(s2, UT(l[2], c[2], d2));
    s3 = __dadd_rn(s3, UT(l[3], c[3], d3));
    s0 = __dadd_rn(s0, UT(l[4], c[4], d0));
    s1 = __dadd_rn(s1, UT(l[5], c[5], d1));
    s2 = __dadd_rn(s2, UT(l[6], c[6], d2));
    s3 = __dadd_rn(s3, UT(l[7], c[7], d3));
  }
  for (; p + 96 < n; p += 128) {
    s0 = __dadd_rn(s0, UT(lam[p], col[p], d0));
    s1 = __dadd_rn(s1, UT(lam[p + 32], col[p + 32], d1));
    s2 = __dadd_rn(s2, UT(lam[p + 64], col[p + 64], d2));
    s3 = __dadd_rn(s3, UT(lam[p + 96], col[p + 96], d3));
  }
  if (p < n) s0 = __dadd_rn(s0, UT(lam[p], col[p], d0));
  if (p + 32 < n) s1 = __dadd_rn(s1, UT(lam[p + 32], col[p + 32], d1));
  if (p + 64 < n) s2 = __dadd_rn(s2, UT(lam[p + 64], col[p + 64], d2));
#undef UT
  if (D) *dsum = warp_reduce_sum((d0 + d1) + (d2 + d3));
  return warp_reduce_sum(__dadd_rn(__dadd_rn(s0, s1), __dadd_rn(s2, s3)));
}

__device__ __forceinline__ double warp_usum(const double* lam, const double* col, int n,
                                            double k, int lane) {
  return warp_usum_t<false>(lam, col, n, k, lane, nullptr);
}

template <bool D>
__device__ __forceinline__ double warp_ssum_t(const double* lam, const double* col,
                                              const double* nd, int n, double k, int lane,
                                              double* dsum) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;  // derivative partials
#define ST(l_, c_, w_, d_) (D ? sterm_d(l_, c_, w_, k, &d_) : sterm(l_, c_, w_, k))
  int p = lane;
  for (; p + 224 < n; p += 256) {
    double c[8], l[8], w[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      c[q] = col[p + 32 * q];
      l[q] = lam[p + 32 * q];
      w[q] = nd[p + 32 * q];
    }
    s0 = __dadd_rn(s0, ST(l[0], c[0], w[0], d0));
    s1 = __dadd_rn(s1, ST(l[1], c[1], w[1], d1));
    s2 = __dadd_rn(s2, ST(l[2], c[2], w[2], d2));
    s3 = __dadd_rn(s3, ST(l[3], c[3], w[3], d3));
    s0 = __dadd_rn(s0, ST(l[4], c[4], w[4], d0));
    s1 = __dadd_rn(s1, ST(l[5], c[5], w[5], d1));
    s2 = __dadd_rn(s2, ST(l[6], c[6], w[6], d2));
    s3 = __dadd_rn(s3, ST(l[7], c[7], w[7], d3));
  }
  for (; p + 96 < n; p += 128) {
    s0 = __dadd_rn(s0, ST(lam[p], col[p], nd[p], d0));
    s1 = __dadd_rn(s1, ST(lam[p + 32], col[p + 32], nd[p + 32], d1));
    s2 = __dadd_rn(s2, ST(lam[p + 64], col[p + 64], nd[p + 64], d2));
    s3 = __dadd_rn(s3, ST(lam[p + 96], col[p + 96], nd[p + 96], d3));
  }
  if (p < n) s0 = __dadd_rn(s0, ST(lam[p], col[p], nd[p], d0));
  if (p + 32 < n) s1 = __dadd_rn(s1, ST(lam[p + 32], col[p + 32], nd[p + 32], d1));
  if (p + 64 < n) s2 = __dadd_rn(s2, ST(lam[p + 64], col[p + 64], nd[p + 64], d2));
#undef ST
  if (D) *dsum = warp_reduce_sum((d0 + d1) + (d2 + d3));
  return warp_reduce_sum(__dadd_rn(__dadd_rn(s0, s1), __dadd_rn(s2, s3)));
}

__device__ __forceinline__ double warp_ssum(const double* lam, const double* col,
                                            const double* nd, int n, double k, int lane) {
  return warp_ssum_t<false>(lam, col, nd, n, k, lane, nullptr);
}

// U or S at kappa k.
__device__ __forceinline__ double warp_us(bool UnotS, const double* lam, const double* col,
                                          const double* nd, int n, double k, double C,
                                          int lane) {
  if (UnotS) {
    double usum = warp_usum(lam, col, n, k, lane);
    return __ddiv_rn(__dsub_rn(C, __ddiv_rn(usum, 4.0)), C);
  }
  return __ddiv_rn(warp_ssum(lam, col, nd, n, k, lane), 4.0);
}

// U/S evaluator that streams the pixel's P column (any n).
struct StreamCol {
  const double* lam;
  const double* col;
  const double* nd;
  int n;
  bool U;
  double C;
  __device__ __forceinline__ double operator()(double k, int lane) const {
    return warp_us(U, lam, col, nd, n, k, C, lane);
  }
  // U or S at kappa k (the value operator() returns, bit for bit) and its
  // derivative with respect to x = log10(kappa) in *dx.
  __device__ __forceinline__ double eval_d(double k, int lane, double* dx) const {
    constexpr double LN10 = 2.302585092994046;
    double d;
    if (U) {
      const double usum = warp_usum_t<true>(lam, col, n, k, lane, &d);
      *dx = LN10 * k * k / (2.0 * C) * d;
      return __ddiv_rn(__dsub_rn(C, __ddiv_rn(usum, 4.0)), C);
    }
    const double ssum = warp_ssum_t<true>(lam, col, nd, n, k, lane, &d);
    *dx = -0.5 * LN10 * k * d;
    return __ddiv_rn(ssum, 4.0);
  }
};

// U/S evaluator shared by the four warps of a CTA: warp w sums the modes
// p = lane + 32 j with j = w (mod 4), in increasing j -- exactly partial sum
// s_w of warp_usum_t / warp_ssum_t --, the partials meet in shared memory and
// every warp combines them as (s0 + s1) + (s2 + s3) and the lane butterfly.
// So every warp gets the one-warp evaluator's value bit for bit, with a
// quarter of the terms in each warp's dependent chain.  One barrier per
// evaluation (double-buffered partials); all four warps must call it with
// the same arguments.
template <bool D, bool U>
__device__ __forceinline__ double cta_partial(const double* lam, const double* col,
                                              const double* nd, int n, double k, int lane,
                                              int w, double* dpart) {
  constexpr int B = U ? 6 : 4;  // terms whose loads are in flight together
  const double k2 = __dmul_rn(2.0, k);
  double s = 0.0, d0 = 0.0, d1 = 0.0;
  int j = w;
  for (; lane + 32 * (j + 4 * (B - 1)) < n; j += 4 * B) {
    double c[B], l[B], wv[B];
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int p = lane + 32 * (j + 4 * q);
      c[q] = col[p];
      l[q] = lam[p];
      if (!U) wv[q] = nd[p];
    }
#pragma unroll
    for (int q = 0; q < B; ++q) {
      double t;
      if (U)
        t = D ? uterm_d(l[q], c[q], k, k2, (q & 1) ? &d1 : &d0) : uterm(l[q], c[q], k, k2);
      else
        t = D ? sterm_d(l[q], c[q], wv[q], k, (q & 1) ? &d1 : &d0) : sterm(l[q], c[q], wv[q], k);
      s = __dadd_rn(s, t);
    }
  }
  for (; lane + 32 * j < n; j += 4) {
    const int p = lane + 32 * j;
    double t;
    if (U)
      t = D ? uterm_d(lam[p], col[p], k, k2, &d0) : uterm(lam[p], col[p], k, k2);
    else
      t = D ? sterm_d(lam[p], col[p], nd[p], k, &d0) : sterm(lam[p], col[p], nd[p], k);
    s = __dadd_rn(s, t);
  }
  if (D) *dpart = d0 + d1;
  return s;
}

struct CtaCol {
  const double* lam;
  const double* col;
  const double* nd;
  int n;
  bool U;
  double C;
  double* red;  // shared, 2 x 2 x 4 x 32 doubles: buffer, value/derivative, warp, lane
  int warp;
  mutable int buf;

  template <bool D>
  __device__ __forceinline__ double sum(double k, int lane, double* dsum) const {
    double dw = 0.0;
    const double sw = U ? cta_partial<D, true>(lam, col, nd, n, k, lane, warp, &dw)
                        : cta_partial<D, false>(lam, col, nd, n, k, lane, warp, &dw);
    double* r = red + buf * 256;
    buf ^= 1;
    r[warp * 32 + lane] = sw;
    if (D) r[128 + warp * 32 + lane] = dw;
    __syncthreads();
    const double tot = __dadd_rn(__dadd_rn(r[lane], r[32 + lane]), __dadd_rn(r[64 + lane], r[96 + lane]));
    if (D) *dsum = warp_reduce_sum((r[128 + lane] + r[160 + lane]) + (r[192 + lane] + r[224 + lane]));
    return warp_reduce_sum(tot);
  }
  __device__ __forceinline__ double operator()(double k, int lane) const {
    if (U) return __ddiv_rn(__dsub_rn(C, __ddiv_rn(sum<false>(k, lane, nullptr), 4.0)), C);
    return __ddiv_rn(sum<false>(k, lane, nullptr), 4.0);
  }
  // the value operator() returns, bit for bit, and d/dx at x = log10(kappa)
  __device__ __forceinline__ double eval_d(double k, int lane, double* dx) const {
    constexpr double LN10 = 2.302585092994046;
    double d;
    const double s = sum<true>(k, lane, &d);
    if (U) {
      *dx = LN10 * k * k / (2.0 * C) * d;
      return __ddiv_rn(__dsub_rn(C, __ddiv_rn(s, 4.0)), C);
    }
    *dx = -0.5 * LN10 * k * d;
    return __ddiv_rn(s, 4.0);
  }
};

// U/S evaluator with the pixel's column resident in its warp: the weights
// w_p = P_p^2 (U mode) or Ndiag_p P_p^2 (S mode, the reference's product
// formed once) for modes p = lane + 32 j, j < RES_R in registers and
// RES_R <= j < RES_R + RES_S in shared memory.  Terms are added to partial
// sum j mod 4 in increasing j, exactly as warp_usum / warp_ssum do, so both
// evaluators give bit-identical U and S.
constexpr int RES_R = 64;
constexpr int RES_S = 64;
constexpr int RES_MAX_N = 32 * (RES_R + RES_S);  // 4096

struct ResCol {
  double r[RES_R];
  const double* sm;   // this warp's slice: sm[(j - RES_R) * 32 + lane]
  const double* lam;  // eigenvalues
  int n, jn;
  bool U;
  double C;

  __device__ __forceinline__ void load(const double* col, const double* nd, int lane,
                                       double* smw) {
#pragma unroll
    for (int j = 0; j < RES_R; ++j) {
      const int p = lane + 32 * j;
      double v = 0.0;
      if (p < n) {
        const double pp = col[p];
        v = __dmul_rn(pp, pp);
        if (!U) v = __dmul_rn(nd[p], v);
      }
      r[j] = v;
    }
    for (int j = RES_R; j < jn; ++j) {
      const int p = lane + 32 * j;
      double v = 0.0;
      if (p < n) {
        const double pp = col[p];
        v = __dmul_rn(pp, pp);
        if (!U) v = __dmul_rn(nd[p], v);
      }
      smw[(j - RES_R) * 32 + lane] = v;
    }
    sm = smw;
  }

  __device__ __forceinline__ double term(double l, double w, double k, double k2) const {
    const double t = __dadd_rn(l, k);
    const double num = U ? __dmul_rn(__dadd_rn(l, k2), w) : w;
    return __dmul_rn(num, rcp_nr(__dmul_rn(t, t)));
  }

  __device__ __forceinline__ double operator()(double k, int lane) const {
    const double k2 = __dmul_rn(2.0, k);
    double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < RES_R; ++j) {
      const int p = lane + 32 * j;
      if (p < n) s[j & 3] = __dadd_rn(s[j & 3], term(lam[p], r[j], k, k2));
    }
    for (int j = RES_R; j < jn; j += 4) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int p = lane + 32 * (j + q);
        if (j + q < jn && p < n)
          s[q] = __dadd_rn(s[q], term(lam[p], sm[(j + q - RES_R) * 32 + lane], k, k2));
      }
    }
    const double sum = warp_reduce_sum(__dadd_rn(__dadd_rn(s[0], s[1]), __dadd_rn(s[2], s[3])));
    if (U) return __ddiv_rn(__dsub_rn(C, __ddiv_rn(sum, 4.0)), C);
    return __ddiv_rn(sum, 4.0);
  }
};

// Launch shape of the resident kernels: one CTA per SM holding the
// eigenvalues (RES_MAX_N doubles) and RES_S * 32 doubles per warp.  8 warps
// (2 per SM sub-partition) leave 255 registers per thread for the 64
// register-resident weights; with 3 warps on a sub-partition the limit drops
// to 168 and the column spills.
constexpr int RES_WARPS_PLAIN = 8;    // 32 KB + 8 x 16 KB = 160 KB
// Resident kernel for this problem?  mode: IMCOM_BISECT_* option value.
// Automatic choice: streaming.  With the Newton reciprocal the per-term
// chain is short and the streaming kernel's ~28 warps per SM hide L2
// latency; the resident kernel's 8 warps do not hide the FP64 latency
// (n = m = 4096: 0.47 vs 1.03 ms).
inline bool use_resident(int mode, int n) {
  if (n > RES_MAX_N) return false;
  return mode == 2;
}

inline size_t res_smem_bytes(int warps) {
  return (size_t)RES_MAX_N * sizeof(double) + (size_t)warps * RES_S * 32 * sizeof(double);
}

// Shared-memory plan of the per-pixel kernels: the eigenvalues (n) plus one
// P column per warp when they fit, else the eigenvalues only, else nothing.
struct PixelSmem {
  int warps;       // warps per CTA
  bool lam_smem;   // L staged in shared memory
  bool col_smem;   // P(:, a) staged per warp
  size_t bytes;
};

// CTAs of 4 warps.  The eigenvalues and one P column per warp are staged in
// shared memory when five columns fit in 52 KB (n <= 1331), which keeps at
// least 4 CTAs (16 pixel warps) per SM.  Otherwise nothing is staged: the
// eigenvalues (read by every warp) stay in L1, the columns stream from L2,
// and ~28 pixel warps per SM run the n = m = 4096 case in a single wave.
// The pixel kernels' dynamic shared-memory limit is set once to this ceiling
// (the attribute is process-wide: contexts solving on several host threads
// must not set it under one another's launches).
constexpr size_t kPixelSmemMax = 52 * 1024;

inline PixelSmem plan_pixel_smem(int n, size_t limit = kPixelSmemMax) {
  PixelSmem p;
  const size_t col = (size_t)n * sizeof(double);
  p.warps = 4;
  if (col * 5 <= limit) {
    p.lam_smem = p.col_smem = true;
    p.bytes = col * 5;
    return p;
  }
  p.col_smem = false;
  p.lam_smem = false;
  p.bytes = 0;
  return p;
}

}  // namespace imcom
