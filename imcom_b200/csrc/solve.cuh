// solve.cuh -- per-pixel bisection pieces shared by the plain and the
// learned-kappa kernels.
#pragma once

#include "common.cuh"
#include "usum.cuh"

namespace imcom {

struct BisectArgs {
  const double* L;
  const double* P;
  long long ldp;
  const double* Nd;
  double* Pt;  // P~ = P(:, a) / (L + K_a), may be null
  long long ldt;
  double* K;
  double* US;
  int* nev;
  double* margin;   // per pixel: smallest |f - threshold| over the evaluations, may be null
  const int* list;  // pixels to solve (count of them), or null for all m
  int count;
  int n, m;
  int UnotS;
  double US_max, k_min, k_max, tol, C, eps;
  double lg_min, lg_max;  // log10(k_min), log10(k_max) from the host libm
  int maxnits;
};

// Distance of f = U - U_max (or S - S_max) to the thresholds the bisection
// compares it with (0, tol, C eps): a perturbation of f smaller than this
// cannot change any decision taken on it.
__device__ __forceinline__ double decision_margin(double f, double tol, double ceps) {
  const double af = fabs(f);
  return fmin(af, fmin(fabs(af - tol), fabs(af - ceps)));
}

// The reference's bisection for one pixel (imcom_bisect_by_U / _by_S);
// ev(k, lane) is U or S at kappa k (StreamCol or ResCol).  *mg_out receives
// the smallest decision margin over the evaluations.
template <class Eval>
__device__ __forceinline__ void bisect_pixel(const BisectArgs& a, const Eval& ev, int lane,
                                             int* nev_out, double* k_out, double* us_out,
                                             double* mg_out) {
  const bool U = a.UnotS != 0;
  int nev = 0;
  double k_root, us;
  const double ceps = __dmul_rn(a.C, a.eps);
  // imcom_bisect_by_U: U(k_min) first; imcom_bisect_by_S: S(k_max) first.
  double k0 = U ? a.k_min : a.k_max;
  us = ev(k0, lane);
  nev = 1;
  double f = __dsub_rn(us, a.US_max);
  double mg = fabs(f);
  if (!(f < 0.0)) {
    k_root = k0;
  } else {
    double lo = U ? a.lg_min : a.lg_max;
    double hi = U ? a.lg_max : a.lg_min;
    double root = lo, dx = __dsub_rn(hi, lo);
    for (int i = 1; i <= a.maxnits; ++i) {
      dx = __dmul_rn(0.5, dx);
      double mid = __dadd_rn(root, dx);
      double fmid = __dsub_rn(ev(pow(10.0, mid), lane), a.US_max);
      ++nev;
      mg = fmin(mg, decision_margin(fmid, a.tol, ceps));
      if (fmid < 0.0) {
        root = mid;
        us = __dadd_rn(fmid, a.US_max);
        if (fabs(fmid) < a.tol) break;
      }
      if (fabs(fmid) < ceps) break;
    }
    k_root = pow(10.0, root);
  }
  *nev_out = nev;
  *k_out = k_root;
  *us_out = us;
  *mg_out = mg;
}

// Outputs of one pixel, written by the nw warps that solved it together
// (warp wid of them; one warp: wid 0, nw 1).
__device__ __forceinline__ void write_pixel(const BisectArgs& a, const double* lam, const double* col, int pix,
                            int lane, int nev, double k, double us, double mg, int wid = 0,
                            int nw = 1) {
  if (lane == 0 && wid == 0) {
    a.K[pix] = k;
    a.US[pix] = us;
    if (a.nev) a.nev[pix] = nev;
    if (a.margin) a.margin[pix] = mg;
  }
  if (a.Pt) {
    double* dst = a.Pt + (size_t)pix * a.ldt;
    for (int p = lane + 32 * wid; p < a.n; p += 32 * nw)
      dst[p] = __ddiv_rn(col[p], __dadd_rn(lam[p], k));
  }
}

int fill_bisect_args(imcom_ctx* ctx, BisectArgs& a, int UnotS, double US_max, double k_min,
                     double k_max, double tol, int maxnits, double C_a);
int pixel_grid(imcom_ctx* ctx, const PixelSmem& plan, int m);
int copy_pixel_outputs(imcom_ctx* ctx, double* K_out, double* US_out, int* nev_out);
int make_Pt(imcom_ctx* ctx);
// Plain bisection over a.list (or all pixels).
int launch_bisect(imcom_ctx* ctx, const BisectArgs& a);
// Split-precision P: per-pixel margin buffer before the bisection, and the
// error audit with FP64 recomputation of the failing pixels after it
// (split.cu).
int split_margin_buffer(imcom_ctx* ctx, BisectArgs& a);
int split_audit(imcom_ctx* ctx, const BisectArgs& a);

}  // namespace imcom
