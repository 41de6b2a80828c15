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
  int n, m;
  int UnotS;
  double US_max, k_min, k_max, tol, C, eps;
  double lg_min, lg_max;  // log10(k_min), log10(k_max) from the host libm
  int maxnits;
};

// The reference's bisection for one pixel (imcom_bisect_by_U / _by_S).
__device__ __forceinline__ void bisect_pixel(const BisectArgs& a, const double* lam,
                                             const double* col, int lane, int* nev_out,
                                             double* k_out, double* us_out) {
  const bool U = a.UnotS != 0;
  int nev = 0;
  double k_root, us;
  // imcom_bisect_by_U: U(k_min) first; imcom_bisect_by_S: S(k_max) first.
  double k0 = U ? a.k_min : a.k_max;
  us = warp_us(U, lam, col, a.Nd, a.n, k0, a.C, lane);
  nev = 1;
  double f = __dsub_rn(us, a.US_max);
  if (!(f < 0.0)) {
    k_root = k0;
  } else {
    double lo = U ? a.lg_min : a.lg_max;
    double hi = U ? a.lg_max : a.lg_min;
    double root = lo, dx = __dsub_rn(hi, lo);
    for (int i = 1; i <= a.maxnits; ++i) {
      dx = __dmul_rn(0.5, dx);
      double mid = __dadd_rn(root, dx);
      double fmid = __dsub_rn(warp_us(U, lam, col, a.Nd, a.n, pow(10.0, mid), a.C, lane), a.US_max);
      ++nev;
      if (fmid < 0.0) {
        root = mid;
        us = __dadd_rn(fmid, a.US_max);
        if (fabs(fmid) < a.tol) break;
      }
      if (fabs(fmid) < __dmul_rn(a.C, a.eps)) break;
    }
    k_root = pow(10.0, root);
  }
  *nev_out = nev;
  *k_out = k_root;
  *us_out = us;
}

__device__ __forceinline__ void write_pixel(const BisectArgs& a, const double* lam, const double* col, int pix,
                            int lane, int nev, double k, double us) {
  if (lane == 0) {
    a.K[pix] = k;
    a.US[pix] = us;
    if (a.nev) a.nev[pix] = nev;
  }
  if (a.Pt) {
    double* dst = a.Pt + (size_t)pix * a.ldt;
    for (int p = lane; p < a.n; p += 32) dst[p] = __ddiv_rn(col[p], __dadd_rn(lam[p], k));
  }
}

int fill_bisect_args(imcom_ctx* ctx, BisectArgs& a, int UnotS, double US_max, double k_min,
                     double k_max, double tol, int maxnits, double C_a);
int pixel_grid(imcom_ctx* ctx, const PixelSmem& plan, int m);
int copy_pixel_outputs(imcom_ctx* ctx, double* K_out, double* US_out, int* nev_out);
int make_Pt(imcom_ctx* ctx);

}  // namespace imcom
