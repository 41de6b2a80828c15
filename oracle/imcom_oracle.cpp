// imcom_oracle.cpp -- CPU restatement of the IMCOM solve path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the timed
// CPU baseline for the GPU library in imcom_b200/.  Only tests/, the smoke
// check in __graft_entry__.py and the CPU-baseline leg of bench.py may load
// it.  The product path never calls it.
//
// What it restates (reference = barnabytprowe/imcom, Fortran 95):
//   imcom_proc.f90   imcom_rotate_image (:184-250), imcom_polint (:351-394),
//                    imcom_polin2 (:398-429), imcom_iminloc (:338-347),
//                    imcom_ft_r2c (:433-475) incl. the Hermitian fill.
//   imcom_matrix.f90 imcom_build_Alookup (:361-430), imcom_build_Blookup
//                    (:434-493), imcom_interp_lookup (:497-542), imcom_calc_C
//                    (:546-552), imcom_build_Ndiag (:556-582), imcom_lookup_A
//                    (:206-284), imcom_lookup_B (:288-357), imcom_eigen_A
//                    (:586-678), imcom_build_P (:682-712), imcom_build_T
//                    (:716-750), imcom_build_image (:754-790), imcom_build_U
//                    (:795-835), imcom_build_S (:839-877), imcom_U_from_kappa
//                    (:904-922), imcom_S_from_kappa (:955-970).
//   imcom_bisect.f90 imcom_bisect_kappa (:78-170), imcom_bisect_by_U
//                    (:174-222), imcom_bisect_by_S (:226-267).
//
// Third-party arithmetic: the reference links LAPACK DSYEVR/DLAMCH and BLAS
// DGEMM/DGEMV/DDOT (unpinned; macOS Accelerate in its Makefile:17) and FFTW
// >= 3.2.2.  Here the LAPACK/BLAS calls are the real routines, linked from
// the OpenBLAS that scipy bundles (scipy_dsyevr_, scipy_dgemm_, ...).  FFTW
// is replaced by the exact mixed-radix DFT below (same sign and
// normalisation conventions as FFTW: forward -1, backward +1, unnormalised),
// which the tests pin against numpy.fft.
//
// Parity status: PARITY UNPINNED against reference outputs.  The reference
// ships no golden vectors or tests for this path and cannot be compiled in
// this environment (no Fortran compiler, FFTW or CFITSIO).  The pieces are
// pinned instead by known-answer tests: Neville reproduces polynomials of
// degree <= 7 exactly, the FFT matches numpy.fft, DSYEVR is LAPACK's own, the
// table builder reproduces the analytic Gaussian autocorrelation, and the
// bisection obeys its own termination contract.
//
// Compiled with -ffp-contract=off so every expression rounds as written, as
// the reference does when built by gfortran for baseline x86-64.
// Arrays are Fortran column-major; indices inside loops are 1-based where the
// reference's arithmetic depends on it.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <omp.h>

extern "C" {
double scipy_dlamch_(const char* cmach, size_t len);
void scipy_dsyevr_(const char* jobz, const char* range, const char* uplo,
                   const int* n, double* a, const int* lda, const double* vl,
                   const double* vu, const int* il, const int* iu,
                   const double* abstol, int* m, double* w, double* z,
                   const int* ldz, int* isuppz, double* work, const int* lwork,
                   int* iwork, const int* liwork, int* info, size_t, size_t,
                   size_t);
void scipy_dgemm_(const char* ta, const char* tb, const int* m, const int* n,
                  const int* k, const double* alpha, const double* a,
                  const int* lda, const double* b, const int* ldb,
                  const double* beta, double* c, const int* ldc, size_t,
                  size_t);
void scipy_dgemv_(const char* t, const int* m, const int* n,
                  const double* alpha, const double* a, const int* lda,
                  const double* x, const int* incx, const double* beta,
                  double* y, const int* incy, size_t);
double scipy_ddot_(const int* n, const double* x, const int* incx,
                   const double* y, const int* incy);
void scipy_openblas_set_num_threads(int);
}

namespace {

typedef std::complex<double> cplx;

// Plain complex product (a+bi)(c+di) = (ac-bd) + (ad+bc)i, the expression
// Fortran evaluates for complex(KIND=8) multiplication.
inline cplx cmul(cplx a, cplx b) {
  double ar = a.real(), ai = a.imag(), br = b.real(), bi = b.imag();
  return cplx(ar * br - ai * bi, ar * bi + ai * br);
}

int g_threads = 0;  // 0 = all cores

void set_blas_threads(int n) { scipy_openblas_set_num_threads(n); }

int omp_threads() { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

double dlamch(char c) { return scipy_dlamch_(&c, 1); }

// ---------------------------------------------------------------------------
// Mixed-radix DFT (stand-in for FFTW's DFT; any length).
// ---------------------------------------------------------------------------
struct FftPlan {
  int n = 0;
  int sign = -1;
  std::vector<int> factors;
  std::vector<cplx> tw;  // tw[j] = exp(sign * 2 pi i j / n)
};

FftPlan make_plan(int n, int sign) {
  FftPlan p;
  p.n = n;
  p.sign = sign;
  int r = n;
  const int pref[] = {4, 2, 3, 5};
  for (int f : pref) {
    while (r % f == 0) {
      p.factors.push_back(f);
      r /= f;
    }
  }
  for (int f = 7; r > 1; f += 2) {
    while (r % f == 0) {
      p.factors.push_back(f);
      r /= f;
    }
  }
  p.tw.resize(n);
  for (int j = 0; j < n; ++j) {
    long double ang = (long double)sign * 2.0L * 3.14159265358979323846264338327950288L *
                      (long double)j / (long double)n;
    p.tw[j] = cplx((double)cosl(ang), (double)sinl(ang));
  }
  return p;
}

// Decimation in time: out[k + q*m] = sum_r W_n^{r(k+qm)} Y_r[k].
void fft_rec(const FftPlan& p, const cplx* in, int istride, cplx* out, int n,
             size_t level, cplx* scratch) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int f = p.factors[level];
  int m = n / f;
  for (int r = 0; r < f; ++r)
    fft_rec(p, in + (size_t)r * istride, istride * f, out + (size_t)r * m, m,
            level + 1, scratch);
  int tstep = p.n / n;  // W_n^j = tw[j * tstep]
  cplx t[64];
  std::vector<cplx> tbig;
  cplx* tt = t;
  if (f > 64) {
    tbig.resize(f);
    tt = tbig.data();
  }
  for (int k = 0; k < m; ++k) {
    for (int r = 0; r < f; ++r) {
      size_t idx = ((size_t)r * k % n) * tstep;
      tt[r] = cmul(out[(size_t)r * m + k], p.tw[idx]);
    }
    for (int q = 0; q < f; ++q) {
      cplx s(0.0, 0.0);
      int step = (p.n / f);  // W_f^{rq} = tw[(r*q mod f) * n_total/f]
      for (int r = 0; r < f; ++r) {
        s += cmul(tt[r], p.tw[(size_t)((r * q) % f) * step]);
      }
      scratch[(size_t)q * m + k] = s;
    }
    for (int q = 0; q < f; ++q) out[(size_t)q * m + k] = scratch[(size_t)q * m + k];
  }
}

void fft1d(const FftPlan& p, const cplx* in, int istride, cplx* out) {
  std::vector<cplx> scratch(p.n);
  fft_rec(p, in, istride, out, p.n, 0, scratch.data());
}

// 2-D DFT of a column-major (n1, n2) complex array, in place.
void fft2d(cplx* a, int n1, int n2, int sign) {
  FftPlan p1 = make_plan(n1, sign), p2 = make_plan(n2, sign);
#pragma omp parallel num_threads(omp_threads())
  {
    std::vector<cplx> buf(std::max(n1, n2)), res(std::max(n1, n2));
#pragma omp for schedule(static)
    for (int j = 0; j < n2; ++j) {
      fft1d(p1, a + (size_t)j * n1, 1, res.data());
      std::memcpy(a + (size_t)j * n1, res.data(), sizeof(cplx) * n1);
    }
#pragma omp for schedule(static)
    for (int i = 0; i < n1; ++i) {
      for (int j = 0; j < n2; ++j) buf[j] = a[i + (size_t)j * n1];
      fft1d(p2, buf.data(), 1, res.data());
      for (int j = 0; j < n2; ++j) a[i + (size_t)j * n1] = res[j];
    }
  }
}

// Fortran CSHIFT index: cshift(X, s)(i) = X(1 + mod(i - 1 + s, n)), 1-based.
inline int cshift_src(int i1, int s, int n) { return 1 + ((i1 - 1 + s) % n + n) % n; }

// ---------------------------------------------------------------------------
// Neville interpolation: imcom_polint / imcom_polin2 (imcom_proc.f90:351-429)
// ---------------------------------------------------------------------------
// Returns 0, or 1 when two abscissae coincide (the reference stops there).
int polint(const double* xa, const double* ya, int n, double x, double* y,
           double* dy, double eps) {
  double c[16], d[16], den[16], ho[16];
  for (int i = 0; i < n; ++i) {
    c[i] = ya[i];
    d[i] = ya[i];
    ho[i] = xa[i] - x;
  }
  // imcom_iminloc(abs(x - xa)): first index of the minimum, 1-based.
  int ns = 1;
  double best = std::fabs(x - xa[0]);
  for (int i = 1; i < n; ++i) {
    double v = std::fabs(x - xa[i]);
    if (v < best) {
      best = v;
      ns = i + 1;
    }
  }
  *y = ya[ns - 1];
  ns = ns - 1;
  for (int m = 1; m <= n - 1; ++m) {
    for (int i = 1; i <= n - m; ++i) den[i - 1] = ho[i - 1] - ho[i + m - 1];
    for (int i = 1; i <= n - m; ++i)
      if (std::fabs(den[i - 1]) <= eps) return 1;
    for (int i = 1; i <= n - m; ++i) den[i - 1] = (c[i] - d[i - 1]) / den[i - 1];
    for (int i = 1; i <= n - m; ++i) {
      d[i - 1] = ho[i + m - 1] * den[i - 1];
      c[i - 1] = ho[i - 1] * den[i - 1];
    }
    if (2 * ns < n - m) {
      *dy = c[ns];  // c(ns + 1)
    } else {
      *dy = d[ns - 1];  // d(ns)
      ns = ns - 1;
    }
    *y = *y + *dy;
  }
  return 0;
}

// ya is the column-major window ya(1:m1, 1:m2) taken from a parent array with
// leading dimension ld.
int polin2(const double* x1a, int m1, const double* x2a, int m2,
           const double* ya, int ld, double x1, double x2, double* y,
           double* dy, double eps) {
  double ymtmp[16], yntmp[16];
  for (int j = 0; j < m1; ++j) {
    for (int k = 0; k < m2; ++k) yntmp[k] = ya[j + (size_t)k * ld];
    if (polint(x2a, yntmp, m2, x2, &ymtmp[j], dy, eps)) return 1;
  }
  return polint(x1a, ymtmp, m1, x1, y, dy, eps);
}

}  // namespace

extern "C" {

// Threads used by the OpenMP loops (0 = all host cores).
void oracle_set_threads(int n) { g_threads = n; }

int oracle_get_threads(void) { return omp_threads(); }

double oracle_dlamch(const char* c) { return dlamch(c[0]); }

// Exposed for the FFT known-answer test: 2-D DFT of a column-major complex
// (n1, n2) array (interleaved re/im), in place.
void oracle_fft2d(int n1, int n2, int sign, double* a) {
  fft2d(reinterpret_cast<cplx*>(a), n1, n2, sign);
}

// imcom_polint restated (imcom_proc.f90:351-394).  Returns the trap status.
int oracle_polint(int n, const double* xa, const double* ya, double x,
                  double* y) {
  double dy;
  return polint(xa, ya, n, x, y, &dy, dlamch('E'));
}

// imcom_rotate_image (imcom_proc.f90:184-250).  cost/sint are taken from the
// caller when use_cs != 0 (so GPU and oracle can share one libm result);
// otherwise they are computed here exactly as the reference does.
int oracle_rotate_image(int nim1, int nim2, const double* im_in,
                        double theta_deg, int npoly_in, int conserve_flux,
                        double* im_out) {
  const double pi = 3.141592653589793;  // imcom_data.f90 parameter pi
  int npoly = npoly_in;
  if (npoly % 2 == 0) npoly = npoly - 1;
  int npm = npoly / 2;
  double theta_rad = std::fmod(theta_deg, 360.0) * pi / 180.0;
  double cost = std::cos(theta_rad);
  double sint = std::sin(theta_rad);
  double x_cent = (double)(nim1 + 1) / 2.0;
  double y_cent = (double)(nim2 + 1) / 2.0;
  double eps = dlamch('E');
  int bad = 0;
#pragma omp parallel for num_threads(omp_threads()) reduction(| : bad)
  for (int iout = 1; iout <= nim1; ++iout) {
    double xout = (double)iout - x_cent;
    double xa[16], ya[16];
    for (int jout = 1; jout <= nim2; ++jout) {
      double yout = (double)jout - y_cent;
      double xs = xout * cost + yout * sint + x_cent;
      double ys = -xout * sint + yout * cost + y_cent;
      int is_floor = (int)std::floor(xs), js_floor = (int)std::floor(ys);
      int is_ceil = (int)std::ceil(xs), js_ceil = (int)std::ceil(ys);
      double f = 0.0, df;
      if (is_floor >= 1 && js_floor >= 1 && is_ceil <= nim1 && js_ceil <= nim2) {
        int imin = std::max(1, is_floor - npm), jmin = std::max(1, js_floor - npm);
        int imax = std::min(nim1, is_ceil + npm), jmax = std::min(nim2, js_ceil + npm);
        for (int ii = imin; ii <= imax; ++ii) xa[ii - imin] = (double)ii;
        for (int jj = jmin; jj <= jmax; ++jj) ya[jj - jmin] = (double)jj;
        bad |= polin2(xa, imax - imin + 1, ya, jmax - jmin + 1,
                      im_in + (imin - 1) + (size_t)(jmin - 1) * nim1, nim1, xs,
                      ys, &f, &df, eps);
      }
      im_out[(iout - 1) + (size_t)(jout - 1) * nim1] = f;
    }
  }
  if (conserve_flux != 0) {
    // im_out = sum(im_in) * im_out / sum(im_out): gfortran's SUM is a plain
    // sequential loop in array-element order.
    double sin_ = 0.0, sout = 0.0;
    size_t tot = (size_t)nim1 * nim2;
    for (size_t k = 0; k < tot; ++k) sin_ += im_in[k];
    for (size_t k = 0; k < tot; ++k) sout += im_out[k];
    for (size_t k = 0; k < tot; ++k) im_out[k] = sin_ * im_out[k] / sout;
  }
  return bad;
}

// imcom_ft_r2c (imcom_proc.f90:433-475): forward DFT of a real (n1, n2) array
// and the reference's Hermitian fill of the full complex array.  Ft is
// interleaved complex, column-major (n1, n2).
void oracle_ft_r2c(int n1, int n2, const double* F, double* Ft_out) {
  std::vector<cplx> full((size_t)n1 * n2);
  for (size_t k = 0; k < full.size(); ++k) full[k] = cplx(F[k], 0.0);
  fft2d(full.data(), n1, n2, -1);
  // Ft_tmp(0:n1/2, 0:n2-1) is the r2c half spectrum.
  cplx* Ft = reinterpret_cast<cplx*>(Ft_out);
  auto tmp = [&](int i, int j) { return full[i + (size_t)j * n1]; };
  for (int j = 0; j < n2; ++j)
    for (int i = 0; i <= n1 / 2; ++i) Ft[i + (size_t)j * n1] = tmp(i, j);
  // Ft_dum(n1/2+1 : n1-1, 0) = conj(Ft_tmp((n1-1)/2 : 1 : -1, 0))
  for (int t = 0; t < n1 - 1 - n1 / 2; ++t)
    Ft[n1 / 2 + 1 + t] = std::conj(tmp((n1 - 1) / 2 - t, 0));
  for (int i = 1; i <= (n1 - 1) / 2; ++i) {
    int src = (n1 % 2 == 0) ? (n1 / 2 - i) : (n1 / 2 + 1 - i);
    for (int j = 1; j <= n2 - 1; ++j)
      Ft[(n1 / 2 + i) + (size_t)j * n1] = std::conj(tmp(src, n2 - j));
  }
}

// imcom_build_Alookup (imcom_matrix.f90:361-430) and imcom_build_Blookup
// (:434-493) share this body.  Gt: interleaved complex (nps, nps, nexppsf).
// For A (gammat == nullptr): one table per packed pair ial = e + f(f-1)/2,
// e <= f.  For B: one table per exposure, from conj(Gammat) * Gt_e, times -2.
static void build_lookup(int nps, int npad, int nexppsf, const double* Gt_in,
                         const double* Gammat_in, double* lookup) {
  const cplx* Gt = reinterpret_cast<const cplx*>(Gt_in);
  const cplx* Gam = reinterpret_cast<const cplx*>(Gammat_in);
  int nbig = nps * npad;
  int nmin = (nbig - nps) / 2 + 1;
  size_t big2 = (size_t)nbig * nbig, ps2 = (size_t)nps * nps;
  std::vector<std::pair<int, int>> jobs;
  if (Gam == nullptr) {
    for (int iexp = 1; iexp <= nexppsf; ++iexp)
      for (int jexp = iexp; jexp <= nexppsf; ++jexp) jobs.push_back({iexp, jexp});
  } else {
    for (int iexp = 1; iexp <= nexppsf; ++iexp) jobs.push_back({iexp, 0});
  }
  std::vector<cplx> ufunc(big2), ufunc2(big2);
  for (auto& jb : jobs) {
    int iexp = jb.first, jexp = jb.second;
    int ial = (Gam == nullptr) ? iexp + jexp * (jexp - 1) / 2 : iexp;
    std::fill(ufunc.begin(), ufunc.end(), cplx(0.0, 0.0));
    // ufunc(nmin:nmax, nmin:nmax) = cshift(cshift(X, nps/2, 2), nps/2, 1)
    for (int j = 1; j <= nps; ++j) {
      int sj = cshift_src(j, nps / 2, nps);
      for (int i = 1; i <= nps; ++i) {
        int si = cshift_src(i, nps / 2, nps);
        size_t s = (size_t)(si - 1) + (size_t)(sj - 1) * nps;
        cplx x = (Gam == nullptr)
                     ? cmul(std::conj(Gt[s + (iexp - 1) * ps2]), Gt[s + (jexp - 1) * ps2])
                     : cmul(std::conj(Gam[s]), Gt[s + (iexp - 1) * ps2]);
        x = cmul(x, cplx(1.0, 0.0));  // imcom_upsilon2D(ux, uy, 1) == 1
        ufunc[(size_t)(nmin + i - 2) + (size_t)(nmin + j - 2) * nbig] = x;
      }
    }
    // ufunc = cshift(cshift(ufunc, nbig/2, 2), nbig/2, 1)
    for (int q = 1; q <= nbig; ++q) {
      int sq = cshift_src(q, nbig / 2, nbig);
      for (int p = 1; p <= nbig; ++p) {
        int sp = cshift_src(p, nbig / 2, nbig);
        ufunc2[(size_t)(p - 1) + (size_t)(q - 1) * nbig] =
            ufunc[(size_t)(sp - 1) + (size_t)(sq - 1) * nbig];
      }
    }
    fft2d(ufunc2.data(), nbig, nbig, +1);  // FFTW_BACKWARD, unnormalised
    double* out = lookup + (size_t)(ial - 1) * big2;
    for (int q = 1; q <= nbig; ++q) {
      int sq = cshift_src(q, nbig / 2, nbig);
      for (int p = 1; p <= nbig; ++p) {
        int sp = cshift_src(p, nbig / 2, nbig);
        double v = ufunc2[(size_t)(sp - 1) + (size_t)(sq - 1) * nbig].real();
        if (Gam != nullptr) v = -2.0 * v;
        out[(size_t)(p - 1) + (size_t)(q - 1) * nbig] = v;
      }
    }
  }
  // Alookup = Alookup / real(n1psf) / real(n2psf)
  size_t ntab = jobs.size();
  for (size_t k = 0; k < ntab * big2; ++k) lookup[k] = lookup[k] / (double)nps / (double)nps;
}

void oracle_build_Alookup(int nps, int npad, int nexppsf, const double* Gt,
                          double* Alookup) {
  build_lookup(nps, npad, nexppsf, Gt, nullptr, Alookup);
}

void oracle_build_Blookup(int nps, int npad, int nexppsf, const double* Gt,
                          const double* Gammat, double* Blookup) {
  build_lookup(nps, npad, nexppsf, Gt, Gammat, Blookup);
}

// imcom_calc_C (imcom_matrix.f90:546-552): sum(real(Gammat*conj(Gammat)*1))
// / n1psf / n2psf, summed in array-element order.
double oracle_calc_C(int nps, const double* Gammat_in) {
  const cplx* G = reinterpret_cast<const cplx*>(Gammat_in);
  double s = 0.0;
  size_t tot = (size_t)nps * nps;
  for (size_t k = 0; k < tot; ++k) {
    cplx v = cmul(cmul(G[k], std::conj(G[k])), cplx(1.0, 0.0));
    s += v.real();
  }
  return s / (double)nps / (double)nps;
}

// imcom_build_Ndiag (imcom_matrix.f90:556-582): contiguous blocks of n/nexp.
void oracle_build_Ndiag(int n, int nexp, const double* noise, double* Ndiag) {
  for (int i = 0; i < n; ++i) Ndiag[i] = 0.0;
  for (int i = 1; i <= nexp; ++i) {
    int n_i = 1 + (i - 1) * (n / nexp);
    int n_f = (i != nexp) ? i * (n / nexp) : n;
    for (int k = n_i; k <= n_f; ++k) Ndiag[k - 1] = noise[i - 1];
  }
}

// imcom_interp_lookup (imcom_matrix.f90:497-542).  *window receives
// (imin, imax, jmin, jmax) (1-based), or zeros when out of range; *status is
// set to 1 if Neville trapped.
double oracle_interp_lookup(int n1, int n2, const double* lookup, double xarg,
                            double yarg, int npoly_in, int* window,
                            int* status) {
  int npoly = npoly_in;
  if (npoly % 2 == 0) npoly = npoly - 1;
  int npm = npoly / 2;
  double icent = (double)(n1 / 2 + 1), jcent = (double)(n2 / 2 + 1);
  double iarg = icent + xarg, jarg = jcent + yarg;
  int ia_floor = (int)std::floor(iarg), ja_floor = (int)std::floor(jarg);
  int ia_ceil = (int)std::ceil(iarg), ja_ceil = (int)std::ceil(jarg);
  if (ia_floor >= 1 && ja_floor >= 1 && ia_ceil <= n1 && ja_ceil <= n2) {
    int imin = std::max(1, ia_floor - npm), jmin = std::max(1, ja_floor - npm);
    int imax = std::min(n1, ia_ceil + npm), jmax = std::min(n2, ja_ceil + npm);
    double xa[16], ya[16], f, df;
    for (int ii = imin; ii <= imax; ++ii) xa[ii - imin] = (double)ii;
    for (int jj = jmin; jj <= jmax; ++jj) ya[jj - jmin] = (double)jj;
    if (window) {
      window[0] = imin; window[1] = imax; window[2] = jmin; window[3] = jmax;
    }
    int st = polin2(xa, imax - imin + 1, ya, jmax - jmin + 1,
                    lookup + (imin - 1) + (size_t)(jmin - 1) * n1, n1, iarg,
                    jarg, &f, &df, dlamch('E'));
    if (status) *status |= st;
    return f;
  }
  if (window) window[0] = window[1] = window[2] = window[3] = 0;
  return 0.0;
}

// imcom_lookup_A (imcom_matrix.f90:206-284).  exp_i is 1-based.  Alookup is
// (nbig, nbig, ntab).  Returns the Neville trap status.
int oracle_lookup_A(int n, const double* x_i, const double* y_i,
                    const int* exp_i, int psfconst, int nps, int npad,
                    double psfxscale, double psfyscale, int npoly,
                    const double* Alookup, double* A) {
  int nbig = nps * npad;
  size_t big2 = (size_t)nbig * nbig;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(omp_threads()) reduction(| : bad)
  for (int i = 1; i <= n; ++i) {
    for (int j = i; j <= n; ++j) {
      int ial = (psfconst == 1)
                    ? 1
                    : exp_i[i - 1] + exp_i[j - 1] * (exp_i[j - 1] - 1) / 2;
      double Delx = (double)npad * (x_i[j - 1] - x_i[i - 1]) / psfxscale;
      double Dely = (double)npad * (y_i[j - 1] - y_i[i - 1]) / psfyscale;
      int st = 0;
      A[(size_t)(i - 1) + (size_t)(j - 1) * n] = oracle_interp_lookup(
          nbig, nbig, Alookup + (size_t)(ial - 1) * big2, Delx, Dely, npoly,
          nullptr, &st);
      bad |= st;
    }
  }
#pragma omp parallel for num_threads(omp_threads())
  for (int i = 2; i <= n; ++i)
    for (int j = 1; j <= i - 1; ++j)
      A[(size_t)(i - 1) + (size_t)(j - 1) * n] = A[(size_t)(j - 1) + (size_t)(i - 1) * n];
  return bad;
}

// imcom_lookup_B (imcom_matrix.f90:288-357).
int oracle_lookup_B(int n, int m, const double* x_i, const double* y_i,
                    const int* exp_i, const double* X_a, const double* Y_a,
                    int psfconst, int nps, int npad, double psfxscale,
                    double psfyscale, int npoly, const double* Blookup,
                    double* B) {
  int nbig = nps * npad;
  size_t big2 = (size_t)nbig * nbig;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(omp_threads()) reduction(| : bad)
  for (int i = 1; i <= n; ++i) {
    int itab = (psfconst == 1) ? 1 : exp_i[i - 1];
    for (int a = 1; a <= m; ++a) {
      double Delx = (double)npad * (x_i[i - 1] - X_a[a - 1]) / psfxscale;
      double Dely = (double)npad * (y_i[i - 1] - Y_a[a - 1]) / psfyscale;
      int st = 0;
      B[(size_t)(i - 1) + (size_t)(a - 1) * n] = oracle_interp_lookup(
          nbig, nbig, Blookup + (size_t)(itab - 1) * big2, Delx, Dely, npoly,
          nullptr, &st);
      bad |= st;
    }
  }
  return bad;
}

// imcom_eigen_A (imcom_matrix.f90:586-678): DSYEVR('V','A','U') with
// abstol = DLAMCH('Safe minimum'), then reversal into descending order.
// Returns LAPACK's info.
int oracle_eigen_A(int n, const double* A, double* Q, double* L,
                   double* condition) {
  std::vector<double> Atmp(A, A + (size_t)n * n);
  std::vector<int> isupport(2 * (size_t)n);
  double abstol = dlamch('S');
  double vl = 0.0, vu = 0.0, worktest[1];
  int il = 0, iu = 0, n_out = 0, info = 0, lwork = -1, liwork = -1, iworktest[1];
  set_blas_threads(omp_threads());
  scipy_dsyevr_("V", "A", "U", &n, Atmp.data(), &n, &vl, &vu, &il, &iu, &abstol,
                &n_out, L, Q, &n, isupport.data(), worktest, &lwork, iworktest,
                &liwork, &info, 1, 1, 1);
  if (info != 0) return info;
  lwork = (int)std::lround(worktest[0]);
  liwork = iworktest[0];
  std::vector<double> work(lwork);
  std::vector<int> iwork(liwork);
  n_out = n;
  scipy_dsyevr_("V", "A", "U", &n, Atmp.data(), &n, &vl, &vu, &il, &iu, &abstol,
                &n_out, L, Q, &n, isupport.data(), work.data(), &lwork,
                iwork.data(), &liwork, &info, 1, 1, 1);
  if (info != 0) return info;
  // L_i = L_i(n:1:-1); Q_ij = Q_ij(:, n:1:-1)
  for (int k = 0; k < n / 2; ++k) {
    std::swap(L[k], L[n - 1 - k]);
    std::swap_ranges(Q + (size_t)k * n, Q + (size_t)(k + 1) * n,
                     Q + (size_t)(n - 1 - k) * n);
  }
  double lmax = L[0], lmin = L[0];
  for (int k = 1; k < n; ++k) {
    lmax = std::max(lmax, L[k]);
    lmin = std::min(lmin, L[k]);
  }
  *condition = lmax / lmin;
  return 0;
}

// imcom_build_P (imcom_matrix.f90:682-712): P = Q^T B (DGEMM), P2 = P * P.
void oracle_build_P(int n, int m, const double* Q, const double* B, double* P,
                    double* P2) {
  double one = 1.0, zero = 0.0;
  set_blas_threads(omp_threads());
  scipy_dgemm_("T", "N", &n, &m, &n, &one, Q, &n, B, &n, &zero, P, &n, 1, 1);
  if (P2) {
    size_t tot = (size_t)n * m;
    for (size_t k = 0; k < tot; ++k) P2[k] = P[k] * P[k];
  }
}

// imcom_U_from_kappa (imcom_matrix.f90:904-922).  P2a is the column P2(:, a).
double oracle_U_from_kappa(int n, const double* L, const double* P2a, double C,
                           double k) {
  std::vector<double> v(n), ones(n, 1.0);
  for (int p = 0; p < n; ++p) {
    double denom = (L[p] + k) * (L[p] + k);
    v[p] = (L[p] + 2.0 * k) * P2a[p] / denom;
  }
  int inc = 1;
  double Usum = scipy_ddot_(&n, v.data(), &inc, ones.data(), &inc);
  return (C - Usum / 4.0) / C;
}

// imcom_S_from_kappa (imcom_matrix.f90:955-970).  Ndiag is indexed by
// eigenmode, as in the reference.
double oracle_S_from_kappa(int n, const double* L, const double* P2a,
                           const double* Ndiag, double k) {
  std::vector<double> v(n), ones(n, 1.0);
  for (int p = 0; p < n; ++p) {
    double denom = (L[p] + k) * (L[p] + k);
    v[p] = Ndiag[p] * P2a[p] / denom;
  }
  int inc = 1;
  double Ssum = scipy_ddot_(&n, v.data(), &inc, ones.data(), &inc);
  return Ssum / 4.0;
}

// imcom_bisect_by_U (imcom_bisect.f90:174-222).  *nevals counts U
// evaluations (1 + bisection steps taken).
static void bisect_by_U(int n, const double* L, const double* P2a, double C,
                        double k_min, double k_max, double U_max, double tol,
                        int maxnits, double* k_root, double* U_out,
                        int* nevals) {
  double eps = dlamch('E');
  *U_out = oracle_U_from_kappa(n, L, P2a, C, k_min);
  *nevals = 1;
  double f = *U_out - U_max, lo, hi;
  if (f < 0.0) {
    lo = std::log10(k_min);
    hi = std::log10(k_max);
  } else {
    *k_root = k_min;
    return;
  }
  double root = lo, dx = hi - lo;
  for (int i = 1; i <= maxnits; ++i) {
    dx = 0.5 * dx;
    double mid = root + dx;
    double fmid = oracle_U_from_kappa(n, L, P2a, C, std::pow(10.0, mid)) - U_max;
    *nevals += 1;
    if (fmid < 0.0) {
      root = mid;
      *U_out = fmid + U_max;
      if (std::fabs(fmid) < tol) break;
    }
    if (std::fabs(fmid) < C * eps) break;
  }
  *k_root = std::pow(10.0, root);
}

// imcom_bisect_by_S (imcom_bisect.f90:226-267).
static void bisect_by_S(int n, const double* L, const double* P2a,
                        const double* Ndiag, double C, double k_min,
                        double k_max, double S_max, double tol, int maxnits,
                        double* k_root, double* S_out, int* nevals) {
  double eps = dlamch('E');
  *S_out = oracle_S_from_kappa(n, L, P2a, Ndiag, k_max);
  *nevals = 1;
  double f = *S_out - S_max, lo, hi;
  if (f < 0.0) {
    lo = std::log10(k_max);
    hi = std::log10(k_min);
  } else {
    *k_root = k_max;
    return;
  }
  double root = lo, dx = hi - lo;
  for (int i = 1; i <= maxnits; ++i) {
    dx = 0.5 * dx;
    double mid = root + dx;
    double fmid = oracle_S_from_kappa(n, L, P2a, Ndiag, std::pow(10.0, mid)) - S_max;
    *nevals += 1;
    if (fmid < 0.0) {
      root = mid;
      *S_out = fmid + S_max;
      if (std::fabs(fmid) < tol) break;
    }
    if (std::fabs(fmid) < C * eps) break;
  }
  *k_root = std::pow(10.0, root);
}

// imcom_bisect_kappa (imcom_bisect.f90:78-170): per output pixel, OpenMP
// dynamic,64.  US_out receives U_a (UnotS != 0) or S_a.  nevals may be null.
void oracle_bisect_kappa(int UnotS, int n, int m, const double* L,
                         const double* P2, const double* Ndiag, double C,
                         double US, double k_min, double k_max, double tol,
                         int maxnits, double* K, double* US_out, int* nevals) {
  set_blas_threads(1);
#pragma omp parallel for schedule(dynamic, 64) num_threads(omp_threads())
  for (int a = 1; a <= m; ++a) {
    int ne = 0;
    const double* P2a = P2 + (size_t)(a - 1) * n;
    if (UnotS)
      bisect_by_U(n, L, P2a, C, k_min, k_max, US, tol, maxnits, &K[a - 1],
                  &US_out[a - 1], &ne);
    else
      bisect_by_S(n, L, P2a, Ndiag, C, k_min, k_max, US, tol, maxnits,
                  &K[a - 1], &US_out[a - 1], &ne);
    if (nevals) nevals[a - 1] = ne;
  }
  set_blas_threads(omp_threads());
}

// imcom_build_T (imcom_matrix.f90:716-750): T(:,a) = Q (P(:,a) / (L + K_a))
// by DGEMV, then T = -T / 2.
void oracle_build_T(int n, int m, const double* Q, const double* P,
                    const double* L, const double* K, double* T) {
  set_blas_threads(1);
#pragma omp parallel num_threads(omp_threads())
  {
    std::vector<double> x(n);
    double one = 1.0, zero = 0.0;
    int inc = 1;
#pragma omp for schedule(dynamic, 64)
    for (int a = 1; a <= m; ++a) {
      const double* Pa = P + (size_t)(a - 1) * n;
      for (int p = 0; p < n; ++p) x[p] = Pa[p] / (L[p] + K[a - 1]);
      scipy_dgemv_("N", &n, &n, &one, Q, &n, x.data(), &inc, &zero,
                   T + (size_t)(a - 1) * n, &inc, 1);
    }
  }
  size_t tot = (size_t)n * m;
  for (size_t k = 0; k < tot; ++k) T[k] = -T[k] / 2.0;
  set_blas_threads(omp_threads());
}

// imcom_build_image (imcom_matrix.f90:754-790): H = T^T I (DGEMV 'T').
void oracle_build_image(int n, int m, const double* T, const double* I,
                        double* H) {
  double one = 1.0, zero = 0.0;
  int inc = 1;
  scipy_dgemv_("T", &n, &m, &one, T, &n, I, &inc, &zero, H, &inc, 1);
}

// imcom_build_U (imcom_matrix.f90:795-835).
void oracle_build_U(int n, int m, const double* L, const double* P2, double C,
                    const double* K, double* U) {
  set_blas_threads(1);
#pragma omp parallel for num_threads(omp_threads())
  for (int a = 1; a <= m; ++a)
    U[a - 1] = oracle_U_from_kappa(n, L, P2 + (size_t)(a - 1) * n, C, K[a - 1]);
  set_blas_threads(omp_threads());
}

// imcom_build_S (imcom_matrix.f90:839-877): S_a = sum(T(:,a) * TN(:,a)),
// TN(i,:) = T(i,:) * Ndiag(i); SUM in element order.
void oracle_build_S(int n, int m, const double* T, const double* Ndiag,
                    double* S) {
#pragma omp parallel for num_threads(omp_threads())
  for (int a = 1; a <= m; ++a) {
    const double* Ta = T + (size_t)(a - 1) * n;
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += Ta[i] * (Ta[i] * Ndiag[i]);
    S[a - 1] = s;
  }
}

}  // extern "C"
