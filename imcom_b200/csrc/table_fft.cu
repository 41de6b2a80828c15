// table_fft.cu -- the lookup tables' inverse 2-D FFT, pruned and fused.
//
// imcom_build_Alookup / imcom_build_Blookup (imcom_matrix.f90:400-416,
// 467-480) embed conj(Gt_e) Gt_f (or conj(Gammat) Gt_e) in the middle of an
// npad-times larger frequency grid (side L = npad nps), inverse-FFT the grid
// (imcom_invft_c2c, imcom_proc.f90:498-512, an FFTW backward DFT) and keep the
// cshifted, scaled real part as the table.  The cuFFT path does that as
// embed_kernel -> cuFFT Z2Z -> shift_scale_kernel (tables.cu).  This file does
// the same in two passes over HBM, using that only nps of the grid's L lines
// are non-zero (for nps = 576, npad = 3 by the register path further down,
// the default there; elsewhere by the Stockham stages below, opt-in):
//   pass 1  the nps non-zero lines, computed from the spectra straight into
//           shared memory and transformed along p; the result W (nps x L per
//           table) is 1/npad of the grid.
//   pass 2  TP columns of W at a time, scattered into zero lines of length L,
//           transformed along q and written as the shifted, scaled real table.
// Per table element that is ~16/npad bytes written and read back plus the
// 8-byte table, against a full complex grid written by the embedding, the
// FFT's passes over it and the shift's read of it.
//
// The line transforms are the Stockham autosort formulation (Govindaraju et
// al., "High performance discrete Fourier transforms on graphics
// processors", SC 2008), stage by stage in place in shared memory: every
// thread reads its butterflies' inputs into registers, the block
// synchronises, and the outputs go to their autosorted places.  Radices 4, 2,
// 3, 5, 7, 11, 13; the twiddles come from a table of exp(2 pi i t / L) computed
// on the host in extended precision.  Sides with another prime factor, or longer
// than a block's shared memory holds, stay on cuFFT.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace imcom {

namespace {

constexpr int FFT_THREADS = 512;
constexpr int FFT_MAX_ELEMS = 8192;  // TP x LS complex values in shared memory (128 KiB)

// Elements a block may hold when its plan has a stage of radix R: each thread
// keeps the inputs of cap / (R x FFT_THREADS) butterflies (16, 16, 12, 10, 7,
// 11 and 13 complex values for R = 2, 4, 3, 5, 7, 11, 13) in registers between
// a stage's reads and writes, inside the 128 registers of a thread of a
// 512-thread block.
constexpr int fft_cap(int R) {
  return R == 3    ? 6144
         : R == 5  ? 5120
         : R == 7  ? 3584
         : R == 11 ? 5632
         : R == 13 ? 6656
                   : FFT_MAX_ELEMS;
}

struct FftPlan {
  int L = 0;   // transform length (grid side)
  int LS = 0;  // shared-memory stride of a line: L rounded up to odd (no bank conflicts
               // between the lines of a column read)
  int TP = 0;  // lines per block (TP x LS <= fft_cap of every radix of the plan)
  int count[7] = {};  // stages of radix 4, 2, 3, 5, 7, 11, 13 (run in that order)
};

constexpr int kRadices[7] = {4, 2, 3, 5, 7, 11, 13};

bool make_plan(int L, FftPlan* p) {
  if (L < 1) return false;
  p->L = L;
  p->LS = (L % 2 == 0) ? L + 1 : L;
  if (p->LS > FFT_MAX_ELEMS) return false;
  int n = L, cap = FFT_MAX_ELEMS;
  for (int i = 0; i < 7; ++i) {
    const int r = kRadices[i];
    p->count[i] = 0;
    while (n % r == 0) {
      ++p->count[i];
      n /= r;
    }
    if (p->count[i] > 0 && fft_cap(r) < cap) cap = fft_cap(r);
  }
  if (n != 1) return false;
  p->TP = cap / p->LS < 8 ? cap / p->LS : 8;
  return p->TP >= 1;
}

// Fortran CSHIFT source index (1-based): cshift(X, s)(i) = X(1 + mod(i-1+s, n)).
__device__ __forceinline__ int cshift_src(int i1, int s, int n) {
  return 1 + ((i1 - 1 + s) % n + n) % n;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// The embedded grid value: conj(Gt_e) Gt_f (A) or conj(Gammat) Gt_e (B) times
// imcom_upsilon2D = (1, 0), rounded step by step as embed_kernel does.
__device__ __forceinline__ double2 pair_product(const double2* __restrict__ Gt,
                                                const double2* __restrict__ Gammat, int2 pr,
                                                size_t s, int nps) {
  const size_t plane = (size_t)nps * nps;
  double2 a, b;
  if (pr.y > 0) {
    a = Gt[s + (size_t)(pr.x - 1) * plane];
    b = Gt[s + (size_t)(pr.y - 1) * plane];
  } else {
    a = Gammat[s];
    b = Gt[s + (size_t)(pr.x - 1) * plane];
  }
  const double ar = a.x, ai = -a.y;
  const double xr = __dsub_rn(__dmul_rn(ar, b.x), __dmul_rn(ai, b.y));
  const double xi = __dadd_rn(__dmul_rn(ar, b.y), __dmul_rn(ai, b.x));
  return make_double2(__dsub_rn(__dmul_rn(xr, 1.0), __dmul_rn(xi, 0.0)),
                      __dadd_rn(__dmul_rn(xr, 0.0), __dmul_rn(xi, 1.0)));
}

// DFT of length R with the + sign, y_r = sum_s v_s exp(2 pi i r s / R),
// stored to y[r Ns] as each output is formed (no output array is held).  Odd
// R uses the symmetric pairs: with a_s = v_s + v_{R-s}, b_s = v_s - v_{R-s}
// (s = 1 .. (R-1)/2), y_r and y_{R-r} = v_0 + sum_s a_s cos(2 pi r s / R)
// +- i sum_s b_s sin(2 pi r s / R); v is overwritten with the a_s and b_s.
template <int R>
__device__ __forceinline__ void dft_store(double2 (&v)[R], const double2* __restrict__ tw, int L,
                                          double2* y, int Ns) {
  if constexpr (R == 2) {
    y[0] = make_double2(v[0].x + v[1].x, v[0].y + v[1].y);
    y[Ns] = make_double2(v[0].x - v[1].x, v[0].y - v[1].y);
  } else if constexpr (R == 4) {
    const double2 s0 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
    const double2 d0 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
    const double2 s1 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
    const double2 d1 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
    y[0] = make_double2(s0.x + s1.x, s0.y + s1.y);
    y[2 * Ns] = make_double2(s0.x - s1.x, s0.y - s1.y);
    // d0 +- i d1, i (x, y) = (-y, x)
    y[Ns] = make_double2(d0.x - d1.y, d0.y + d1.x);
    y[3 * Ns] = make_double2(d0.x + d1.y, d0.y - d1.x);
  } else {
    constexpr int H = (R - 1) / 2;
    const int step = L / R;
    double2 y0 = v[0];
#pragma unroll
    for (int s = 1; s <= H; ++s) {
      const double2 a = make_double2(v[s].x + v[R - s].x, v[s].y + v[R - s].y);
      const double2 b = make_double2(v[s].x - v[R - s].x, v[s].y - v[R - s].y);
      v[s] = a;
      v[R - s] = b;
      y0.x += a.x;
      y0.y += a.y;
    }
    y[0] = y0;
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      double2 A = v[0], B = make_double2(0.0, 0.0);
#pragma unroll
      for (int s = 1; s <= H; ++s) {
        const double2 w = tw[((r * s) % R) * step];  // (cos, sin) of 2 pi r s / R
        A.x += v[s].x * w.x;
        A.y += v[s].y * w.x;
        B.x += v[R - s].x * w.y;
        B.y += v[R - s].y * w.y;
      }
      y[r * Ns] = make_double2(A.x - B.y, A.y + B.x);
      y[(R - r) * Ns] = make_double2(A.x + B.y, A.y - B.x);
    }
  }
}

// One Stockham stage of radix R over the block's TP lines (span Ns before
// the stage).  Butterfly j of a line reads x[j + r L/R], multiplies input r by
// exp(2 pi i k r / (Ns R)) (k = j mod Ns) and writes x[(j div Ns) Ns R + k + r Ns].
template <int R>
__device__ __forceinline__ void fft_stage(double2* buf, const FftPlan& plan, int Ns,
                                          const double2* __restrict__ tw) {
  // butterflies per thread: TP x L / R <= fft_cap(R) / R = JM x FFT_THREADS
  constexpr int JM = fft_cap(R) / (R * FFT_THREADS);
  static_assert(JM * R * FFT_THREADS == fft_cap(R), "cap is a whole number of butterflies");
  const int L = plan.L, LS = plan.LS;
  const int per = L / R;
  const int B = plan.TP * per;
  double2 v[JM][R];
#pragma unroll
  for (int i = 0; i < JM; ++i) {
    const int b = threadIdx.x + i * FFT_THREADS;
    if (b < B) {
      const int line = b / per, j = b - line * per;
      const double2* x = buf + line * LS + j;
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = x[r * per];
    }
  }
  __syncthreads();  // every input is in registers before any output lands
  const int tstep = L / (Ns * R);
#pragma unroll
  for (int i = 0; i < JM; ++i) {
    const int b = threadIdx.x + i * FFT_THREADS;
    if (b < B) {
      const int line = b / per, j = b - line * per;
      const int k = j % Ns;
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[i][r] = cmul(v[i][r], tw[k * r * tstep]);
      }
      dft_store<R>(v[i], tw, L, buf + line * LS + (j / Ns) * Ns * R + k, Ns);
    }
  }
  __syncthreads();
}

// The plan's stages in its order (all radix-4 stages, then 2, 3, 5, 7, 11,
// 13): one counted loop per radix, so each stage body is compiled once.
__device__ __forceinline__ void run_stages(double2* buf, const FftPlan& plan,
                                           const double2* __restrict__ tw) {
  int Ns = 1;
  for (int i = 0; i < plan.count[0]; ++i, Ns *= 4) fft_stage<4>(buf, plan, Ns, tw);
  for (int i = 0; i < plan.count[1]; ++i, Ns *= 2) fft_stage<2>(buf, plan, Ns, tw);
  for (int i = 0; i < plan.count[2]; ++i, Ns *= 3) fft_stage<3>(buf, plan, Ns, tw);
  for (int i = 0; i < plan.count[3]; ++i, Ns *= 5) fft_stage<5>(buf, plan, Ns, tw);
  for (int i = 0; i < plan.count[4]; ++i, Ns *= 7) fft_stage<7>(buf, plan, Ns, tw);
  for (int i = 0; i < plan.count[5]; ++i, Ns *= 11) fft_stage<11>(buf, plan, Ns, tw);
  for (int i = 0; i < plan.count[6]; ++i, Ns *= 13) fft_stage<13>(buf, plan, Ns, tw);
}

// Pass 1: lines u0 .. u0+TP-1 of the nps non-zero grid lines (grid row
// sq = nmin + u) of table blockIdx.y, transformed along p, into W.
__global__ void __launch_bounds__(FFT_THREADS, 1)
table_fft_pass1(FftPlan plan, const double2* __restrict__ Gt, const double2* __restrict__ Gammat,
                const int2* __restrict__ pairs, const double2* __restrict__ tw,
                double2* __restrict__ W, int nps) {
  extern __shared__ double2 buf[];
  const int L = plan.L, LS = plan.LS, TP = plan.TP;
  const int t = blockIdx.y;
  const int u0 = blockIdx.x * TP;
  const int s = L / 2, nmin = (L - nps) / 2 + 1;
  const int2 pr = pairs[t];
  for (int e = threadIdx.x; e < TP * L; e += FFT_THREADS) {
    const int line = e / L, p0 = e - line * L;
    const int u = u0 + line;
    double2 v = make_double2(0.0, 0.0);
    if (u < nps) {
      const int sp = cshift_src(p0 + 1, s, L);
      if (sp >= nmin && sp < nmin + nps) {
        const int si = cshift_src(sp - nmin + 1, nps / 2, nps);
        const int sj = cshift_src(u + 1, nps / 2, nps);
        v = pair_product(Gt, Gammat, pr, (size_t)(si - 1) + (size_t)(sj - 1) * nps, nps);
      }
    }
    buf[line * LS + p0] = v;
  }
  __syncthreads();
  run_stages(buf, plan, tw);
  for (int e = threadIdx.x; e < TP * L; e += FFT_THREADS) {
    const int line = e / L, k1 = e - line * L;
    const int u = u0 + line;
    if (u < nps) W[((size_t)t * nps + u) * L + k1] = buf[line * LS + k1];
  }
}

// Pass 2: columns c0 .. c0+TP-1 of W for table blockIdx.y, each scattered
// into a zero line of length L at the grid rows of its nps entries,
// transformed along q and written to the table through the cshifts:
// tab(p, q) = s Re F(cshift(p), cshift(q)), s = 1/nps^2 (A) or -2/nps^2 (B).
__global__ void __launch_bounds__(FFT_THREADS, 1)
table_fft_pass2(FftPlan plan, const double2* __restrict__ W, const double2* __restrict__ tw,
                double* __restrict__ tab, int nps, int isB) {
  extern __shared__ double2 buf[];
  const int L = plan.L, LS = plan.LS, TP = plan.TP;
  const int t = blockIdx.y;
  const int c0 = blockIdx.x * TP;
  const int s = L / 2, nmin = (L - nps) / 2 + 1;
  for (int e = threadIdx.x; e < TP * L; e += FFT_THREADS) {
    const int line = e / L, q0 = e - line * L;
    buf[line * LS + q0] = make_double2(0.0, 0.0);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nps * TP; e += FFT_THREADS) {
    const int u = e / TP, c = e - u * TP;
    const int k1 = c0 + c;
    if (k1 < L) {
      const int q0 = ((nmin + u - 1 - s) % L + L) % L;
      buf[c * LS + q0] = W[((size_t)t * nps + u) * L + k1];
    }
  }
  __syncthreads();
  run_stages(buf, plan, tw);
  const size_t tbase = (size_t)t * L * L;
  for (int e = threadIdx.x; e < TP * L; e += FFT_THREADS) {
    const int k2 = e / TP, c = e - k2 * TP;
    const int k1 = c0 + c;
    if (k1 < L) {
      double v = buf[c * LS + k2].x;
      if (isB) v = -2.0 * v;
      const int p0 = ((k1 - s) % L + L) % L, q0 = ((k2 - s) % L + L) % L;
      tab[tbase + (size_t)q0 * L + p0] = v / (double)nps / (double)nps;
    }
  }
}

// ---------------------------------------------------------------------------
// The PSF spectra's real-to-complex transform (imcom_ft_r2c,
// imcom_proc.f90:433-475: FFTW's forward r2c of an nps x nps image, the first
// axis halved to nps/2 + 1), in two passes with the same line transforms.
// The forward transform is the conjugate of the backward one of the
// conjugated input: pass 1 transforms the real lines along the first axis and
// keeps k = 0 .. nps/2 (stored column-major by k, H[b][k][j]), pass 2
// transforms those columns along the second axis and writes the half
// spectrum half[b][j][k] (k fastest), the layout the Hermitian fill reads.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(FFT_THREADS, 1)
r2c_pass1(FftPlan plan, const double* __restrict__ in, const double2* __restrict__ tw,
          double2* __restrict__ H) {
  extern __shared__ double2 buf[];
  const int n = plan.L, LS = plan.LS, TP = plan.TP;
  const int nh = n / 2 + 1;
  const int b = blockIdx.y;
  const int j0 = blockIdx.x * TP;
  const double* src = in + (size_t)b * n * n;
  for (int e = threadIdx.x; e < TP * n; e += FFT_THREADS) {
    const int line = e / n, k = e - line * n;
    const int j = j0 + line;
    buf[line * LS + k] = make_double2(j < n ? src[(size_t)j * n + k] : 0.0, 0.0);
  }
  __syncthreads();
  run_stages(buf, plan, tw);
  for (int e = threadIdx.x; e < TP * nh; e += FFT_THREADS) {
    const int k = e / TP, line = e - k * TP;
    const int j = j0 + line;
    if (j < n) {
      const double2 v = buf[line * LS + k];
      H[((size_t)b * nh + k) * n + j] = make_double2(v.x, -v.y);
    }
  }
}

__global__ void __launch_bounds__(FFT_THREADS, 1)
r2c_pass2(FftPlan plan, const double2* __restrict__ H, const double2* __restrict__ tw,
          double2* __restrict__ half) {
  extern __shared__ double2 buf[];
  const int n = plan.L, LS = plan.LS, TP = plan.TP;
  const int nh = n / 2 + 1;
  const int b = blockIdx.y;
  const int k0 = blockIdx.x * TP;
  for (int e = threadIdx.x; e < TP * n; e += FFT_THREADS) {
    const int line = e / n, j = e - line * n;
    const int k = k0 + line;
    double2 v = make_double2(0.0, 0.0);
    if (k < nh) {
      v = H[((size_t)b * nh + k) * n + j];
      v.y = -v.y;
    }
    buf[line * LS + j] = v;
  }
  __syncthreads();
  run_stages(buf, plan, tw);
  for (int e = threadIdx.x; e < TP * n; e += FFT_THREADS) {
    const int j = e / TP, line = e - j * TP;
    const int k = k0 + line;
    if (k < nh) {
      const double2 v = buf[line * LS + j];
      half[((size_t)b * n + j) * nh + k] = make_double2(v.x, -v.y);
    }
  }
}

// ---------------------------------------------------------------------------
// Register path for nps = 576, npad = 3 (L = 1728), the n = 4096 workload's
// sides.  The grid's non-zero block is the spectrum X(u1, u2) at signed
// frequencies m(u) = u (u < nps/2) or u - nps, so with k = 3 j + b
//   sum_u X(u) exp(2 pi i m(u) k / L) = DFT_nps[X(u) exp(2 pi i m(u) b / L)](j)
// along each axis: three length-576 transforms of pre-twiddled copies
// replace one length-1728 transform of a zero-padded line.  One warp holds a
// line, 18 values per lane (element 32 n1 + lane), and transforms it in
// registers by four steps (576 = 18 x 32): a DFT-18 per lane, the twiddles
// exp(2 pi i lane k1 / 576), and a DFT-32 across the lanes by five radix-2
// decimation-in-frequency stages on shuffles, after which lane L's value k1
// is output k1 + 18 bitrev5(L).  Blocks of 16 (pass 1) or 8 (pass 2) lines
// stage their outputs in shared memory and write them in row segments:
//   pass 1  lines u2 of one table, along u1: W[t][3 j + b][u2]
//   pass 2  columns k1 of W, along u2: the table's real part, shifted and
//           scaled like the other paths, one 8-column row segment per j.
// All twiddles come from the table of exp(2 pi i t / 1728) (those of 576 at
// t multiple of 3).
// ---------------------------------------------------------------------------
constexpr int FX_N1 = 18, FX_N2 = 32, FX_N = FX_N1 * FX_N2, FX_L = 3 * FX_N;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}

// In-place DFT-3 with the + sign: (a, b, c) <- (a + b + c, a + w b + w^2 c,
// a + w^2 b + w c), w = exp(2 pi i / 3); h3 = sqrt(3) / 2.
__device__ __forceinline__ void dft3p(double2& a, double2& b, double2& c, double h3) {
  const double2 t1 = cadd(b, c);
  const double2 d = csub(b, c);
  const double2 t2 = make_double2(-d.y * h3, d.x * h3);  // i h3 (b - c)
  const double2 m = make_double2(a.x - 0.5 * t1.x, a.y - 0.5 * t1.y);
  a = cadd(a, t1);
  b = cadd(m, t2);
  c = csub(m, t2);
}

// The register path's twiddles in shared memory, laid out so that a warp's
// reads are consecutive (no bank conflicts) or one broadcast address:
//   pl[b 32 + lane]   exp(2 pi i lane b / L)  (b < 3)
//   lt[lane]          exp(2 pi i lane / 576)
//   st[i 32 + lane]   exp(2 pi i (lane mod h) / (2 h)), h = 16 >> i (i < 3)
//   cst[k] = w18^k (k < 9), cst[9 + i] = w9^(1, 2, 4), cst[12].y = sin(2 pi / 3),
//   cst[13 + b] = exp(2 pi i 32 b / L)
// The other twiddles are products of these (a few ulps at most).
constexpr int FX_TW = 3 * 32 + 32 + 3 * 32 + 16;  // double2 entries
struct FxTw {
  const double2 *pl, *lt, *st, *cst;
};

// DFT-9 (+ sign) of z[0..8] as 3 x 3; output s + 3 t is left in z[3 s + t].
__device__ __forceinline__ void dft9p(double2 (&z)[9], const double2* __restrict__ cst, double h3) {
#pragma unroll
  for (int r = 0; r < 3; ++r) dft3p(z[r], z[r + 3], z[r + 6], h3);
  z[4] = cmul(z[4], cst[9]);       // r = 1, s = 1: w9
  z[7] = cmul(z[7], cst[10]);      // r = 1, s = 2: w9^2
  z[5] = cmul(z[5], cst[10]);      // r = 2, s = 1: w9^2
  z[8] = cmul(z[8], cst[11]);      // r = 2, s = 2: w9^4
#pragma unroll
  for (int s = 0; s < 3; ++s) dft3p(z[3 * s], z[3 * s + 1], z[3 * s + 2], h3);
}

// DFT-576 (+ sign) of the warp's line: lane holds y[n1] = x[32 n1 + lane];
// on return y[k1] = X[k1 + 18 bitrev5(lane)].
__device__ __forceinline__ void dft576_warp(double2 (&y)[FX_N1], const FxTw& tw, int lane) {
  const double h3 = tw.cst[12].y;  // sin(2 pi / 3)
  // DFT-18 per lane: even and odd halves by DFT-9, joined with w18^k
  double2 e[9], o[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    e[i] = y[2 * i];
    o[i] = y[2 * i + 1];
  }
  dft9p(e, tw.cst, h3);
  dft9p(o, tw.cst, h3);
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int at = 3 * (k % 3) + k / 3;  // output k of dft9p
    const double2 t = cmul(o[at], tw.cst[k]);  // w18^k
    y[k] = cadd(e[at], t);
    y[k + 9] = csub(e[at], t);
  }
  // twiddles exp(2 pi i lane k1 / 576)
#pragma unroll
  // as powers of w576^lane (one shared read instead of 17; 16 more products,
  // ~2e-15 relative at k1 = 17)
  {
    const double2 w1 = tw.lt[lane];
    double2 wk = w1;
#pragma unroll
    for (int k1 = 1; k1 < FX_N1; ++k1) {
      y[k1] = cmul(y[k1], wk);
      if (k1 + 1 < FX_N1) wk = cmul(wk, w1);
    }
  }
  // DFT-32 across the lanes (element index = lane), decimation in frequency:
  // lower lane y + p, upper lane (p - y) w_{2h}^(lane mod h), formed as
  // (s y + p) w with s = -1 and w = 1 on the lower lanes; the last two
  // stages' twiddles are 1 and i (a swap), so they need no product.
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    const bool upper = (lane & h) != 0;
    const double sgn = upper ? -1.0 : 1.0;
    const double2 w =
        (upper && h >= 4) ? tw.st[(h == 16 ? 0 : h == 8 ? 1 : 2) * 32 + lane] : make_double2(1.0, 0.0);
    const bool rot = h == 2 && upper && (lane & 1);  // w_4^1 = i
#pragma unroll
    for (int k1 = 0; k1 < FX_N1; ++k1) {
      const double px = __shfl_xor_sync(0xffffffffu, y[k1].x, h);
      const double py = __shfl_xor_sync(0xffffffffu, y[k1].y, h);
      const double2 r = make_double2(fma(sgn, y[k1].x, px), fma(sgn, y[k1].y, py));
      if (h >= 4) y[k1] = cmul(r, w);
      else if (h == 2) y[k1] = rot ? make_double2(-r.y, r.x) : r;
      else y[k1] = r;
    }
  }
}

__device__ __forceinline__ int fx_brev5(int x) { return (int)(__brev((unsigned)x) >> 27); }

// The shared twiddle tables from the global table g[t] = exp(2 pi i t / L),
// by every thread of the block (FX_TW entries at sm).
__device__ __forceinline__ FxTw fx_fill(const double2* __restrict__ g, double2* sm) {
  double2 *pl = sm, *lt = pl + 3 * 32, *st = lt + 32, *cst = st + 3 * 32;
  for (int i = threadIdx.x; i < 3 * 32; i += blockDim.x) pl[i] = g[(i >> 5) * (i & 31)];
  for (int i = threadIdx.x; i < 32; i += blockDim.x) lt[i] = g[3 * i];
  for (int i = threadIdx.x; i < 3 * 32; i += blockDim.x) {
    const int h = 16 >> (i >> 5), L = i & 31;
    st[i] = g[54 * (16 / h) * (L & (h - 1))];  // w_{2h}^(L mod h) = w_32^((16/h)(L mod h))
  }
  if (threadIdx.x < 9) cst[threadIdx.x] = g[96 * threadIdx.x];  // w18^k
  if (threadIdx.x == 9) cst[9] = g[192];                        // w9
  if (threadIdx.x == 10) cst[10] = g[384];                      // w9^2
  if (threadIdx.x == 11) cst[11] = g[768];                      // w9^4
  if (threadIdx.x == 12) cst[12] = g[576];                      // w3: (-1/2, sin(2 pi / 3))
  if (threadIdx.x >= 13 && threadIdx.x < 16) cst[threadIdx.x] = g[32 * (threadIdx.x - 13)];
  return FxTw{pl, lt, st, cst};
}

// y[n1] *= exp(2 pi i m(u) b / L), u = 32 n1 + lane: powers of w_L^(32 b)
// from w_L^(lane b) up for n1 < 9 (m = u) and from w_L^((lane - 32) b) down
// for n1 >= 9 (m = u - nps).
__device__ __forceinline__ void fx_pretwiddle(double2 (&y)[FX_N1], const FxTw& tw, int lane,
                                              int b) {
  if (b == 0) return;
  const double2 step = tw.cst[13 + b], stepm = make_double2(step.x, -step.y);
  const double2 base = tw.pl[b * 32 + lane];
  double2 c = base;
#pragma unroll
  for (int n1 = 0; n1 < FX_N1 / 2; ++n1) {
    y[n1] = cmul(y[n1], c);
    if (n1 + 1 < FX_N1 / 2) c = cmul(c, step);
  }
  c = cmul(base, stepm);
#pragma unroll
  for (int n1 = FX_N1 - 1; n1 >= FX_N1 / 2; --n1) {
    y[n1] = cmul(y[n1], c);
    if (n1 > FX_N1 / 2) c = cmul(c, stepm);
  }
}

constexpr int FX1_LINES = 8, FX2_LINES = 8;
constexpr size_t FX1_SMEM = ((size_t)FX_TW + 2 * (size_t)FX_N * FX1_LINES) * sizeof(double2);
constexpr size_t FX2_SMEM = (size_t)FX_TW * sizeof(double2) + (size_t)FX_N * FX2_LINES * sizeof(double);

// Pass 1: spectrum columns u2 = 8 blockIdx.x + warp of table blockIdx.y,
// along u1, into W[t][k1][u2] (ld nps).
__global__ void __launch_bounds__(FX1_LINES * 32, 1)
fx_pass1(const double2* __restrict__ Gt, const double2* __restrict__ Gammat,
         const int2* __restrict__ pairs, const double2* __restrict__ twg, double2* __restrict__ W) {
  extern __shared__ double2 fx_smem[];
  const FxTw tw = fx_fill(twg, fx_smem);
  double2* S = fx_smem + FX_TW;               // [FX_N][FX1_LINES]
  double2* X = S + (size_t)FX_N * FX1_LINES;  // [FX1_LINES][FX_N]: the lines' values
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.y, u2 = blockIdx.x * FX1_LINES + warp;
  const int2 pr = pairs[t];
  double2* xl = X + (size_t)warp * FX_N;
  for (int u = lane; u < FX_N; u += 32)
    xl[u] = pair_product(Gt, Gammat, pr, (size_t)u + (size_t)u2 * FX_N, FX_N);
  __syncthreads();  // twiddles and the lines in place
  for (int b = 0; b < 3; ++b) {
    double2 y[FX_N1];
#pragma unroll
    for (int n1 = 0; n1 < FX_N1; ++n1) y[n1] = xl[32 * n1 + lane];
    fx_pretwiddle(y, tw, lane, b);
    dft576_warp(y, tw, lane);
    const int j0 = FX_N1 * fx_brev5(lane);
#pragma unroll
    for (int k1 = 0; k1 < FX_N1; ++k1) S[(j0 + k1) * FX1_LINES + warp] = y[k1];
    __syncthreads();
    double2* dst = W + ((size_t)t * FX_L + b) * FX_N + (size_t)blockIdx.x * FX1_LINES;
    for (int e = threadIdx.x; e < FX_N * FX1_LINES; e += blockDim.x) {
      const int j = e / FX1_LINES, c = e - j * FX1_LINES;
      dst[(size_t)(3 * j) * FX_N + c] = S[e];
    }
    __syncthreads();
  }
}

// Pass 2: columns k1 = 8 blockIdx.x + warp of W for table blockIdx.y, along
// u2, written as tab(p, q) = scale Re F(cshift(p), cshift(q)).
__global__ void __launch_bounds__(FX2_LINES * 32, 2)
fx_pass2(const double2* __restrict__ W, const double2* __restrict__ twg, double* __restrict__ tab,
         int isB) {
  extern __shared__ double2 fx_smem[];
  const FxTw tw = fx_fill(twg, fx_smem);
  double* R = reinterpret_cast<double*>(fx_smem + FX_TW);  // [FX_N][FX2_LINES]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.y, k1 = blockIdx.x * FX2_LINES + warp;
  const double2* src = W + ((size_t)t * FX_L + k1) * FX_N;
  __syncthreads();
  constexpr int s = FX_L / 2;
  // the block's 8 columns map to 8 consecutive p (s is a multiple of 8)
  const int p0 = (blockIdx.x * FX2_LINES - s + FX_L) % FX_L;
  double* tt = tab + (size_t)t * FX_L * FX_L;
  for (int b = 0; b < 3; ++b) {
    double2 y[FX_N1];
#pragma unroll
    for (int n1 = 0; n1 < FX_N1; ++n1)
      y[n1] = __ldg(src + 32 * n1 + lane);
    fx_pretwiddle(y, tw, lane, b);
    dft576_warp(y, tw, lane);
    const int j0 = FX_N1 * fx_brev5(lane);
#pragma unroll
    for (int q = 0; q < FX_N1; ++q) {
      double v = y[q].x;
      if (isB) v = -2.0 * v;
      R[(j0 + q) * FX2_LINES + warp] = v / (double)FX_N / (double)FX_N;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < FX_N * FX2_LINES; e += blockDim.x) {
      const int j = e / FX2_LINES, c = e - j * FX2_LINES;
      const int q0 = (3 * j + b - s + FX_L) % FX_L;
      tt[(size_t)q0 * FX_L + p0 + c] = R[e];
    }
    __syncthreads();
  }
}

// exp(2 pi i t / L), t < L, rounded from extended precision; the parts that
// are exactly 0 (where 4t is a multiple of L) come out as exact zeros.
std::vector<double2> twiddles(int L) {
  const long double two_pi = 6.283185307179586476925286766559005768L;
  std::vector<double2> tw(L);
  for (int t = 0; t < L; ++t) {
    const long double a = two_pi * (long double)t / (long double)L;
    long double c = cosl(a), s = sinl(a);
    if (fabsl(c) < 1e-18L) c = 0.0L;
    if (fabsl(s) < 1e-18L) s = 0.0L;
    tw[t] = make_double2((double)c, (double)s);
  }
  return tw;
}

}  // namespace

int psf_r2c_own(imcom_ctx* ctx, int n, int count, const double* in, double2* H, double2* half,
                bool* done) {
  *done = false;
  FftPlan plan;
  if (n < 2 || !make_plan(n, &plan)) return 0;
  if (ctx->r2c_tw_L != n) {
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));  // no launch still reads the old table
    IMC_TRY(ensure_buf(ctx, (void**)&ctx->r2c_tw, ctx->r2c_tw_bytes, (size_t)n * sizeof(double2)));
    const std::vector<double2> tw = twiddles(n);
    IMC_CUDA(cudaMemcpyAsync(ctx->r2c_tw, tw.data(), (size_t)n * sizeof(double2),
                             cudaMemcpyHostToDevice, ctx->stream));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->r2c_tw_L = n;
  }
  const int smem = plan.TP * plan.LS * (int)sizeof(double2);
  // limits set to the largest plan's need: the attribute is process-wide and
  // contexts on several host threads must not lower it under each other
  constexpr int kMax = FFT_MAX_ELEMS * (int)sizeof(double2);
  IMC_CUDA(cudaFuncSetAttribute(r2c_pass1, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax));
  IMC_CUDA(cudaFuncSetAttribute(r2c_pass2, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax));
  const int nh = n / 2 + 1;
  const dim3 g1((unsigned)((n + plan.TP - 1) / plan.TP), (unsigned)count);
  r2c_pass1<<<g1, FFT_THREADS, smem, ctx->stream>>>(plan, in, ctx->r2c_tw, H);
  IMC_LAUNCH();
  const dim3 g2((unsigned)((nh + plan.TP - 1) / plan.TP), (unsigned)count);
  r2c_pass2<<<g2, FFT_THREADS, smem, ctx->stream>>>(plan, H, ctx->r2c_tw, half);
  IMC_LAUNCH();
  *done = true;
  return 0;
}

bool table_fft_fast(int nps, int L) { return nps == FX_N && L == FX_L; }

int table_fft_inverse(imcom_ctx* ctx, int nps, int L, int ntab, const int2* dpairs, double2* W,
                      double* tab, int isB, bool* done) {
  *done = false;
  FftPlan plan;
  if (nps <= 0 || (L - nps) % 2 != 0 || L < nps || !make_plan(L, &plan)) return 0;
  if (ctx->fft_tw_L != L) {
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));  // no launch still reads the old table
    IMC_TRY(ensure_buf(ctx, (void**)&ctx->fft_tw, ctx->fft_tw_bytes, (size_t)L * sizeof(double2)));
    const std::vector<double2> tw = twiddles(L);
    IMC_CUDA(cudaMemcpyAsync(ctx->fft_tw, tw.data(), (size_t)L * sizeof(double2),
                             cudaMemcpyHostToDevice, ctx->stream));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->fft_tw_L = L;
  }
  if (table_fft_fast(nps, L)) {  // the register path
    IMC_CUDA(cudaFuncSetAttribute(fx_pass1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)FX1_SMEM));
    IMC_CUDA(cudaFuncSetAttribute(fx_pass2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)FX2_SMEM));
    fx_pass1<<<dim3(FX_N / FX1_LINES, (unsigned)ntab), FX1_LINES * 32, FX1_SMEM, ctx->stream>>>(
        ctx->Gt, ctx->Gammat, dpairs, ctx->fft_tw, W);
    IMC_LAUNCH();
    fx_pass2<<<dim3(FX_L / FX2_LINES, (unsigned)ntab), FX2_LINES * 32, FX2_SMEM, ctx->stream>>>(
        W, ctx->fft_tw, tab, isB);
    IMC_LAUNCH();
    *done = true;
    return 0;
  }
  const int smem = plan.TP * plan.LS * (int)sizeof(double2);
  constexpr int kMax = FFT_MAX_ELEMS * (int)sizeof(double2);  // see psf_r2c_own
  IMC_CUDA(cudaFuncSetAttribute(table_fft_pass1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kMax));
  IMC_CUDA(cudaFuncSetAttribute(table_fft_pass2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kMax));
  const dim3 g1((unsigned)((nps + plan.TP - 1) / plan.TP), (unsigned)ntab);
  table_fft_pass1<<<g1, FFT_THREADS, smem, ctx->stream>>>(plan, ctx->Gt, ctx->Gammat, dpairs,
                                                          ctx->fft_tw, W, nps);
  IMC_LAUNCH();
  const dim3 g2((unsigned)((L + plan.TP - 1) / plan.TP), (unsigned)ntab);
  table_fft_pass2<<<g2, FFT_THREADS, smem, ctx->stream>>>(plan, W, ctx->fft_tw, tab, nps, isB);
  IMC_LAUNCH();
  *done = true;
  return 0;
}

}  // namespace imcom
