// tables.cu -- PSF rotation, PSF spectra and the FFT-built lookup tables.
//
// Compiled with --fmad=false: every expression here rounds as written, like
// the reference's gfortran build, so rotation indices and table values follow
// imcom_proc.f90 / imcom_matrix.f90 operation by operation.  The FFTs are
// cuFFT (the reference calls FFTW for the same transforms).
//
//   rotate_psf_kernel     imcom_rotate_image   imcom_proc.f90:184-250 (Lagrange form)
//   hermitian_fill_kernel imcom_ft_r2c         imcom_proc.f90:433-475
//   csum_kernel           imcom_calc_C         imcom_matrix.f90:546-552
//   embed_kernel          imcom_build_Alookup  imcom_matrix.f90:395-411
//                         imcom_build_Blookup  imcom_matrix.f90:468-476
//   shift_scale_kernel    (same, :412-413, :427-429 / :477-478, :490-492)
#include <cmath>
#include <vector>

#include "common.cuh"

namespace imcom {
namespace {

// Lagrange weights of the m consecutive integer nodes x0, x0+1, ... at t:
// w_k = prod_{j != k} (t - x_j) / prod_{j != k} (k - j), from prefix and
// suffix products (the denominators are exact integers); a node hit exactly
// gets weight 1 and the others 0.
__device__ __forceinline__ void lagrange_weights(double t, int x0, int m, double (&w)[16]) {
  double sv[16], pre[16];
  bool node = false;
  double acc = 1.0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    sv[j] = (j < m) ? t - (double)(x0 + j) : 1.0;
    node |= (j < m) && (sv[j] == 0.0);
    pre[j] = acc;
    acc = acc * sv[j];
  }
  acc = 1.0;
#pragma unroll
  for (int k = 15; k >= 0; --k) {
    // prod_{j != k} (k - j) = (-1)^(m-1-k) k! (m-1-k)!
    double den = 1.0;
    for (int q = 2; q <= k; ++q) den = den * (double)q;
    for (int q = 2; q <= m - 1 - k; ++q) den = den * (double)q;
    if ((m - 1 - k) & 1) den = -den;
    w[k] = (k < m) ? pre[k] * acc / den : 0.0;
    acc = acc * sv[k];
  }
  if (node) {
#pragma unroll
    for (int k = 0; k < 16; ++k) w[k] = (k < m && sv[k] == 0.0) ? 1.0 : 0.0;
  }
}

// One output pixel of imcom_rotate_image per thread.  cost/sint come from
// the host (same libm as the reference's runtime), so the source coordinate,
// its floor/ceiling and the interpolation window [floor - npm, ceil + npm]
// clipped to the image are bit-identical.  The reference interpolates on that
// window with imcom_polin2 (Neville's tableau along the second axis for each
// window row, then along the first; imcom_proc.f90:351-429); the
// interpolating polynomial on those nodes is unique, and this kernel
// evaluates it in Lagrange form, f = sum_j wx_j sum_k wy_k in(x_j, y_k):
// equal up to rounding, with no divisions by data.  Neville's
// duplicate-abscissa trap cannot fire on distinct integer nodes.
__global__ void rotate_psf_kernel(const double* __restrict__ in, double* __restrict__ out,
                                  int nim, int npm, double cost, double sint) {
  int iout = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int jout = blockIdx.y + 1;
  if (iout > nim) return;
  double x_cent = (double)(nim + 1) / 2.0, y_cent = x_cent;
  double xout = (double)iout - x_cent;
  double yout = (double)jout - y_cent;
  double xs = xout * cost + yout * sint + x_cent;
  double ys = -xout * sint + yout * cost + y_cent;
  int is_floor = (int)floor(xs), js_floor = (int)floor(ys);
  int is_ceil = (int)ceil(xs), js_ceil = (int)ceil(ys);
  double f = 0.0;
  if (is_floor >= 1 && js_floor >= 1 && is_ceil <= nim && js_ceil <= nim) {
    int imin = max(1, is_floor - npm), jmin = max(1, js_floor - npm);
    int imax = min(nim, is_ceil + npm), jmax = min(nim, js_ceil + npm);
    int m1 = imax - imin + 1, m2 = jmax - jmin + 1;
    double wx[16], wy[16];
    lagrange_weights(xs, imin, m1, wx);
    lagrange_weights(ys, jmin, m2, wy);
    const double* base = in + (size_t)(imin - 1) + (size_t)(jmin - 1) * nim;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      if (k < m2) {
        const double* row = base + (size_t)k * nim;
        double g = 0.0;
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (j < m1) g = g + wx[j] * __ldg(row + j);
        f = f + wy[k] * g;
      }
    }
  }
  out[(size_t)(iout - 1) + (size_t)(jout - 1) * nim] = f;
}

// Block sums of a real array (tree order); the host finishes the sum.
__global__ void partial_sum_kernel(const double* __restrict__ a, size_t count,
                                   double* __restrict__ partial) {
  __shared__ double sh[256];
  double s = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < count;
       k += (size_t)gridDim.x * blockDim.x)
    s += a[k];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void finish_sum_kernel(const double* __restrict__ partial, int np, double* out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) s += partial[k];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// Sum of |z_k|^2 = re^2 + im^2 over k = 0 .. count-1 with the rounding of the
// sequential loop s = s + |z_k|^2 (Fortran's SUM without reassociation, as
// in imcom_calc_C, imcom_matrix.f90:546-552), in parallel.  While s stays in
// one binade [2^(E-1), 2^E), every step rounds to a multiple of the same ulp
// u = 2^(E-53): s_k = s_(k-1) + rint(t_k / u) u, unless t_k / u is exactly
// half-way (a tie, decided by the parity of s) or s leaves the binade.  The
// terms are non-negative, so s only grows: a block of terms whose rounded
// quotients sum to Q with s / u + Q < 2^53 and no tie advances s by Q u
// exactly.  One CTA walks the terms in chunks of SQ_CHUNK; a chunk that
// crosses a binade or holds a tie is split into 32-term sub-chunks and only
// those sub-chunks are added term by term.  Result bit-identical to the
// sequential loop (a binade's worth of terms is an exact integer sum).
constexpr int SQ_THREADS = 1024, SQ_PER = 4, SQ_CHUNK = SQ_THREADS * SQ_PER, SQ_SUB = 32;
constexpr int SQ_NSUB = SQ_CHUNK / SQ_SUB;

__global__ void __launch_bounds__(SQ_THREADS, 1)
    seq_abs2_sum_kernel(const double2* __restrict__ z, size_t count, double* __restrict__ out) {
  __shared__ double st[SQ_CHUNK];     // the chunk's terms in order
  __shared__ double sq[SQ_NSUB];      // rounded-quotient sums per sub-chunk
  __shared__ int stie[SQ_NSUB];       // a tie in the sub-chunk
  __shared__ double sS;               // the running sum
  __shared__ int s_start, s_done;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double two53 = 9007199254740992.0, tiny = 4.450147717014403e-308;  // 2^53, 2^-1021
  if (tid == 0) sS = 0.0;
  // term r * 1024 + tid of a chunk (coalesced); sub-chunk r * 32 + warp.  The
  // next chunk's values are loaded while this one is reduced.
  double2 vn[SQ_PER];
#pragma unroll
  for (int r = 0; r < SQ_PER; ++r) {
    const size_t k = (size_t)r * SQ_THREADS + tid;
    vn[r] = k < count ? z[k] : make_double2(0.0, 0.0);
  }
  for (size_t base = 0; base < count; base += SQ_CHUNK) {
    double t[SQ_PER];
#pragma unroll
    for (int r = 0; r < SQ_PER; ++r) {
      t[r] = __dadd_rn(__dmul_rn(vn[r].x, vn[r].x), __dmul_rn(vn[r].y, vn[r].y));
      st[r * SQ_THREADS + tid] = t[r];
    }
#pragma unroll
    for (int r = 0; r < SQ_PER; ++r) {
      const size_t k = base + SQ_CHUNK + (size_t)r * SQ_THREADS + tid;
      vn[r] = k < count ? z[k] : make_double2(0.0, 0.0);
    }
    if (tid == 0) s_start = 0;
    __syncthreads();
    while (true) {
      const double S = sS;
      const int start = s_start;
      const bool normal = S >= tiny;
      int E = 0;
      if (normal) frexp(S, &E);
#pragma unroll
      for (int r = 0; r < SQ_PER; ++r) {
        const int sub = r * 32 + warp;
        double q = 0.0;
        int tie = 0;
        if (sub >= start) {
          if (normal) {
            const double x = ldexp(t[r], 53 - E);
            q = rint(x);
            tie = (x - floor(x) == 0.5) ? 1 : 0;
          } else {
            tie = 1;  // no binade yet: term by term
          }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
          q += __shfl_xor_sync(0xffffffffu, q, o);
          tie |= __shfl_xor_sync(0xffffffffu, tie, o);
        }
        if (lane == 0) {
          sq[sub] = q;
          stie[sub] = tie;
        }
      }
      __syncthreads();
      if (warp == 0) {
        // the whole chunk at once when it stays in the binade without a tie
        double tot = 0.0;
        int anytie = 0;
#pragma unroll
        for (int r = 0; r < SQ_NSUB / 32; ++r) {
          tot += sq[r * 32 + lane];
          anytie |= stie[r * 32 + lane];
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
          tot += __shfl_xor_sync(0xffffffffu, tot, o);
          anytie |= __shfl_xor_sync(0xffffffffu, anytie, o);
        }
        if (lane == 0) {
          s_done = 1;
          const double M = normal ? ldexp(S, 53 - E) : 0.0;
          if (normal && !anytie && M + tot < two53) {
            sS = ldexp(M + tot, E - 53);
          } else {
            // sub-chunk walk
            double Mw = M, Sw = S;
            int Ew = E;
            bool nw = normal;
            for (int idx = start; idx < SQ_NSUB; ++idx) {
              if (nw && !stie[idx] && Mw + sq[idx] < two53) {
                Mw += sq[idx];
                continue;
              }
              if (nw) Sw = ldexp(Mw, Ew - 53);
              for (int i = 0; i < SQ_SUB; ++i) Sw = __dadd_rn(Sw, st[idx * SQ_SUB + i]);
              if (Sw >= tiny) {
                int E2;
                frexp(Sw, &E2);
                if (!nw || E2 != Ew) {
                  // a new binade: the later sub-chunks' quotients are stale
                  if (idx + 1 < SQ_NSUB) {
                    s_start = idx + 1;
                    s_done = 0;
                  }
                  nw = false;  // Sw is authoritative
                  break;
                }
                Mw = ldexp(Sw, 53 - Ew);
              } else {
                nw = false;
              }
            }
            sS = nw ? ldexp(Mw, Ew - 53) : Sw;
          }
        }
      }
      __syncthreads();
      if (s_done) break;
    }
  }
  if (tid == 0) *out = sS;
}

// im_out = sum(im_in) * im_out / sum(im_out)  (imcom_proc.f90:249)
__global__ void flux_scale_kernel(double* __restrict__ out, size_t count,
                                  const double* __restrict__ sums) {
  double sin_ = sums[0], sout = sums[1];
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < count;
       k += (size_t)gridDim.x * blockDim.x)
    out[k] = sin_ * out[k] / sout;
}

// Full spectrum from the r2c half spectrum with the reference's fill:
// Ft(k, j) = half(k, j) for k <= n1/2, else conj(half(n1 - k, (n2 - j) mod n2)).
// half is [b][j][0..n1/2], full is [b][j][0..n1-1] (x fastest).
__global__ void hermitian_fill_kernel(const double2* __restrict__ half, double2* __restrict__ full,
                                      int n1, int n2) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  int b = blockIdx.z;
  if (k >= n1) return;
  int nh = n1 / 2 + 1;
  const double2* hb = half + (size_t)b * nh * n2;
  double2 v;
  if (k <= n1 / 2) {
    v = hb[(size_t)j * nh + k];
  } else {
    double2 s = hb[(size_t)((n2 - j) % n2) * nh + (n1 - k)];
    v = make_double2(s.x, -s.y);
  }
  full[(size_t)b * n1 * n2 + (size_t)j * n1 + k] = v;
}


// Fortran CSHIFT source index (1-based): cshift(X, s)(i) = X(1 + mod(i-1+s, n)).
__device__ __forceinline__ int cshift_src(int i1, int s, int n) {
  return 1 + ((i1 - 1 + s) % n + n) % n;
}

// Embedding of conj(Gt_e) * Gt_f (A) or conj(Gammat) * Gt_e (B) into the
// npad-times larger frequency grid, with both cshifts of the reference
// composed into one gather.  Output grid [t][q][p], p fastest.
__global__ void embed_kernel(const double2* __restrict__ Gt, const double2* __restrict__ Gammat,
                             const int2* __restrict__ pairs, double2* __restrict__ grid,
                             int nps, int nbig) {
  int p = blockIdx.x * blockDim.x + threadIdx.x + 1;  // 1-based
  int q = blockIdx.y + 1;
  int t = blockIdx.z;
  if (p > nbig) return;
  int nmin = (nbig - nps) / 2 + 1, nmax = (nbig + nps) / 2;
  int sp = cshift_src(p, nbig / 2, nbig), sq = cshift_src(q, nbig / 2, nbig);
  double2 v = make_double2(0.0, 0.0);
  if (sp >= nmin && sp <= nmax && sq >= nmin && sq <= nmax) {
    int si = cshift_src(sp - nmin + 1, nps / 2, nps);
    int sj = cshift_src(sq - nmin + 1, nps / 2, nps);
    size_t s = (size_t)(si - 1) + (size_t)(sj - 1) * nps;
    int2 pr = pairs[t];
    double2 a, b;
    if (pr.y > 0) {  // A: conj(Gt_e) * Gt_f
      a = Gt[s + (size_t)(pr.x - 1) * nps * nps];
      b = Gt[s + (size_t)(pr.y - 1) * nps * nps];
    } else {  // B: conj(Gammat) * Gt_e
      a = Gammat[s];
      b = Gt[s + (size_t)(pr.x - 1) * nps * nps];
    }
    double ar = a.x, ai = -a.y;  // conj(a)
    double xr = ar * b.x - ai * b.y;
    double xi = ar * b.y + ai * b.x;
    // times imcom_upsilon2D(ux, uy, 1) = (1, 0)
    v = make_double2(xr * 1.0 - xi * 0.0, xr * 0.0 + xi * 1.0);
  }
  grid[(size_t)t * nbig * nbig + (size_t)(q - 1) * nbig + (p - 1)] = v;
}

// table(p, q) = Re(tmp(cshift(p), cshift(q))) / nps / nps   (A)
//             = (-2 * Re(...)) / nps / nps                   (B)
__global__ void shift_scale_kernel(const double2* __restrict__ grid, double* __restrict__ tab,
                                   int nbig, int nps, int isB) {
  int p = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int q = blockIdx.y + 1;
  int t = blockIdx.z;
  if (p > nbig) return;
  int sp = cshift_src(p, nbig / 2, nbig), sq = cshift_src(q, nbig / 2, nbig);
  double v = grid[(size_t)t * nbig * nbig + (size_t)(sq - 1) * nbig + (sp - 1)].x;
  if (isB) v = -2.0 * v;
  tab[(size_t)t * nbig * nbig + (size_t)(q - 1) * nbig + (p - 1)] = v / (double)nps / (double)nps;
}

int sum_device(imcom_ctx* ctx, const double* a, size_t count, double* dst, double* scratch) {
  partial_sum_kernel<<<256, 256, 0, ctx->stream>>>(a, count, scratch);
  IMC_LAUNCH();
  finish_sum_kernel<<<1, 256, 0, ctx->stream>>>(scratch, 256, dst);
  IMC_LAUNCH();
  return 0;
}

}  // namespace

// Build the lookup tables for A (isB = 0: all pairs e <= f, packed index
// ial = e + f(f-1)/2) or B (isB = 1: one per exposure) into ctx->tables.
static int build_tables_body(imcom_ctx* ctx, int npad, int isB) {
  int nps = ctx->nps, E = ctx->nexppsf;
  int nbig = nps * npad;
  std::vector<int2> pairs;
  if (!isB) {
    pairs.resize(E * (E + 1) / 2);
    for (int iexp = 1; iexp <= E; ++iexp)
      for (int jexp = iexp; jexp <= E; ++jexp) pairs[iexp + jexp * (jexp - 1) / 2 - 1] = make_int2(iexp, jexp);
  } else {
    for (int iexp = 1; iexp <= E; ++iexp) pairs.push_back(make_int2(iexp, 0));
  }
  int ntab = (int)pairs.size();
  size_t big2 = (size_t)nbig * nbig;
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->fftbuf, ctx->fftbuf_bytes,
                     big2 * ntab * sizeof(double2) + 4096));
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->tables, ctx->tables_bytes, big2 * ntab * sizeof(double)));
  int2* dpairs = reinterpret_cast<int2*>(reinterpret_cast<char*>(ctx->fftbuf) +
                                         big2 * ntab * sizeof(double2));
  IMC_CUDA(cudaMemcpyAsync(dpairs, pairs.data(), ntab * sizeof(int2), cudaMemcpyHostToDevice,
                           ctx->stream));
  // the own transform: always when asked for, by default where it is faster
  // than cuFFT (the register path, nps = 576 with npad = 3)
  if (ctx->table_fft == IMCOM_TABLE_FFT_OWN ||
      (ctx->table_fft == IMCOM_TABLE_FFT_AUTO && table_fft_fast(nps, nbig))) {
    bool done = false;
    IMC_TRY(table_fft_inverse(ctx, nps, nbig, ntab, dpairs, ctx->fftbuf, ctx->tables, isB, &done));
    if (done) return 0;
  }
  dim3 blk(128), grd((nbig + 127) / 128, nbig, ntab);
  embed_kernel<<<grd, blk, 0, ctx->stream>>>(ctx->Gt, ctx->Gammat, dpairs, ctx->fftbuf, nps, nbig);
  IMC_LAUNCH();
  IMC_TRY(fft_z2z(ctx, nbig, ntab, ctx->fftbuf, CUFFT_INVERSE));
  shift_scale_kernel<<<grd, blk, 0, ctx->stream>>>(ctx->fftbuf, ctx->tables, nbig, nps, isB);
  IMC_LAUNCH();
  return 0;
}

// The table build between two events (imcom_gpu_table_times).
int build_tables(imcom_ctx* ctx, int npad, int isB) {
  cudaEvent_t* ev = ctx->tab_ev[isB ? 1 : 0];
  if (!ev[0]) {
    IMC_CUDA(cudaEventCreate(&ev[0]));
    IMC_CUDA(cudaEventCreate(&ev[1]));
  }
  IMC_CUDA(cudaEventRecord(ev[0], ctx->stream));
  IMC_TRY(build_tables_body(ctx, npad, isB));
  IMC_CUDA(cudaEventRecord(ev[1], ctx->stream));
  ctx->tab_used[isB ? 1 : 0] = true;
  return 0;
}

}  // namespace imcom

using namespace imcom;

extern "C" int imcom_gpu_psf_spectra(imcom_ctx* ctx, int npoly_in, double* C_out, double* Gt_out,
                                     double* Gammat_out) {
  if (!ctx) return -1;
  if (!ctx->have_psf) return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_set_psfs has not run");
  cudaSetDevice(ctx->device);
  int npoly = npoly_in;
  if (npoly % 2 == 0) npoly = npoly - 1;  // imcom_proc.f90:201-205
  if (npoly < 1 || npoly > 15) return set_err(ctx, -2, "npoly must be in 1..16");
  int npm = npoly / 2;
  int nps = ctx->nps, E = ctx->nexppsf;
  size_t ps2 = (size_t)nps * nps;
  int nh = nps / 2 + 1;
  // scratch: real inputs (E+1) ps2 | half spectra (E+1) nh nps | sums
  // each region starts on a 256-byte boundary (complex data needs 16 bytes)
  size_t real_b = ((E + 1) * ps2 * sizeof(double) + 255) / 256 * 256;
  size_t half_b = ((size_t)(E + 1) * nh * nps * sizeof(double2) + 255) / 256 * 256;
  // own transform: its intermediate (same size as the half spectra) follows
  const bool own = ctx->table_fft == IMCOM_TABLE_FFT_OWN;
  size_t need = real_b + half_b + 8192 + (own ? half_b : 0);
  stage_begin(ctx, ST_SPECTRA);
  IMC_TRY(ensure_buf(ctx, (void**)&ctx->fftbuf, ctx->fftbuf_bytes, need));
  double* rin = reinterpret_cast<double*>(ctx->fftbuf);
  double2* half = reinterpret_cast<double2*>(reinterpret_cast<char*>(ctx->fftbuf) + real_b);
  double* sums = reinterpret_cast<double*>(reinterpret_cast<char*>(ctx->fftbuf) + real_b + half_b);
  double* scratch = sums + 16;
  const double pi = 3.141592653589793;  // imcom_data.f90 parameter
  const double eps = 1.1102230246251565e-16;  // DLAMCH('Epsilon')
  IMC_CUDA(cudaMemsetAsync(ctx->flags, 0, sizeof(int), ctx->stream));
  for (int e = 0; e < E; ++e) {
    const double* src = ctx->G + (size_t)e * ps2;
    double* dst = rin + (size_t)e * ps2;
    double ang = ctx->rot[e];
    if (fabs(ang) > 2.0 * pi * eps) {  // imcom.f90:102
      double theta_rad = std::fmod(ang, 360.0) * pi / 180.0;
      double cost = std::cos(theta_rad), sint = std::sin(theta_rad);
      dim3 blk(128), grd((nps + 127) / 128, nps);
      rotate_psf_kernel<<<grd, blk, 0, ctx->stream>>>(src, dst, nps, npm, cost, sint);
      IMC_LAUNCH();
      IMC_TRY(sum_device(ctx, src, ps2, sums + 0, scratch));
      IMC_TRY(sum_device(ctx, dst, ps2, sums + 1, scratch + 256));
      flux_scale_kernel<<<296, 256, 0, ctx->stream>>>(dst, ps2, sums);
      IMC_LAUNCH();
    } else {
      IMC_CUDA(cudaMemcpyAsync(dst, src, ps2 * sizeof(double), cudaMemcpyDeviceToDevice,
                               ctx->stream));
    }
  }
  IMC_CUDA(cudaMemcpyAsync(rin + (size_t)E * ps2, ctx->Gamma, ps2 * sizeof(double),
                           cudaMemcpyDeviceToDevice, ctx->stream));
  bool done = false;
  if (own) {
    double2* H = reinterpret_cast<double2*>(reinterpret_cast<char*>(ctx->fftbuf) + real_b +
                                            half_b + 8192);
    IMC_TRY(psf_r2c_own(ctx, nps, E + 1, rin, H, half, &done));
  }
  if (!done) IMC_TRY(fft_d2z(ctx, nps, E + 1, rin, half));
  {
    dim3 blk(128), grd((nps + 127) / 128, nps, E);
    hermitian_fill_kernel<<<grd, blk, 0, ctx->stream>>>(half, ctx->Gt, nps, nps);
    IMC_LAUNCH();
    dim3 grd1((nps + 127) / 128, nps, 1);
    hermitian_fill_kernel<<<grd1, blk, 0, ctx->stream>>>(half + (size_t)E * nh * nps,
                                                         ctx->Gammat, nps, nps);
    IMC_LAUNCH();
  }
  // C_a's sum in the reference's order: its rounding moves U by about
  // count * eps / 2 relative at U ~ 1e-6 (about 1e-12 absolute)
  seq_abs2_sum_kernel<<<1, SQ_THREADS, 0, ctx->stream>>>(ctx->Gammat, ps2, sums + 2);
  IMC_LAUNCH();
  double hs[3];
  int flag = 0;
  IMC_CUDA(cudaMemcpyAsync(hs, sums, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(&flag, ctx->flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  if (Gt_out)
    IMC_CUDA(cudaMemcpyAsync(Gt_out, ctx->Gt, ps2 * E * sizeof(double2), cudaMemcpyDeviceToHost,
                             ctx->stream));
  if (Gammat_out)
    IMC_CUDA(cudaMemcpyAsync(Gammat_out, ctx->Gammat, ps2 * sizeof(double2),
                             cudaMemcpyDeviceToHost, ctx->stream));
  stage_end(ctx, ST_SPECTRA);
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (flag)
    return set_err(ctx, IMCOM_ERR_NEVILLE,
                   "IMCOM ERROR: Two or more identical x input locations to IMCOM_POLINT");
  // C_a = sum(real(Gammat * conj(Gammat))) / n1psf / n2psf
  ctx->C_a = hs[2] / (double)nps / (double)nps;
  if (C_out) *C_out = ctx->C_a;
  ctx->have_spectra = true;
  return 0;
}
