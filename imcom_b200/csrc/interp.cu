// interp.cu -- A and B assembly by lookup-table interpolation.
//
// Reference: imcom_lookup_A (imcom_matrix.f90:206-284), imcom_lookup_B
// (:288-357), imcom_interp_lookup (:497-542), imcom_polin2/imcom_polint
// (imcom_proc.f90:351-429).
//
// Per element the reference takes the table window [floor-npm, ceil+npm]
// clipped to [1, L] (8 x 8 points for a non-integer argument, 7 x 7 for an
// integer one), interpolates along y for each window row, then along x.
// The argument, floor/ceiling and window bounds are computed here with the
// same floating-point operations, so they are bit-identical.  The
// interpolating polynomial on those nodes is unique; this kernel evaluates
// it in Lagrange form (weights from prefix/suffix products of (t - x_j) and
// exact integer denominators) instead of Neville's tableau: ~8x fewer flops
// and no divisions, equal to the reference up to rounding (tests bound the
// difference at 1e-13 of the table scale).
//
// Mapping: 8 lanes per element.  Lane k owns window column x_k and sums the
// y-interpolation g_k = sum_l wy_l T(x_k, y_l) over its 8 rows; three xor
// shuffles form f = sum_k wx_k g_k.  Each warp load instruction touches 4
// elements x 1 row = 4 contiguous 64-byte row segments, so a window costs 8
// row fetches instead of 64 scattered ones.  A CTA computes a 32 x 32 tile
// into shared memory and writes it (and, for A, its mirror) coalesced.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace imcom {

int build_tables(imcom_ctx* ctx, int npad, int isB);

namespace {

// 1 / prod_{j != k} (k - j) for a window of K consecutive integer nodes.
__constant__ double c_invd[9][8];

constexpr int TILE = 32;
constexpr int WARPS = 8;

struct InterpGeom {
  const double* tables;
  long long L;     // table side
  long long L2;    // L * L
  double cent;     // L/2 + 1
  int npm;
};

// Interpolate one element; called by the 8 lanes of a group with the same
// (xarg, yarg, table).  Returns f in every lane of the group.
__device__ __forceinline__ double interp8(const InterpGeom& g, const double* __restrict__ tab,
                                          double xarg, double yarg, int k) {
  double iarg = __dadd_rn(g.cent, xarg);
  double jarg = __dadd_rn(g.cent, yarg);
  int ia_floor = (int)floor(iarg), ja_floor = (int)floor(jarg);
  int ia_ceil = (int)ceil(iarg), ja_ceil = (int)ceil(jarg);
  double contrib = 0.0;
  bool inside = (ia_floor >= 1) && (ja_floor >= 1) && (ia_ceil <= g.L) && (ja_ceil <= g.L);
  if (inside) {
    int imin = max(1, ia_floor - g.npm), jmin = max(1, ja_floor - g.npm);
    int imax = min((int)g.L, ia_ceil + g.npm), jmax = min((int)g.L, ja_ceil + g.npm);
    int Kx = imax - imin + 1, Ky = jmax - jmin + 1;
    // y weights (all lanes need all of them)
    double sy[8], pre[8], wy[8];
    bool ynode = false;
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      sy[l] = (l < Ky) ? jarg - (double)(jmin + l) : 1.0;
      ynode |= (l < Ky) && (sy[l] == 0.0);
    }
    double acc = 1.0;
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      pre[l] = acc;
      acc *= sy[l];
    }
    acc = 1.0;
#pragma unroll
    for (int l = 7; l >= 0; --l) {
      wy[l] = pre[l] * acc * c_invd[Ky][l];
      acc *= sy[l];
    }
    if (ynode) {
#pragma unroll
      for (int l = 0; l < 8; ++l) wy[l] = (l < Ky && sy[l] == 0.0) ? 1.0 : 0.0;
    }
    // x weight of this lane's node
    double wx = 0.0;
    if (k < Kx) {
      double p = 1.0;
      bool xnode = false;
      for (int j = 0; j < Kx; ++j) {
        double s = iarg - (double)(imin + j);
        xnode |= (s == 0.0);
        if (j != k) p *= s;
      }
      wx = p * c_invd[Kx][k];
      if (xnode) wx = (iarg - (double)(imin + k) == 0.0) ? 1.0 : 0.0;
      const double* col = tab + (size_t)(imin - 1 + k) + (size_t)(jmin - 1) * g.L;
      double gk = 0.0;
#pragma unroll
      for (int l = 0; l < 8; ++l)
        if (l < Ky) gk += wy[l] * __ldg(col + (size_t)l * g.L);
      contrib = wx * gk;
    }
  }
  contrib += __shfl_xor_sync(0xffffffffu, contrib, 1);
  contrib += __shfl_xor_sync(0xffffffffu, contrib, 2);
  contrib += __shfl_xor_sync(0xffffffffu, contrib, 4);
  return contrib;
}

// A: upper-triangle tiles (bj >= bi); writes the tile and its mirror.
__global__ void __launch_bounds__(WARPS * 32)
lookup_A_kernel(InterpGeom g, const double* __restrict__ x, const double* __restrict__ y,
                const int* __restrict__ expi, int n, int psfconst, double npad, double psfx,
                double psfy, double* __restrict__ A, long long lda) {
  int bi = blockIdx.x, bj = blockIdx.y;
  if (bj < bi) return;
  __shared__ double tile[TILE][TILE + 1];  // tile[jj][ii]
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int k = lane & 7, grp = lane >> 3;
  for (int c = 0; c < TILE / WARPS; ++c) {
    int jj = warp + WARPS * c;
    int j = bj * TILE + jj;
    for (int s = 0; s < TILE / 4; ++s) {
      int ii = 4 * s + grp;
      int i = bi * TILE + ii;
      bool valid = (i < n) && (j < n) && (j >= i);
      // every lane runs the shuffles; invalid groups interpolate at 0 offset
      int ie = valid ? i : 0, je = valid ? j : 0;
      double xj = x[je], xi = x[ie], yj = y[je], yi = y[ie];
      int ial = 1;
      if (psfconst != 1) {
        int ei = expi[ie], ej = expi[je];
        ial = ei + ej * (ej - 1) / 2;
      }
      double Delx = __ddiv_rn(__dmul_rn(npad, __dsub_rn(xj, xi)), psfx);
      double Dely = __ddiv_rn(__dmul_rn(npad, __dsub_rn(yj, yi)), psfy);
      double f = interp8(g, g.tables + (size_t)(ial - 1) * g.L2, Delx, Dely, k);
      if (k == 0) tile[jj][ii] = valid ? f : 0.0;
    }
  }
  __syncthreads();
  // A(i, j) for j >= i from the tile; below the diagonal use the mirror.
  for (int e = threadIdx.x; e < TILE * TILE; e += WARPS * 32) {
    int ii = e & 31, jj = e >> 5;
    int i = bi * TILE + ii, j = bj * TILE + jj;
    if (i < n && j < n) {
      double v = (bi == bj && jj < ii) ? tile[ii][jj] : tile[jj][ii];
      A[(size_t)i + (size_t)j * lda] = v;
    }
  }
  if (bi != bj) {
    // A(j, i) = A(i, j): column i of the mirror block, rows j.
    for (int e = threadIdx.x; e < TILE * TILE; e += WARPS * 32) {
      int jj = e & 31, ii = e >> 5;
      int i = bi * TILE + ii, j = bj * TILE + jj;
      if (i < n && j < n) A[(size_t)j + (size_t)i * lda] = tile[jj][ii];
    }
  }
}

// B(i, a): tile of 32 input pixels x 32 output pixels.
__global__ void __launch_bounds__(WARPS * 32)
lookup_B_kernel(InterpGeom g, const double* __restrict__ x, const double* __restrict__ y,
                const int* __restrict__ expi, const double* __restrict__ X,
                const double* __restrict__ Y, int n, int m, int psfconst, double npad,
                double psfx, double psfy, double* __restrict__ B, long long ldb) {
  int bi = blockIdx.x, ba = blockIdx.y;
  __shared__ double tile[TILE][TILE + 1];  // tile[aa][ii]
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int k = lane & 7, grp = lane >> 3;
  for (int c = 0; c < TILE / WARPS; ++c) {
    int aa = warp + WARPS * c;
    int a = ba * TILE + aa;
    for (int s = 0; s < TILE / 4; ++s) {
      int ii = 4 * s + grp;
      int i = bi * TILE + ii;
      bool valid = (i < n) && (a < m);
      int ie = valid ? i : 0, ae = valid ? a : 0;
      int itab = (psfconst == 1) ? 1 : expi[ie];
      double Delx = __ddiv_rn(__dmul_rn(npad, __dsub_rn(x[ie], X[ae])), psfx);
      double Dely = __ddiv_rn(__dmul_rn(npad, __dsub_rn(y[ie], Y[ae])), psfy);
      double f = interp8(g, g.tables + (size_t)(itab - 1) * g.L2, Delx, Dely, k);
      if (k == 0) tile[aa][ii] = valid ? f : 0.0;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < TILE * TILE; e += WARPS * 32) {
    int ii = e & 31, aa = e >> 5;
    int i = bi * TILE + ii, a = ba * TILE + aa;
    if (i < n && a < m) B[(size_t)i + (size_t)a * ldb] = tile[aa][ii];
  }
}

bool g_invd_ready[64] = {false};

int upload_invd(imcom_ctx* ctx) {
  if (ctx->device >= 0 && ctx->device < 64 && g_invd_ready[ctx->device]) return 0;
  double h[9][8] = {};
  for (int K = 1; K <= 8; ++K)
    for (int k = 0; k < K; ++k) {
      double d = 1.0;
      for (int j = 0; j < K; ++j)
        if (j != k) d *= (double)(k - j);
      h[K][k] = 1.0 / d;
    }
  IMC_CUDA(cudaMemcpyToSymbol(c_invd, h, sizeof h));
  if (ctx->device >= 0 && ctx->device < 64) g_invd_ready[ctx->device] = true;
  return 0;
}

int check_interp_args(imcom_ctx* ctx, int npoly_in, int npad, int* npm) {
  if (!ctx->have_spectra)
    return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_psf_spectra has not run");
  if (ctx->n <= 0) return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_set_inputs has not run");
  int npoly = npoly_in;
  if (npoly % 2 == 0) npoly = npoly - 1;  // imcom_matrix.f90:515-519
  if (npoly < 1 || npoly > 7)
    return set_err(ctx, -2, "npoly must be 1..8 (window of at most 8 points)");
  if (npad < 1) return set_err(ctx, -3, "npad must be >= 1");
  *npm = npoly / 2;
  if (ctx->psfconst == 0 && ctx->max_exp > ctx->nexppsf)
    return set_err(ctx, IMCOM_ERR_STATE, "exp_i reaches %d but only %d PSFs were set",
                   ctx->max_exp, ctx->nexppsf);
  return 0;
}

}  // namespace
}  // namespace imcom

using namespace imcom;

extern "C" int imcom_gpu_build_A(imcom_ctx* ctx, int npoly, int npad, double* A_out) {
  if (!ctx) return -1;
  int npm = 0;
  IMC_TRY(check_interp_args(ctx, npoly, npad, &npm));
  cudaSetDevice(ctx->device);
  IMC_TRY(upload_invd(ctx));
  stage_begin(ctx, ST_A);
  IMC_TRY(build_tables(ctx, npad, 0));
  IMC_TRY(ensure_mat(ctx, ctx->A, ctx->n, ctx->n));
  int L = ctx->nps * npad;
  InterpGeom g{ctx->tables, L, (long long)L * L, (double)(L / 2 + 1), npm};
  int nt = (ctx->n + TILE - 1) / TILE;
  dim3 grd(nt, nt);
  lookup_A_kernel<<<grd, WARPS * 32, 0, ctx->stream>>>(g, ctx->x, ctx->y, ctx->exp_i, ctx->n,
                                                       ctx->psfconst, (double)npad, ctx->psfx,
                                                       ctx->psfy, ctx->A.p, ctx->A.ld);
  IMC_LAUNCH();
  stage_end(ctx, ST_A);
  ctx->have_A = true;
  ctx->have_QL = false;
  if (A_out) {
    IMC_TRY(download_mat(ctx, ctx->A, A_out));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}

extern "C" int imcom_gpu_build_B(imcom_ctx* ctx, int npoly, int npad, double* B_out) {
  if (!ctx) return -1;
  int npm = 0;
  IMC_TRY(check_interp_args(ctx, npoly, npad, &npm));
  cudaSetDevice(ctx->device);
  IMC_TRY(upload_invd(ctx));
  stage_begin(ctx, ST_B);
  IMC_TRY(build_tables(ctx, npad, 1));
  IMC_TRY(ensure_mat(ctx, ctx->B, ctx->n, ctx->m));
  int L = ctx->nps * npad;
  InterpGeom g{ctx->tables, L, (long long)L * L, (double)(L / 2 + 1), npm};
  dim3 grd((ctx->n + TILE - 1) / TILE, (ctx->m + TILE - 1) / TILE);
  lookup_B_kernel<<<grd, WARPS * 32, 0, ctx->stream>>>(g, ctx->x, ctx->y, ctx->exp_i, ctx->X,
                                                       ctx->Y, ctx->n, ctx->m, ctx->psfconst,
                                                       (double)npad, ctx->psfx, ctx->psfy,
                                                       ctx->B.p, ctx->B.ld);
  IMC_LAUNCH();
  stage_end(ctx, ST_B);
  ctx->have_B = true;
  ctx->have_P = false;
  if (B_out) {
    IMC_TRY(download_mat(ctx, ctx->B, B_out));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}
