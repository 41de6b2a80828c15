// eigen_2s.cu -- two-stage reduction of a symmetric matrix to tridiagonal
// form: dense -> band (bandwidth SB) by blocked Householder QR of panels and
// two-sided block updates on the FP64 DMMA GEMM, then band -> tridiagonal by
// bulge chasing.  Alternative to the one-stage dsytrd of eigen_dc.cu for the
// eigensolver that replaces DSYEVR in imcom_eigen_A (imcom_matrix.f90:617-643).
//
// Stage 1 (LAPACK dsytrd_sy2sb structure, lower): for the panel of columns
// k .. k+SB-1 the rows k+SB .. n-1 are factorised, P = Q R with
// Q = I - V T V^T; R goes into the band below the diagonal block, and the
// trailing matrix A22 = A(k+SB:, k+SB:) (full symmetric storage) becomes
// Q^T A22 Q through
//     W = A22 V T,  W <- W - 1/2 V (T^T (V^T W)),  A22 <- A22 - V W^T - W V^T,
// the last on the lower tiles only, its upper triangle mirrored after.
// The panel QR runs in one thread-block cluster: each CTA holds a slice of
// the panel's rows in shared memory, and every column needs one cluster-wide
// exchange of its partial sums (the column's norm below the pivot, its dot
// products with the later columns, and the pivot row) through distributed
// shared memory.
#include <algorithm>
#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "common.cuh"
#include "eigen.cuh"

namespace imcom {

namespace {

constexpr int SB = 32;            // bandwidth of the first stage (panel width)
constexpr int SB_CTAS = 16;       // CTAs of the panel cluster (8 where 16 cannot be placed)
// threads of the panel kernel: 32 columns x 8 row slices with the panel
// staged in shared memory, x 32 row slices when it is updated in place in
// global memory (more loads in flight per column)
__host__ __device__ constexpr int sb_threads(bool staged) { return staged ? 256 : 1024; }

struct PanelArgs {
  double* A;       // full symmetric working matrix
  long long lda;
  double* V;       // reflectors: column k + j, rows k + SB ..; 1 at the pivot, 0 above
  long long ldv;
  double* tau;     // tau[k + j]
  int n, k, per;   // panel columns k .. k + SB - 1; rows per CTA
};

// Householder QR of the panel A(k+SB : n, k : k+SB) (LAPACK dgeqr2 with
// dlarfg's conventions) by a cluster of CTAs.  CTA q holds panel rows
// q*per .. q*per + per - 1 in shared memory (column-major, stride per).  For
// column j every CTA forms, over its rows, S_c = sum_{i > j} P(i,j) P(i,c)
// (c >= j; S_j is the squared norm below the pivot) and contributes the pivot
// row R_c = P(j, c) if it holds it; the 2 SB values of every CTA are stored
// into every CTA's shared memory (alternating buffers by column parity) and
// summed after one cluster barrier.  Then, in every CTA,
//   beta = -sign(alpha) sqrt(alpha^2 + S_j), tau = (beta - alpha) / beta,
//   v = [1; P(j+1:, j) / (alpha - beta)],  w_c = tau (R_c + S_c / (alpha - beta)),
// and the later columns are updated, P(:, c) -= v w_c.
// STAGED: the CTA's rows are copied into shared memory first (panels of up to
// a few hundred rows per CTA); otherwise the columns are updated in place in
// global memory (stride lda), which only the reduction buffers need shared
// memory for.
template <bool STAGED>
__global__ void __launch_bounds__(sb_threads(STAGED), 1) sb_panel_kernel(PanelArgs a) {
  constexpr int SB_THREADS = sb_threads(STAGED), SB_SLICES = SB_THREADS / SB;
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int q = (int)cl.block_rank(), nct = (int)cl.num_blocks();
  const int N = a.n - a.k - SB;  // panel rows
  const int per = a.per;
  const int rb = q * per, nr = max(0, min(per, N - rb));
  const int jmax = min(SB, N);
  extern __shared__ __align__(16) double psm[];
  const size_t row0 = (size_t)a.k + SB + rb;
  // P(i, c) = P[c * ldp + i]: the CTA's rows of the panel
  const long long ldp = STAGED ? per : a.lda;
  double* P = STAGED ? psm : a.A + row0 + (size_t)a.k * a.lda;
  double* part = psm + (STAGED ? (size_t)SB * per : 0);  // [2][SB_CTAS][2 SB] from every CTA
  double* red = part + 2 * SB_CTAS * 2 * SB;              // [SB_SLICES][2 SB]
  double* fin = red + SB_SLICES * 2 * SB;                 // [2 SB] cluster totals
  const int c = threadIdx.x & (SB - 1), slice = threadIdx.x / SB;
  if (STAGED)
    for (int e = threadIdx.x; e < SB * nr; e += SB_THREADS) {
      const int cc = e / nr, i = e - cc * nr;
      P[(size_t)cc * per + i] = a.A[row0 + i + (size_t)(a.k + cc) * a.lda];
    }
  cl.sync();  // every CTA runs before any stores into its shared memory
  for (int j = 0; j < jmax; ++j) {
    double sdot = 0.0, rowv = 0.0;
    if (c >= j) {
      const double* pj = P + (size_t)j * ldp;
      const double* pc = P + (size_t)c * ldp;
      for (int i = slice; i < nr; i += SB_SLICES) {
        const int gi = rb + i;
        if (gi > j) sdot = fma(pj[i], pc[i], sdot);
        else if (gi == j) rowv = pc[i];
      }
    }
    red[slice * 2 * SB + c] = sdot;
    red[slice * 2 * SB + SB + c] = rowv;
    __syncthreads();
    double* mine = part + (size_t)(j & 1) * SB_CTAS * 2 * SB;
    if (threadIdx.x < 2 * SB) {
      double s = 0.0;
      for (int h = 0; h < SB_SLICES; ++h) s += red[h * 2 * SB + threadIdx.x];
      for (int r = 0; r < nct; ++r) cl.map_shared_rank(mine, r)[q * 2 * SB + threadIdx.x] = s;
    }
    cl.sync();
    if (threadIdx.x < 2 * SB) {
      double s = 0.0;
      for (int r = 0; r < nct; ++r) s += mine[r * 2 * SB + threadIdx.x];
      fin[threadIdx.x] = s;
    }
    __syncthreads();
    const double alpha = fin[SB + j], sig2 = fin[j];
    double t = 0.0, beta = alpha, scl = 0.0;
    if (sig2 != 0.0) {
      beta = -copysign(sqrt(alpha * alpha + sig2), alpha);
      t = (beta - alpha) / beta;
      scl = 1.0 / (alpha - beta);
    }
    if (c > j) {
      const double w = t * (fin[SB + c] + scl * fin[c]);
      const double* pj = P + (size_t)j * ldp;
      double* pc = P + (size_t)c * ldp;
      for (int i = slice; i < nr; i += SB_SLICES) {
        const int gi = rb + i;
        if (gi > j) pc[i] -= (pj[i] * scl) * w;
        else if (gi == j) pc[i] -= w;
      }
    }
    __syncthreads();
    if (c == j) {
      // column j: v below the pivot (kept in P until the write-back), beta on it
      double* pj = P + (size_t)j * ldp;
      for (int i = slice; i < nr; i += SB_SLICES) {
        const int gi = rb + i;
        if (gi > j) pj[i] *= scl;
        else if (gi == j) pj[i] = beta;
      }
    }
    if (q == 0 && threadIdx.x == 0) a.tau[a.k + j] = t;
    __syncthreads();
  }
  if (q == 0 && threadIdx.x < SB && threadIdx.x >= jmax) a.tau[a.k + threadIdx.x] = 0.0;
  // write back: R on and above the pivot into the band, zeros below; v into V
  for (int e = threadIdx.x; e < SB * nr; e += SB_THREADS) {
    const int cc = e / nr, i = e - cc * nr;
    const int gi = rb + i;
    const double p = P[(size_t)cc * ldp + i];
    const size_t col = (size_t)(a.k + cc);
    a.A[row0 + i + col * a.lda] = gi <= cc ? p : 0.0;
    a.V[row0 + i + col * a.ldv] = gi < cc ? 0.0 : (gi == cc ? 1.0 : p);
  }
}

inline size_t panel_smem(int per, bool staged) {
  return ((staged ? (size_t)SB * per : 0) + 2 * SB_CTAS * 2 * SB +
          (size_t)(sb_threads(staged) / SB) * 2 * SB + 2 * SB) *
         sizeof(double);
}

// The panel's two-sided update factors from X1 = A22 V (N x SB):
//   W = X1 T - 1/2 V M2,  M2 = T^T (V^T X1) T     (V^T W = (V^T X1) T),
// in three launches.  wy_partial_kernel: S_b = V_b^T X1_b for blocks b of
// WY_ROWS rows.  wy_m2_kernel (one CTA): S = sum_b S_b in a fixed order and
// M2.  wy_finish_kernel: for its rows, W and the packed operands of the
// update A22 -= X Y^T, X = [V | W] and Y = [W | V] (ld ldx, 2 SB columns),
// written over X1's storage (the block's rows of X1 are read first; X1 lives
// in X's first SB columns).
constexpr int WY_ROWS = 48, WY_THREADS = 256;

__global__ void __launch_bounds__(WY_THREADS) wy_partial_kernel(
    const double* __restrict__ V, long long ldv, const double* __restrict__ X1, long long ldx,
    int N, double* __restrict__ Spart) {
  __shared__ double sV[WY_ROWS][SB + 1], sX[WY_ROWS][SB + 1];
  const int r0 = blockIdx.x * WY_ROWS;
  for (int e = threadIdx.x; e < WY_ROWS * SB; e += WY_THREADS) {
    const int r = e % WY_ROWS, c = e / WY_ROWS;
    const bool in = r0 + r < N;
    sV[r][c] = in ? V[(size_t)(r0 + r) + (size_t)c * ldv] : 0.0;
    sX[r][c] = in ? X1[(size_t)(r0 + r) + (size_t)c * ldx] : 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < SB * SB; e += WY_THREADS) {
    const int i = e % SB, j = e / SB;
    double acc = 0.0;
    for (int r = 0; r < WY_ROWS; ++r) acc = fma(sV[r][i], sX[r][j], acc);
    Spart[(size_t)blockIdx.x * SB * SB + e] = acc;
  }
}

// One CTA of SB * SB threads: M2 = T^T S T (column-major, ld SB).
__global__ void __launch_bounds__(SB * SB) wy_m2_kernel(const double* __restrict__ Spart, int nb,
                                                        const double* __restrict__ T,
                                                        double* __restrict__ M2) {
  __shared__ double sS[SB][SB + 1], sT[SB][SB + 1], sU[SB][SB + 1];
  const int e = threadIdx.x, i = e % SB, j = e / SB;
  double acc = 0.0;
  for (int b = 0; b < nb; ++b) acc += Spart[(size_t)b * SB * SB + e];
  sS[i][j] = acc;
  sT[i][j] = T[e];  // T(i, j) at i + j SB, upper triangular
  __syncthreads();
  double u = 0.0;
  for (int h = 0; h <= j; ++h) u = fma(sS[i][h], sT[h][j], u);
  sU[i][j] = u;
  __syncthreads();
  double m = 0.0;
  for (int h = 0; h <= i; ++h) m = fma(sT[h][i], sU[h][j], m);
  M2[e] = m;
}

// One CTA of SB * SB threads: G = sum_b Spart_b (the panel's Gram matrix
// V^T V from wy_partial_kernel's blocks, in a fixed order) and T from G and
// tau (LAPACK dlarft, forward, columnwise: T(j,j) = tau_j,
// T(0:j, j) = -tau_j T(0:j, 0:j) G(0:j, j)), by warp 0.
__global__ void __launch_bounds__(SB * SB) gram_larft_kernel(const double* __restrict__ Spart,
                                                             int nb,
                                                             const double* __restrict__ tau,
                                                             double* __restrict__ T) {
  __shared__ double sG[SB][SB + 1];  // sG[j][h] = G(h, j)
  __shared__ double sT[SB][SB + 1];
  const int e = threadIdx.x, i = e % SB, j = e / SB;
  double acc = 0.0;
  for (int b = 0; b < nb; ++b) acc += Spart[(size_t)b * SB * SB + e];
  sG[j][i] = acc;
  sT[i][j] = 0.0;
  __syncthreads();
  if (threadIdx.x < SB) {
    const int r = threadIdx.x;
    for (int jj = 0; jj < SB; ++jj) {
      const double tj = tau[jj];
      double sum = 0.0;
      if (r < jj)
        for (int h = r; h < jj; ++h) sum += sT[r][h] * sG[jj][h];
      __syncwarp();
      if (r < jj) sT[r][jj] = -tj * sum;
      if (r == jj) sT[jj][jj] = tj;
      __syncwarp();
    }
  }
  __syncthreads();
  T[e] = sT[i][j];  // column-major: T(i, j) at i + j SB
}

__global__ void __launch_bounds__(WY_THREADS) wy_finish_kernel(
    const double* __restrict__ T, const double* __restrict__ M2, const double* __restrict__ V,
    long long ldv, double* __restrict__ XY, long long ldx, int N) {
  __shared__ double sT[SB][SB + 1], sM[SB][SB + 1];
  __shared__ double sV[WY_ROWS][SB + 1], sX[WY_ROWS][SB + 1];
  const int r0 = blockIdx.x * WY_ROWS;
  for (int e = threadIdx.x; e < SB * SB; e += WY_THREADS) {
    sT[e % SB][e / SB] = T[e];
    sM[e % SB][e / SB] = M2[e];
  }
  for (int e = threadIdx.x; e < WY_ROWS * SB; e += WY_THREADS) {
    const int r = e % WY_ROWS, c = e / WY_ROWS;
    const bool in = r0 + r < N;
    sV[r][c] = in ? V[(size_t)(r0 + r) + (size_t)c * ldv] : 0.0;
    sX[r][c] = in ? XY[(size_t)(r0 + r) + (size_t)c * ldx] : 0.0;
  }
  __syncthreads();
  double* X = XY;
  double* Y = XY + (size_t)ldx * 2 * SB;
  for (int e = threadIdx.x; e < WY_ROWS * SB; e += WY_THREADS) {
    const int r = e % WY_ROWS, j = e / WY_ROWS;
    if (r0 + r >= N) continue;
    double w1 = 0.0, w2 = 0.0;
    for (int h = 0; h <= j; ++h) w1 = fma(sX[r][h], sT[h][j], w1);
    for (int h = 0; h < SB; ++h) w2 = fma(sV[r][h], sM[h][j], w2);
    const double w = w1 - 0.5 * w2;
    const double v = sV[r][j];
    const size_t row = (size_t)(r0 + r);
    X[row + (size_t)j * ldx] = v;
    X[row + (size_t)(SB + j) * ldx] = w;
    Y[row + (size_t)j * ldx] = w;
    Y[row + (size_t)(SB + j) * ldx] = v;
  }
}

// A(i, j) = A(j, i) for i < j: the strictly upper triangle of the N x N
// matrix at ld from its lower triangle, through 32 x 32 shared tiles
// (block (x, y) writes tile row y, tile column x >= y; reads only the lower
// tile (x, y), so blocks never touch each other's data).
__global__ void mirror_lower_kernel(double* __restrict__ A, long long ld, int N) {
  __shared__ double t[32][33];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bi > bj) return;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int k = ty; k < 32; k += 8) {
    const int r = bj * 32 + tx, c = bi * 32 + k;  // source A(r, c), r >= c
    t[k][tx] = (r < N && c < N) ? A[r + (size_t)c * ld] : 0.0;
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    const int r = bi * 32 + tx, c = bj * 32 + k;  // destination A(r, c) = A(c, r)
    if (r < c && c < N) A[r + (size_t)c * ld] = t[tx][k];
  }
}

// Band storage for the second stage: AB[d + c * ldb] = A(c + d, c) for
// d <= SB, zero for SB < d < ldb.
__global__ void band_extract_kernel(const double* __restrict__ A, long long lda, int n,
                                    double* __restrict__ AB, int ldb) {
  const int c = blockIdx.x;
  for (int d = threadIdx.x; d < ldb; d += blockDim.x)
    AB[d + (size_t)c * ldb] = (d <= SB && c + d < n) ? A[(c + d) + (size_t)c * lda] : 0.0;
}


// ---- Stage 2: band -> tridiagonal by bulge chasing ------------------------
// The band (bandwidth SB, lower) is reduced column by column (LAPACK
// dsb2st's scheme): sweep s annihilates A(s+2 :, s) with a reflector on rows
// s+1 .. s+SB (task 0), whose right application fills a triangle below the
// band; task t > 0 of the sweep annihilates the first column of that bulge
// (column r0 - SB, rows r0 = s + 1 + t SB ..) and applies its reflector from
// the left to the bulge's other columns, two-sidedly to the diagonal block
// and from the right to the rows below, pushing the bulge SB rows further.
// Task (s, t) touches columns s + 1 + (t-1) SB .. s + (t+2) SB only, so task
// t of sweep s + 1 may run beside task t + 3 of sweep s: a warp per sweep,
// CH_K consecutive sweeps per CTA ("group") in lock step, each warp CH_LAG
// tasks behind the one before it.  The group's live columns sit in a
// circular shared-memory window (band and bulge, 2 SB rows per column);
// columns it has finished are written back to AB and published by a
// watermark, which the next group waits for before it loads them.  Two
// more warps move the columns while the four task warps compute: in step
// tau one writes back and publishes the columns the previous step finished,
// the other fetches the columns step tau + 1 adds, so the global round trips
// stay off the tasks' path; one barrier per step.
constexpr int CH_K = 4;                 // sweeps per group, one warp each
constexpr int CH_THREADS = 32 * (CH_K + 2);  // + a storing and a loading warp
constexpr int CH_LAG = 3;               // tasks between consecutive sweeps
constexpr int CH_LDB = 2 * SB;          // rows of band storage: band and bulge
// columns of the window: a group's tasks span < 11 SB columns; the columns
// being written back (one step behind) and fetched (one step ahead) add 2 SB
constexpr int CH_WCOLS = 13 * SB;
constexpr size_t CH_SMEM = (size_t)CH_WCOLS * CH_LDB * sizeof(double);

struct ChaseArgs {
  double* AB;       // AB[d + c * CH_LDB] = A(c + d, c)
  int n, ngroups;
  double* V;        // V[(t n + s) SB + i]: reflector of task t of sweep s, V[0] = 1
  double* tau;      // tau[t n + s]
  int* wm;          // wm[g]: AB holds group g's final values of columns < wm[g]
  int* next_group;  // groups are taken in order
  int* err;         // a wait ran out
  long long spin;   // polls per wait
};

__host__ __device__ __forceinline__ int chase_ntasks(int n, int s) {
  return (n - s - 3) >= 0 ? (n - s - 3) / SB + 1 : 0;
}

// A(r, c), r >= c, in the window
__device__ __forceinline__ double& wb_at(double* W, int r, int c) {
  return W[(size_t)(c % CH_WCOLS) * CH_LDB + (r - c)];
}

// One task, by one warp (lane i: row r0 + i of the reflector).
__device__ void chase_task(const ChaseArgs& a, double* W, int s, int t, int lane, double* sv,
                           double* sw) {
  const int n = a.n;
  const int r0 = s + 1 + t * SB;
  const int c0 = t == 0 ? s : r0 - SB;
  const int L = min(SB, n - r0);
  // reflector from A(r0 : r0 + L, c0) (dlarfg)
  const double x = lane < L ? wb_at(W, r0 + lane, c0) : 0.0;
  double sig2 = lane >= 1 ? x * x : 0.0;
#pragma unroll
  for (int o = 16; o; o >>= 1) sig2 += __shfl_xor_sync(0xffffffffu, sig2, o);
  const double alpha = __shfl_sync(0xffffffffu, x, 0);
  double beta = alpha, tau = 0.0, scl = 0.0;
  if (sig2 != 0.0) {
    beta = -copysign(sqrt(alpha * alpha + sig2), alpha);
    tau = (beta - alpha) / beta;
    scl = 1.0 / (alpha - beta);
  }
  const double v = lane == 0 ? 1.0 : (lane < L ? x * scl : 0.0);
  sv[lane] = v;
  if (lane < L) wb_at(W, r0 + lane, c0) = lane == 0 ? beta : 0.0;
  a.V[((size_t)t * n + s) * SB + lane] = v;
  if (lane == 0) a.tau[(size_t)t * n + s] = tau;
  __syncwarp();
  if (tau == 0.0) return;
  // left: the bulge's other columns c0 + 1 .. r0 - 1, rows r0 .. r0 + L - 1
  if (t > 0 && lane < SB - 1) {
    const int c = c0 + 1 + lane;
    double w = 0.0;
    for (int i = 0; i < L; ++i) w = fma(sv[i], wb_at(W, r0 + i, c), w);
    w *= tau;
    for (int i = 0; i < L; ++i) wb_at(W, r0 + i, c) -= sv[i] * w;
  }
  // two-sided on the diagonal block D: D - v w^T - w v^T,
  // p = tau D v, w = p - tau/2 (p^T v) v (dlarfy)
  double y = 0.0;
  if (lane < L)
    for (int j = 0; j < L; ++j) {
      const double dij = j <= lane ? wb_at(W, r0 + lane, r0 + j) : wb_at(W, r0 + j, r0 + lane);
      y = fma(dij, sv[j], y);
    }
  const double p = tau * y;
  double pv = p * v;
#pragma unroll
  for (int o = 16; o; o >>= 1) pv += __shfl_xor_sync(0xffffffffu, pv, o);
  const double wv = p - 0.5 * tau * pv * v;
  sw[lane] = wv;
  __syncwarp();
  if (lane < L)
    for (int j = 0; j <= lane; ++j) wb_at(W, r0 + lane, r0 + j) -= v * sw[j] + wv * sv[j];
  // right: rows r0 + L .. r0 + L + L2 - 1 (the new bulge), columns r0 .. r0 + L - 1
  const int L2 = min(SB, n - (r0 + L));
  if (lane < L2) {
    const int r = r0 + L + lane;
    double z = 0.0;
    for (int j = 0; j < L; ++j) z = fma(wb_at(W, r, r0 + j), sv[j], z);
    z *= tau;
    for (int j = 0; j < L; ++j) wb_at(W, r, r0 + j) -= z * sv[j];
  }
  __syncwarp();
}

// Columns [lo, hi) group g's tasks at step tau touch; lo also covers the
// group's sweeps that have not started (they begin at their own column).
__device__ __forceinline__ void chase_span(const ChaseArgs& a, int g, int step, int& lo,
                                           int& hi) {
  lo = 0x7fffffff;
  hi = 0;
  for (int k = 0; k < CH_K; ++k) {
    const int s = g * CH_K + k;
    if (s > a.n - 3) break;
    const int t = step - CH_LAG * k;
    if (t < 0) {
      lo = min(lo, s);
      continue;
    }
    if (t >= chase_ntasks(a.n, s)) continue;
    const int r0 = s + 1 + t * SB;
    lo = min(lo, t == 0 ? s : r0 - SB);
    hi = max(hi, min(a.n, r0 + SB));
  }
}

// Waits (bounded) until group g has published columns below need.
__device__ bool wait_wm(const ChaseArgs& a, int g, int need) {
  if (g < 0) return true;
  for (long long it = 0;; ++it) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(a.wm + g) : "memory");
    if (v >= need) return true;
    if (*(volatile int*)a.err) return false;
    if (it >= a.spin) {
      atomicExch(a.err, 1);
      return false;
    }
  }
}

__device__ __forceinline__ void publish_wm(const ChaseArgs& a, int g, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(a.wm + g), "r"(v) : "memory");
}

// Columns [c_lo, c_hi) of the window back to AB, by one warp.
__device__ __forceinline__ void window_store_warp(const ChaseArgs& a, const double* W, int c_lo,
                                                  int c_hi, int lane) {
  for (int e = lane; e < (c_hi - c_lo) * CH_LDB; e += 32) {
    const int c = c_lo + e / CH_LDB, d = e % CH_LDB;
    a.AB[(size_t)c * CH_LDB + d] = W[(size_t)(c % CH_WCOLS) * CH_LDB + d];
  }
}

// Columns [c_lo, c_hi) of AB into the window, by one warp.
__device__ __forceinline__ void window_load_warp(const ChaseArgs& a, double* W, int c_lo,
                                                 int c_hi, int lane) {
  for (int e = lane; e < (c_hi - c_lo) * CH_LDB; e += 32) {
    const int c = c_lo + e / CH_LDB, d = e % CH_LDB;
    W[(size_t)(c % CH_WCOLS) * CH_LDB + d] = __ldcg(a.AB + (size_t)c * CH_LDB + d);
  }
}

// Persistent: every CTA takes groups in order until none is left.  Launched
// cooperatively, so all CTAs are resident and the group a CTA waits for is
// always held by a running CTA.  Warps 0 .. CH_K-1 run the sweeps' tasks,
// warp CH_K writes back and publishes, warp CH_K + 1 fetches.
__global__ void __launch_bounds__(CH_THREADS, 1) chase_kernel(ChaseArgs a) {
  extern __shared__ __align__(16) double W[];
  __shared__ double sv[CH_K][SB], sw[CH_K][SB];
  __shared__ int s_g, s_ok;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int STORER = CH_K, LOADER = CH_K + 1;
  while (true) {
    if (threadIdx.x == 0) {
      s_g = atomicAdd(a.next_group, 1);
      s_ok = 1;
    }
    __syncthreads();
    const int g = s_g;
    if (g >= a.ngroups) return;
    const int s0 = g * CH_K;
    int steps = 0;
    for (int k = 0; k < CH_K && s0 + k <= a.n - 3; ++k)
      steps = max(steps, CH_LAG * k + chase_ntasks(a.n, s0 + k));
    int loaded = s0, lo_prev = s0;
    {
      int lo, hi;
      chase_span(a, g, 0, lo, hi);
      if (warp == LOADER && hi > loaded) {
        bool ok = true;
        if (lane == 0) ok = wait_wm(a, g - 1, hi);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok) window_load_warp(a, W, loaded, hi, lane);
        else if (lane == 0) s_ok = 0;
      }
      loaded = max(loaded, hi);
    }
    __syncthreads();
    if (!s_ok) return;
    for (int step = 0; step < steps; ++step) {
      int lo, hi, lo1, hi1;
      chase_span(a, g, step, lo, hi);
      chase_span(a, g, step + 1, lo1, hi1);
      const int lo_next = min(lo, loaded);
      if (warp < CH_K) {
        const int s = s0 + warp, t = step - CH_LAG * warp;
        if (s <= a.n - 3 && t >= 0 && t < chase_ntasks(a.n, s))
          chase_task(a, W, s, t, lane, sv[warp], sw[warp]);
      } else if (warp == STORER) {
        // columns the previous step finished: no task of this step touches them
        if (lo_next > lo_prev) {
          window_store_warp(a, W, lo_prev, lo_next, lane);
          __threadfence();
          __syncwarp();
          if (lane == 0) publish_wm(a, g, lo_next);
        }
      } else if (hi1 > loaded) {
        // the columns the next step adds: beyond every column in use, and
        // their slots held columns already written back
        bool ok = true;
        if (lane == 0) ok = wait_wm(a, g - 1, hi1);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok) window_load_warp(a, W, loaded, hi1, lane);
        else if (lane == 0) s_ok = 0;
      }
      if (lo_next > lo_prev) lo_prev = lo_next;
      loaded = max(loaded, hi1);
      __syncthreads();
      if (!s_ok) return;
    }
    // the rest of the window; columns this group never loaded are final once
    // the previous group's are
    if (warp == STORER) {
      window_store_warp(a, W, lo_prev, loaded, lane);
      __threadfence();
      __syncwarp();
      if (lane == 0) {
        if (wait_wm(a, g - 1, a.n)) publish_wm(a, g, a.n);
        else s_ok = 0;
      }
    }
    __syncthreads();
    if (!s_ok) return;
  }
}

__global__ void band_tridiag_kernel(const double* __restrict__ AB, int n, double* __restrict__ d,
                                    double* __restrict__ e) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  d[c] = AB[(size_t)c * CH_LDB];
  e[c] = c + 1 < n ? AB[(size_t)c * CH_LDB + 1] : 0.0;
}

// ---- Q2 back-transformation ----------------------------------------------
// Z <- Q2 Z with Q2 the product of all tasks' reflectors in the order they
// were applied.  Block B(g, t) holds task t of the BT_G consecutive sweeps
// g BT_G .. g BT_G + BT_G - 1: sweep j of the block reflects rows
// R0 + j .. R0 + j + SB - 1 (R0 = g BT_G + 1 + t SB), so V of the block is a
// parallelogram of SB + BT_G - 1 rows, and H_j ... H_{j+G-1} = I - V T V^T (forward
// dlarft).  Reflectors of different t within a block range never overlap
// and later sweeps act below earlier ones, so the blocks apply in the order
// g descending, t ascending.  Every CTA owns a strip of BT_CW columns of Z
// and applies all blocks to it; no CTA waits for another.
constexpr int BT_G = SB;
constexpr int BT_CW = 32;
constexpr int BT_THREADS = 256;
__host__ __device__ __forceinline__ int bt_ntasks(int n, int g) { return chase_ntasks(n, g * BT_G); }

// T of block (t, g) = (blockIdx.x, blockIdx.y), column-major BT_G x BT_G.
__global__ void bt_tfactor_kernel(const double* __restrict__ V, const double* __restrict__ tau,
                                  int n, int tmax, double* __restrict__ T) {
  const int t = blockIdx.x, g = blockIdx.y, lane = threadIdx.x;
  if (t >= bt_ntasks(n, g)) return;
  __shared__ double sv[BT_G][SB + 1];
  __shared__ double sT[BT_G][BT_G + 1];
  __shared__ double stau[BT_G], sg[BT_G];
  for (int j = 0; j < BT_G; ++j) {
    const int s = g * BT_G + j;
    const bool ok = s <= n - 3 && t < chase_ntasks(n, s);
    sv[j][lane] = ok ? V[((size_t)t * n + s) * SB + lane] : 0.0;
    if (lane == 0) stau[j] = ok ? tau[(size_t)t * n + s] : 0.0;
  }
  __syncwarp();
  for (int j = 0; j < BT_G; ++j) {
    // G(h, j) = v_h^T v_j over the rows both reach (h < j): rows j .. h + SB - 1
    double gv = 0.0;
    if (lane < j)
      for (int r = j; r < lane + SB; ++r) gv = fma(sv[lane][r - lane], sv[j][r - j], gv);
    sg[lane] = gv;
    __syncwarp();
    double x = 0.0;
    if (lane < j)
      for (int h = lane; h < j; ++h) x = fma(sT[lane][h], sg[h], x);
    sT[lane][j] = lane < j ? -stau[j] * x : (lane == j ? stau[j] : 0.0);
    __syncwarp();
  }
  double* Tb = T + ((size_t)g * tmax + t) * BT_G * BT_G;
  for (int c = 0; c < BT_G; ++c) Tb[(size_t)c * BT_G + lane] = sT[lane][c];
}

__device__ __forceinline__ void dmma(double (&d)[4], double a0, double a1, double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b));
}

// Row strides of the shared tiles (doubles), chosen so that the DMMA operand
// loads of a half-warp (4 x 4 lanes) hit 16 distinct 8-byte banks.
constexpr int BT_SVS = 37;  // sv[j][i]: V(j) element i; (S - 1) = 4 mod 16
constexpr int BT_TS = 36;   // sT[i][h] = T(i, h)
constexpr int BT_YS = 36;   // sY[j][c]
constexpr int BT_ZS = 36;   // sZ[slot][row][c]

constexpr size_t BT_SMEM =
    ((size_t)BT_G * BT_SVS + (size_t)BT_G * BT_TS + 2 * (size_t)BT_G * BT_YS +
     2 * 32 * (size_t)BT_ZS) * sizeof(double);

// One CTA (8 warps) per strip of BT_CW = 32 columns of Z.  For block (g, tb)
// the 64 rows R0 .. R0 + 63 of the strip sit in shared memory as two 32-row
// segments (segment k of the sweep group: rows g G + 1 + 32 k ..); block tb
// uses segments tb and tb + 1, so after it segment tb is final and is
// written back and segment tb + 2 takes its slot.  The next block's V, T and
// new segment are loaded into registers while this block computes.  The three
// products are FP64 DMMA tiles (m16n8k4):
//   Y = V^T Z (32 x 32, K over the parallelogram's 47 rows per 16-row tile),
//   -Y2 = -T Y (T upper triangular), Z += V (-Y2) (64 x 32).
__global__ void __launch_bounds__(BT_THREADS, 2) bt_apply_kernel(
    const double* __restrict__ V, const double* __restrict__ T, int n, int ngroups, int tmax,
    double* __restrict__ Z, long long ldz) {
  extern __shared__ __align__(16) double bsm[];
  double* sv = bsm;                        // [BT_G][BT_SVS]
  double* sT = sv + BT_G * BT_SVS;         // [BT_G][BT_TS]
  double* sY = sT + BT_G * BT_TS;          // [BT_G][BT_YS]
  double* sY2 = sY + BT_G * BT_YS;         // [BT_G][BT_YS], holds -Y2
  double* sZ = sY2 + BT_G * BT_YS;         // [2][32][BT_ZS]
  const int c0 = blockIdx.x * BT_CW;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  // element e = tid + 256 q (q < 4) of a 32 x 32 tile: (row e % 32, column e / 32)
  auto vload = [&](int g, int tb, double (&r)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + BT_THREADS * q, jj = e >> 5, i = e & 31, sw = g * BT_G + jj;
      r[q] = (sw <= n - 3 && tb < chase_ntasks(n, sw)) ? V[((size_t)tb * n + sw) * SB + i] : 0.0;
    }
  };
  auto tload = [&](int g, int tb, double (&r)[4]) {
    const double* Tb = T + ((size_t)g * tmax + tb) * BT_G * BT_G;
#pragma unroll
    for (int q = 0; q < 4; ++q) r[q] = Tb[tid + BT_THREADS * q];
  };
  // rows row0 .. row0 + 31 of the strip (zero beyond n)
  auto zload = [&](int row0, double (&r)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + BT_THREADS * q, rr = e & 31, c = e >> 5;
      const int gr = row0 + rr, gc = c0 + c;
      r[q] = (gr < n && gc < n) ? Z[(size_t)gc * ldz + gr] : 0.0;
    }
  };
  auto zput = [&](int slot, const double (&r)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + BT_THREADS * q;
      sZ[((size_t)slot * 32 + (e & 31)) * BT_ZS + (e >> 5)] = r[q];
    }
  };
  auto zstore = [&](int slot, int row0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + BT_THREADS * q, rr = e & 31, c = e >> 5;
      const int gr = row0 + rr, gc = c0 + c;
      if (gr < n && gc < n) Z[(size_t)gc * ldz + gr] = sZ[((size_t)slot * 32 + rr) * BT_ZS + c];
    }
  };
  auto vput = [&](const double (&r)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + BT_THREADS * q;
      sv[(e >> 5) * BT_SVS + (e & 31)] = r[q];
    }
  };
  auto tput = [&](const double (&r)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + BT_THREADS * q;  // T(i, h) at column-major e = h 32 + i
      sT[(e & 31) * BT_TS + (e >> 5)] = r[q];
    }
  };
  // the first block
  int g = ngroups - 1, tb = 0;
  {
    double rv[4], rt[4], z0[4], z1[4];
    vload(g, tb, rv);
    tload(g, tb, rt);
    zload(g * BT_G + 1, z0);
    zload(g * BT_G + 1 + 32, z1);
    vput(rv);
    tput(rt);
    zput(0, z0);
    zput(1, z1);
  }
  __syncthreads();
  while (g >= 0) {
    const int nt = bt_ntasks(n, g);
    const int R0 = g * BT_G + 1 + tb * SB;
    const bool last = tb + 1 >= nt;
    const int ng = last ? g - 1 : g, ntb = last ? 0 : tb + 1;  // the next block
    // prefetch: the next block's V and T, and the segment it adds (for the
    // next sweep group its first segment, which this group never touches;
    // its second is this group's first and is read after the write-back)
    double pv[4], pt[4], pz[4];
    if (ng >= 0) {
      vload(ng, ntb, pv);
      tload(ng, ntb, pt);
      zload(last ? ng * BT_G + 1 : R0 + 64, pz);
    }
    const int slot0 = tb & 1, slot1 = (tb + 1) & 1;
    auto zrow = [&](int r) { return sZ + ((size_t)((r >> 5) ? slot1 : slot0) * 32 + (r & 31)) * BT_ZS; };
    // Y = V^T Z: warp -> 16 x 8 tile (rows 16 mt of Y, columns 8 nt)
    {
      const int mt = warp & 1, nt8 = warp >> 1, m0 = 16 * mt, n0 = 8 * nt8;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int kb = 0; kb < 48; kb += 4) {
        const int r = m0 + kb + tq;
        const int i0 = r - (m0 + gq), i1 = i0 - 8;
        const double a0 = (i0 >= 0 && i0 < SB) ? sv[(m0 + gq) * BT_SVS + i0] : 0.0;
        const double a1 = (i1 >= 0 && i1 < SB) ? sv[(m0 + gq + 8) * BT_SVS + i1] : 0.0;
        dmma(acc, a0, a1, zrow(r)[n0 + gq]);
      }
      double* y0 = sY + (m0 + gq) * BT_YS + n0 + 2 * tq;
      y0[0] = acc[0];
      y0[1] = acc[1];
      y0[8 * BT_YS] = acc[2];
      y0[8 * BT_YS + 1] = acc[3];
    }
    __syncthreads();
    // -Y2 = -T Y
    {
      const int mt = warp & 1, nt8 = warp >> 1, m0 = 16 * mt, n0 = 8 * nt8;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int kb = 0; kb < 32; kb += 4) {
        if (kb + 4 <= m0) continue;  // T(i, h) = 0 for h < i
        dmma(acc, sT[(m0 + gq) * BT_TS + kb + tq], sT[(m0 + gq + 8) * BT_TS + kb + tq],
             sY[(kb + tq) * BT_YS + n0 + gq]);
      }
      double* y0 = sY2 + (m0 + gq) * BT_YS + n0 + 2 * tq;
      y0[0] = -acc[0];
      y0[1] = -acc[1];
      y0[8 * BT_YS] = -acc[2];
      y0[8 * BT_YS + 1] = -acc[3];
    }
    __syncthreads();
    // Z += V (-Y2): warp -> rows 16 mt, two 8-column tiles
    {
      const int mt = warp & 3, m0 = 16 * mt, n0 = 16 * (warp >> 2);
      double acc[2][4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const double* zr0 = zrow(m0 + gq);
        const double* zr1 = zrow(m0 + gq + 8);
        const int cc = n0 + 8 * h + 2 * tq;
        acc[h][0] = zr0[cc];
        acc[h][1] = zr0[cc + 1];
        acc[h][2] = zr1[cc];
        acc[h][3] = zr1[cc + 1];
      }
      const int jlo = m0 >= SB ? m0 - SB + 1 : 0, jhi = min(BT_G - 1, m0 + 15);
#pragma unroll
      for (int kb = 0; kb < 32; kb += 4) {
        if (kb + 3 < jlo || kb > jhi) continue;
        const int jj = kb + tq;
        const int i0 = m0 + gq - jj, i1 = i0 + 8;
        const double a0 = (i0 >= 0 && i0 < SB) ? sv[jj * BT_SVS + i0] : 0.0;
        const double a1 = (i1 >= 0 && i1 < SB) ? sv[jj * BT_SVS + i1] : 0.0;
#pragma unroll
        for (int h = 0; h < 2; ++h) dmma(acc[h], a0, a1, sY2[jj * BT_YS + n0 + 8 * h + gq]);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        double* zr0 = zrow(m0 + gq);
        double* zr1 = zrow(m0 + gq + 8);
        const int cc = n0 + 8 * h + 2 * tq;
        zr0[cc] = acc[h][0];
        zr0[cc + 1] = acc[h][1];
        zr1[cc] = acc[h][2];
        zr1[cc + 1] = acc[h][3];
      }
    }
    __syncthreads();
    // segment tb is final; the next block's operands take the freed space
    // (each thread writes back and refills the same elements: no barrier)
    zstore(slot0, R0);
    if (last) zstore(slot1, R0 + 32);
    if (ng >= 0) {
      vput(pv);
      tput(pt);
      if (last) {
        // rows ng G + 33 .. ng G + 64 are this group's first segment, written
        // back by this thread (at block 0, or just above when nt = 1)
        double pz2[4];
        zload(ng * BT_G + 1 + 32, pz2);
        zput(0, pz);
        zput(1, pz2);
      } else {
        zput(slot0, pz);
      }
    }
    __syncthreads();
    g = ng;
    tb = ntb;
  }
}

}  // namespace

// X = [V(:, k:k+b) | W(:, 0:b)], Y = [W | V] (eigen_dc.cu)
__global__ void pack_update_kernel(const double* __restrict__ V, long long ldv,
                                   const double* __restrict__ W, long long ldw, int t0, int n,
                                   int b, double* __restrict__ X, double* __restrict__ Y,
                                   long long ldx);

// Sets the panel kernel's attributes (non-portable cluster size; the device's
// shared-memory ceiling, since the attribute is process-wide) and tells
// whether a cluster of cs CTAs with smem bytes each can be placed.
template <bool STAGED>
static bool panel_cluster_fits(imcom_ctx* ctx, int cs, size_t smem, int optin) {
  if (cudaFuncSetAttribute(sb_panel_kernel<STAGED>,
                           cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
      cudaFuncSetAttribute(sb_panel_kernel<STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           optin - 1024) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(sb_threads(STAGED));
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int nc = 0;
  const bool ok = cudaOccupancyMaxActiveClusters(&nc, (void*)sb_panel_kernel<STAGED>, &cfg) ==
                      cudaSuccess && nc >= 1;
  cudaGetLastError();
  (void)ctx;
  return ok;
}

// Cluster size for the panel kernel: 16 CTAs where the device can place them
// (a non-portable size), else 8.  Placement is checked at the largest shared
// memory either variant asks for.
static int panel_cluster(imcom_ctx* ctx, int optin, int* ctas) {
  for (int cs : {16, 8}) {
    if (panel_cluster_fits<true>(ctx, cs, optin - 1024, optin) &&
        panel_cluster_fits<false>(ctx, cs, panel_smem(0, false), optin)) {
      *ctas = cs;
      return 0;
    }
  }
  return set_err(ctx, IMCOM_ERR_CUDA, "the band reduction's panel cluster cannot be placed");
}

// Dense -> band: A (full symmetric, n x n, ld) is overwritten by the band
// matrix (bandwidth SB) below the diagonal and garbage elsewhere; the
// reflectors of panel p go to V (columns p SB ..), their tau to tau and the
// block reflectors' T factors (SB x SB each, column-major) to Tf.  AB
// receives the band in the storage of the second stage (ldb rows).
int sy2sb_gpu(imcom_ctx* ctx, DMat& Aw, DMat& V, double* tau, double* Tf, double* W,
              long long ldw, double* XY, double* AB, int ldb) {
  const int n = (int)Aw.rows;
  const long long ld = Aw.ld;
  IMC_CUDA(cudaMemsetAsync(V.p, 0, V.bytes(), ctx->stream));
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
  int ctas = 16;
  IMC_TRY(panel_cluster(ctx, optin, &ctas));
  double* M2 = Tf + (size_t)((n + SB - 1) / SB) * SB * SB;  // SB x SB scratch after the T factors
  double* Spart = W;  // per-block partials of V^T X1: ceil(N / WY_ROWS) SB^2 <= SB ldw
  for (int k = 0; k + SB < n - 1; k += SB) {
    const int N = n - k - SB;
    const int pc = std::max(1, (N + ctas - 1) / ctas);
    // panels whose slices fit are staged in shared memory, taller ones run in place
    const bool staged = panel_smem(pc, true) <= (size_t)optin - 1024;
    PanelArgs pa{Aw.p, ld, V.p, V.ld, tau, n, k, pc};
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(sb_threads(staged));
    cfg.dynamicSmemBytes = panel_smem(pc, staged);
    cfg.stream = ctx->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (staged)
      IMC_CUDA(cudaLaunchKernelEx(&cfg, sb_panel_kernel<true>, pa));
    else
      IMC_CUDA(cudaLaunchKernelEx(&cfg, sb_panel_kernel<false>, pa));
    IMC_LAUNCH();
    const size_t r0 = (size_t)k + SB;
    const double* Vp = V.p + r0 + (size_t)k * V.ld;  // N x SB
    double* T = Tf + (size_t)(k / SB) * SB * SB;
    double* A22 = Aw.p + r0 + r0 * (size_t)ld;
    // T from the Gram matrix V^T V (block partials, then one CTA)
    const int nbg = (N + WY_ROWS - 1) / WY_ROWS;
    wy_partial_kernel<<<nbg, WY_THREADS, 0, ctx->stream>>>(Vp, V.ld, Vp, V.ld, N, Spart);
    IMC_LAUNCH();
    gram_larft_kernel<<<1, SB * SB, 0, ctx->stream>>>(Spart, nbg, tau + k, T);
    IMC_LAUNCH();
    // X1 = A22 V into the first SB columns of XY, then W and the packed
    // operands X = [V | W], Y = [W | V] of the update A22 -= X Y^T
    double* X1 = XY;
    IMC_TRY(dgemm_nn_skinny32(ctx, N, N, A22, ld, Vp, V.ld, X1, ldw));
    const int nb = (N + WY_ROWS - 1) / WY_ROWS;
    wy_partial_kernel<<<nb, WY_THREADS, 0, ctx->stream>>>(Vp, V.ld, X1, ldw, N, Spart);
    IMC_LAUNCH();
    wy_m2_kernel<<<1, SB * SB, 0, ctx->stream>>>(Spart, nb, T, M2);
    IMC_LAUNCH();
    wy_finish_kernel<<<nb, WY_THREADS, 0, ctx->stream>>>(T, M2, Vp, V.ld, XY, ldw, N);
    IMC_LAUNCH();
    double* X = XY;
    double* Y = XY + (size_t)ldw * 2 * SB;
    // the update on the tiles on and below the diagonal only; the next panel's
    // product A22 V reads the whole trailing matrix, so its upper triangle is
    // then mirrored from the lower
    IMC_TRY(dgemm_lower_nt(ctx, N, 2 * SB, -1.0, X, ldw, Y, ldw, 1.0, A22, ld));
    const int Nn = N - SB;  // the next trailing matrix
    if (k + 2 * SB < n - 1 && Nn > 0) {
      dim3 grd((Nn + 31) / 32, (Nn + 31) / 32);
      mirror_lower_kernel<<<grd, dim3(32, 8), 0, ctx->stream>>>(A22 + SB + (size_t)SB * ld, ld,
                                                                Nn);
      IMC_LAUNCH();
    }
  }
  band_extract_kernel<<<n, 128, 0, ctx->stream>>>(Aw.p, ld, n, AB, ldb);
  IMC_LAUNCH();
  return 0;
}


// ---- two-stage driver -----------------------------------------------------

namespace {

struct TwoStage {
  double* AB;    // band + bulge storage, CH_LDB x n
  double* V2;    // stage-2 reflectors, tmax x n x SB
  double* tau2;  // tmax x n
  double* T2;    // T factors of the Q2 blocks, ng_bt x tmax x BT_G^2
  int* sync;     // [0] group counter, [1] error, [16 ..] watermarks
  double* Tf;    // stage-1 T factors and scratch
  int tmax, ng_chase, ng_bt;
};

inline size_t r256(size_t b) { return (b + 255) / 256 * 256; }

inline void twostage_dims(int n, int& tmax, int& ng_chase, int& ng_bt) {
  tmax = std::max(1, chase_ntasks(n, 0));
  ng_chase = std::max(1, (n - 2 + CH_K - 1) / CH_K);
  ng_bt = std::max(1, (n - 2 + BT_G - 1) / BT_G);
}

TwoStage carve(int n, void* scratch) {
  TwoStage ts;
  twostage_dims(n, ts.tmax, ts.ng_chase, ts.ng_bt);
  char* p = (char*)scratch;
  auto take = [&](size_t bytes) {
    char* r = p;
    p += r256(bytes);
    return r;
  };
  ts.AB = (double*)take((size_t)CH_LDB * n * 8);
  ts.V2 = (double*)take((size_t)ts.tmax * n * SB * 8);
  ts.tau2 = (double*)take((size_t)ts.tmax * n * 8);
  ts.T2 = (double*)take((size_t)ts.ng_bt * ts.tmax * BT_G * BT_G * 8);
  ts.sync = (int*)take((size_t)ts.ng_chase * 4 + 64);
  ts.Tf = (double*)take(((size_t)(n / SB + 1) * SB * SB + 3 * SB * SB) * 8);
  return ts;
}

}  // namespace

size_t twostage_bytes(int n) {
  int tmax, ngc, ngb;
  twostage_dims(n, tmax, ngc, ngb);
  return r256((size_t)CH_LDB * n * 8) + r256((size_t)tmax * n * SB * 8) +
         r256((size_t)tmax * n * 8) + r256((size_t)ngb * tmax * BT_G * BT_G * 8) +
         r256((size_t)ngc * 4 + 64) + r256(((size_t)(n / SB + 1) * SB * SB + 3 * SB * SB) * 8);
}

// Tridiagonal (d, e) of the full symmetric Aw through the band: the stage-1
// reflectors go to Vall (column c, unit at row c + SB) and tau, so the
// one-stage back-transformation applies Q1 unchanged; the stage-2
// reflectors stay in scratch for twostage_backtransform2.
int twostage_tridiag(imcom_ctx* ctx, DMat& Aw, DMat& Vall, double* d, double* e, double* tau,
                     double* W, long long ldw, double* XY, void* scratch, long long spin) {
  const int n = (int)Aw.rows;
  TwoStage ts = carve(n, scratch);
  IMC_CUDA(cudaMemsetAsync(tau, 0, (size_t)n * 8, ctx->stream));
  IMC_TRY(sy2sb_gpu(ctx, Aw, Vall, tau, ts.Tf, W, ldw, XY, ts.AB, CH_LDB));
  IMC_CUDA(cudaMemsetAsync(ts.sync, 0, (size_t)ts.ng_chase * 4 + 64, ctx->stream));
  if (n >= 3) {
    IMC_CUDA(cudaMemsetAsync(ts.V2, 0, (size_t)ts.tmax * n * SB * 8, ctx->stream));
    IMC_CUDA(cudaMemsetAsync(ts.tau2, 0, (size_t)ts.tmax * n * 8, ctx->stream));
    IMC_CUDA(cudaFuncSetAttribute(chase_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)CH_SMEM));
    int per_sm = 0;
    IMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chase_kernel, CH_THREADS,
                                                           CH_SMEM));
    if (per_sm < 1)
      return set_err(ctx, IMCOM_ERR_CUDA, "bulge chasing: the kernel cannot be placed");
    const int grid = std::min(sm_count(ctx) * per_sm, ts.ng_chase);
    ChaseArgs ca{ts.AB, n, ts.ng_chase, ts.V2, ts.tau2, ts.sync + 16, ts.sync, ts.sync + 1,
                 std::min<long long>(spin, 4000000LL)};
    void* args[] = {&ca};
    IMC_CUDA(cudaLaunchCooperativeKernel((void*)chase_kernel, dim3(grid), dim3(CH_THREADS), args,
                                         CH_SMEM, ctx->stream));
    IMC_LAUNCH();
  }
  band_tridiag_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(ts.AB, n, d, e);
  IMC_LAUNCH();
  int h = 0;
  IMC_CUDA(cudaMemcpyAsync(&h, ts.sync + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h) return set_err(ctx, IMCOM_ERR_EIGEN, "bulge chasing: a wait between sweep groups timed out");
  return 0;
}

// Z <- Q2 Z (n x n, ld ldz) with the reflectors twostage_tridiag left in scratch.
int twostage_backtransform2(imcom_ctx* ctx, int n, void* scratch, double* Z, long long ldz) {
  if (n < 3) return 0;
  TwoStage ts = carve(n, scratch);
  bt_tfactor_kernel<<<dim3(ts.tmax, ts.ng_bt), 32, 0, ctx->stream>>>(ts.V2, ts.tau2, n, ts.tmax,
                                                                     ts.T2);
  IMC_LAUNCH();
  IMC_CUDA(cudaFuncSetAttribute(bt_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)BT_SMEM));
  bt_apply_kernel<<<(n + BT_CW - 1) / BT_CW, BT_THREADS, BT_SMEM, ctx->stream>>>(
      ts.V2, ts.T2, n, ts.ng_bt, ts.tmax, Z, ldz);
  IMC_LAUNCH();
  return 0;
}

}  // namespace imcom

using namespace imcom;

// First stage alone, for tests: the band matrix of the resident A (loaded or
// built), SB + 1 diagonals in band storage AB_out[d + c * ldb], d <= SB.
extern "C" int imcom_gpu_band_reduce(imcom_ctx* ctx, double* AB_out, int ldb) {
  if (!ctx) return -1;
  if (!AB_out) return -2;
  if (ldb < SB + 1) return -3;
  if (!ctx->have_A) return set_err(ctx, IMCOM_ERR_STATE, "A has not been built or loaded");
  cudaSetDevice(ctx->device);
  const int n = ctx->n;
  EigWork* ew = eig_work(ctx);
  IMC_TRY(ensure_mat(ctx, ew->Z, n, n));
  IMC_TRY(ensure_mat(ctx, ew->V, n, n));
  IMC_TRY(copy_mat(ctx, ctx->A.p, ctx->A.ld, ew->Z.p, ew->Z.ld, n, n));
  const long long ldw = pad_ld(n);
  const int LDB = 2 * SB;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_tau = take((size_t)n * 8), o_T = take(((size_t)(n / SB + 1) * SB * SB + 3 * SB * SB) * 8);
  const size_t o_W = take((size_t)ldw * SB * 8), o_XY = take((size_t)ldw * 4 * SB * 8);
  const size_t o_AB = take((size_t)LDB * n * 8);
  IMC_TRY(eig_buf(ctx, off + 256));
  char* base = (char*)ew->buf;
  double* AB = (double*)(base + o_AB);
  IMC_TRY(sy2sb_gpu(ctx, ew->Z, ew->V, (double*)(base + o_tau), (double*)(base + o_T),
                    (double*)(base + o_W), ldw, (double*)(base + o_XY), AB, LDB));
  IMC_CUDA(cudaMemcpy2DAsync(AB_out, (size_t)ldb * 8, AB, (size_t)LDB * 8, (size_t)(SB + 1) * 8, n,
                             cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}
