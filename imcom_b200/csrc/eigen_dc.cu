// eigen_dc.cu -- FP64 symmetric eigensolver: blocked Householder
// tridiagonalisation, divide and conquer on the tridiagonal matrix, and
// blocked back-transformation.  Replaces LAPACK DSYEVR in imcom_eigen_A
// (imcom_matrix.f90:617-643); results are returned in ascending order and
// reversed by the caller (imcom_matrix.f90:656-662).
//
// 1. Tridiagonalisation (LAPACK dsytrd/dlatrd, lower).  Panels of NB = 32
//    columns; only the lower triangle of the trailing matrix is read or
//    updated.  Inside a panel every column needs the trailing symmetric
//    matrix-vector product y0 = A22 v and the panel corrections
//    y = y0 - V (W^T v) - W (V^T v).  One persistent cooperative kernel per
//    panel runs the whole panel with two grid-wide barriers per column:
//      phase A: A22 x for the raw column x = A(j+1:n, j) (so the tiles need
//               not wait for the reflector), from 64 x 16 lower-triangle
//               tiles staged through shared memory by cp.async: row sums
//               and column sums per tile, and x^T A22 x (one atomic per CTA);
//      phase B: y0 = scl A22 x + delta A22(:, j+1) for v = scl x +
//               delta e_{j+1}, then w = tau (y - 1/2 tau (y^T v) v) row by
//               row, using v^T y = v^T y0 - 2 (V^T v).(W^T v), the update of
//               the next column, its norm and its dot products with the
//               panel's W and V (the rows already hold them in registers).
//    The trailing update A22 -= V W^T + W V^T runs on the DMMA GEMM as one
//    product with K = 2 NB ([V W] [W V]^T), over the tiles on or below the
//    diagonal (LAPACK dsyr2k 'L').
//    Grid barriers spin with a bound and report a timeout instead of hanging.
// 2. Divide and conquer (LAPACK dstedc / dlaed0-4 structure).  Leaves of at
//    most 32 rows are diagonalised by a cyclic Jacobi sweep in one CTA each.
//    Each merge level runs batched over all nodes: z vector and sort (merge
//    ranks), deflation scan (one thread per node, LAPACK dlaed2 tests and
//    Givens rotations), the secular equation roots (one warp per root; in
//    tau = lambda - d_org the nearest pole is kept exact and the rest
//    linearised, so each step solves a quadratic), the
//    Gu-Eisenstat z-hat (dlaed3) and the eigenvector columns (one warp each),
//    then Q_node = Q_old(:, nondeflated) U as one DMMA GEMM per node.
// 3. Back-transformation (dormtr): Z <- (I - V T V^T) Z over blocks of 256
//    reflectors, three GEMMs per block.  T is built from V^T V: dlarft on
//    each 128-reflector half, joined by T12 = -T1 (V1^T V2) T2.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include <cooperative_groups.h>

#include "common.cuh"
#include "dgemm_tile.cuh"
#include "eigen.cuh"

namespace imcom {

namespace {

constexpr int NB = 32;            // tridiagonalisation panel width
constexpr int TRD_THREADS = 256;  // threads per CTA of the panel kernel
constexpr int TRD_SLOTS = 3;      // tiles staged per warp (two in flight ahead)
constexpr int CW = 16;            // columns per symv tile
constexpr int TR = 64;            // rows per symv tile (two per lane)
constexpr int CPB = TR / CW;      // column chunks per row block along the diagonal
// one staging slot: a CW x TR tile, then the TR rows and CW columns of the
// reflector column it multiplies
constexpr int TRD_SLOT = CW * TR + TR + CW;
constexpr size_t TRD_SMEM = (size_t)(TRD_THREADS / 32) * TRD_SLOTS * TRD_SLOT * sizeof(double);
constexpr int LEAF = 32;          // largest leaf of the divide-and-conquer tree
constexpr int NBB = 128;          // reflectors per back-transformation block
constexpr double EPS = 1.1102230246251565e-16;
constexpr size_t LARFT_SMEM = (size_t)NBB * (NBB + 1) * sizeof(double);

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// 16-byte global -> shared copy; bytes < 16 zero-fill the rest (0: all zero)
__device__ __forceinline__ void cp_async16(double* dst, const double* src, int bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async8(double* dst, const double* src, int bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_2() { asm volatile("cp.async.wait_group 2;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ double ld_cg(const double* p) {
  double v;
  asm volatile("ld.global.cg.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// ---------------------------------------------------------------------------
// Bounded grid barrier (cooperative launch guarantees co-residency).
// ---------------------------------------------------------------------------
struct GridSync {
  unsigned count;  // arrivals so far (monotonic; one barrier = gridDim.x arrivals)
  unsigned pad0;
  int err;
  int pad1;
};

// Arrive with a release add, wait with acquire loads until every CTA of this
// barrier generation has arrived.  The wait gives up after `limit` polls and
// sets the error word instead of spinning forever.  `extra` > 0 (a test of
// that bound) waits for arrivals that never come.
__device__ __forceinline__ bool grid_barrier(GridSync* s, long long limit, int extra = 0) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned nb = gridDim.x;
    unsigned old;
    asm volatile("atom.add.release.gpu.u32 %0, [%1], 1;" : "=r"(old) : "l"(&s->count) : "memory");
    const unsigned target = (old / nb + 1) * nb + (unsigned)extra;
    int ok = 1;
    long long it = 0;
    while (true) {
      unsigned cur;
      asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(cur) : "l"(&s->count) : "memory");
      if ((int)(cur - target) >= 0) break;
      if ((++it & 31) == 0) {
        if (*(volatile int*)&s->err) {
          ok = 0;
          break;
        }
        if (it > limit) {
          atomicExch(&s->err, 1);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// 1. Tridiagonalisation
// ---------------------------------------------------------------------------
struct TrdAcc {
  double SW[NB];  // sum_{r >= j+2} A(r, j) W(r, p) for the column j this parity serves
  double SV[NB];  // sum_{r >= j+2} A(r, j) V(r, p)
  double vty0;    // x^T A22 x of the raw column x = A(j+1:n, j)
  double nrm;     // squared norm of the column below its subdiagonal
};

struct TrdArgs {
  double* A;
  long long lda;
  double* V;  // n x n: column j holds v_j (zero above row j+1, 1 at row j+1)
  long long ldv;
  double* W;  // n x NB panel
  long long ldw;
  double *d, *e, *tau;
  double* ypart;  // [chunk][ldy]: row sums of the tiles of one column chunk
  double* ycol;   // [row block][ldy]: column sums of the tiles of one row block
  long long ldy;
  TrdAcc* acc;  // [2] by column parity
  GridSync* sync;
  int n, k, b;
  long long spin;
  int stall;  // test of the bounded barrier: the first barrier never completes
};

template <bool CACHED>
__global__ void __launch_bounds__(TRD_THREADS, 1) trd_panel_kernel(TrdArgs a) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  constexpr int WPB = TRD_THREADS / 32;
  constexpr int HP = (NB + WPB - 1) / WPB;  // panel columns per warp in phase B
  const long long gw = (long long)blockIdx.x * WPB + wib;
  const long long GW = (long long)gridDim.x * WPB;
  const int n = a.n, k = a.k;
  double* A = a.A;
  const long long lda = a.lda, ldv = a.ldv, ldw = a.ldw;
  __shared__ double s_pq[2 * NB];            // p = W^T v, q = V^T v of the current column
  __shared__ double s_rowV[NB], s_rowW[NB];  // row j+1 of V and W
  __shared__ double s_alpha2;                  // -1/2 tau^2 v^T y of the current column
  __shared__ double sm_y[WPB][32], sm_c[WPB][32], sm_u[WPB][32];
  extern __shared__ __align__(16) double trd_tiles[];  // [warp][slot][TRD_SLOT]
  double* wbuf = trd_tiles + (size_t)wib * TRD_SLOTS * TRD_SLOT;
  if (*(volatile int*)&a.sync->err) return;  // an earlier panel failed

  // Column k: d(k) and the norm of A(k+2:n, k) (one atomic per CTA).
  {
    double part = 0.0;
    for (long long r0 = k + 2 + gw * 32; r0 < n; r0 += GW * 32) {
      long long r = r0 + lane;
      double v = (r < n) ? A[r + k * lda] : 0.0;
      part += v * v;
    }
    part = warp_sum(part);
    if (lane == 0) sm_y[wib][0] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < WPB; ++w) s += sm_y[w][0];
      if (s != 0.0) atomicAdd(&a.acc[0].nrm, s);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.d[k] = A[k + k * lda];
  if (!grid_barrier(a.sync, a.spin, a.stall)) return;

  for (int i = 0; i < a.b; ++i) {
    const int j = k + i;
    const int par = i & 1;
    TrdAcc* cur = a.acc + par;
    TrdAcc* nxt = a.acc + (par ^ 1);
    // The tiles cover the trailing matrix of column jg: this column, or for
    // the cached variant the panel's first column k, so that every warp
    // keeps the same tiles (in its shared-memory slots) through the panel
    // and only x changes; x is zero left of and above column j+1 there, and
    // the chunks wholly left of it (ch < chf) are skipped.
    const long long jg = CACHED ? k : j;
    const long long chf = (j - jg) / CW;
    // rows handled in pairs from an even base row so the loads are 16-byte
    const long long rbase = (jg + 1) & ~1LL;
    const long long R = n - (jg + 1);
    const long long RB = (n - rbase + TR - 1) / TR, NC = (R + CW - 1) / CW;
    // Tiles on or below the diagonal: row block rb (TR rows from rbase +
    // TR rb) with column chunks ch < min(NC, CPB (rb + 1)), counted row block
    // by row block; rb < rbc has CPB (rb + 1) chunks, the rest NC.
    const long long rbc = min(RB, max(0LL, (NC - 1) / CPB));
    const long long tri = (long long)CPB * rbc * (rbc + 1) / 2;
    const long long ntiles = tri + (RB - rbc) * NC;

    // tiles are staged through a TRD_SLOTS-slot shared-memory buffer per warp
    // by cp.async (zero-filled outside the triangle and below row n), together
    // with the segments of column j they multiply, so the next two tiles are
    // in flight while this one is summed
    const double* colj = A + (long long)j * lda;
    // tile counts stay far below 2^31 (n^2 / 2048), so 32-bit arithmetic; the
    // float square root is only a first guess that the loops correct
    auto decode = [&](int tile, int& rb, int& ch) {
      if (tile < (int)tri) {
        // largest rb with CPB rb (rb + 1) / 2 <= tile
        int q = (int)((sqrtf(1.0f + 8.0f * (float)tile / CPB) - 1.0f) * 0.5f);
        while (CPB * (q + 1) * (q + 2) / 2 <= tile) ++q;
        while (q > 0 && CPB * q * (q + 1) / 2 > tile) --q;
        rb = q;
        ch = tile - CPB * q * (q + 1) / 2;
      } else {
        const unsigned t2 = (unsigned)(tile - (int)tri), nc = (unsigned)NC;
        const unsigned qq = t2 / nc;
        rb = (int)rbc + (int)qq;
        ch = (int)(t2 - qq * nc);
      }
    };
    // x's segments for tile (rb, ch): rows r, r + 1 and columns c0 ..
    auto issue_x = [&](int rb, int ch, int slot) {
      const long long r = rbase + (long long)rb * TR + 2 * lane;
      const long long c0 = jg + 1 + (long long)ch * CW, c1 = min((long long)n, c0 + CW);
      double* dst = wbuf + slot * TRD_SLOT + 2 * lane;
      const bool okr = r < n;
      cp_async16(dst + CW * TR, okr ? colj + r : A, okr ? (r + 1 < n ? 16 : 8) : 0);
      if (lane < CW) {
        const bool okc = c0 + lane < c1;
        cp_async8(wbuf + slot * TRD_SLOT + CW * TR + TR + lane, okc ? colj + c0 + lane : A,
                  okc ? 8 : 0);
      }
    };
    auto issue = [&](int rb, int ch, int slot) {
      const long long r = rbase + (long long)rb * TR + 2 * lane;
      const long long c0 = jg + 1 + (long long)ch * CW, c1 = min((long long)n, c0 + CW);
      double* dst = wbuf + slot * TRD_SLOT + 2 * lane;
#pragma unroll
      for (int u = 0; u < CW; ++u) {
        const long long c = c0 + u;
        // a row of the pair on or below the diagonal; the second row only
        // if it exists
        const bool ok = c < c1 && r + 1 >= c && r < n;
        cp_async16(dst + u * TR, ok ? A + r + c * lda : A, ok ? (r + 1 < n ? 16 : 8) : 0);
      }
      const bool okr = r < n;
      cp_async16(dst + CW * TR, okr ? colj + r : A, okr ? (r + 1 < n ? 16 : 8) : 0);
      if (lane < CW) {
        const bool okc = c0 + lane < c1;
        cp_async8(wbuf + slot * TRD_SLOT + CW * TR + TR + lane, okc ? colj + c0 + lane : A,
                  okc ? 8 : 0);
      }
    };
    // Phase A forms A22 x for the raw column x = A(j+1:n, j); the reflector
    // v = scl x + delta e_{j+1} (delta = 1 - scl x(j+1)) only enters in
    // phase B, y0 = A22 v = scl (A22 x) + delta A22(:, j+1), so the tiles do
    // not wait for the reflector.  Its loads are issued now, used after the
    // tile loop.
    // decoded indices of this warp's next two tiles
    int rb_n = 0, ch_n = 0, rb_m = 0, ch_m = 0;
    if constexpr (CACHED) {
      // the warp's tiles (at most TRD_SLOTS) sit in slots 0, 1, .. for the
      // whole panel: the first column loads them, every column its x
      int q = 0;
      for (long long tile = gw; tile < ntiles; tile += GW, ++q) {
        int rb, ch;
        decode((int)tile, rb, ch);
        if (i == 0) issue(rb, ch, q);
        else issue_x(rb, ch, q);
      }
      cp_commit();
    } else {
      if (gw < ntiles) {
        decode((int)gw, rb_n, ch_n);
        issue(rb_n, ch_n, 0);
      }
      cp_commit();
      if (gw + GW < ntiles) {
        decode((int)(gw + GW), rb_m, ch_m);
        issue(rb_m, ch_m, 1);
      }
      cp_commit();
    }
    const double alpha = ld_cg(A + (j + 1) + (long long)j * lda);
    const double xn2 = ld_cg(&cur->nrm);
    // A(j+1, j+1) before this column's phase B rewrites column j+1
    const double a11 = (wib == 0) ? ld_cg(A + (j + 1) + (long long)(j + 1) * lda) : 0.0;
    if (blockIdx.x == 0 && threadIdx.x < 2 * NB + 2) {
      // clear the other parity's accumulators (last read one phase ago)
      if (threadIdx.x < NB) nxt->SW[threadIdx.x] = 0.0;
      else if (threadIdx.x < 2 * NB) nxt->SV[threadIdx.x - NB] = 0.0;
      else if (threadIdx.x == 2 * NB) nxt->vty0 = 0.0;
      else nxt->nrm = 0.0;
    }
    // Row j+1 of V and W, and p = W^T v = W(j+1, :) + scl * SW, q = V^T v
    // likewise (sums from the previous column's phase B); loaded now, kept
    // in shared memory for phase B after the tile loop
    double wr1 = 0.0, vr1 = 0.0, sw1 = 0.0, sv1 = 0.0;
    if (wib == 0 && lane < i) {
      wr1 = ld_cg(a.W + (j + 1) + lane * ldw);
      vr1 = ld_cg(a.V + (j + 1) + (k + lane) * ldv);
      sw1 = ld_cg(&cur->SW[lane]);
      sv1 = ld_cg(&cur->SV[lane]);
    }
    // ---- phase A: A22 x from the lower triangle (LAPACK dsymv 'L').
    // Tile (rb, ch) reads A(r, c) for r >= c once and gives the row sums
    // sum_c A(r, c) x(c) (to ypart[ch]) and the column sums
    // sum_{r > c} A(r, c) x(r) (to ycol[rb]); (A22 x)(r) is the sum of both
    // kinds.  x^T A22 x is summed per warp, then per CTA, and added with one
    // atomic per CTA. ----
    double vty_part = 0.0;
    // Tile (rb, ch) in `slot`: row sums to ypart[ch], column sums to
    // ycol[rb], its share of x^T A22 x to vty_part.
    auto sum_tile = [&](int rb, int ch, int slot) {
      const long long r = rbase + (long long)rb * TR + 2 * lane;
      const long long c0 = jg + 1 + (long long)ch * CW, c1 = min((long long)n, c0 + CW);
      const double* sl = wbuf + slot * TRD_SLOT;
      const double2 vraw = reinterpret_cast<const double2*>(sl + CW * TR)[lane];
      // raw column-j values at rows r, r + 1 and at columns c0 .. c0 + CW - 1
      // (zero-filled past row n); rows at or above j lie above x (only row j
      // when rbase = j; the cached tiles' columns at or left of j are zeroed
      // before the tile is summed)
      const double* vcol = sl + CW * TR + TR;
      const double v0 = (r <= j) ? 0.0 : vraw.x, v1 = (r + 1 <= j) ? 0.0 : vraw.y;
      const double2* av = reinterpret_cast<const double2*>(sl) + lane;
      const int dr = (int)(r - c0);  // this lane's first row relative to column c0
      double acc0 = 0.0, acc1 = 0.0, vtz = 0.0;
      // two halves of CW / 2 columns: row sums, then the column sums of the
      // half transpose-reduced over the warp (lane L ends with the sum for
      // column c0 + H + (L >> 2)), so only CW / 2 partials are live at once.
      // Tiles crossing the diagonal mask A(r, c) with r < c from the row sums
      // and r <= c from the column sums; the others need no mask.
      auto tile_sums = [&](auto masked) {
#pragma unroll
        for (int H = 0; H < CW; H += CW / 2) {
          double z[CW / 2];
#pragma unroll
          for (int u = 0; u < CW / 2; ++u) {
            const int cu = H + u;
            const double2 e2 = av[cu * (TR / 2)];
            const double vc = vcol[cu];
            double ax = e2.x, zx = e2.x, zy = e2.y;
            if (decltype(masked)::value) {
              ax = (dr >= cu) ? e2.x : 0.0;
              zx = (dr > cu) ? e2.x : 0.0;
              zy = (dr + 1 > cu) ? e2.y : 0.0;
            }
            acc0 = fma(ax, vc, acc0);
            acc1 = fma(e2.y, vc, acc1);
            z[u] = fma(zy, v1, zx * v0);
          }
#pragma unroll
          for (int h = CW / 4, m = 16; h >= 1; h >>= 1, m >>= 1) {
            const bool hi = (lane & m) != 0;
#pragma unroll
            for (int q = 0; q < h; ++q) {
              const double send = hi ? z[q] : z[q + h];
              const double keep = hi ? z[q + h] : z[q];
              z[q] = keep + __shfl_xor_sync(0xffffffffu, send, m);
            }
          }
          double zc = z[0] + __shfl_xor_sync(0xffffffffu, z[0], 2);
          zc += __shfl_xor_sync(0xffffffffu, zc, 1);
          const long long cz = c0 + H + (lane >> 2);
          if (!(lane & 3) && cz < c1) {
            a.ycol[(long long)rb * a.ldy + cz] = zc;
            vtz += vcol[H + (lane >> 2)] * zc;
          }
        }
      };
      if (rbase + (long long)rb * TR <= c0 + CW - 1) tile_sums(std::true_type{});
      else tile_sums(std::false_type{});
      if (r >= j + 1 && r < n) a.ypart[(long long)ch * a.ldy + r] = acc0;
      if (r + 1 >= j + 1 && r + 1 < n) a.ypart[(long long)ch * a.ldy + r + 1] = acc1;
      vty_part += v0 * acc0 + v1 * acc1 + vtz;
    };
    if constexpr (CACHED) {
      cp_wait_0();
      __syncwarp();
      int q = 0;
      for (long long tile = gw; tile < ntiles; tile += GW, ++q) {
        int rb, ch;
        decode((int)tile, rb, ch);
        if (ch < chf) continue;  // every column left of j+1: x is zero
        const long long c0 = jg + 1 + (long long)ch * CW;
        double* vc = wbuf + q * TRD_SLOT + CW * TR + TR;
        if (lane < CW && c0 + lane <= j) vc[lane] = 0.0;
        __syncwarp();
        sum_tile(rb, ch, q);
      }
    } else {
      int slot = 0;
      for (long long tile = gw; tile < ntiles; tile += GW, slot = (slot + 1) % TRD_SLOTS) {
        const int rb = rb_n, ch = ch_n;
        rb_n = rb_m;
        ch_n = ch_m;
        if (tile + 2 * GW < ntiles) {
          decode((int)(tile + 2 * GW), rb_m, ch_m);
          issue(rb_m, ch_m, (slot + 2) % TRD_SLOTS);
        }
        cp_commit();
        cp_wait_2();
        sum_tile(rb, ch, slot);
      }
    }
    cp_wait_0();
    // Householder reflector of x = A(j+1:n, j) (LAPACK dlarfg)
    double beta, t, scl;
    if (xn2 == 0.0) {
      t = 0.0;
      beta = alpha;
      scl = 0.0;
    } else {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      t = (beta - alpha) / beta;
      scl = 1.0 / (alpha - beta);
    }
    const double delta = 1.0 - scl * alpha;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.e[j] = beta;
      a.tau[j] = t;
    }
    if (wib == 0 && lane < i) {
      s_rowW[lane] = wr1;
      s_rowV[lane] = vr1;
      s_pq[lane] = wr1 + scl * sw1;
      s_pq[NB + lane] = vr1 + scl * sv1;
    }
    vty_part = warp_sum(vty_part);
    if (lane == 0) sm_u[wib][0] = vty_part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < WPB; ++w) s += sm_u[w][0];
      if (s != 0.0) atomicAdd(&cur->vty0, s);
    }
    if (!grid_barrier(a.sync, a.spin)) return;

    // ---- phase B: w, the next column, its norm and dot products ----
    const bool next = (i + 1 < a.b);
    bool have_w1 = false;
    // one 32-row block per CTA at a time; the warps split the chunk partials
    // and the panel columns, then reduce through shared memory
    // warp 0: this lane's share of y0(j+1), loaded alongside the first row
    // block's partial sums
    double y1 = 0.0;
    if (wib == 0) {
      if (lane >= chf && lane < min(NC, (long long)CPB))
        y1 = __ldcg(a.ypart + lane * a.ldy + (j + 1));
      for (long long q = lane; q < RB; q += 32) y1 += __ldcg(a.ycol + q * a.ldy + (j + 1));
    }
    for (long long rb = blockIdx.x; j + 1 + rb * 32 < n; rb += gridDim.x) {
      const long long r = j + 1 + rb * 32 + lane;
      const bool valid = r < n;
      // issue every load of the row block first
      double ys = 0.0, vp[HP] = {}, wp[HP] = {};
      double vr = 0.0, aold = 0.0;
      const double vty0 = __ldcg(&cur->vty0);
      if (valid) {
        // row sums of the chunks its row block covers, column sums of the
        // row blocks below its chunk
        const long long ncr = min(NC, (long long)CPB * ((r - rbase) / TR + 1));
        const long long rb0 = (r - (jg + 1)) / CW / CPB;
#pragma unroll 4
        for (long long ch = chf + wib; ch < ncr; ch += WPB) ys += __ldcg(a.ypart + ch * a.ldy + r);
#pragma unroll 4
        for (long long q = rb0 + wib; q < RB; q += WPB) ys += __ldcg(a.ycol + q * a.ldy + r);
#pragma unroll
        for (int h = 0; h < HP; ++h) {
          const int p = wib + WPB * h;
          if (p < i) {
            vp[h] = __ldcg(a.V + r + (k + p) * ldv);
            wp[h] = __ldcg(a.W + r + p * ldw);
          }
        }
        vr = (r == j + 1) ? 1.0 : __ldcg(colj + r) * scl;
        aold = __ldcg(A + r + (long long)(j + 1) * lda);
      }
      if (!have_w1 && wib == 0) {
        // v^T y0 = scl^2 x^T A22 x + 2 scl delta (A22 x)(j+1) + delta^2 A(j+1, j+1),
        // alpha2 = -1/2 tau^2 v^T y with v^T y = v^T y0 - 2 (V^T v).(W^T v), and
        // w(j+1) (the new entry of row j+1 of W)
        const double s1 = warp_sum(y1);
        double qp = 0.0;
        for (int p = 0; p < i; ++p) qp += s_pq[NB + p] * s_pq[p];
        const double vty = scl * scl * vty0 + 2.0 * scl * delta * s1 + delta * delta * a11;
        const double al2 = -0.5 * t * t * (vty - 2.0 * qp);
        double corr = (lane < i) ? s_rowV[lane] * s_pq[lane] + s_rowW[lane] * s_pq[NB + lane] : 0.0;
        corr = warp_sum(corr);
        if (lane == 0) {
          s_alpha2 = al2;
          if (next) {
            s_rowW[i] = t * ((scl * s1 + delta * a11) - corr) + al2;
            s_rowV[i] = 1.0;
          }
        }
      }
      have_w1 = true;
      double cs = 0.0, us = 0.0;
#pragma unroll
      for (int h = 0; h < HP; ++h) {
        const int p = wib + WPB * h;
        if (p < i) {
          cs += vp[h] * s_pq[p] + wp[h] * s_pq[NB + p];
          us += vp[h] * s_rowW[p] + wp[h] * s_rowV[p];
        }
      }
      sm_y[wib][lane] = ys;
      sm_c[wib][lane] = cs;
      sm_u[wib][lane] = us;
      __syncthreads();
      double y0 = 0.0, corr = 0.0, upd = 0.0;
#pragma unroll
      for (int w = 0; w < WPB; ++w) {
        y0 += sm_y[w][lane];
        corr += sm_c[w][lane];
        upd += sm_u[w][lane];
      }
      y0 = scl * y0 + delta * aold;  // A22 v from A22 x
      const double wr = t * (y0 - corr) + s_alpha2 * vr;
      if (valid && wib == 0) {
        a.V[r + (long long)j * ldv] = vr;
        a.W[r + i * ldw] = wr;
      }
      if (next) {
        double anew = 0.0;
        if (valid) {
          upd += vr * s_rowW[i] + wr * s_rowV[i];
          anew = aold - upd;
          if (wib == 0) {
            A[r + (long long)(j + 1) * lda] = anew;
            if (r == j + 1) a.d[j + 1] = anew;
          }
        }
        // column j+1's dot products with W, V over rows >= j+3 and its norm
        const double am = (valid && r >= j + 3) ? anew : 0.0;
#pragma unroll
        for (int h = 0; h < HP; ++h) {
          const int p = wib + WPB * h;
          if (p <= i) {
            const double wv = (p == i) ? wr : wp[h];
            const double vv = (p == i) ? vr : vp[h];
            const double sw = warp_sum(am * wv), sv = warp_sum(am * vv);
            if (lane == 0) {
              atomicAdd(&nxt->SW[p], sw);
              atomicAdd(&nxt->SV[p], sv);
            }
          }
        }
        if (wib == 0) {
          const double nr = warp_sum(am * am);
          if (lane == 0) atomicAdd(&nxt->nrm, nr);
        }
      }
      __syncthreads();
    }
    if (!grid_barrier(a.sync, a.spin)) return;
  }

}

// ---------------------------------------------------------------------------
// 1b. The last columns of the tridiagonalisation in one thread-block cluster.
//
// Once the trailing matrix is small, every column of the panel kernel is a
// chain of dependent L2 round trips and two grid barriers (~9 us whatever
// the size).  From trailing size S <= tail_max the rest of the matrix is
// factorised by one cluster of up to 16 CTAs holding it in distributed
// shared memory: full symmetric rows, CTA q owning rows [q rpc, (q+1) rpc).
// Unblocked LAPACK dsytd2 'L', per column j:
//   the owner of row j applies the previous column's update to row j, forms
//   the reflector of x = A(j+1:S, j) (= its row j) and stores v and tau into
//   every CTA's shared memory;                            cluster barrier 1
//   every CTA applies the previous column's update to its other rows and,
//   in the same pass, forms p = tau A22 v on them; it stores p and its part
//   of p^T v into every CTA;                              cluster barrier 2
//   w = p - 1/2 tau (p^T v) v is formed where the next pass needs it.
// Values move by remote stores before a barrier, never by remote loads after
// it, so no step waits on a distributed-shared-memory round trip; one pass
// over the rows per column both updates them and multiplies them by v.
// The reflectors go to V (column j: 1 at row j+1, v below), d, e and tau to
// global memory; the hardware cluster barrier needs no poll limit.
// ---------------------------------------------------------------------------
constexpr int TAIL_THREADS = 512;
constexpr int TAIL_MAX_CTAS = 16;
constexpr int TAIL_RPW = 4;  // rows per warp: rpc <= TAIL_RPW * (TAIL_THREADS / 32)

struct TailArgs {
  const double* A;  // lower triangle valid for rows and columns k0 .. n-1
  long long lda;
  double* V;
  long long ldv;
  double *d, *e, *tau;
  int n, k0, rpc;  // rows per CTA
};

__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  return t;
}

__global__ void __launch_bounds__(TAIL_THREADS, 1) trd_tail_kernel(TailArgs a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int q = (int)cl.block_rank(), nct = (int)cl.num_blocks();
  const int S = a.n - a.k0, rpc = a.rpc, k0 = a.k0;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NW = TAIL_THREADS / 32;
  extern __shared__ __align__(16) double tsm[];
  // Buffers written by other CTAs alternate with the column's parity: the
  // owner of column j+1 may push v while a CTA still updates with column j's.
  double* Ar = tsm;                     // [rpc][S] this CTA's rows
  double* vb = Ar + (size_t)rpc * S;    // [2][S] v of the column (pushed by its owner)
  double* pb = vb + 2 * (size_t)S;      // [2][S] p of the column (pushed by each row's owner)
  double* tb = pb + 2 * (size_t)S;      // [2] tau of the column
  double* pvb = tb + 2;                 // [2][TAIL_MAX_CTAS] each CTA's part of p^T v
  __shared__ double red[TAIL_THREADS / 32];
  const int r0 = q * rpc;
  const int nrow = max(0, min(rpc, S - r0));

  // rows r0 .. r0+nrow-1: entries on and right of the diagonal from the
  // lower triangle's columns (coalesced), then the entries left of it from
  // the owners of those columns' rows
  for (int idx = tid; idx < nrow * S; idx += TAIL_THREADS) {
    const int i = idx / S, c = idx - i * S;
    if (c >= r0 + i) Ar[idx] = a.A[(long long)(k0 + c) + (long long)(k0 + r0 + i) * a.lda];
  }
  cl.sync();
  for (int idx = tid; idx < nrow * S; idx += TAIL_THREADS) {
    const int i = idx / S, c = idx - i * S;
    if (c < r0 + i) {
      const int o = c / rpc;
      const double* rem = cl.map_shared_rank(Ar, o);
      Ar[idx] = rem[(size_t)(c - o * rpc) * S + (r0 + i)];
    }
  }
  cl.sync();

  // Column j's update A22 -= v w^T + w v^T is applied lazily: the owner of
  // row j+1 applies it to that row first (the next reflector needs it), the
  // other rows receive it in the same pass that forms their part of the next
  // column's p = tau A22 v.  w = p + a2 v comes from the parity buffers.
  double a2 = 0.0;  // -1/2 tau (p^T v) of the pending (previous) column
  for (int jl = 0; jl < S - 1; ++jl) {
    const int j = k0 + jl, par = jl & 1;
    double* v = vb + (size_t)par * S;
    const double* vq = vb + (size_t)(par ^ 1) * S;  // pending column's v
    const double* pq = pb + (size_t)(par ^ 1) * S;  // pending column's p
    const int o = jl / rpc;
    if (q == o) {
      // row j: the pending update, then the Householder reflector of
      // x = A(j+1:n, j) (LAPACK dlarfg)
      double* row = Ar + (size_t)(jl - r0) * S;
      double part = 0.0;
      if (jl > 0) {
        const double vr = vq[jl], wr = pq[jl] + a2 * vr;
        for (int c = jl + tid; c < S; c += TAIL_THREADS) {
          const double vc = vq[c];
          const double nv = row[c] - (vr * (pq[c] + a2 * vc) + wr * vc);
          row[c] = nv;
          if (c >= jl + 2) part += nv * nv;
        }
      } else {
        for (int c = 2 + tid; c < S; c += TAIL_THREADS) part += row[c] * row[c];
      }
      const double xn2 = block_sum(part, red);  // also orders the row's new values
      const double alpha = row[jl + 1];
      double beta, t, scl;
      if (xn2 == 0.0) {
        t = 0.0;
        beta = alpha;
        scl = 0.0;
      } else {
        beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        t = (beta - alpha) / beta;
        scl = 1.0 / (alpha - beta);
      }
      // push v and tau into every CTA (stores complete before the barrier)
      for (int c = jl + 1 + tid; c < S; c += TAIL_THREADS) {
        const double vc = (c == jl + 1) ? 1.0 : row[c] * scl;
        for (int r = 0; r < nct; ++r) cl.map_shared_rank(v, r)[c] = vc;
        a.V[(long long)(k0 + c) + (long long)j * a.ldv] = vc;
      }
      if (tid < nct) cl.map_shared_rank(tb, tid)[par] = t;
      if (tid == 0) {
        a.d[j] = row[jl];
        a.e[j] = beta;
        a.tau[j] = t;
      }
    }
    cl.sync();
    const double t = tb[par];
    // this CTA's rows below row j: the pending update (columns >= j) and
    // p = tau A22 v (columns > j) in one pass; a warp takes rows wid,
    // wid + NW, ... together with one independent chain per row
    double pv = 0.0;
    {
      double* rowp[TAIL_RPW];
      bool act[TAIL_RPW];
      double acc[TAIL_RPW], vr[TAIL_RPW], wr[TAIL_RPW];
#pragma unroll
      for (int h = 0; h < TAIL_RPW; ++h) {
        const int i = wid + NW * h;
        act[h] = i < nrow && r0 + i > jl;
        rowp[h] = Ar + (size_t)min(i, rpc - 1) * S;
        acc[h] = 0.0;
        vr[h] = (act[h] && jl > 0) ? vq[r0 + i] : 0.0;
        wr[h] = (act[h] && jl > 0) ? pq[r0 + i] + a2 * vr[h] : 0.0;
      }
      for (int c = jl + lane; c < S; c += 32) {
        const double vc = vq[c], wc = pq[c] + a2 * vc;  // zero terms when jl = 0
        const double vn = (c > jl) ? v[c] : 0.0;
#pragma unroll
        for (int h = 0; h < TAIL_RPW; ++h) {
          if (!act[h]) continue;
          double nv = rowp[h][c];
          if (jl > 0) {
            nv -= vr[h] * wc + wr[h] * vc;
            rowp[h][c] = nv;
          }
          acc[h] = fma(nv, vn, acc[h]);
        }
      }
#pragma unroll
      for (int h = 0; h < TAIL_RPW; ++h) {
        if (!act[h]) continue;
        const int rr = r0 + wid + NW * h;
        const double ph = t * warp_sum(acc[h]);  // every lane holds the sum
        if (lane < nct) cl.map_shared_rank(pb + (size_t)par * S, lane)[rr] = ph;
        if (lane == 0) pv += ph * v[rr];
      }
    }
    pv = block_sum(pv, red);
    if (tid < nct) cl.map_shared_rank(pvb, tid)[par * TAIL_MAX_CTAS + q] = pv;
    cl.sync();
    double ptv = 0.0;
    for (int r = 0; r < nct; ++r) ptv += pvb[par * TAIL_MAX_CTAS + r];
    a2 = -0.5 * t * ptv;
  }
  // the last diagonal entry receives the last column's update
  if (S >= 2 && q == (S - 1) / rpc && tid == 0) {
    const int par = (S - 2) & 1;
    const double* vl = vb + (size_t)par * S;
    const double* pl = pb + (size_t)par * S;
    const double vr = vl[S - 1], wr = pl[S - 1] + a2 * vr;
    a.d[k0 + S - 1] = Ar[(size_t)(S - 1 - r0) * S + (S - 1)] - (vr * wr + wr * vr);
  } else if (S == 1 && q == 0 && tid == 0) {
    a.d[k0] = Ar[0];
  }
}

// Shared memory of the cluster tail for trailing size S with `ctas` CTAs.
inline size_t tail_smem(int S, int ctas) {
  const int rpc = (S + ctas - 1) / ctas;
  return ((size_t)rpc * S + 4 * (size_t)S + 2 + 2 * TAIL_MAX_CTAS) * sizeof(double);
}

__global__ void set_last_diag_kernel(const double* A, long long lda, int n, double* d) {
  d[n - 1] = A[(n - 1) + (long long)(n - 1) * lda];
}

// ---------------------------------------------------------------------------
// 2. Divide and conquer
// ---------------------------------------------------------------------------
struct Node {
  int s, n1, nm;  // first row, left child size, node size
};

// Tearing: d(s-1) -= |e(s-1)|, d(s) -= |e(s-1)| at every split point.
__global__ void tear_kernel(double* dt, const double* e, const int* splits, int nsplit) {
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (int q = 0; q < nsplit; ++q) {
      int s = splits[q];
      double b = fabs(e[s - 1]);
      dt[s - 1] -= b;
      dt[s] -= b;
    }
}

// Cyclic Jacobi on one leaf (tridiagonal block), sorted ascending output.
__global__ void __launch_bounds__(256) leaf_jacobi_kernel(const Node* nodes, const double* dt,
                                                          const double* e, double* w, double* Z,
                                                          long long ldz, int max_sweeps,
                                                          int* err) {
  const Node nd = nodes[blockIdx.x];
  const int m = nd.nm, s0 = nd.s;
  __shared__ double Am[LEAF][LEAF + 1];
  __shared__ double Zm[LEAF][LEAF + 1];
  __shared__ double cs[LEAF / 2][2];
  __shared__ int pr[LEAF / 2][2];
  __shared__ int s_done;
  __shared__ double s_val[LEAF];
  __shared__ int s_idx[LEAF];
  const int tid = threadIdx.x;
  for (int q = tid; q < LEAF * LEAF; q += blockDim.x) {
    int r = q % LEAF, c = q / LEAF;
    double v = 0.0;
    if (r < m && c < m) {
      if (r == c) v = dt[s0 + r];
      else if (r == c + 1) v = e[s0 + c];
      else if (c == r + 1) v = e[s0 + r];
    }
    Am[r][c] = v;
    Zm[r][c] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int mp = (m + 1) & ~1;  // even number of players (a dummy when m is odd)
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    // convergence: off-diagonal mass below eps^2 of the total
    if (tid == 0) {
      double off = 0.0, tot = 0.0;
      for (int r = 0; r < m; ++r)
        for (int c = 0; c < m; ++c) {
          double v = Am[r][c] * Am[r][c];
          tot += v;
          if (r != c) off += v;
        }
      s_done = (off <= 64.0 * EPS * EPS * tot) ? 1 : 0;
    }
    __syncthreads();
    if (s_done) break;
    for (int rnd = 0; rnd < mp - 1; ++rnd) {
      if (tid < mp / 2) {
        auto idx = [&](int x) { return x == 0 ? 0 : 1 + (x - 1 + rnd) % (mp - 1); };
        int p = idx(tid), q = idx(mp - 1 - tid);
        if (p > q) { int tt = p; p = q; q = tt; }
        double c = 1.0, sn = 0.0;
        if (q < m) {
          double apq = Am[p][q];
          if (apq != 0.0) {
            double theta = (Am[q][q] - Am[p][p]) / (2.0 * apq);
            double tt = copysign(1.0, theta) / (fabs(theta) + sqrt(1.0 + theta * theta));
            c = 1.0 / sqrt(1.0 + tt * tt);
            sn = tt * c;
          }
        }
        pr[tid][0] = p;
        pr[tid][1] = q;
        cs[tid][0] = c;
        cs[tid][1] = sn;
      }
      __syncthreads();
      // columns: A <- A J, Z <- Z J
      for (int item = tid; item < (mp / 2) * LEAF; item += blockDim.x) {
        int pi = item / LEAF, r = item % LEAF;
        int p = pr[pi][0], q = pr[pi][1];
        if (q >= m || r >= m) continue;
        double c = cs[pi][0], sn = cs[pi][1];
        double ap = Am[r][p], aq = Am[r][q];
        Am[r][p] = c * ap - sn * aq;
        Am[r][q] = sn * ap + c * aq;
        double zp = Zm[r][p], zq = Zm[r][q];
        Zm[r][p] = c * zp - sn * zq;
        Zm[r][q] = sn * zp + c * zq;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int item = tid; item < (mp / 2) * LEAF; item += blockDim.x) {
        int pi = item / LEAF, col = item % LEAF;
        int p = pr[pi][0], q = pr[pi][1];
        if (q >= m || col >= m) continue;
        double c = cs[pi][0], sn = cs[pi][1];
        double ap = Am[p][col], aq = Am[q][col];
        Am[p][col] = c * ap - sn * aq;
        Am[q][col] = sn * ap + c * aq;
      }
      __syncthreads();
      // the rotation annihilates a_pq exactly in exact arithmetic
      if (tid < mp / 2 && pr[tid][1] < m && cs[tid][1] != 0.0) {
        Am[pr[tid][0]][pr[tid][1]] = 0.0;
        Am[pr[tid][1]][pr[tid][0]] = 0.0;
      }
      __syncthreads();
    }
    if (sweep == max_sweeps - 1 && tid == 0) atomicOr(err, 2);
    __syncthreads();
  }
  // sort ascending (insertion sort of m values)
  if (tid == 0) {
    for (int c = 0; c < m; ++c) {
      s_val[c] = Am[c][c];
      s_idx[c] = c;
    }
    for (int c = 1; c < m; ++c) {
      double v = s_val[c];
      int ix = s_idx[c], p = c - 1;
      while (p >= 0 && s_val[p] > v) {
        s_val[p + 1] = s_val[p];
        s_idx[p + 1] = s_idx[p];
        --p;
      }
      s_val[p + 1] = v;
      s_idx[p + 1] = ix;
    }
  }
  __syncthreads();
  for (int q = tid; q < m * m; q += blockDim.x) {
    int r = q % m, c = q / m;
    Z[(s0 + r) + (long long)(s0 + c) * ldz] = Zm[r][s_idx[c]];
  }
  for (int c = tid; c < m; c += blockDim.x) w[s0 + c] = s_val[c];
}

struct DcWork {
  // per element (offset by node start s)
  double *ds, *zs, *dl, *zz, *defd, *tau, *lam, *zhat;
  int *perm, *ndcol, *defcol, *org, *rank;
  // rotations (offset s): columns and (c, s)
  int2* rcol;
  double2* rcs;
  // per node
  int *kcnt, *ndef, *nrot;
  double* rho;
};

// z, merge ranks of the two sorted child lists, scatter into sorted order.
__global__ void dc_prep_kernel(const Node* nodes, const double* w, const double* Z, long long ldz,
                               const double* e, DcWork wk) {
  const Node nd = nodes[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd.nm) return;
  const int s = nd.s, n1 = nd.n1, n2 = nd.nm - nd.n1;
  const double beta = e[s + n1 - 1];
  const double sq = 0.70710678118654752440;  // 1/sqrt(2)
  double v = w[s + i], z;
  int pos;
  if (i < n1) {
    z = Z[(s + n1 - 1) + (long long)(s + i) * ldz] * sq;
    // number of right-list values strictly below v
    int lo = 0, hi = n2;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (w[s + n1 + mid] < v) lo = mid + 1; else hi = mid;
    }
    pos = i + lo;
  } else {
    int jj = i - n1;
    z = copysign(1.0, beta) * Z[(s + n1) + (long long)(s + i) * ldz] * sq;
    // number of left-list values <= v
    int lo = 0, hi = n1;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (w[s + mid] <= v) lo = mid + 1; else hi = mid;
    }
    pos = jj + lo;
  }
  wk.ds[s + pos] = v;
  wk.zs[s + pos] = z;
  wk.perm[s + pos] = i;
  if (i == 0) wk.rho[blockIdx.y] = 2.0 * fabs(beta);
}

// Deflation (LAPACK dlaed2): one CTA per node; reductions in parallel, the
// scan by thread 0.
// The scan is sequential (LAPACK dlaed2): one thread walks the node's sorted
// (d, z) pairs, carrying the previous non-deflated entry (possibly rotated)
// in registers.  The other warps stage the input into shared memory one
// chunk ahead, so the walk never waits on a global-memory round trip.
constexpr int DEF_CH = 1024;

__global__ void __launch_bounds__(256) dc_deflate_kernel(const Node* nodes, DcWork wk) {
  const Node nd = nodes[blockIdx.x];
  const int s = nd.s, nm = nd.nm;
  const double rho = wk.rho[blockIdx.x];
  __shared__ double sh_d[256], sh_z[256];
  __shared__ double cd[2][DEF_CH], cz[2][DEF_CH];
  __shared__ int cpm[2][DEF_CH];
  double md = 0.0, mz = 0.0;
  for (int q = threadIdx.x; q < nm; q += blockDim.x) {
    md = fmax(md, fabs(wk.ds[s + q]));
    mz = fmax(mz, fabs(wk.zs[s + q]));
  }
  sh_d[threadIdx.x] = md;
  sh_z[threadIdx.x] = mz;
  for (int q = threadIdx.x; q < min(nm, DEF_CH); q += blockDim.x) {
    cd[0][q] = wk.ds[s + q];
    cz[0][q] = wk.zs[s + q];
    cpm[0][q] = wk.perm[s + q];
  }
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sh_d[threadIdx.x] = fmax(sh_d[threadIdx.x], sh_d[threadIdx.x + o]);
      sh_z[threadIdx.x] = fmax(sh_z[threadIdx.x], sh_z[threadIdx.x + o]);
    }
    __syncthreads();
  }
  const double tol = 8.0 * EPS * fmax(sh_d[0], rho * sh_z[0]);
  // Fast path: when the cheap test below keeps every non-deflated pair (no
  // pair needs the exact rotation test), the scan keeps the non-deflated and
  // the z-deflated entries each in their order, so the output positions are
  // prefix counts and every thread writes its own chunk.  Otherwise the
  // sequential scan further down.
  {
    __shared__ int s_last[256], s_nk[256], s_nz[256], s_slow;
    const int per = (nm + (int)blockDim.x - 1) / (int)blockDim.x;
    const int a0 = min(nm, (int)threadIdx.x * per), a1 = min(nm, a0 + per);
    const double* ds = wk.ds + s;
    const double* zs = wk.zs + s;
    int last = -1, nk = 0, nz = 0;
    for (int q = a0; q < a1; ++q) {
      if (rho * fabs(zs[q]) <= tol) {
        ++nz;
      } else {
        ++nk;
        last = q;
      }
    }
    s_last[threadIdx.x] = last;
    s_nk[threadIdx.x] = nk;
    s_nz[threadIdx.x] = nz;
    if (threadIdx.x == 0) s_slow = 0;
    __syncthreads();
    // the previous non-deflated entry before this chunk and the chunk's
    // output offsets
    int prev = -1, ko = 0, zo = 0;
    for (int u = 0; u < (int)threadIdx.x; ++u) {
      if (s_last[u] >= 0) prev = s_last[u];
      ko += s_nk[u];
      zo += s_nz[u];
    }
    bool slow = false;
    for (int q = a0; q < a1; ++q) {
      const double zj = zs[q];
      if (rho * fabs(zj) <= tol) continue;
      if (prev >= 0) {  // the same test as the scan's, against the raw previous entry
        const double zpv = zs[prev], t = ds[q] - ds[prev];
        const double far = 4.0 * tol * fma(zj, zj, zpv * zpv);
        if (!(far >= 2.2250738585072014e-308 && fabs(t * zj * zpv) > far)) slow = true;
      }
      prev = q;
    }
    if (slow) s_slow = 1;
    __syncthreads();
    if (!s_slow) {
      const int* pm = wk.perm + s;
      for (int q = a0; q < a1; ++q) {
        const double zj = zs[q];
        if (rho * fabs(zj) <= tol) {
          wk.defd[s + zo] = ds[q];
          wk.defcol[s + zo] = pm[q];
          ++zo;
        } else {
          wk.dl[s + ko] = ds[q];
          wk.zz[s + ko] = zj;
          wk.ndcol[s + ko] = pm[q];
          ++ko;
        }
      }
      if (threadIdx.x == 0) {
        int kt = 0, zt = 0;
        for (int u = 0; u < (int)blockDim.x; ++u) {
          kt += s_nk[u];
          zt += s_nz[u];
        }
        wk.kcnt[blockIdx.x] = kt;
        wk.ndef[blockIdx.x] = zt;
        wk.nrot[blockIdx.x] = 0;
      }
      return;
    }
  }
  int k = 0, ndef = 0, nrot = 0;
  bool have = false;      // a previous non-deflated entry exists
  double dp = 0.0, zp = 0.0;
  int pp = 0;
  for (int c0 = 0, b = 0; c0 < nm; c0 += DEF_CH, b ^= 1) {
    if (threadIdx.x >= 32) {
      const int n0 = c0 + DEF_CH;
      for (int q = threadIdx.x - 32; q < min(DEF_CH, nm - n0); q += blockDim.x - 32) {
        cd[b ^ 1][q] = wk.ds[s + n0 + q];
        cz[b ^ 1][q] = wk.zs[s + n0 + q];
        cpm[b ^ 1][q] = wk.perm[s + n0 + q];
      }
    } else if (threadIdx.x == 0) {
      const int cn = min(DEF_CH, nm - c0);
      for (int jj = 0; jj < cn; ++jj) {
        const double dj = cd[b][jj], zj = cz[b][jj];
        const int pj = cpm[b][jj];
        if (rho * fabs(zj) <= tol) {
          wk.defd[s + ndef] = dj;
          wk.defcol[s + ndef] = pj;
          ++ndef;
          continue;
        }
        if (!have) {
          have = true;
          dp = dj;
          zp = zj;
          pp = pj;
          continue;
        }
        const double t = dj - dp;
        // |t c s| = |t zj zp| / (zj^2 + zp^2).  Far above tol (the usual
        // case) the pair is kept without the square root and divisions; the
        // factor 4 covers the rounding of both sides (a normal right-hand
        // side keeps the products out of the subnormal range), so the
        // decision is the one the exact test below makes.
        const double far = 4.0 * tol * fma(zj, zj, zp * zp);
        bool rotate = false;
        double cv = zj, sv = zp, tau = 0.0;
        if (!(far >= 2.2250738585072014e-308 && fabs(t * zj * zp) > far)) {
          tau = hypot(cv, sv);
          cv /= tau;
          sv = -sv / tau;
          rotate = fabs(t * cv * sv) <= tol;
        }
        if (rotate) {
          wk.rcol[s + nrot] = make_int2(pp, pj);
          wk.rcs[s + nrot] = make_double2(cv, sv);
          ++nrot;
          const double tt = dp * cv * cv + dj * sv * sv;
          const double dn = dp * sv * sv + dj * cv * cv;
          wk.defd[s + ndef] = tt;
          wk.defcol[s + ndef] = pp;
          ++ndef;
          dp = dn;
          zp = tau;
          pp = pj;
        } else {
          wk.dl[s + k] = dp;
          wk.zz[s + k] = zp;
          wk.ndcol[s + k] = pp;
          ++k;
          dp = dj;
          zp = zj;
          pp = pj;
        }
      }
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  if (have) {
    wk.dl[s + k] = dp;
    wk.zz[s + k] = zp;
    wk.ndcol[s + k] = pp;
    ++k;
  }
  wk.kcnt[blockIdx.x] = k;
  wk.ndef[blockIdx.x] = ndef;
  wk.nrot[blockIdx.x] = nrot;
}

// Apply each node's deflation rotations, in order, to its columns of Z.
__global__ void dc_rotate_kernel(const Node* nodes, double* Z, long long ldz, DcWork wk) {
  const Node nd = nodes[blockIdx.y];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nd.nm) return;
  const int s = nd.s, nrot = wk.nrot[blockIdx.y];
  double* row = Z + (s + r);
  for (int q = 0; q < nrot; ++q) {
    int2 cc = wk.rcol[s + q];
    double2 t = wk.rcs[s + q];
    double* pp = row + (long long)(s + cc.x) * ldz;
    double* pj = row + (long long)(s + cc.y) * ldz;
    double a = *pp, b = *pj;
    *pp = t.x * a + t.y * b;
    *pj = t.x * b - t.y * a;
  }
}

// Secular equation 1 + rho sum z_i^2 / (d_i - lambda) = 0: root j of each node.
__global__ void dc_secular_kernel(const Node* nodes, DcWork wk, int maxit, int* err) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int b = blockIdx.y;
  const int k = wk.kcnt[b];
  if (j >= k) return;
  const int s = nodes[b].s;
  const double rho = wk.rho[b];
  const double* dl = wk.dl + s;
  const double* zz = wk.zz + s;
  int org;
  double lo, hi;
  if (j < k - 1) {
    const double mid = 0.5 * (dl[j + 1] - dl[j]);
    double f = 0.0;
    for (int q = lane; q < k; q += 32) f += zz[q] * zz[q] / ((dl[q] - dl[j]) - mid);
    f = 1.0 + rho * warp_sum(f);
    if (f > 0.0) {
      org = j;
      lo = 0.0;
      hi = mid;
    } else {
      org = j + 1;
      lo = -mid;
      hi = 0.0;
    }
  } else {
    org = k - 1;
    double z2 = 0.0;
    for (int q = lane; q < k; q += 32) z2 += zz[q] * zz[q];
    lo = 0.0;
    hi = rho * warp_sum(z2) * (1.0 + 8.0 * EPS) + 1e-300;
  }
  const double dorg = dl[org];
  const double zo = rho * zz[org] * zz[org];
  double tau = 0.5 * (lo + hi);
  int it = 0;
  for (; it < maxit; ++it) {
    // g = 1 + rho sum z_i^2 / (s_i - tau); the org pole is treated exactly:
    // 1 + phi + phi' (t - tau) - zo / t = 0 is solved for the next t.
    double g = 0.0, gabs = 0.0, phi = 0.0, dphi = 0.0;
    for (int q = lane; q < k; q += 32) {
      double del = (dl[q] - dorg) - tau;
      double r = zz[q] / del;
      double term = zz[q] * r;
      g += term;
      gabs += fabs(term);
      if (q != org) {
        phi += term;
        dphi += r * r;
      }
    }
    g = 1.0 + rho * warp_sum(g);
    gabs = 1.0 + rho * warp_sum(gabs);
    phi = rho * warp_sum(phi);
    dphi = rho * warp_sum(dphi);
    if (fabs(g) <= 4.0 * k * EPS * gabs) break;  // at the rounding level of g
    if (g > 0.0) hi = tau; else lo = tau;
    const double qa = dphi, qb = 1.0 + phi - dphi * tau, qc = -zo;
    double tn;
    if (qa == 0.0) {
      tn = -qc / qb;
    } else {
      const double sq = sqrt(fmax(qb * qb - 4.0 * qa * qc, 0.0));
      const double qq = -0.5 * (qb + copysign(sq, qb));
      const double r1 = qq != 0.0 ? qq / qa : 0.0;
      const double r2 = qq != 0.0 ? qc / qq : 0.0;
      const bool ok1 = r1 > lo && r1 < hi, ok2 = r2 > lo && r2 < hi;
      if (ok1 && ok2) tn = fabs(r1 - tau) < fabs(r2 - tau) ? r1 : r2;
      else if (ok1) tn = r1;
      else if (ok2) tn = r2;
      else tn = 0.5 * (lo + hi);
    }
    if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
    if (fabs(tn - tau) <= 2.0 * EPS * fabs(tn) ||
        hi - lo <= 2.0 * EPS * fmax(fabs(lo), fabs(hi))) {
      tau = tn;
      break;
    }
    tau = tn;
  }
  if (lane == 0) {
    wk.org[s + j] = org;
    wk.tau[s + j] = tau;
    wk.lam[s + j] = dorg + tau;
    if (it >= maxit) atomicOr(err, 4);
  }
}

// Gu-Eisenstat z-hat (LAPACK dlaed3): zhat_i^2 = -delta_ii prod_{j!=i}
// delta_ij / (d_i - d_j) / rho, with delta_ij = (d_i - d_org_j) - tau_j.
__global__ void dc_zhat_kernel(const Node* nodes, DcWork wk, int* err) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int b = blockIdx.y;
  const int k = wk.kcnt[b];
  if (i >= k) return;
  const int s = nodes[b].s;
  const double* dl = wk.dl + s;
  const double di = dl[i];
  double prod = 1.0;
  for (int q = lane; q < k; q += 32) {
    double del = (di - dl[wk.org[s + q]]) - wk.tau[s + q];
    prod *= (q == i) ? -del : del / (di - dl[q]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) prod *= __shfl_xor_sync(0xffffffffu, prod, o);
  if (lane == 0) {
    double v = prod / wk.rho[b];
    if (!isfinite(v)) atomicOr(err, 8);
    wk.zhat[s + i] = copysign(sqrt(fmax(v, 0.0)), wk.zz[s + i]);
  }
}

// Eigenvector j of D + rho zhat zhat^T: U(:, j) = zhat / delta(:, j), normalised.
__global__ void dc_vectors_kernel(const Node* nodes, DcWork wk, double* U, long long ldu) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int b = blockIdx.y;
  const int k = wk.kcnt[b];
  if (j >= k) return;
  const int s = nodes[b].s;
  const double* dl = wk.dl + s;
  const double dorg = dl[wk.org[s + j]], tau = wk.tau[s + j];
  double* col = U + s + (long long)(s + j) * ldu;
  double nrm = 0.0;
  for (int q = lane; q < k; q += 32) {
    double v = wk.zhat[s + q] / ((dl[q] - dorg) - tau);
    col[q] = v;
    nrm += v * v;
  }
  nrm = sqrt(warp_sum(nrm));
  __syncwarp();
  for (int q = lane; q < k; q += 32) col[q] = col[q] / nrm;
}

// G(:, jj) = Z(node rows, ndcol(jj)) for the non-deflated columns.
__global__ void dc_gather_kernel(const Node* nodes, const double* Z, long long ldz, DcWork wk,
                                 double* G, long long ldg) {
  const Node nd = nodes[blockIdx.z];
  const int jj = blockIdx.y;
  if (jj >= wk.kcnt[blockIdx.z]) return;
  const int s = nd.s;
  const int col = wk.ndcol[s + jj];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nd.nm; r += gridDim.x * blockDim.x)
    G[(s + r) + (long long)(s + jj) * ldg] = Z[(s + r) + (long long)(s + col) * ldz];
}

// The merge products of one level in one launch: OUT(node) = G(node) U(node)
// for node z = blockIdx.z, M = its size, N = K = its non-deflated count read
// on the device, so the level needs no host synchronisation.  Tiles past a
// node's extent are skipped at once.
template <int VEC>
__global__ void __launch_bounds__(gemm::THREADS, 1)
dc_gemm_kernel(const Node* nodes, const int* kcnt, const double* G, const double* U, double* OUT,
               long long ld, int tiles, int nn) {
  // one tile per CTA, or (a context on a share of the SMs, grid.x below the
  // tile count) tiles b, b + gridDim.x, ... of tiles x tiles x nn
  const long long total = (long long)tiles * tiles * nn;
  for (long long b = blockIdx.x; b < total; b += gridDim.x) {
    const int z = (int)(b / ((long long)tiles * tiles));
    const int xy = (int)(b - (long long)z * tiles * tiles);
    const Node nd = nodes[z];
    const long long k = kcnt[z];
    const long long m0 = (long long)(xy % tiles) * gemm::BM, n0 = (long long)(xy / tiles) * gemm::BN;
    if (m0 >= nd.nm || n0 >= k) continue;  // uniform over the CTA
    __syncthreads();  // every warp is done with the previous tile's shared stages
    const size_t off = (size_t)nd.s + (size_t)nd.s * ld;
    gemm::dgemm_tile<false, true, VEC>(nd.nm, k, k, 1.0, G + off, ld, U + off, ld, 0.0,
                                       OUT + off, ld, k, m0, n0, 0, 1);
  }
}

// Rank of each new eigenvalue within its node (stable, O(nm) per element).
// One warp per element: the lanes split the comparisons and add their counts.
__global__ void dc_rank_kernel(const Node* nodes, DcWork wk) {
  const Node nd = nodes[blockIdx.y];
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= nd.nm) return;
  const int s = nd.s, k = wk.kcnt[blockIdx.y];
  auto val = [&](int q) { return q < k ? wk.lam[s + q] : wk.defd[s + (q - k)]; };
  const double v = val(i);
  int rank = 0;
  for (int q = lane; q < nd.nm; q += 32) {
    const double u = val(q);
    rank += (u < v) || (u == v && q < i);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) rank += __shfl_xor_sync(0xffffffffu, rank, o);
  if (lane == 0) wk.rank[s + i] = rank;
}

// New node block: column rank(q) <- OUT(:, q) (q < k) or Z_old(:, defcol).
__global__ void dc_assemble_kernel(const Node* nodes, DcWork wk, const double* OUT, long long ldo,
                                   const double* Zold, long long ldz, double* Znew,
                                   long long ldn, double* w) {
  const Node nd = nodes[blockIdx.z];
  const int q = blockIdx.y;
  if (q >= nd.nm) return;
  const int s = nd.s, k = wk.kcnt[blockIdx.z];
  const int dst = wk.rank[s + q];
  const double* src = (q < k) ? OUT + s + (long long)(s + q) * ldo
                              : Zold + s + (long long)(s + wk.defcol[s + (q - k)]) * ldz;
  double* out = Znew + s + (long long)(s + dst) * ldn;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nd.nm; r += gridDim.x * blockDim.x)
    out[r] = src[r];
  if (blockIdx.x == 0 && threadIdx.x == 0)
    w[s + dst] = (q < k) ? wk.lam[s + q] : wk.defd[s + (q - k)];
}

// ---------------------------------------------------------------------------
// 3. Back-transformation: T factor of a block of reflectors (dlarft)
// ---------------------------------------------------------------------------
// T(i,i) = tau_i, T(0:i, i) = -tau_i T(0:i, 0:i) G(0:i, i), G = V^T V.
// T (upper triangle) and G (strict upper triangle, stored transposed in the
// lower triangle) share one shared-memory tile, so the recurrence reads no
// global memory.
// One CTA per block of NBB reflectors: block b holds reflectors
// b NBB .. b NBB + jb - 1 (jb = min(NBB, nref - b NBB)).
// The Gram matrices and T factors are stored per pair of blocks (2 NBB x
// 2 NBB, leading dimension ldg = ldt = 2 NBB): block b is the diagonal
// sub-block b % 2 of pair b / 2.
__global__ void __launch_bounds__(NBB) larft_kernel(const double* Gall, long long ldg,
                                                    const double* tau_all, int nref,
                                                    double* Tall, long long ldt) {
  extern __shared__ double smem_t[];
  double(*S)[NBB + 1] = reinterpret_cast<double(*)[NBB + 1]>(smem_t);
  const int r = threadIdx.x;
  const int j0 = blockIdx.x * NBB, jb = min(NBB, nref - j0);
  if (jb <= 0) return;
  const int pr = blockIdx.x >> 1, h = blockIdx.x & 1;
  const double* G = Gall + (size_t)pr * 2 * NBB * ldg + (size_t)h * NBB * (ldg + 1);
  const double* tau = tau_all + j0;
  double* T = Tall + (size_t)pr * 2 * NBB * ldt + (size_t)h * NBB * (ldt + 1);
  // S[c][r] = G(r, c) for r < c (lower triangle); the upper triangle holds T
  for (int c = 0; c < jb; ++c) {
    if (r <= c) S[r][c] = 0.0;                          // T part: upper triangle
    else S[r][c] = G[c + (long long)r * ldg];           // G(c, r), c < r: lower triangle
  }
  __syncthreads();
  for (int i = 0; i < jb; ++i) {
    const double ti = tau[i];
    double s = 0.0;
    if (r < i)
      for (int c = r; c < i; ++c) s += S[r][c] * S[i][c];
    __syncthreads();
    if (r < i) S[r][i] = -ti * s;
    if (r == i) S[i][i] = ti;
    __syncthreads();
  }
  for (int c = 0; c < jb; ++c)
    if (r < jb) T[r + (long long)c * ldt] = (r <= c) ? S[r][c] : 0.0;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
// X = [V(:, k:k+b) | W(:, 0:b)] and Y = [W | V], rows t0..n-1 (ld ldx): the
// operands of the fused trailing update A22 -= X Y^T = V W^T + W V^T.
__global__ void pack_update_kernel(const double* __restrict__ V, long long ldv,
                                   const double* __restrict__ W, long long ldw, int t0, int n,
                                   int b, double* __restrict__ X, double* __restrict__ Y,
                                   long long ldx) {
  const int c = blockIdx.y;  // 0 .. b-1
  for (int r = t0 + blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double v = V[r + (long long)c * ldv], w = W[r + (long long)c * ldw];
    X[r + (long long)c * ldx] = v;
    X[r + (long long)(b + c) * ldx] = w;
    Y[r + (long long)c * ldx] = w;
    Y[r + (long long)(b + c) * ldx] = v;
  }
}

// Where the cluster tail starts and with how many CTAs (host-side queries,
// made before any stream capture).
static void tail_config(imcom_ctx* ctx, int* tail_ctas_out, int* tail_max_out) {
  const int dev = ctx->device;
  int tail_ctas = 0, tail_max = 0;
  // 16 CTAs (non-portable cluster size) if the device can co-schedule them,
  // else 8 (or as IMCOM_OPT_TAIL_CTAS asks); tail_max = the largest trailing
  // size whose rows fit the cluster's shared memory
  {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t limit = optin > 2048 ? (size_t)optin - 1024 : 0;  // room for static shared
    cudaFuncSetAttribute(trd_tail_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(trd_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)limit);
    const int want = ctx->tail_ctas;
    for (int c : {16, 8}) {
      if (want < 0 || (want == 8 && c == 16)) continue;
      int smax = 1024;
      while (smax > 32 && (tail_smem(smax, c) > limit ||
                           (smax + c - 1) / c > TAIL_RPW * (TAIL_THREADS / 32)))
        --smax;
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = c;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(c);
      cfg.blockDim = dim3(TAIL_THREADS);
      cfg.dynamicSmemBytes = tail_smem(smax, c);
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int nc = 0;
      if (cudaOccupancyMaxActiveClusters(&nc, (void*)trd_tail_kernel, &cfg) == cudaSuccess &&
          nc >= 1) {
        tail_ctas = c;
        tail_max = smax;
        break;
      }
    }
    cudaGetLastError();  // an unsupported cluster size only disables the tail
  }
  *tail_ctas_out = tail_ctas;
  *tail_max_out = tail_max;
}

// The launch sequence of the tridiagonalisation: panels, their trailing
// updates and the cluster tail.  `capturing`: recorded into a graph, so the
// periodic host check of the barrier's error word is left to the caller.
static int sytrd_launches(imcom_ctx* ctx, DMat& Aw, DMat& Vall, double* d, double* e,
                          double* tau, double* W, long long ldw, double* ypart, double* ycol,
                          long long ldy, void* accbuf, long long spin, double* XY, int tail_ctas,
                          int tail_max, bool capturing) {
  const int n = (int)Aw.rows;
  int grid = sm_count(ctx);  // one CTA per SM: the cheapest grid barrier
  TrdAcc* acc = (TrdAcc*)accbuf;
  GridSync* sync = (GridSync*)((char*)accbuf + 2 * sizeof(TrdAcc) + 64);
  int* flag = &sync->err;
  IMC_CUDA(cudaMemsetAsync(sync, 0, sizeof(GridSync), ctx->stream));
  bool tail_done = false;
  for (int k = 0; k < n - 1; k += NB) {
    if (tail_ctas && n - k <= tail_max) {
      const int S = n - k;
      TailArgs ta{Aw.p, Aw.ld, Vall.p, Vall.ld, d, e, tau, n, k, (S + tail_ctas - 1) / tail_ctas};
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = tail_ctas;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(tail_ctas);
      cfg.blockDim = dim3(TAIL_THREADS);
      cfg.dynamicSmemBytes = tail_smem(S, tail_ctas);
      cfg.stream = ctx->stream;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      IMC_CUDA(cudaLaunchKernelEx(&cfg, trd_tail_kernel, ta));
      IMC_LAUNCH();
      tail_done = true;
      break;
    }
    const int b = std::min(NB, n - 1 - k);
    IMC_CUDA(cudaMemsetAsync(accbuf, 0, 2 * sizeof(TrdAcc), ctx->stream));
    static_assert(2 * sizeof(TrdAcc) + 64 + sizeof(GridSync) <= 4096, "panel scratch");
    TrdArgs a{Aw.p, Aw.ld, Vall.p, Vall.ld, W, ldw, d, e, tau, ypart, ycol, ldy, acc, sync, n,
              k, b, spin, (ctx->stall_test & IMCOM_STALL_TRIDIAG) ? 1 : 0};
    void* args[] = {&a};
    // Tiles of the panel's first trailing matrix: when every warp has at
    // most TRD_SLOTS of them, they stay in shared memory for the panel's
    // columns (read from L2 once per panel instead of once per column).
    const long long rbase = (k + 1) & ~1LL, R = n - (k + 1);
    const long long RB = (n - rbase + TR - 1) / TR, NC = (R + CW - 1) / CW;
    const long long rbc = std::min(RB, std::max(0LL, (NC - 1) / CPB));
    const long long ntiles = (long long)CPB * rbc * (rbc + 1) / 2 + (RB - rbc) * NC;
    const bool cached = ntiles <= (long long)TRD_SLOTS * grid * (TRD_THREADS / 32);
    IMC_CUDA(cudaLaunchCooperativeKernel(
        cached ? (void*)trd_panel_kernel<true> : (void*)trd_panel_kernel<false>, grid,
        TRD_THREADS, args, TRD_SMEM, ctx->stream));
    IMC_LAUNCH();
    const int t0 = k + b, rem = n - t0;
    if (rem > 0) {
      // A22 -= V W^T + W V^T as one K = 2b product over the lower triangle
      // (the only part the panel kernel reads)
      const long long ldx = ldw;
      double* X = XY;
      double* Y = XY + (size_t)ldx * 2 * NB;
      dim3 grd((rem + 255) / 256, b);
      pack_update_kernel<<<grd, 256, 0, ctx->stream>>>(Vall.p + (long long)k * Vall.ld, Vall.ld,
                                                       W, ldw, t0, n, b, X, Y, ldx);
      IMC_LAUNCH();
      IMC_TRY(dgemm_lower_nt(ctx, rem, 2 * b, -1.0, X + t0, ldx, Y + t0, ldx, 1.0,
                             Aw.p + t0 + (long long)t0 * Aw.ld, Aw.ld));
    }
    // a timed-out barrier ends the factorisation with an error
    if (!capturing && (k / NB) % 16 == 15) {
      int h = 0;
      IMC_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      IMC_CUDA(cudaStreamSynchronize(ctx->stream));
      if (h) return set_err(ctx, IMCOM_ERR_EIGEN, "tridiagonalisation grid barrier timed out");
    }
  }
  if (!tail_done) {  // the tail writes the last diagonal entry itself
    set_last_diag_kernel<<<1, 1, 0, ctx->stream>>>(Aw.p, Aw.ld, n, d);
    IMC_LAUNCH();
  }
  return 0;
}

// Householder tridiagonalisation (lower) of Aw into d, e, tau and the
// reflectors Vall.  The launch sequence (about four launches per panel) is
// replayed as a CUDA graph once the same size and buffers come back: the
// first call at a key runs it directly, the second captures and instantiates
// it, later calls launch the graph.  A capture the driver refuses leaves the
// direct path in place.
static int sytrd_gpu(imcom_ctx* ctx, DMat& Aw, DMat& Vall, double* d, double* e, double* tau,
                     double* W, long long ldw, double* ypart, double* ycol, long long ldy,
                     void* accbuf, long long spin, double* XY) {
  const int n = (int)Aw.rows;
  int dev = ctx->device, coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (!coop) return set_err(ctx, IMCOM_ERR_CUDA, "device lacks cooperative launch");
  int per_sm = 0, per_sm_c = 0;
  IMC_CUDA(cudaFuncSetAttribute(trd_panel_kernel<false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRD_SMEM));
  IMC_CUDA(cudaFuncSetAttribute(trd_panel_kernel<true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRD_SMEM));
  IMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trd_panel_kernel<false>,
                                                         TRD_THREADS, TRD_SMEM));
  IMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_c, trd_panel_kernel<true>,
                                                         TRD_THREADS, TRD_SMEM));
  if (per_sm < 1 || per_sm_c < 1)
    return set_err(ctx, IMCOM_ERR_CUDA, "panel kernel does not fit on an SM");
  int tail_ctas = 0, tail_max = 0;
  tail_config(ctx, &tail_ctas, &tail_max);
  GridSync* sync = (GridSync*)((char*)accbuf + 2 * sizeof(TrdAcc) + 64);
  EigWork* ew = eig_work(ctx);
  const long long key[] = {n, (long long)(uintptr_t)Aw.p, Aw.ld, (long long)(uintptr_t)Vall.p,
                           Vall.ld, (long long)(uintptr_t)d, (long long)(uintptr_t)e,
                           (long long)(uintptr_t)tau, (long long)(uintptr_t)W, ldw,
                           (long long)(uintptr_t)ypart, (long long)(uintptr_t)ycol, ldy,
                           (long long)(uintptr_t)accbuf, spin, (long long)(uintptr_t)XY,
                           sm_count(ctx), tail_ctas, tail_max, ctx->stall_test};
  constexpr int NKEY = (int)(sizeof(key) / sizeof(key[0]));
  static_assert(NKEY <= EigWork::kTrdKey, "graph key size");
  const bool same = std::equal(key, key + NKEY, ew->trd_key);
  if (!same) {
    if (ew->trd_exec) cudaGraphExecDestroy((cudaGraphExec_t)ew->trd_exec);
    ew->trd_exec = nullptr;
    std::copy(key, key + NKEY, ew->trd_key);
  }
  if (ew->trd_exec) {
    IMC_CUDA(cudaGraphLaunch((cudaGraphExec_t)ew->trd_exec, ctx->stream));
    __atomic_fetch_add(&g_launches, ew->trd_launches, __ATOMIC_RELAXED);
  } else if (same && !ew->trd_graph_off) {
    // second call at this key: capture, instantiate, launch
    cudaGraph_t graph = nullptr;
    const unsigned long long l0 = __atomic_load_n(&g_launches, __ATOMIC_RELAXED);
    bool ok;
    {
      // no other thread frees, allocates or plans while this stream captures
      std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
      ok = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed) == cudaSuccess;
      int st = 0;
      if (ok) {
        st = sytrd_launches(ctx, Aw, Vall, d, e, tau, W, ldw, ypart, ycol, ldy, accbuf, spin,
                            XY, tail_ctas, tail_max, true);
        ok = cudaStreamEndCapture(ctx->stream, &graph) == cudaSuccess && st == 0 && graph;
      }
    }
    cudaGraphExec_t exec = nullptr;
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (ok) {
      ew->trd_exec = exec;
      ew->trd_launches = __atomic_load_n(&g_launches, __ATOMIC_RELAXED) - l0;
      IMC_CUDA(cudaGraphLaunch(exec, ctx->stream));
    } else {
      ew->trd_graph_off = true;  // run directly from now on
      ctx->err.clear();
      IMC_TRY(sytrd_launches(ctx, Aw, Vall, d, e, tau, W, ldw, ypart, ycol, ldy, accbuf, spin,
                             XY, tail_ctas, tail_max, false));
    }
  } else {
    IMC_TRY(sytrd_launches(ctx, Aw, Vall, d, e, tau, W, ldw, ypart, ycol, ldy, accbuf, spin, XY,
                           tail_ctas, tail_max, false));
  }
  // a timed-out grid barrier ends the factorisation with an error
  int h = 0;
  IMC_CUDA(cudaMemcpyAsync(&h, &sync->err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h) return set_err(ctx, IMCOM_ERR_EIGEN, "tridiagonalisation grid barrier timed out");
  return 0;
}

int eigen_dc(imcom_ctx* ctx, const DMat& A, DMat& Wout, double* wout) {
  EigWork* ew = eig_work(ctx);
  const int n = (int)A.rows;
  if (n == 1) {
    IMC_CUDA(cudaMemcpyAsync(wout, A.p, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    double one = 1.0;
    IMC_CUDA(cudaMemcpyAsync(Wout.p, &one, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
    return 0;
  }
  const long long spin = ctx->eig_maxiter > 0 ? ctx->eig_maxiter : 20000000LL;
  // Buffers: Aw (copy of A, ld), Vall (n x n), Z (ping-pong with Wout), G, U, OUT.
  IMC_TRY(ensure_mat(ctx, ew->Z, n, n));
  IMC_TRY(ensure_mat(ctx, ew->V, n, n));
  DMat& Aw = ew->Z;     // first the working copy of A, later a D&C buffer
  DMat& Vall = ew->V;   // reflectors; later reused as the GEMM output block
  const long long ld = Wout.ld;
  const size_t nn = (size_t)ld * n;
  // scratch vectors and small matrices in one allocation
  const long long ldw = pad_ld(n), ldy = pad_ld(n);
  const long long nch = (n + CW - 1) / CW + 1, nrb = (n + TR - 1) / TR + 1;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  size_t o_d = take(n * 8), o_e = take(n * 8), o_tau = take(n * 8), o_dt = take(n * 8);
  size_t o_W = take((size_t)ldw * NB * 8), o_y = take((size_t)ldy * (nch + nrb) * 8);
  size_t o_XY = take((size_t)ldw * 4 * NB * 8);
  size_t o_acc = take(4096);
  size_t o_split = take((size_t)n * 4), o_nodes = take((size_t)n * sizeof(Node));
  size_t o_wk = take(((size_t)n * 8 + 16) * 9 + ((size_t)n * 4 + 16) * 8 + ((size_t)n * 24 + 32) +
                     4096);
  const size_t nblk_bt = (size_t)(n - 1 + NBB - 1) / NBB + 1;
  const size_t npair_bt = (nblk_bt + 1) / 2;
  size_t o_T = take(npair_bt * 4 * NBB * NBB * 8), o_G = take(npair_bt * 4 * NBB * NBB * 8);
  size_t o_X = take((size_t)2 * NBB * ld * 8 * 2);
  size_t o_err = take(64);
  const bool two = ctx->eig_mode == IMCOM_EIGH_TWOSTAGE;
  size_t o_2s = take(two ? twostage_bytes(n) : 0);
  IMC_TRY(eig_buf(ctx, off + 256));
  char* base = (char*)ew->buf;
  double* d = (double*)(base + o_d);
  double* e = (double*)(base + o_e);
  double* tau = (double*)(base + o_tau);
  double* dt = (double*)(base + o_dt);
  double* Wp = (double*)(base + o_W);
  double* yp = (double*)(base + o_y);
  int* dsplit = (int*)(base + o_split);
  Node* dnodes = (Node*)(base + o_nodes);
  double* Tb = (double*)(base + o_T);
  double* Gb = (double*)(base + o_G);
  double* Xb = (double*)(base + o_X);
  int* derr = (int*)(base + o_err);
  IMC_CUDA(cudaMemsetAsync(derr, 0, 64, ctx->stream));

  // ---- 1. tridiagonalisation ----
  stage_begin(ctx, ST_EIG_TRD);
  IMC_TRY(copy_mat(ctx, A.p, A.ld, Aw.p, Aw.ld, n, n));
  IMC_CUDA(cudaMemsetAsync(Vall.p, 0, Vall.bytes(), ctx->stream));
  IMC_CUDA(cudaMemsetAsync(Wp, 0, (size_t)ldw * NB * 8, ctx->stream));
  if (two)
    IMC_TRY(twostage_tridiag(ctx, Aw, Vall, d, e, tau, Wp, ldw, (double*)(base + o_XY),
                             base + o_2s, spin));
  else
    IMC_TRY(sytrd_gpu(ctx, Aw, Vall, d, e, tau, Wp, ldw, yp, yp + (size_t)ldy * nch, ldy,
                      base + o_acc, spin, (double*)(base + o_XY)));
  stage_end(ctx, ST_EIG_TRD);
  stage_begin(ctx, ST_EIG_DC);

  // ---- 2. divide and conquer on (d, e) ----
  // tree of nodes: split ranges in halves until they hold at most LEAF rows
  std::vector<std::vector<Node>> levels;
  levels.push_back({Node{0, n / 2, n}});
  while (true) {
    const auto& last = levels.back();
    if (last[0].nm <= LEAF && std::all_of(last.begin(), last.end(), [](const Node& x) { return x.nm <= LEAF; }))
      break;
    std::vector<Node> nxt;
    for (const Node& x : last) {
      int l = x.nm / 2, r = x.nm - l;
      nxt.push_back(Node{x.s, l / 2, l});
      nxt.push_back(Node{x.s + l, r / 2, r});
    }
    levels.push_back(nxt);
  }
  std::vector<int> splits;
  for (size_t L = 0; L + 1 < levels.size(); ++L)
    for (const Node& x : levels[L]) splits.push_back(x.s + x.n1);
  IMC_CUDA(cudaMemcpyAsync(dt, d, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  if (!splits.empty()) {
    IMC_CUDA(cudaMemcpyAsync(dsplit, splits.data(), splits.size() * 4, cudaMemcpyHostToDevice,
                             ctx->stream));
    tear_kernel<<<1, 1, 0, ctx->stream>>>(dt, e, dsplit, (int)splits.size());
    IMC_LAUNCH();
  }
  // Z buffers: ZA = Wout, ZB = Aw (the A copy is no longer needed after sytrd...
  // but Aw holds nothing the back-transformation needs: the reflectors are in Vall)
  double* ZA = Wout.p;
  double* ZB = Aw.p;
  IMC_CUDA(cudaMemsetAsync(ZA, 0, nn * 8, ctx->stream));
  IMC_CUDA(cudaMemsetAsync(ZB, 0, nn * 8, ctx->stream));
  // D&C work arrays
  DcWork wk;
  {
    // every array starts on a 16-byte boundary whatever n is
    char* p = base + o_wk;
    auto adv = [&](size_t bytes) { p += (bytes + 15) / 16 * 16; };
    auto dv = [&](void) { double* r = (double*)p; adv((size_t)n * 8); return r; };
    auto iv = [&](void) { int* r = (int*)p; adv((size_t)n * 4); return r; };
    wk.ds = dv(); wk.zs = dv(); wk.dl = dv(); wk.zz = dv(); wk.defd = dv(); wk.tau = dv();
    wk.lam = dv(); wk.zhat = dv();
    wk.perm = iv(); wk.ndcol = iv(); wk.defcol = iv(); wk.org = iv(); wk.rank = iv();
    wk.rcs = (double2*)p; adv((size_t)n * 16);
    wk.rcol = (int2*)p; adv((size_t)n * 8);
    wk.kcnt = iv(); wk.ndef = iv(); wk.nrot = iv();
    wk.rho = dv();
  }
  double* w = wout;
  // leaves
  {
    const auto& leaves = levels.back();
    IMC_CUDA(cudaMemcpyAsync(dnodes, leaves.data(), leaves.size() * sizeof(Node),
                             cudaMemcpyHostToDevice, ctx->stream));
    leaf_jacobi_kernel<<<(unsigned)leaves.size(), 256, 0, ctx->stream>>>(dnodes, dt, e, w, ZA, ld,
                                                                         60, derr);
    IMC_LAUNCH();
  }
  // merges, deepest level first
  double* Zcur = ZA;
  double* Znxt = ZB;
  // node blocks of U (k x k), G (gathered columns) and OUT = G U, each n x n
  DMat& UO = ew->U;
  IMC_TRY(ensure_mat(ctx, UO, n, 3 * (long long)n));
  double* Ub = UO.p;
  double* Gm = UO.p + (size_t)UO.ld * n;
  double* OUT = UO.p + 2 * (size_t)UO.ld * n;
  for (int L = (int)levels.size() - 2; L >= 0; --L) {
    const auto& nodes = levels[L];
    const int nn_ = (int)nodes.size();
    int maxnm = 0;
    for (const Node& x : nodes) maxnm = std::max(maxnm, x.nm);
    IMC_CUDA(cudaMemcpyAsync(dnodes, nodes.data(), nn_ * sizeof(Node), cudaMemcpyHostToDevice,
                             ctx->stream));
    dim3 ge((maxnm + 255) / 256, nn_);
    dc_prep_kernel<<<ge, 256, 0, ctx->stream>>>(dnodes, w, Zcur, ld, e, wk);
    IMC_LAUNCH();
    dc_deflate_kernel<<<nn_, 256, 0, ctx->stream>>>(dnodes, wk);
    IMC_LAUNCH();
    dc_rotate_kernel<<<ge, 256, 0, ctx->stream>>>(dnodes, Zcur, ld, wk);
    IMC_LAUNCH();
    dim3 gw((maxnm + 7) / 8, nn_);
    dc_secular_kernel<<<gw, 256, 0, ctx->stream>>>(dnodes, wk,
                                                   ctx->dc_maxiter > 0 ? ctx->dc_maxiter : 100,
                                                   derr);
    IMC_LAUNCH();
    dc_zhat_kernel<<<gw, 256, 0, ctx->stream>>>(dnodes, wk, derr);
    IMC_LAUNCH();
    dc_vectors_kernel<<<gw, 256, 0, ctx->stream>>>(dnodes, wk, Ub, UO.ld);
    IMC_LAUNCH();
    dim3 gg((maxnm + 255) / 256, maxnm, nn_);
    dc_gather_kernel<<<gg, 256, 0, ctx->stream>>>(dnodes, Zcur, ld, wk, Gm, UO.ld);
    IMC_LAUNCH();
    // OUT(node) = G(node) U(node): the new non-deflated eigenvectors, every
    // node of the level in one launch (16-byte copies when every node block
    // starts on a 16-byte boundary)
    {
      bool even = (UO.ld % 2 == 0) && (((uintptr_t)UO.p & 15) == 0);
      for (const Node& x : nodes) even = even && (x.s % 2 == 0);
      const unsigned tiles = (unsigned)((maxnm + gemm::BM - 1) / gemm::BM);
      const unsigned total = tiles * tiles * (unsigned)nn_;
      // a context on a share of the SMs: at most one CTA per SM of its share
      const unsigned gd = ctx->sm_share > 0 ? std::min(total, (unsigned)sm_count(ctx)) : total;
      if (even) {
        IMC_CUDA(cudaFuncSetAttribute(dc_gemm_kernel<2>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)gemm::SMEM_BYTES));
        dc_gemm_kernel<2><<<gd, gemm::THREADS, gemm::SMEM_BYTES, ctx->stream>>>(
            dnodes, wk.kcnt, Gm, Ub, OUT, UO.ld, (int)tiles, nn_);
      } else {
        IMC_CUDA(cudaFuncSetAttribute(dc_gemm_kernel<1>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)gemm::SMEM_BYTES));
        dc_gemm_kernel<1><<<gd, gemm::THREADS, gemm::SMEM_BYTES, ctx->stream>>>(
            dnodes, wk.kcnt, Gm, Ub, OUT, UO.ld, (int)tiles, nn_);
      }
      IMC_LAUNCH();
    }
    dc_rank_kernel<<<dim3((maxnm + 7) / 8, nn_), 256, 0, ctx->stream>>>(dnodes, wk);
    IMC_LAUNCH();
    // Znxt(node) = [OUT | rotated deflated columns of Zcur] in eigenvalue order
    dim3 ga((maxnm + 255) / 256, maxnm, nn_);
    dc_assemble_kernel<<<ga, 256, 0, ctx->stream>>>(dnodes, wk, OUT, UO.ld, Zcur, ld, Znxt, ld, w);
    IMC_LAUNCH();
    std::swap(Zcur, Znxt);
  }
  {
    int h = 0;
    IMC_CUDA(cudaMemcpyAsync(&h, derr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    IMC_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h) return set_err(ctx, IMCOM_ERR_EIGEN, "divide and conquer did not converge (flags %d)", h);
  }

  stage_end(ctx, ST_EIG_DC);
  // ---- 3. back-transformation Z <- Q_T Z (Q_T = H_0 H_1 ... H_{n-2}) ----
  stage_begin(ctx, ST_EIG_BT);
  // two-stage: Z <- Q2 Z first; Q1 (reflectors in Vall, unit at row c + SB
  // of column c) then applies like the one-stage Q
  if (two) IMC_TRY(twostage_backtransform2(ctx, n, base + o_2s, Zcur, ld));
  const int nref = n - 1;
  const int nblk = (nref + NBB - 1) / NBB;
  const int NB2 = 2 * NBB, npair = (nblk + 1) / 2;
  IMC_CUDA(cudaFuncSetAttribute(larft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)LARFT_SMEM));
  double* X = Xb;
  double* X2 = Xb + (size_t)NB2 * ld;
  // Blocks of 2 NBB reflectors: the Gram matrix of each pair, the T factors of
  // its two halves in one launch (one CTA per half: the T recurrences run
  // concurrently), then T12 = -T1 (V1^T V2) T2 joins them (H1 H2 = I - V T V^T
  // with V = [V1 V2], T = [T1 T12; 0 T2]).  Pairs halve the passes over Z and
  // double the inner dimension of the update product.
  for (int pi = 0; pi < npair; ++pi) {
    const int j0 = pi * NB2, jb = std::min(NB2, nref - j0);
    const int r0 = j0, K = n - r0;
    const double* Vb = Vall.p + r0 + (size_t)j0 * Vall.ld;
    IMC_TRY(dgemm(ctx, 'T', 'N', jb, jb, K, 1.0, Vb, Vall.ld, Vb, Vall.ld, 0.0,
                  Gb + (size_t)pi * NB2 * NB2, NB2));
  }
  IMC_CUDA(cudaMemsetAsync(Tb, 0, (size_t)npair * NB2 * NB2 * sizeof(double), ctx->stream));
  larft_kernel<<<nblk, NBB, LARFT_SMEM, ctx->stream>>>(Gb, NB2, tau, nref, Tb, NB2);
  IMC_LAUNCH();
  for (int pi = 0; pi < npair; ++pi) {
    const int j0 = pi * NB2, jb = std::min(NB2, nref - j0);
    if (jb <= NBB) continue;  // a single block: no T12
    const int jb2 = jb - NBB;
    double* T = Tb + (size_t)pi * NB2 * NB2;
    const double* G = Gb + (size_t)pi * NB2 * NB2;
    // X = G12 T2 (NBB x jb2), then T12 = -T1 X
    IMC_TRY(dgemm(ctx, 'N', 'N', NBB, jb2, jb2, 1.0, G + (size_t)NBB * NB2, NB2,
                  T + NBB + (size_t)NBB * NB2, NB2, 0.0, X, NBB));
    IMC_TRY(dgemm(ctx, 'N', 'N', NBB, jb2, NBB, -1.0, T, NB2, X, NBB, 0.0,
                  T + (size_t)NBB * NB2, NB2));
  }
  for (int pi = npair - 1; pi >= 0; --pi) {
    const int j0 = pi * NB2, jb = std::min(NB2, nref - j0);
    // rows from j0: row j0 of the block's reflectors is zero, and an even
    // first row keeps the GEMM operands 16-byte aligned
    const int r0 = j0, K = n - r0;
    const double* Vb = Vall.p + r0 + (size_t)j0 * Vall.ld;
    const double* Tblk = Tb + (size_t)pi * NB2 * NB2;
    IMC_TRY(dgemm(ctx, 'T', 'N', jb, n, K, 1.0, Vb, Vall.ld, Zcur + r0, ld, 0.0, X, NB2));
    IMC_TRY(dgemm(ctx, 'N', 'N', jb, n, jb, 1.0, Tblk, NB2, X, NB2, 0.0, X2, NB2));
    IMC_TRY(dgemm(ctx, 'N', 'N', K, n, jb, -1.0, Vb, Vall.ld, X2, NB2, 1.0, Zcur + r0, ld));
  }
  if (Zcur != Wout.p) IMC_TRY(copy_mat(ctx, Zcur, ld, Wout.p, Wout.ld, n, n));
  stage_end(ctx, ST_EIG_BT);
  return 0;
}

}  // namespace imcom
