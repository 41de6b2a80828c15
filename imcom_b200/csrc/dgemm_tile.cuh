// dgemm_tile.cuh -- the FP64 DMMA GEMM tile (see dgemm.cu), shared by the
// GEMM launchers of dgemm.cu and the grouped divide-and-conquer products of
// eigen_dc.cu.
#pragma once

#include "common.cuh"

namespace imcom {
namespace gemm {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, THREADS = 256;
constexpr int SKC = BK + 4;   // stride of a k-contiguous tile row
constexpr int SMC = BM + 4;   // stride of an m/n-contiguous tile row
constexpr int TILE_DBL = (BM * SKC > BK * SMC) ? BM * SKC : BK * SMC;  // 4608
constexpr int STAGE_DBL = 2 * TILE_DBL;
constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_DBL * sizeof(double);

__device__ __forceinline__ void cp_async(double* dst, const double* src, int bytes, int vec) {
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  if (vec == 2)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(bytes));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Load one operand tile.  KCONTIG: element (r, k) at P[k + r * ld] (r = m or
// n), stored S[r][k] (stride SKC).  Otherwise element (r, k) at P[r + k * ld],
// stored S[k][r] (stride SMC).  Out-of-range elements are zero-filled.
template <bool KCONTIG, int VEC>
__device__ __forceinline__ void load_tile(double* S, const double* __restrict__ P, long long ld,
                                          long long r0, long long k0, long long R, long long K) {
  constexpr int CHUNKS = BM * BK / VEC;
  for (int c = threadIdx.x; c < CHUNKS; c += THREADS) {
    long long r, k;
    double* dst;
    int valid;
    const double* src;
    if (KCONTIG) {
      constexpr int PER = BK / VEC;
      int rr = c / PER, kk = (c % PER) * VEC;
      r = r0 + rr;
      k = k0 + kk;
      dst = S + rr * SKC + kk;
      valid = (r < R) ? (int)min((long long)VEC, max(0LL, K - k)) : 0;
      src = valid ? P + k + r * ld : P;
    } else {
      constexpr int PER = BM / VEC;
      int kk = c / PER, rr = (c % PER) * VEC;
      r = r0 + rr;
      k = k0 + kk;
      dst = S + kk * SMC + rr;
      valid = (k < K) ? (int)min((long long)VEC, max(0LL, R - r)) : 0;
      src = valid ? P + r + k * ld : P;
    }
    cp_async(dst, src, valid * 8, VEC);
  }
}

// LOWER: only output tiles with a row on or below the diagonal (row >= col)
// are computed; tiles strictly above it are left as they are (the symmetric
// rank-2k update of a matrix kept in its lower triangle, LAPACK dsyr2k 'L').
// One 128 x 128 output tile (rows m0.., columns n0..) of the K slice kz of
// nkz (split-K: partial sums go to slice kz of C when nkz > 1).
template <bool AK, bool BKC, int VEC, bool LOWER = false>
__device__ __forceinline__ void dgemm_tile(long long M, long long N, long long K, double alpha,
                                           const double* __restrict__ A, long long lda,
                                           const double* __restrict__ B, long long ldb,
                                           double beta, double* __restrict__ C, long long ldc,
                                           long long kchunk, long long m0, long long n0, int kz,
                                           int nkz) {
  extern __shared__ __align__(16) double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp & 1, wn = warp >> 1;  // 2 x 4 warps
  const int g = lane >> 2, t = lane & 3;
  if (LOWER && m0 + BM <= n0) return;
  // split-K: this CTA covers k in [kb, ke); partial sums go to slice z of C
  const long long kb = (long long)kz * kchunk;
  const long long ke = min(K, kb + kchunk);
  if (nkz > 1) C += (size_t)kz * (size_t)ldc * (size_t)N;
  const int nk = ke > kb ? (int)((ke - kb + BK - 1) / BK) : 0;

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
  // beta C is added in the epilogue.  Its tile is prefetched into L2 now (a
  // hint, no registers held), so the epilogue's loads hit L2 and the HBM
  // reads overlap the main loop instead of holding up the first MMA.
  const bool readc = nkz == 1 && beta != 0.0;
  if (readc) {
    // 128 columns x 128 rows: 8 lines of 128 bytes per column, 4 per thread
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int line = threadIdx.x + q * THREADS;
      const long long col = n0 + (line >> 3), row = m0 + (line & 7) * 16;
      if (row < M && col < N)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(C + row + col * ldc));
    }
  }

  auto stageA = [&](int s) { return smem + s * STAGE_DBL; };
  auto stageB = [&](int s) { return smem + s * STAGE_DBL + TILE_DBL; };

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) {
      load_tile<AK, VEC>(stageA(s), A, lda, m0, kb + (long long)s * BK, M, ke);
      load_tile<BKC, VEC>(stageB(s), B, ldb, n0, kb + (long long)s * BK, N, ke);
    }
    cp_commit();
  }

  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    const double* As = stageA(kt % STAGES);
    const double* Bs = stageB(kt % STAGES);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[4][2], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        int mr = wm * 64 + i * 16 + g;
        if (AK) {
          af[i][0] = As[mr * SKC + kk + t];
          af[i][1] = As[(mr + 8) * SKC + kk + t];
        } else {
          af[i][0] = As[(kk + t) * SMC + mr];
          af[i][1] = As[(kk + t) * SMC + mr + 8];
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int nc = wn * 32 + j * 8 + g;
        bf[j] = BKC ? Bs[nc * SKC + kk + t] : Bs[(kk + t) * SMC + nc];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
              "{%0,%1,%2,%3};\n"
              : "+d"(acc[i][j][0]), "+d"(acc[i][j][1]), "+d"(acc[i][j][2]), "+d"(acc[i][j][3])
              : "d"(af[i][0]), "d"(af[i][1]), "d"(bf[j]));
    }
    int nxt = kt + STAGES - 1;
    if (nxt < nk) {
      load_tile<AK, VEC>(stageA(nxt % STAGES), A, lda, m0, kb + (long long)nxt * BK, M, ke);
      load_tile<BKC, VEC>(stageB(nxt % STAGES), B, ldb, n0, kb + (long long)nxt * BK, N, ke);
    }
    cp_commit();
  }
  cp_wait<0>();

  // one 16-row band at a time: its 16 C values are loaded together, then
  // combined and stored
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    double cv[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const long long row = m0 + wm * 64 + i * 16 + g + ((r >> 1) ? 8 : 0);
        const long long col = n0 + wn * 32 + j * 8 + 2 * t + (r & 1);
        cv[j][r] = (readc && row < M && col < N) ? C[row + col * ldc] : 0.0;
      }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const long long row = m0 + wm * 64 + i * 16 + g + ((r >> 1) ? 8 : 0);
        const long long col = n0 + wn * 32 + j * 8 + 2 * t + (r & 1);
        if (row < M && col < N)
          C[row + col * ldc] = readc ? fma(beta, cv[j][r], alpha * acc[i][j][r])
                                     : alpha * acc[i][j][r];
      }
  }
}

template <bool AK, bool BKC, int VEC, bool LOWER = false>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_kernel(long long M, long long N, long long K, double alpha, const double* __restrict__ A,
             long long lda, const double* __restrict__ B, long long ldb, double beta,
             double* __restrict__ C, long long ldc, long long kchunk) {
  dgemm_tile<AK, BKC, VEC, LOWER>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kchunk,
                                  (long long)blockIdx.x * BM, (long long)blockIdx.y * BN,
                                  (int)blockIdx.z, (int)gridDim.z);
}

// The same gm x gn x nkz tiles from a grid of at most a context's SM share:
// CTA b takes tiles b, b + gridDim.x, ... (row blocks fastest), so a context
// that shares the GPU with others keeps to about its share of the SMs.
template <bool AK, bool BKC, int VEC>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_persist_kernel(long long M, long long N, long long K, double alpha,
                     const double* __restrict__ A, long long lda, const double* __restrict__ B,
                     long long ldb, double beta, double* __restrict__ C, long long ldc,
                     long long kchunk, int gm, int gn, int nkz) {
  const long long total = (long long)gm * gn * nkz;
  for (long long tile = blockIdx.x; tile < total; tile += gridDim.x) {
    __syncthreads();  // every warp is done with the previous tile's shared stages
    const long long xy = tile % ((long long)gm * gn);
    dgemm_tile<AK, BKC, VEC, false>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kchunk,
                                    (xy % gm) * BM, (xy / gm) * BN,
                                    (int)(tile / ((long long)gm * gn)), nkz);
  }
}

}  // namespace gemm
}  // namespace imcom
