// dgemm.cu -- FP64 GEMM on the B200 double-precision tensor path.
//
// C (M x N) = alpha * op(A) op(B) + beta * C, column-major, any M, N, K.
// Used for P = Q^T B (imcom_build_P, imcom_matrix.f90:699, DGEMM 'T','N'),
// T = Q P~ (imcom_build_T, :732-744, m DGEMVs fused into one GEMM) and the
// eigensolver's blocked updates.
//
// sm_100a has no tcgen05 kind for f64, so the FP64 tensor instruction is the
// warp-level DMMA  mma.sync.m16n8k4.f64.  CTA tile 128 x 128 x 32, 8 warps
// as 2 (M) x 4 (N), warp tile 64 x 32 = 4 x 4 MMAs per k-step of 4.
// Operands stream through a 3-stage cp.async shared-memory pipeline (216 KB,
// one CTA per SM, one barrier per 32 of K); the shared layouts are padded so
// every fragment load is bank-conflict free (stride 36 doubles for
// k-contiguous tiles, 132 for m/n-contiguous ones).
#include <algorithm>

#include "common.cuh"

#include "dgemm_tile.cuh"

namespace imcom {

using namespace gemm;

// C = alpha * sum_z part[z] + beta * C
__global__ void splitk_reduce_kernel(const double* __restrict__ part, long long ldp, int splits,
                                     long long M, long long N, double alpha, double beta,
                                     double* __restrict__ C, long long ldc) {
  long long col = blockIdx.y;
  for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < M;
       row += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int z = 0; z < splits; ++z) s += part[(size_t)z * ldp * N + row + col * ldp];
    double* cp = C + row + col * ldc;
    s = alpha * s;
    *cp = (beta != 0.0) ? s + beta * *cp : s;
  }
}

template <bool AK, bool BKC>
int launch(imcom_ctx* ctx, long long M, long long N, long long K, double alpha, const double* A,
           long long lda, const double* B, long long ldb, double beta, double* C, long long ldc,
           int vec) {
  long long gm = (M + BM - 1) / BM, gn = (N + BN - 1) / BN;
  int sms = sm_count(ctx);
  // Split K when the output tiles cannot fill the GPU and K is long: the
  // number of slices (<= 16, >= 4 k-steps each) that minimises waves x
  // k-steps per CTA (one CTA per SM), plus the reduction's pass over the
  // slices and its launch in the same units (a k-step of BK is ~0.14 BK us,
  // the reduction moves ~6 GB/s per us).
  int splits = 1;
  if (gm * gn < sms && K >= 8 * BK) {
    const long long tiles = gm * gn, ksteps = (K + BK - 1) / BK;
    double best = 0.0;
    for (int s = 1; s <= 16 && ksteps >= 4LL * s; ++s) {
      const long long waves = (tiles * s + sms - 1) / sms;
      const long long per = (ksteps + s - 1) / s;
      double cost = (double)(waves * per);
      const double step_us = 0.14 * BK;
      if (s > 1) cost += (3.3 + (double)(s + 1) * (double)M * (double)N * 8.0 / 6e6) / step_us;
      if (s == 1 || cost < best) {
        best = cost;
        splits = s;
      }
    }
  }
  long long kchunk = (K + splits - 1) / splits;
  kchunk = (kchunk + BK - 1) / BK * BK;
  if (kchunk <= 0) kchunk = BK;
  splits = (int)std::max<long long>(1, (K + kchunk - 1) / kchunk);
  double* out = C;
  long long ldo = ldc;
  if (splits > 1) {
    ldo = pad_ld(M);
    size_t need = (size_t)splits * (size_t)ldo * (size_t)N * sizeof(double);
    IMC_TRY(ensure_buf(ctx, &ctx->gemm_ws, ctx->gemm_ws_bytes, need));
    out = (double*)ctx->gemm_ws;
  }
  dim3 grd((unsigned)gm, (unsigned)gn, (unsigned)splits);
  double a1 = splits > 1 ? 1.0 : alpha;
  if (ctx->sm_share > 0 && gm * gn * splits > sms) {
    // a context on a share of the SMs: at most one CTA per SM of its share
    auto k = vec == 2 ? dgemm_persist_kernel<AK, BKC, 2> : dgemm_persist_kernel<AK, BKC, 1>;
    IMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
    k<<<sms, THREADS, SMEM_BYTES, ctx->stream>>>(M, N, K, a1, A, lda, B, ldb, beta, out, ldo,
                                                 kchunk, (int)gm, (int)gn, splits);
  } else if (vec == 2) {
    auto k = dgemm_kernel<AK, BKC, 2>;
    IMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
    k<<<grd, THREADS, SMEM_BYTES, ctx->stream>>>(M, N, K, a1, A, lda, B, ldb, beta, out, ldo, kchunk);
  } else {
    auto k = dgemm_kernel<AK, BKC, 1>;
    IMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
    k<<<grd, THREADS, SMEM_BYTES, ctx->stream>>>(M, N, K, a1, A, lda, B, ldb, beta, out, ldo, kchunk);
  }
  IMC_LAUNCH();
  if (splits > 1) {
    dim3 g2((unsigned)std::min<long long>((M + 255) / 256, 64), (unsigned)N);
    splitk_reduce_kernel<<<g2, 256, 0, ctx->stream>>>(out, ldo, splits, M, N, alpha, beta, C,
                                                      ldc);
    IMC_LAUNCH();
  }
  return 0;
}

// ---------------------------------------------------------------------------
// C (M x 32) = A (M x K) B (K x 32), A and B column-major ('N', 'N'): the
// tall-skinny product of a symmetric trailing matrix and a panel's 32
// reflectors.  The general tile is 128 x 128, so with 32 output columns six
// of its eight warps would compute nothing; this tile is 128 x 32 with every
// warp on 16 rows x all 32 columns (four m16n8k4 DMMA tiles), K in steps of
// SK_BK through a 3-stage cp.async pipeline, split over K into partial
// slices that splitk_reduce_kernel sums.
// Shared strides: A stored [k][r] (stride SK_SA), B stored [n][k] (stride
// SK_SB); both = 4 (mod 16) doubles, so the fragment loads of a half-warp
// (4 x 4 lanes) hit distinct 8-byte banks.
// ---------------------------------------------------------------------------
constexpr int SK_BM = 128, SK_BN = 32, SK_BK = 32, SK_STAGES = 3, SK_THREADS = 256;
constexpr int SK_SA = SK_BM + 4, SK_SB = SK_BK + 4;
constexpr int SK_STAGE = SK_BK * SK_SA + SK_BN * SK_SB;
constexpr size_t SK_SMEM = (size_t)SK_STAGES * SK_STAGE * sizeof(double);

template <int VEC>
__global__ void __launch_bounds__(SK_THREADS) skinny32_kernel(long long M, long long K,
                                                              const double* __restrict__ A,
                                                              long long lda,
                                                              const double* __restrict__ B,
                                                              long long ldb, double* __restrict__ C,
                                                              long long ldc, long long kchunk) {
  using namespace gemm;
  extern __shared__ __align__(16) double sk[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long long m0 = (long long)blockIdx.x * SK_BM;
  const long long kb = (long long)blockIdx.y * kchunk, ke = min(K, kb + kchunk);
  C += (size_t)blockIdx.y * (size_t)ldc * SK_BN;  // partial slice
  const int nk = ke > kb ? (int)((ke - kb + SK_BK - 1) / SK_BK) : 0;
  auto sA = [&](int st) { return sk + st * SK_STAGE; };
  auto sB = [&](int st) { return sk + st * SK_STAGE + SK_BK * SK_SA; };
  auto load = [&](int st, long long k0) {
    double* a = sA(st);
    for (int c = threadIdx.x; c < SK_BM * SK_BK / VEC; c += SK_THREADS) {
      const int kk = c / (SK_BM / VEC), rr = (c % (SK_BM / VEC)) * VEC;
      const long long r = m0 + rr, k = k0 + kk;
      const int valid = (k < ke) ? (int)min((long long)VEC, max(0LL, M - r)) : 0;
      cp_async(a + kk * SK_SA + rr, valid ? A + r + k * lda : A, valid * 8, VEC);
    }
    double* b = sB(st);
    for (int c = threadIdx.x; c < SK_BN * SK_BK / VEC; c += SK_THREADS) {
      const int nn = c / (SK_BK / VEC), kk = (c % (SK_BK / VEC)) * VEC;
      const long long k = k0 + kk;
      const int valid = (int)min((long long)VEC, max(0LL, ke - k));
      cp_async(b + nn * SK_SB + kk, valid ? B + k + nn * ldb : B, valid * 8, VEC);
    }
  };
  double acc[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[j][r] = 0.0;
#pragma unroll
  for (int st = 0; st < SK_STAGES - 1; ++st) {
    if (st < nk) load(st, kb + (long long)st * SK_BK);
    cp_commit();
  }
  const int mr = warp * 16 + g;
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<SK_STAGES - 2>();
    __syncthreads();
    const double* a = sA(kt % SK_STAGES);
    const double* b = sB(kt % SK_STAGES);
#pragma unroll
    for (int kk = 0; kk < SK_BK; kk += 4) {
      const double a0 = a[(kk + t) * SK_SA + mr], a1 = a[(kk + t) * SK_SA + mr + 8];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double bv = b[(8 * j + g) * SK_SB + kk + t];
        asm volatile(
            "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(acc[j][0]), "+d"(acc[j][1]), "+d"(acc[j][2]), "+d"(acc[j][3])
            : "d"(a0), "d"(a1), "d"(bv));
      }
    }
    const int nxt = kt + SK_STAGES - 1;
    if (nxt < nk) load(nxt % SK_STAGES, kb + (long long)nxt * SK_BK);
    cp_commit();
  }
  cp_wait<0>();
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const long long row = m0 + mr + ((r >> 1) ? 8 : 0);
      const int col = 8 * j + 2 * t + (r & 1);
      if (row < M) C[row + (size_t)col * ldc] = acc[j][r];
    }
}

int dgemm_nn_skinny32(imcom_ctx* ctx, long long M, long long K, const double* A, long long lda,
                      const double* B, long long ldb, double* C, long long ldc) {
  if (M <= 0) return 0;
  const long long gm = (M + SK_BM - 1) / SK_BM;
  const int sms = sm_count(ctx);
  int splits = (int)std::max<long long>(1, std::min<long long>((3LL * sms + gm - 1) / gm,
                                                               K / (2 * SK_BK)));
  splits = std::min(splits, 32);
  long long kchunk = (K + splits - 1) / splits;
  kchunk = std::max<long long>(SK_BK, (kchunk + SK_BK - 1) / SK_BK * SK_BK);
  splits = (int)std::max<long long>(1, (K + kchunk - 1) / kchunk);
  double* out = C;
  long long ldo = ldc;
  if (splits > 1) {
    ldo = pad_ld(M);
    IMC_TRY(ensure_buf(ctx, &ctx->gemm_ws, ctx->gemm_ws_bytes,
                       (size_t)splits * (size_t)ldo * SK_BN * sizeof(double)));
    out = (double*)ctx->gemm_ws;
  }
  auto al16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
  const bool v2 = al16(A) && al16(B) && lda % 2 == 0 && ldb % 2 == 0;
  dim3 grd((unsigned)gm, (unsigned)splits);
  if (v2) {
    IMC_CUDA(cudaFuncSetAttribute(skinny32_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)SK_SMEM));
    skinny32_kernel<2><<<grd, SK_THREADS, SK_SMEM, ctx->stream>>>(M, K, A, lda, B, ldb, out, ldo,
                                                                  kchunk);
  } else {
    IMC_CUDA(cudaFuncSetAttribute(skinny32_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)SK_SMEM));
    skinny32_kernel<1><<<grd, SK_THREADS, SK_SMEM, ctx->stream>>>(M, K, A, lda, B, ldb, out, ldo,
                                                                  kchunk);
  }
  IMC_LAUNCH();
  if (splits > 1) {
    dim3 g2((unsigned)std::min<long long>((M + 255) / 256, 64), (unsigned)SK_BN);
    splitk_reduce_kernel<<<g2, 256, 0, ctx->stream>>>(out, ldo, splits, M, SK_BN, 1.0, 0.0, C,
                                                      ldc);
    IMC_LAUNCH();
  }
  return 0;
}

// ---------------------------------------------------------------------------
// C = alpha (alpha C + A B^T), alpha = +-1, on the tiles on and below the
// diagonal, K <= 64: the rank-2b update of a trailing matrix kept in its
// lower triangle (LAPACK dsyr2k 'L' with A = [V W], B = [W V], alpha = -1).
// With K this short the 128 x 128 tile is bound by its C round trip and the
// start of its operand pipeline (a lone tile takes ~27 us for ~9 us of
// MMAs), and a small trailing matrix has fewer 128-row tiles than SMs.  Here
// the tile is 64 x 64 (four warps of 32 x 32), all of K is loaded at once,
// only the lower tiles are launched (a diagonal tile's upper-right quarter is
// skipped), and three CTAs share an SM so that one's loads overlap another's
// MMAs.  C's tile is prefetched into L2 while the operands arrive and added
// in the epilogue (C + alpha A B^T, alpha = +-1 exact).
// ---------------------------------------------------------------------------
constexpr int LU_T = 64, LU_KMAX = 64, LU_THREADS = 128, LU_S = LU_T + 4;
constexpr size_t LU_SMEM = (size_t)2 * LU_KMAX * LU_S * sizeof(double);

template <int VEC>
__global__ void __launch_bounds__(LU_THREADS, 3)
    lower_update_kernel(long long M, int K, int KP, double alpha, const double* __restrict__ A,
                        long long lda, const double* __restrict__ B, long long ldb,
                        double* __restrict__ C, long long ldc, int ntiles) {
  extern __shared__ __align__(16) double lu[];
  double* sA = lu;                   // sA[k][r]
  double* sB = lu + LU_KMAX * LU_S;  // sB[k][c]
  // one tile per CTA, or (a context on a share of the SMs) tiles b, b + gridDim.x, ...
  for (int b = (int)blockIdx.x; b < ntiles; b += (int)gridDim.x) {
    __syncthreads();  // every warp is done with the previous tile's sA, sB
    // lower tile (ti, tj), ti >= tj, from the linear index b
    int ti = (int)((sqrtf(8.0f * (float)b + 1.0f) - 1.0f) * 0.5f);
    while ((ti + 1) * (ti + 2) / 2 <= b) ++ti;
    while (ti > 0 && ti * (ti + 1) / 2 > b) --ti;
    const int tj = b - ti * (ti + 1) / 2;
    const long long m0 = (long long)ti * LU_T, n0 = (long long)tj * LU_T;
    for (int c = threadIdx.x; c < KP * (LU_T / VEC); c += LU_THREADS) {
      const int kk = c / (LU_T / VEC), rr = (c % (LU_T / VEC)) * VEC;
      const long long ra = m0 + rr, rb = n0 + rr;
      const int va = kk < K ? (int)min((long long)VEC, max(0LL, M - ra)) : 0;
      const int vb = kk < K ? (int)min((long long)VEC, max(0LL, M - rb)) : 0;
      cp_async(sA + kk * LU_S + rr, va ? A + ra + (long long)kk * lda : A, va * 8, VEC);
      cp_async(sB + kk * LU_S + rr, vb ? B + rb + (long long)kk * ldb : B, vb * 8, VEC);
    }
    cp_commit();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp & 1, wn = warp >> 1, g = lane >> 2, t = lane & 3;
    const bool skip = ti == tj && wm < wn;  // above the diagonal
    // C's tile into L2 while the operands arrive (4 lines of 128 bytes per
    // column, 2 per thread); the epilogue's loads of it then hit L2
  #pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int line = threadIdx.x + q * LU_THREADS;
      const long long col = n0 + (line >> 2), row = m0 + (line & 3) * 16;
      if (row < M && col < M && !(ti == tj && row + 15 < col))
        asm volatile("prefetch.global.L2 [%0];" ::"l"(C + row + col * ldc));
    }
    double acc[2][4][4];
  #pragma unroll
    for (int i = 0; i < 2; ++i)
  #pragma unroll
      for (int j = 0; j < 4; ++j)
  #pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
    cp_wait<0>();
    __syncthreads();
    if (skip) continue;
  #pragma unroll 4
    for (int kk = 0; kk < KP; kk += 4) {
      double af[2][2], bf[4];
  #pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int mr = wm * 32 + i * 16 + g;
        af[i][0] = sA[(kk + t) * LU_S + mr];
        af[i][1] = sA[(kk + t) * LU_S + mr + 8];
      }
  #pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = sB[(kk + t) * LU_S + wn * 32 + j * 8 + g];
  #pragma unroll
      for (int i = 0; i < 2; ++i)
  #pragma unroll
        for (int j = 0; j < 4; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
              "{%0,%1,%2,%3};\n"
              : "+d"(acc[i][j][0]), "+d"(acc[i][j][1]), "+d"(acc[i][j][2]), "+d"(acc[i][j][3])
              : "d"(af[i][0]), "d"(af[i][1]), "d"(bf[j]));
    }
  #pragma unroll
    for (int i = 0; i < 2; ++i) {
      double cv[4][4];
  #pragma unroll
      for (int j = 0; j < 4; ++j)
  #pragma unroll
        for (int r = 0; r < 4; ++r) {
          const long long row = m0 + wm * 32 + i * 16 + g + ((r >> 1) ? 8 : 0);
          const long long col = n0 + wn * 32 + j * 8 + 2 * t + (r & 1);
          cv[j][r] = (row < M && col < M) ? C[row + col * ldc] : 0.0;
        }
  #pragma unroll
      for (int j = 0; j < 4; ++j)
  #pragma unroll
        for (int r = 0; r < 4; ++r) {
          const long long row = m0 + wm * 32 + i * 16 + g + ((r >> 1) ? 8 : 0);
          const long long col = n0 + wn * 32 + j * 8 + 2 * t + (r & 1);
          if (row < M && col < M) C[row + col * ldc] = fma(alpha, acc[i][j][r], cv[j][r]);
        }
    }
  }
}

int dgemm_lower_nt(imcom_ctx* ctx, long long M, long long K, double alpha, const double* A,
                   long long lda, const double* B, long long ldb, double beta, double* C,
                   long long ldc) {
  if (M <= 0 || K <= 0) return 0;
  auto al16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
  const bool v2 = al16(A) && al16(B) && lda % 2 == 0 && ldb % 2 == 0;
  if (K <= LU_KMAX && beta == 1.0 && (alpha == 1.0 || alpha == -1.0)) {
    const long long nt = (M + LU_T - 1) / LU_T;
    const unsigned tiles = (unsigned)(nt * (nt + 1) / 2);
    const int KP = (int)((K + 3) / 4 * 4);  // whole k-steps of 4, zero-filled
    auto k = v2 ? lower_update_kernel<2> : lower_update_kernel<1>;
    IMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LU_SMEM));
    IMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    // a context on a share of the SMs keeps to about three CTAs per SM of it
    const unsigned grid =
        ctx->sm_share > 0 ? std::min(tiles, 3u * (unsigned)sm_count(ctx)) : tiles;
    k<<<grid, LU_THREADS, LU_SMEM, ctx->stream>>>(M, (int)K, KP, alpha, A, lda, B, ldb, C, ldc,
                                                  (int)tiles);
    IMC_LAUNCH();
    return 0;
  }
  const long long g = (M + BM - 1) / BM;
  dim3 grd((unsigned)g, (unsigned)g, 1);
  if (v2) {
    auto k = dgemm_kernel<false, false, 2, true>;
    IMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
    k<<<grd, THREADS, SMEM_BYTES, ctx->stream>>>(M, M, K, alpha, A, lda, B, ldb, beta, C, ldc, K);
  } else {
    auto k = dgemm_kernel<false, false, 1, true>;
    IMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
    k<<<grd, THREADS, SMEM_BYTES, ctx->stream>>>(M, M, K, alpha, A, lda, B, ldb, beta, C, ldc, K);
  }
  IMC_LAUNCH();
  return 0;
}

int dgemm(imcom_ctx* ctx, char transA, char transB, long long M, long long N, long long K,
          double alpha, const double* A, long long lda, const double* B, long long ldb,
          double beta, double* C, long long ldc) {
  if (M <= 0 || N <= 0) return 0;
  if (K <= 0) {
    if (beta == 1.0) return 0;
    // C = beta * C through a K = 0 GEMM with zero-filled operands.
    K = 0;
  }
  bool ak = (transA == 'T' || transA == 't');
  bool bk = !(transB == 'T' || transB == 't');
  auto al16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
  int vec = (al16(A) && al16(B) && (lda % 2 == 0) && (ldb % 2 == 0)) ? 2 : 1;
  if (ak && bk) return launch<true, true>(ctx, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, vec);
  if (ak && !bk) return launch<true, false>(ctx, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, vec);
  if (!ak && bk) return launch<false, true>(ctx, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, vec);
  return launch<false, false>(ctx, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, vec);
}

}  // namespace imcom

// ---------------------------------------------------------------------------
// Allocation-free P = Q^T B for callers that must not allocate device memory.
//
// The split-K partial sums live in this fixed array instead of a cudaMalloc'd
// buffer.  It is 32 MiB, allocated when the module loads and held by every
// GPU that loads the library until the process exits.  Host code may not use
// the array's name as a device address; the first call on each device looks
// the address up with cudaGetSymbolAddress (and sets the kernel's shared-
// memory limit), so that first call should come before any stream capture.
// Each call writes every partial-sum element it later reads, so nothing needs
// clearing between calls; calls whose GPU work overlaps (different streams or
// threads) share the array and race.
// ---------------------------------------------------------------------------
namespace {
constexpr long long kNoAllocDoubles = 4LL * 1024 * 1024;  // 32 MiB of partial sums
constexpr int kNoAllocSplits = 2;                         // K slices per call
}  // namespace

static __device__ __align__(256) double g_noalloc_partials[kNoAllocDoubles];

#include <mutex>

namespace {
std::mutex g_noalloc_mu;
double* g_noalloc_addr[64] = {};

int noalloc_setup(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) {
      cudaGetLastError();
      return IMCOM_ERR_CUDA;
    }
    auto k2 = imcom::gemm::dgemm_kernel<true, true, 2>;
    auto k1 = imcom::gemm::dgemm_kernel<true, true, 1>;
    if (cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)imcom::gemm::SMEM_BYTES) != cudaSuccess ||
        cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)imcom::gemm::SMEM_BYTES) != cudaSuccess) {
      cudaGetLastError();
      return IMCOM_ERR_CUDA;
    }
    g_noalloc_addr[dev] = (double*)p;
  }
  *out = g_noalloc_addr[dev];
  return 0;
}
}  // namespace

extern "C" int imcom_gpu_build_P_noalloc(const double* dQ, long long ldq, const double* dB,
                                         long long ldb, double* dP, long long ldp, int n, int m,
                                         void* stream) {
  if (!dQ) return -1;
  if (ldq < n || ldq < 1) return -2;
  if (!dB) return -3;
  if (ldb < n || ldb < 1) return -4;
  if (!dP) return -5;
  if (ldp < n || ldp < 1) return -6;
  if (n <= 0) return -7;
  if (m <= 0) return -8;
  const long long ldo = imcom::pad_ld(n);
  // the reduce kernel's grid has one row of blocks per output column, and a
  // grid's y extent stops at 65,535
  if ((long long)kNoAllocSplits * ldo * (long long)m > kNoAllocDoubles || m > 65535)
    return IMCOM_ERR_NOALLOC_SIZE;
  // an error left by the caller's earlier CUDA work is reported, not cleared
  // (and not mistaken for a failure of this call's launches)
  if (cudaPeekAtLastError() != cudaSuccess) return IMCOM_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return IMCOM_ERR_CUDA;
  }
  double* part = nullptr;
  int st = noalloc_setup(dev, &part);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  using namespace imcom::gemm;
  const long long gm = (n + BM - 1) / BM, gn = (m + BN - 1) / BN;
  long long kchunk = ((long long)n + kNoAllocSplits - 1) / kNoAllocSplits;
  kchunk = (kchunk + BK - 1) / BK * BK;
  const int splits = (int)std::max<long long>(1, (n + kchunk - 1) / kchunk);
  dim3 grd((unsigned)gm, (unsigned)gn, (unsigned)splits);
  auto al16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
  if (al16(dQ) && al16(dB) && ldq % 2 == 0 && ldb % 2 == 0)
    dgemm_kernel<true, true, 2><<<grd, THREADS, SMEM_BYTES, s>>>(
        n, m, n, 1.0, dQ, ldq, dB, ldb, 0.0, part, ldo, kchunk);
  else
    dgemm_kernel<true, true, 1><<<grd, THREADS, SMEM_BYTES, s>>>(
        n, m, n, 1.0, dQ, ldq, dB, ldb, 0.0, part, ldo, kchunk);
  __atomic_fetch_add(&imcom::g_launches, 1ULL, __ATOMIC_RELAXED);
  if (cudaGetLastError() != cudaSuccess) return IMCOM_ERR_CUDA;
  dim3 g2((unsigned)std::min<long long>((n + 255) / 256, 64), (unsigned)m);
  imcom::splitk_reduce_kernel<<<g2, 256, 0, s>>>(part, ldo, splits, n, m, 1.0, 0.0, dP, ldp);
  __atomic_fetch_add(&imcom::g_launches, 1ULL, __ATOMIC_RELAXED);
  if (cudaGetLastError() != cudaSuccess) return IMCOM_ERR_CUDA;
  return 0;
}
