// dgemm.cu -- FP64 GEMM on the B200 double-precision tensor path.
//
// C (M x N) = alpha * op(A) op(B) + beta * C, column-major, any M, N, K.
// Used for P = Q^T B (imcom_build_P, imcom_matrix.f90:699, DGEMM 'T','N'),
// T = Q P~ (imcom_build_T, :732-744, m DGEMVs fused into one GEMM) and the
// eigensolver's blocked updates.
//
// sm_100a has no tcgen05 kind for f64, so the FP64 tensor instruction is the
// warp-level DMMA  mma.sync.m16n8k4.f64.  CTA tile 128 x 128 x 16, 8 warps
// as 2 (M) x 4 (N), warp tile 64 x 32 = 4 x 4 MMAs per k-step of 4.
// Operands stream through a 3-stage cp.async shared-memory pipeline; the
// shared layouts are padded so every fragment load is bank-conflict free
// (stride 20 doubles for k-contiguous tiles, 132 for m/n-contiguous ones).
#include <algorithm>

#include "common.cuh"

namespace imcom {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 3, THREADS = 256;
constexpr int SKC = BK + 4;   // stride of a k-contiguous tile row
constexpr int SMC = BM + 4;   // stride of an m/n-contiguous tile row
constexpr int TILE_DBL = (BM * SKC > BK * SMC) ? BM * SKC : BK * SMC;  // 2560
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
template <bool AK, bool BKC, int VEC, bool LOWER = false>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_kernel(long long M, long long N, long long K, double alpha, const double* __restrict__ A,
             long long lda, const double* __restrict__ B, long long ldb, double beta,
             double* __restrict__ C, long long ldc, long long kchunk) {
  extern __shared__ __align__(16) double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp & 1, wn = warp >> 1;  // 2 x 4 warps
  const int g = lane >> 2, t = lane & 3;
  const long long m0 = (long long)blockIdx.x * BM, n0 = (long long)blockIdx.y * BN;
  if (LOWER && m0 + BM <= n0) return;
  // split-K: this CTA covers k in [kb, ke); partial sums go to slice z of C
  const long long kb = (long long)blockIdx.z * kchunk;
  const long long ke = min(K, kb + kchunk);
  if (gridDim.z > 1) C += (size_t)blockIdx.z * (size_t)ldc * (size_t)N;
  const int nk = ke > kb ? (int)((ke - kb + BK - 1) / BK) : 0;

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
  // C += alpha op(A) op(B) with alpha = +-1 (the updates of the eigensolver):
  // the accumulators start from alpha C, loaded before the operand pipeline
  // so the C reads overlap it; the epilogue then stores alpha acc (sign
  // flips are exact).
  const bool preload = gridDim.z == 1 && beta == 1.0 && (alpha == 1.0 || alpha == -1.0);
  if (preload) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          long long row = m0 + wm * 64 + i * 16 + g + ((r >> 1) ? 8 : 0);
          long long col = n0 + wn * 32 + j * 8 + 2 * t + (r & 1);
          if (row < M && col < N) acc[i][j][r] = alpha * C[row + col * ldc];
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

#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        long long row = m0 + wm * 64 + i * 16 + g + ((r >> 1) ? 8 : 0);
        long long col = n0 + wn * 32 + j * 8 + 2 * t + (r & 1);
        if (row < M && col < N) {
          double* cp = C + row + col * ldc;
          double v = alpha * acc[i][j][r];
          if (!preload && gridDim.z == 1 && beta != 0.0) v += beta * *cp;
          *cp = v;
        }
      }
}

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
  // Split K when the output tiles cannot fill the GPU and K is long.
  int splits = 1;
  if (gm * gn < sms && K >= 8 * BK) {
    splits = (int)std::min<long long>((2LL * sms + gm * gn - 1) / (gm * gn), K / (4 * BK));
    splits = std::max(1, std::min(splits, 16));
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
  if (vec == 2) {
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

int dgemm_lower_nt(imcom_ctx* ctx, long long M, long long K, double alpha, const double* A,
                   long long lda, const double* B, long long ldb, double beta, double* C,
                   long long ldc) {
  if (M <= 0 || K <= 0) return 0;
  const long long g = (M + BM - 1) / BM;
  dim3 grd((unsigned)g, (unsigned)g, 1);
  auto al16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
  if (al16(A) && al16(B) && lda % 2 == 0 && ldb % 2 == 0) {
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
    auto k2 = imcom::dgemm_kernel<true, true, 2>;
    auto k1 = imcom::dgemm_kernel<true, true, 1>;
    if (cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)imcom::SMEM_BYTES) != cudaSuccess ||
        cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)imcom::SMEM_BYTES) != cudaSuccess) {
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
  const long long gm = (n + imcom::BM - 1) / imcom::BM, gn = (m + imcom::BN - 1) / imcom::BN;
  long long kchunk = ((long long)n + kNoAllocSplits - 1) / kNoAllocSplits;
  kchunk = (kchunk + imcom::BK - 1) / imcom::BK * imcom::BK;
  const int splits = (int)std::max<long long>(1, (n + kchunk - 1) / kchunk);
  dim3 grd((unsigned)gm, (unsigned)gn, (unsigned)splits);
  auto al16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
  if (al16(dQ) && al16(dB) && ldq % 2 == 0 && ldb % 2 == 0)
    imcom::dgemm_kernel<true, true, 2><<<grd, imcom::THREADS, imcom::SMEM_BYTES, s>>>(
        n, m, n, 1.0, dQ, ldq, dB, ldb, 0.0, part, ldo, kchunk);
  else
    imcom::dgemm_kernel<true, true, 1><<<grd, imcom::THREADS, imcom::SMEM_BYTES, s>>>(
        n, m, n, 1.0, dQ, ldq, dB, ldb, 0.0, part, ldo, kchunk);
  __atomic_fetch_add(&imcom::g_launches, 1ULL, __ATOMIC_RELAXED);
  if (cudaGetLastError() != cudaSuccess) return IMCOM_ERR_CUDA;
  dim3 g2((unsigned)std::min<long long>((n + 255) / 256, 64), (unsigned)m);
  imcom::splitk_reduce_kernel<<<g2, 256, 0, s>>>(part, ldo, splits, n, m, 1.0, 0.0, dP, ldp);
  __atomic_fetch_add(&imcom::g_launches, 1ULL, __ATOMIC_RELAXED);
  if (cudaGetLastError() != cudaSuccess) return IMCOM_ERR_CUDA;
  return 0;
}
