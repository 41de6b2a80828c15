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
