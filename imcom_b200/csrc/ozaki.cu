// ozaki.cu -- split-precision FP64 products on the sm_100a tensor cores.
//
// C = alpha * A B^T with A (M x K) and B (N x K) given as FP64 matrices is
// computed from int8 digit slices (an Ozaki-style split):
//
//   * every operand row r is scaled by sigma_r = 2^(ilogb(max_k |x_rk|) + 2),
//     so |x / sigma| < 1/2, and x / sigma is rounded to the integer grid
//     N = rint(x / sigma * 2^(7 + 8(S-1))); N is written as S balanced
//     base-256 digits d_0 .. d_{S-1} (d_0 in [-65, 65], the rest in
//     [-128, 127]), x = sigma * sum_k d_k 2^(-7-8k) up to half a unit of the
//     last digit;
//   * the digit products are accumulated exactly in int32 on the tensor
//     cores (tcgen05.mma kind::i8), one TMEM accumulator per diagonal
//     t = k + l, keeping the S diagonals t < S (S(S+1)/2 products);
//   * the epilogue combines the diagonals in FP64 (Horner in 2^-8) and
//     applies alpha * sigma_A(r) * sigma_B(c) * 2^-14.
//
// Exactness of the int32 sums: |d_k d_l| <= 2^14 and a diagonal holds at most
// S <= 8 products per k, so K <= 2^31 / (8 * 2^14) = 16384 is exact for S = 8
// and K <= 18724 for S = 7; larger K is rejected.
//
// Operand layout in HBM (written by the slicing kernels): for every block of
// R operand rows (R = 128 for A, 64 for B) and every 32-byte K block, the S
// digit tiles are contiguous, each in the tcgen05 K-major no-swizzle layout
// (8-row x 16-byte core matrices; byte (r, k) of a tile at
// (r/8)*256 + (k/16)*128 + (r%8)*16 + k%16).  One stage of the GEMM pipeline
// is therefore two contiguous bulk copies (cp.async.bulk, TMA engine).
//
// Kernel: one CTA per 128 x 128 output tile, 10 warps.  Lane 0 of warp 0
// feeds a ring of shared-memory stages with bulk copies completing on
// mbarriers; lane 0 of warp 1 issues the 128 x 128 x 32 MMAs of a stage and
// releases it with tcgen05.commit; warps 2-9 read TMEM (tcgen05.ld 32x32b,
// two warps per 32 lanes, 64 columns each) and write the FP64 tile.  TMEM holds at most four 128-column
// accumulators, so the S digit diagonals are summed in two passes over K
// (see OzPlan).  An MMA of N = 128 takes 64 cycles of tensor time; narrower
// ones are bound by a per-instruction cost of about 50 cycles (measured), so
// one pass with S accumulators of 64 columns would cap the pipe near 64%.
// Every wait is bounded by %globaltimer; a wait that runs out sets an error
// word, the CTA still waits (bounded) for its issued MMAs, frees TMEM and
// returns.
#include <climits>
#include <cmath>

#include "common.cuh"

namespace imcom {

namespace {

constexpr int OZ_BM = 128;
constexpr int OZ_BN = 128;
constexpr int OZ_KB = 32;        // bytes (= int8 elements) of K per block
constexpr int OZ_TILE_A = OZ_BM * OZ_KB;  // 4096 bytes per digit tile
constexpr int OZ_THREADS = 320;  // warp 0 loads, warp 1 issues MMAs, warps 2-9 epilogue
constexpr int OZ_EPI_THREADS = 256;
constexpr int OZ_SMEM_BUDGET = 220 * 1024;
constexpr unsigned long long OZ_WAIT_NS = 2000000000ull;  // 2 s per wait

// ---- slicing -------------------------------------------------------------

// exps[r] = max over k of ilogb(|x_rk|) (INT_MIN / 2 when the row is zero),
// via atomicMax (ilogb is monotone in |x|).
// COLS: operand row r is column r of X (x_rk = X[k + r ld]);
// otherwise operand row r is row r of X (x_rk = X[r + k ld]).
template <bool COLS>
__global__ void oz_exp_kernel(const double* __restrict__ X, long long ld, long long rows,
                              long long K, int* __restrict__ exps) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;  // 8 warps
  const long long k0 = (long long)blockIdx.y * 1024;
  const long long k1 = k0 + 1024 < K ? k0 + 1024 : K;
  if (COLS) {
    // block: 8 rows (one per warp), lanes over k
    const long long r = (long long)blockIdx.x * 8 + w;
    if (r >= rows) return;
    const double* c = X + r * ld;
    double mx = 0.0;
    for (long long k = k0 + lane; k < k1; k += 32) mx = fmax(mx, fabs(c[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0 && mx > 0.0) atomicMax(exps + r, ilogb(mx));
  } else {
    // block: 32 rows (lanes), warps over k
    const long long r = (long long)blockIdx.x * 32 + lane;
    __shared__ double part[8][33];
    double mx = 0.0;
    if (r < rows)
      for (long long k = k0 + w; k < k1; k += 8) mx = fmax(mx, fabs(X[r + k * ld]));
    part[w][lane] = mx;
    __syncthreads();
    if (w == 0 && r < rows) {
#pragma unroll
      for (int q = 1; q < 8; ++q) mx = fmax(mx, part[q][lane]);
      if (mx > 0.0) atomicMax(exps + r, ilogb(mx));
    }
  }
}

// Digits of one (row block, K block): R*32 elements, 16 per thread.
template <bool COLS, int S>
__global__ void oz_digit_kernel(const double* __restrict__ X, long long ld, long long rows,
                                long long K, const int* __restrict__ exps, int R, long long KB,
                                int8_t* __restrict__ dig, double* __restrict__ scale) {
  const int t = threadIdx.x;  // blockDim.x = 2 R
  const int rr = t % R, kh = t / R;
  const long long kb = blockIdx.x, rb = blockIdx.y;
  const long long r = rb * R + rr;
  const long long kbase = kb * OZ_KB + kh * 16;
  int e = 0;
  bool live = r < rows;
  if (live) {
    const int ex = exps[r];
    live = ex > INT_MIN / 2;
    e = live ? ex + 2 : 0;
    if (kb == 0 && kh == 0) scale[r] = scalbn(1.0, e);
  }
  // x 2^(7 + 8 (S-1) - e) in one exact multiply when the power of two is a
  // normal double (always for these operands), else two exact scalings
  const int sh = 7 + 8 * (S - 1) - e;
  const bool one_mul = sh > -1000 && sh < 1000;
  const double mul = one_mul ? scalbn(1.0, sh) : 0.0;
  int8_t d[S][16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const long long k = kbase + j;
    double x = 0.0;
    if (live && k < K) x = COLS ? X[k + r * ld] : X[r + k * ld];
    const double y = one_mul ? x * mul : scalbn(scalbn(x, -e), 7 + 8 * (S - 1));
    long long N = __double2ll_rn(y);
    if (S >= 4 && S <= 7) {
      // |N| < 2^54: N = 2^24 H + L with 0 <= L < 2^24 and |H| < 2^30, so the
      // three lowest balanced digits come from L in 32-bit arithmetic and
      // carry into H (the same digits as the 64-bit recursion below)
      int c = (int)(N & 0xFFFFFF);
      int hi = (int)(N >> 24);
#pragma unroll
      for (int s = S - 1; s >= 1; --s) {
        if (s >= S - 3) {
          const int q = ((c + 128) & 255) - 128;
          d[s][j] = (int8_t)q;
          c = (c - q) >> 8;
          if (s == S - 3) hi += c;  // the carry out of the low 24 bits
        } else {
          const int q = ((hi + 128) & 255) - 128;
          d[s][j] = (int8_t)q;
          hi = (hi - q) >> 8;
        }
      }
      d[0][j] = (int8_t)hi;
    } else {
#pragma unroll
      for (int s = S - 1; s >= 1; --s) {
        const long long q = ((N + 128) & 255) - 128;
        d[s][j] = (int8_t)q;
        N = (N - q) >> 8;
      }
      d[0][j] = (int8_t)N;
    }
  }
  const size_t tile = (size_t)R * OZ_KB;
  int8_t* base = dig + ((size_t)(rb * KB + kb) * S) * tile + (rr >> 3) * 256 + kh * 128 +
                 (rr & 7) * 16;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    uint4 v;
    uint32_t w4[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      w4[q] = (uint32_t)(uint8_t)d[s][4 * q] | ((uint32_t)(uint8_t)d[s][4 * q + 1] << 8) |
              ((uint32_t)(uint8_t)d[s][4 * q + 2] << 16) |
              ((uint32_t)(uint8_t)d[s][4 * q + 3] << 24);
    v.x = w4[0];
    v.y = w4[1];
    v.z = w4[2];
    v.w = w4[3];
    *reinterpret_cast<uint4*>(base + s * tile) = v;
  }
}

// ---- PTX wrappers ----------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of the given parity; false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = gtimer();
  for (unsigned it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 1023u) == 0 && gtimer() - t0 > OZ_WAIT_NS) return false;
  }
}

// Bounded wait for long waits (the epilogue warps wait through the whole
// main loop): lane 0 alone polls, suspending in try_wait and sleeping between
// polls, so that the waiting warps take no shared-memory bandwidth from the
// tensor core.  Warp-uniform result.
__device__ __forceinline__ bool mbar_wait_warp(uint32_t bar, uint32_t parity) {
  uint32_t ok = 0;
  if ((threadIdx.x & 31) == 0) {
    const unsigned long long t0 = gtimer();
    for (;;) {
      uint32_t r;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}\n"
          : "=r"(r)
          : "r"(bar), "r"(parity), "r"(20000u)
          : "memory");
      if (r) {
        ok = 1;
        break;
      }
      if (gtimer() - t0 > OZ_WAIT_NS) break;
      __nanosleep(2000);
    }
  }
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// K-major, no swizzle: LBO = 128 B (second 16-byte K half), SBO = 256 B
// (next 8-row group), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(256 >> 4) << 32) | (1ull << 46);
}

// kind::i8 instruction descriptor: D s32, A s8, B s8, both K-major,
// N = 128, M = 128.
constexpr uint32_t OZ_IDESC = (2u << 4) | (1u << 7) | (1u << 10) |
                              ((uint32_t)(OZ_BN >> 3) << 17) | ((uint32_t)(OZ_BM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dt),
      "l"(ad), "l"(bd), "r"(OZ_IDESC), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

// ---- the GEMM ---------------------------------------------------------------

struct OzArgs {
  const int8_t* A;  // digits, 128-row blocks
  const int8_t* B;  // digits, 128-row blocks
  const double* sa;
  const double* sb;
  double* C;
  long long ldc;
  long long M, N, KB;
  int mblocks, nblocks;
  double alpha;
  int nst;
  int stall;  // test of the bounded waits: the producer issues no copies
  int* err;
};

constexpr int OZ_GROUP_M = 8;  // tile raster: groups of 8 row blocks
constexpr int OZ_MAXACC = 512 / OZ_BN;  // accumulators of 128 columns in TMEM

// Diagonals t = k + l < S are split into a low group (t >= H) and a high
// group (t < H), each of at most 4 accumulators, and the K loop runs once
// per group: first the low group, whose partial Horner sum
//   lo = (((D_{S-1}) 2^-8 + D_{S-2}) 2^-8 + ... ) + D_H
// is parked in the output tile, then the high group, which continues the
// same sequence (lo 2^-8 + D_{H-1}) ... + D_0.  The result is bit-identical
// to one Horner pass over all S diagonals.
template <int S>
struct OzPlan {
  static constexpr int H = S < OZ_MAXACC ? S : OZ_MAXACC;  // high group t = 0 .. H-1
  static constexpr int NLOW = S - H;                       // low group t = H .. S-1
  static_assert(NLOW <= OZ_MAXACC, "at most 8 slices");
  static constexpr int NPHASE = NLOW > 0 ? 2 : 1;
};

// Issue the MMAs of one stage for the diagonals T0 <= t < T1 (accumulator
// slot t - T0); first MMA of every accumulator overwrites it when `fresh`.
template <int S, int T0, int T1>
__device__ __forceinline__ void oz_issue_stage(uint32_t tmem, uint64_t da, uint64_t db, bool fresh) {
#pragma unroll
  for (int t = T0; t < T1; ++t) {
#pragma unroll
    for (int k = 0; k <= t; ++k) {
      const int l = t - k;
      // descriptors address 16-byte units: slice k starts k * 256 units later
      mma_i8(tmem + (uint32_t)((t - T0) * OZ_BN), da + (uint64_t)(k * (OZ_TILE_A >> 4)),
             db + (uint64_t)(l * (OZ_TILE_A >> 4)), (fresh && k == 0) ? 0u : 1u);
    }
  }
}

// Sum the TMEM accumulator slots NSLOT-1 .. 0 of 16 columns (one tcgen05.ld
// per slot, one wait) into acc by Horner in 2^-8; acc enters as the sum of
// the lower-order diagonals (or is ignored when `start`).
template <int NSLOT>
__device__ __forceinline__ void oz_horner16(uint32_t taddr, double (&acc)[16], bool start) {
  uint32_t r[NSLOT > 0 ? NSLOT : 1][16];
#pragma unroll
  for (int q = 0; q < NSLOT; ++q)
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[q][0]), "=r"(r[q][1]), "=r"(r[q][2]), "=r"(r[q][3]), "=r"(r[q][4]),
          "=r"(r[q][5]), "=r"(r[q][6]), "=r"(r[q][7]), "=r"(r[q][8]), "=r"(r[q][9]),
          "=r"(r[q][10]), "=r"(r[q][11]), "=r"(r[q][12]), "=r"(r[q][13]), "=r"(r[q][14]),
          "=r"(r[q][15])
        : "r"(taddr + (uint32_t)(q * OZ_BN)));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = NSLOT - 1; q >= 0; --q) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const double d = (double)(int)r[q][j];
      acc[j] = (start && q == NSLOT - 1) ? d : __dadd_rn(__dmul_rn(acc[j], 0x1p-8), d);
    }
  }
}

template <int S>
__global__ void __launch_bounds__(OZ_THREADS, 1) oz_gemm_kernel(OzArgs g) {
  using Plan = OzPlan<S>;
  constexpr int H = Plan::H, NLOW = Plan::NLOW, NPHASE = Plan::NPHASE;
  extern __shared__ uint8_t oz_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // grouped raster of the output tiles (row blocks fastest within a group)
  const int per_group = OZ_GROUP_M * g.nblocks;
  const int grp = blockIdx.x / per_group;
  const int first_m = grp * OZ_GROUP_M;
  const int gm = min(g.mblocks - first_m, OZ_GROUP_M);
  const int rem = blockIdx.x % per_group;
  const int mb = first_m + rem % gm, nb = rem / gm;

  constexpr uint32_t SLICE = OZ_TILE_A;  // 128 rows x 32 bytes, A and B alike
  constexpr uint32_t HALF = S * SLICE;   // A part (or B part) of a stage
  constexpr uint32_t STAGE = 2 * HALF;
  const uint32_t raw = smem_u32(oz_smem);
  const uint32_t base = (raw + 1023u) & ~1023u;
  const int nst = g.nst;
  const uint32_t bars = base + (uint32_t)nst * STAGE;
  const uint32_t accf0 = bars + 16u * nst;  // low-group accumulators complete
  const uint32_t accf1 = accf0 + 8u;        // high-group accumulators complete
  const uint32_t tfree = accf0 + 16u;       // low group read out of TMEM
  const uint32_t holder = accf0 + 24u;

  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mbar_init(bars + 8u * s, 1);
      mbar_init(bars + 8u * (nst + s), 1);
    }
    mbar_init(accf0, 1);
    mbar_init(accf1, 1);
    mbar_init(tfree, OZ_EPI_THREADS);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(holder),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  uint32_t tmem;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(tmem) : "r"(holder) : "memory");

  const int KB = (int)g.KB;
  if (warp == 0 && lane == 0) {
    // producer: phase 0 = low group (needs all S slices), last phase = high
    // group (needs slices 0 .. H-1, a prefix of each block)
    const int8_t* srcA = g.A + (size_t)mb * KB * HALF;
    const int8_t* srcB = g.B + (size_t)nb * KB * HALF;
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    int it = 0;
    if (g.stall) {  // nothing arrives on the stages: the issuer's wait runs out
      atomicOr(g.err, 16);
      ok = false;
    }
    for (int phase = 0; phase < NPHASE && ok; ++phase) {
      const uint32_t bytes = ((NPHASE == 2 && phase == 0) ? S : H) * SLICE;
      for (int kb = 0; kb < KB; ++kb, ++it) {
        if (it >= nst && !mbar_wait(bars + 8u * (nst + s), ph ^ 1u)) {
          atomicOr(g.err, 1);
          ok = false;
          break;
        }
        const uint32_t sA = base + (uint32_t)s * STAGE;
        const uint32_t fb = bars + 8u * s;
        mbar_expect_tx(fb, 2 * bytes);
        bulk_g2s(sA, srcA + (size_t)kb * HALF, bytes, fb);
        bulk_g2s(sA + HALF, srcB + (size_t)kb * HALF, bytes, fb);
        if (++s == nst) {
          s = 0;
          ph ^= 1u;
        }
      }
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint64_t dbase = smem_desc(base);
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    for (int phase = 0; phase < NPHASE; ++phase) {
      const bool low = NPHASE == 2 && phase == 0;
      if (NPHASE == 2 && phase == 1) {
        // the epilogue warps must have read the low group out of TMEM
        if (!mbar_wait(tfree, 0)) {
          atomicOr(g.err, 8);
          ok = false;
        }
        tc_fence_after();
      }
      for (int kb = 0; ok && kb < KB; ++kb) {
        if (!mbar_wait(bars + 8u * s, ph)) {
          atomicOr(g.err, 2);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t da = dbase + (uint64_t)((s * STAGE) >> 4);
        const uint64_t db = da + (uint64_t)(HALF >> 4);
        if (low)
          oz_issue_stage<S, H, S>(tmem, da, db, kb == 0);
        else
          oz_issue_stage<S, 0, H>(tmem, da, db, kb == 0);
        mma_commit(bars + 8u * (nst + s));
        if (++s == nst) {
          s = 0;
          ph ^= 1u;
        }
      }
      mma_commit(low ? accf0 : accf1);
    }
  }
  __syncwarp();

  // epilogue warps 2..9: warp w reads TMEM lanes 32 (w % 4) .. +31 (tile rows)
  // and handles columns 64 ((w - 2) / 4) .. +63 of the tile
  if (warp >= 2) {
    const long long row = (long long)mb * OZ_BM + (warp & 3) * 32 + lane;
    const int c0 = ((warp - 2) >> 2) * (OZ_BN / 2);
    const bool rv = row < g.M;
    const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0;
    double* crow = g.C + row;
    const long long col0 = (long long)nb * OZ_BN + c0;
    bool ok = true;
    if (NPHASE == 2) {
      // low group: partial Horner sum parked in C
      ok = mbar_wait_warp(accf0, 0);
      tc_fence_after();
      if (ok) {
#pragma unroll 1
        for (int cc = 0; cc < OZ_BN / 32; ++cc) {
          double acc[16];
          oz_horner16<NLOW>(lane_base + (uint32_t)(cc * 16), acc, true);
          if (rv) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const long long col = col0 + cc * 16 + j;
              if (col < g.N) crow[col * g.ldc] = acc[j];
            }
          }
        }
      } else if (lane == 0) {
        atomicOr(g.err, 4);
      }
      tc_fence_before();
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tfree) : "memory");
    }
    ok = ok && mbar_wait_warp(accf1, 0);
    tc_fence_after();
    if (ok) {
      const double srow = rv ? g.alpha * g.sa[row] * 0x1p-14 : 0.0;
      // the parked low-group sums of the next chunk load while this one is
      // combined
      double nxt[16];
      if (NPHASE == 2) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const long long col = col0 + j;
          nxt[j] = (rv && col < g.N) ? crow[col * g.ldc] : 0.0;
        }
      }
#pragma unroll 1
      for (int cc = 0; cc < OZ_BN / 32; ++cc) {
        double acc[16];
        if (NPHASE == 2) {
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[j] = nxt[j];
          if (cc + 1 < OZ_BN / 32) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const long long col = col0 + (cc + 1) * 16 + j;
              nxt[j] = (rv && col < g.N) ? crow[col * g.ldc] : 0.0;
            }
          }
        }
        oz_horner16<H>(lane_base + (uint32_t)(cc * 16), acc, NPHASE == 1);
        if (rv) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const long long col = col0 + cc * 16 + j;
            if (col < g.N) crow[col * g.ldc] = srow * g.sb[col] * acc[j];
          }
        }
      }
    } else if (lane == 0) {
      atomicOr(g.err, 4);
    }
  }  // epilogue warps
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512)
                 : "memory");
  }
}

template <int S>
int launch_gemm(imcom_ctx* ctx, OzArgs g, cudaStream_t st) {
  const size_t stage = (size_t)S * 2 * OZ_TILE_A;
  int nst = (int)(OZ_SMEM_BUDGET / stage);
  if (nst > 8) nst = 8;
  if (nst < 2) nst = 2;
  g.nst = nst;
  const size_t smem = 1024 + nst * stage + 16 * nst + 32;
  IMC_CUDA(cudaFuncSetAttribute(oz_gemm_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  const long long tiles = (long long)g.mblocks * g.nblocks;
  oz_gemm_kernel<S><<<(unsigned)tiles, OZ_THREADS, smem, st>>>(g);
  IMC_LAUNCH();
  return 0;
}

template <bool COLS, int S>
int launch_digits(imcom_ctx* ctx, const double* X, long long ld, long long rows, long long K,
                  const int* exps, SplitOp& op, cudaStream_t st) {
  dim3 grd((unsigned)op.kb, (unsigned)op.rb);
  oz_digit_kernel<COLS, S><<<grd, 2 * op.R, 0, st>>>(X, ld, rows, K, exps, op.R, op.kb, op.dig,
                                                     op.scale);
  IMC_LAUNCH();
  return 0;
}

}  // namespace

long long split_max_k(int S) { return (long long)(2147483647.0 / ((double)S * 16384.0)); }

int split_operand(imcom_ctx* ctx, const double* X, long long ld, long long rows, long long K,
                  bool cols, int S, int R, SplitOp& op) {
  if (S < 2 || S > 8) return set_err(ctx, IMCOM_ERR_SPLIT, "split: slices must be 2..8 (got %d)", S);
  if (R != OZ_BM) return set_err(ctx, IMCOM_ERR_SPLIT, "split: bad row block %d", R);
  if (K > split_max_k(S))
    return set_err(ctx, IMCOM_ERR_SPLIT, "split: K = %lld exceeds the exact int32 range (%lld)", K,
                   split_max_k(S));
  const long long rb = (rows + R - 1) / R, kb = (K + OZ_KB - 1) / OZ_KB;
  const size_t dig_bytes = (size_t)rb * kb * S * R * OZ_KB;
  IMC_TRY(ensure_buf(ctx, reinterpret_cast<void**>(&op.dig), op.dig_bytes, dig_bytes));
  IMC_TRY(ensure_buf(ctx, reinterpret_cast<void**>(&op.scale), op.scale_bytes,
                     (size_t)rb * R * sizeof(double)));
  IMC_TRY(ensure_buf(ctx, reinterpret_cast<void**>(&op.exps), op.exps_bytes,
                     (size_t)rb * R * sizeof(int)));
  op.rows = rows;
  op.K = K;
  op.S = S;
  op.R = R;
  op.rb = rb;
  op.kb = kb;
  cudaStream_t st = ctx->stream;
  // 0x80 bytes: every int is -2139062144 < INT_MIN / 2 (zero row)
  IMC_CUDA(cudaMemsetAsync(op.exps, 0x80, (size_t)rb * R * sizeof(int), st));
  IMC_CUDA(cudaMemsetAsync(op.scale, 0, (size_t)rb * R * sizeof(double), st));
  const unsigned ky = (unsigned)((K + 1023) / 1024);
  if (cols) {
    oz_exp_kernel<true><<<dim3((unsigned)((rows + 7) / 8), ky), 256, 0, st>>>(X, ld, rows, K,
                                                                              op.exps);
  } else {
    oz_exp_kernel<false><<<dim3((unsigned)((rows + 31) / 32), ky), 256, 0, st>>>(X, ld, rows, K,
                                                                                 op.exps);
  }
  IMC_LAUNCH();
#define OZ_DIG_CASE(SS)                                                                   \
  case SS:                                                                                \
    return cols ? launch_digits<true, SS>(ctx, X, ld, rows, K, op.exps, op, st)           \
                : launch_digits<false, SS>(ctx, X, ld, rows, K, op.exps, op, st);
  switch (S) {
    OZ_DIG_CASE(2)
    OZ_DIG_CASE(3)
    OZ_DIG_CASE(4)
    OZ_DIG_CASE(5)
    OZ_DIG_CASE(6)
    OZ_DIG_CASE(7)
    OZ_DIG_CASE(8)
  }
#undef OZ_DIG_CASE
  return set_err(ctx, IMCOM_ERR_SPLIT, "split: slices must be 2..8");
}

int split_gemm(imcom_ctx* ctx, const SplitOp& a, const SplitOp& b, double alpha, double* C,
               long long ldc) {
  if (a.R != OZ_BM || b.R != OZ_BN) return set_err(ctx, IMCOM_ERR_SPLIT, "split_gemm: operand blocks");
  if (a.S != b.S) return set_err(ctx, IMCOM_ERR_SPLIT, "split_gemm: slice counts differ");
  if (a.kb != b.kb || a.K != b.K) return set_err(ctx, IMCOM_ERR_SPLIT, "split_gemm: K differs");
  if (a.rows <= 0 || b.rows <= 0 || a.K <= 0) return 0;
  // error word: zeroed by split_reset_error, read by split_check_error at
  // the caller's next synchronisation point (no sync here)
  int* err = ctx->flags + 16;
  OzArgs g;
  g.A = a.dig;
  g.B = b.dig;
  g.sa = a.scale;
  g.sb = b.scale;
  g.C = C;
  g.ldc = ldc;
  g.M = a.rows;
  g.N = b.rows;
  g.KB = a.kb;
  g.mblocks = (int)a.rb;
  g.nblocks = (int)b.rb;
  g.alpha = alpha;
  g.err = err;
  g.stall = (ctx->stall_test & IMCOM_STALL_SPLIT) != 0;
  switch (a.S) {
    case 2: IMC_TRY(launch_gemm<2>(ctx, g, ctx->stream)); break;
    case 3: IMC_TRY(launch_gemm<3>(ctx, g, ctx->stream)); break;
    case 4: IMC_TRY(launch_gemm<4>(ctx, g, ctx->stream)); break;
    case 5: IMC_TRY(launch_gemm<5>(ctx, g, ctx->stream)); break;
    case 6: IMC_TRY(launch_gemm<6>(ctx, g, ctx->stream)); break;
    case 7: IMC_TRY(launch_gemm<7>(ctx, g, ctx->stream)); break;
    case 8: IMC_TRY(launch_gemm<8>(ctx, g, ctx->stream)); break;
    default: return set_err(ctx, IMCOM_ERR_SPLIT, "split_gemm: slices must be 2..8");
  }
  return 0;
}

int split_reset_error(imcom_ctx* ctx) {
  IMC_CUDA(cudaMemsetAsync(ctx->flags + 16, 0, sizeof(int), ctx->stream));
  return 0;
}

int split_check_error(imcom_ctx* ctx) {
  int h = 0;
  IMC_CUDA(cudaMemcpyAsync(&h, ctx->flags + 16, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h)
    return set_err(ctx, IMCOM_ERR_SPLIT, "split product: a pipeline wait ran out (code %d)", h);
  return 0;
}

void split_free(SplitOp& op) {
  std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
  if (op.dig) cudaFree(op.dig);
  if (op.scale) cudaFree(op.scale);
  if (op.exps) cudaFree(op.exps);
  op = SplitOp();
}

}  // namespace imcom
