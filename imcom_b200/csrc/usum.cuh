// usum.cuh -- per-output-pixel U(kappa) and S(kappa) on one warp.
//
// imcom_U_from_kappa (imcom_matrix.f90:904-922):
//   U = (C - 1/4 sum_p (L_p + 2k) P2_pa / ((L_p + k)(L_p + k))) / C
// imcom_S_from_kappa (imcom_matrix.f90:955-970):
//   S = 1/4 sum_p Ndiag_p P2_pa / ((L_p + k)(L_p + k))
// Each term is formed with the reference's operations in the reference's
// order (explicit _rn intrinsics: no FMA contraction); the sum over p is a
// per-lane sequential sum followed by an xor-butterfly, which leaves the
// bit-identical total in every lane so control flow stays warp-uniform.
#pragma once

namespace imcom {

// lam / col / nd may point to shared or global memory.  col holds P(:, a)
// (P2 = P * P is formed here, bit-identical to the reference's P2_ia).
// Each lane keeps four independent partial sums (modes p = lane + 32 j with
// j mod 4 selecting the sum) so that four divisions are in flight per lane;
// the partials are added as (s0 + s1) + (s2 + s3) before the butterfly.
__device__ __forceinline__ double uterm(double l, double pp, double k, double k2) {
  const double p2 = __dmul_rn(pp, pp);
  const double t = __dadd_rn(l, k);
  return __ddiv_rn(__dmul_rn(__dadd_rn(l, k2), p2), __dmul_rn(t, t));
}

__device__ __forceinline__ double sterm(double l, double pp, double nd, double k) {
  const double p2 = __dmul_rn(pp, pp);
  const double t = __dadd_rn(l, k);
  return __ddiv_rn(__dmul_rn(nd, p2), __dmul_rn(t, t));
}

__device__ __forceinline__ double warp_reduce_sum(double s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
}

__device__ __forceinline__ double warp_usum(const double* lam, const double* col, int n,
                                            double k, int lane) {
  const double k2 = __dmul_rn(2.0, k);
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int p = lane;
  for (; p + 96 < n; p += 128) {
    s0 = __dadd_rn(s0, uterm(lam[p], col[p], k, k2));
    s1 = __dadd_rn(s1, uterm(lam[p + 32], col[p + 32], k, k2));
    s2 = __dadd_rn(s2, uterm(lam[p + 64], col[p + 64], k, k2));
    s3 = __dadd_rn(s3, uterm(lam[p + 96], col[p + 96], k, k2));
  }
  for (; p < n; p += 32) s0 = __dadd_rn(s0, uterm(lam[p], col[p], k, k2));
  return warp_reduce_sum(__dadd_rn(__dadd_rn(s0, s1), __dadd_rn(s2, s3)));
}

__device__ __forceinline__ double warp_ssum(const double* lam, const double* col,
                                            const double* nd, int n, double k, int lane) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int p = lane;
  for (; p + 96 < n; p += 128) {
    s0 = __dadd_rn(s0, sterm(lam[p], col[p], nd[p], k));
    s1 = __dadd_rn(s1, sterm(lam[p + 32], col[p + 32], nd[p + 32], k));
    s2 = __dadd_rn(s2, sterm(lam[p + 64], col[p + 64], nd[p + 64], k));
    s3 = __dadd_rn(s3, sterm(lam[p + 96], col[p + 96], nd[p + 96], k));
  }
  for (; p < n; p += 32) s0 = __dadd_rn(s0, sterm(lam[p], col[p], nd[p], k));
  return warp_reduce_sum(__dadd_rn(__dadd_rn(s0, s1), __dadd_rn(s2, s3)));
}

// U or S at kappa k.
__device__ __forceinline__ double warp_us(bool UnotS, const double* lam, const double* col,
                                          const double* nd, int n, double k, double C,
                                          int lane) {
  if (UnotS) {
    double usum = warp_usum(lam, col, n, k, lane);
    return __ddiv_rn(__dsub_rn(C, __ddiv_rn(usum, 4.0)), C);
  }
  return __ddiv_rn(warp_ssum(lam, col, nd, n, k, lane), 4.0);
}

// Shared-memory plan of the per-pixel kernels: the eigenvalues (n) plus one
// P column per warp when they fit, else the eigenvalues only, else nothing.
struct PixelSmem {
  int warps;       // warps per CTA
  bool lam_smem;   // L staged in shared memory
  bool col_smem;   // P(:, a) staged per warp
  size_t bytes;
};

// CTAs of 4 warps.  The eigenvalues and one P column per warp are staged in
// shared memory when five columns fit in 52 KB (n <= 1331), which keeps at
// least 4 CTAs (16 pixel warps) per SM.  Otherwise nothing is staged: the
// eigenvalues (read by every warp) stay in L1, the columns stream from L2,
// and ~28 pixel warps per SM run the n = m = 4096 case in a single wave.
inline PixelSmem plan_pixel_smem(int n, size_t limit = 52 * 1024) {
  PixelSmem p;
  const size_t col = (size_t)n * sizeof(double);
  p.warps = 4;
  if (col * 5 <= limit) {
    p.lam_smem = p.col_smem = true;
    p.bytes = col * 5;
    return p;
  }
  p.col_smem = false;
  p.lam_smem = false;
  p.bytes = 0;
  return p;
}

}  // namespace imcom
