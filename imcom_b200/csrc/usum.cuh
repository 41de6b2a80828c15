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
__device__ __forceinline__ double warp_usum(const double* lam, const double* col, int n,
                                            double k, int lane) {
  double s = 0.0;
  double k2 = __dmul_rn(2.0, k);
  for (int p = lane; p < n; p += 32) {
    double l = lam[p];
    double pp = col[p];
    double p2 = __dmul_rn(pp, pp);
    double t = __dadd_rn(l, k);
    double den = __dmul_rn(t, t);
    double num = __dmul_rn(__dadd_rn(l, k2), p2);
    s = __dadd_rn(s, __ddiv_rn(num, den));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
}

__device__ __forceinline__ double warp_ssum(const double* lam, const double* col,
                                            const double* nd, int n, double k, int lane) {
  double s = 0.0;
  for (int p = lane; p < n; p += 32) {
    double l = lam[p];
    double pp = col[p];
    double p2 = __dmul_rn(pp, pp);
    double t = __dadd_rn(l, k);
    double den = __dmul_rn(t, t);
    double num = __dmul_rn(nd[p], p2);
    s = __dadd_rn(s, __ddiv_rn(num, den));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
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

// Staging columns pays only while it leaves >= 8 warps per CTA; otherwise
// the columns stream from L2 and 16 warps per CTA hide the divide latency.
inline PixelSmem plan_pixel_smem(int n, size_t limit = 200 * 1024) {
  PixelSmem p;
  size_t col = (size_t)n * sizeof(double);
  if (col * 9 <= limit) {
    p.warps = 8;
    p.lam_smem = p.col_smem = true;
    p.bytes = col * 9;
    return p;
  }
  p.warps = 16;
  p.col_smem = false;
  p.lam_smem = col <= limit;
  p.bytes = p.lam_smem ? col : 0;
  return p;
}

}  // namespace imcom
