// kappa.cu -- learned-kappa bracket (features, MLP, bracketed bisection).
#include "common.cuh"

using namespace imcom;

extern "C" int imcom_gpu_kappa_features(imcom_ctx* ctx, int UnotS, double US_max, double C_a,
                                        float* feat_out) {
  (void)UnotS; (void)US_max; (void)C_a; (void)feat_out;
  if (!ctx) return -1;
  return set_err(ctx, IMCOM_ERR_STATE, "learned-kappa features not built");
}

extern "C" int imcom_gpu_mlp_set_weights(imcom_ctx* ctx, const float*, const float*, const float*,
                                         const float*, const float*, const float*, const float*,
                                         const float*) {
  if (!ctx) return -1;
  return set_err(ctx, IMCOM_ERR_STATE, "learned-kappa MLP not built");
}

extern "C" int imcom_gpu_bisect_kappa_learned(imcom_ctx* ctx, int, double, double, double, double,
                                              int, double, double*, double*, int*, int*) {
  if (!ctx) return -1;
  return set_err(ctx, IMCOM_ERR_STATE, "learned-kappa bisection not built");
}
