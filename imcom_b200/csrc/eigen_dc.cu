// eigen_dc.cu -- placeholder entry points of the own eigensolvers.
#include "common.cuh"
#include "eigen.cuh"

namespace imcom {

int eigen_dc(imcom_ctx* ctx, const DMat& A, DMat& W, double* w) {
  (void)A; (void)W; (void)w;
  return set_err(ctx, IMCOM_ERR_STATE, "divide-and-conquer eigensolver not built");
}

int eigen_jacobi(imcom_ctx* ctx, const DMat& A, DMat& W, double* w) {
  (void)A; (void)W; (void)w;
  return set_err(ctx, IMCOM_ERR_STATE, "Jacobi eigensolver not built");
}

}  // namespace imcom
