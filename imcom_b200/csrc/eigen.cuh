// eigen.cuh -- shared state of the eigensolvers.
#pragma once

#include "common.cuh"

namespace imcom {

struct EigWork {
  DMat W;   // ascending eigenvectors (solver output)
  DMat Z;   // scratch matrices
  DMat V;
  DMat U;   // divide-and-conquer node blocks (U | G | OUT)
  double* w = nullptr;  // ascending eigenvalues
  size_t w_cap = 0;
  void* buf = nullptr;  // general scratch
  size_t buf_bytes = 0;
  void* solver = nullptr;  // cuSOLVER handle (comparison baseline only)
  // the tridiagonalisation's launch sequence as a CUDA graph, for the size
  // and buffers of trd_key
  static constexpr int kTrdKey = 24;
  long long trd_key[kTrdKey] = {};
  void* trd_exec = nullptr;              // cudaGraphExec_t
  unsigned long long trd_launches = 0;   // kernel launches one replay stands for
  bool trd_graph_off = false;            // capture refused: launch directly
};

EigWork* eig_work(imcom_ctx* ctx);
int eig_buf(imcom_ctx* ctx, size_t bytes);
int copy_mat(imcom_ctx* ctx, const double* A, long long lda, double* B, long long ldb, int rows,
             int cols);

// Two-stage tridiagonalisation (eigen_2s.cu): scratch bytes for order n,
// the reduction of Aw to (d, e) with the stage-1 reflectors in Vall/tau and
// the stage-2 ones in scratch, and the stage-2 back-transformation Z <- Q2 Z.
size_t twostage_bytes(int n);
int twostage_tridiag(imcom_ctx* ctx, DMat& Aw, DMat& Vall, double* d, double* e, double* tau,
                     double* W, long long ldw, double* XY, void* scratch, long long spin);
int twostage_backtransform2(imcom_ctx* ctx, int n, void* scratch, double* Z, long long ldz);

// Keep-if-large-enough vector allocation.
template <class T>
inline int ensure_vec_keep(imcom_ctx* ctx, T** p, size_t& cap, size_t count) {
  size_t bytes = count * sizeof(T);
  void* v = *p;
  int s = ensure_buf(ctx, &v, cap, bytes);
  *p = (T*)v;
  return s;
}

}  // namespace imcom
