// ctx.cu -- context, module state upload/download and the cache-read branches
// of the reference's imcom_get_* routines.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <mutex>

#include "common.cuh"

namespace imcom {

unsigned long long g_launches = 0;

int set_err(imcom_ctx* c, int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

std::recursive_mutex& alloc_mutex() {
  static std::recursive_mutex mu;
  return mu;
}

int ensure_buf(imcom_ctx* ctx, void** p, size_t& have, size_t need) {
  if (*p && have >= need) return 0;
  std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
  if (*p) cudaFree(*p);
  *p = nullptr;
  have = 0;
  if (need == 0) return 0;
  cudaError_t e = cudaMalloc(p, need);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_err(ctx, IMCOM_ERR_ALLOC, "cudaMalloc(%zu bytes): %s", need,
                   cudaGetErrorString(e));
  }
  have = need;
  return 0;
}

// cuFFT plans shared by every context of the process, keyed by (device,
// type, side, batch).  Planning a size costs tens to hundreds of
// milliseconds of host time (Bluestein sizes included) and the PSF side
// follows each patch's input footprint, so contexts solving a run of patches
// side by side plan each size once between them.  Plans have no work area of
// their own: each execution binds the calling context's work area and stream
// and enqueues under one lock, so two contexts never race on a plan's state.
// Plans live until the last context is destroyed; past kMaxPlans the device
// is synchronised before the least recently used plan is dropped (a plan is
// never destroyed while its kernels may be in flight).
namespace {
struct SharedPlan {
  int dev, type, side, batch;
  cufftHandle h;
  size_t work;
  unsigned long long used;
};
std::mutex g_fft_mu;
std::vector<SharedPlan> g_fft_plans;
unsigned long long g_fft_clock = 0;
int g_fft_contexts = 0;
constexpr size_t kMaxPlans = 512;

int fft_exec(imcom_ctx* ctx, cufftType type, int side, int batch, void* in, void* out, int dir) {
  std::lock_guard<std::mutex> lk(g_fft_mu);
  size_t hit = g_fft_plans.size();
  for (size_t i = 0; i < g_fft_plans.size(); ++i) {
    const SharedPlan& f = g_fft_plans[i];
    if (f.dev == ctx->device && f.type == (int)type && f.side == side && f.batch == batch) hit = i;
  }
  if (hit == g_fft_plans.size()) {
    std::lock_guard<std::recursive_mutex> lk_alloc(alloc_mutex());
    if (g_fft_plans.size() >= kMaxPlans) {
      size_t lru = 0;
      for (size_t i = 1; i < g_fft_plans.size(); ++i)
        if (g_fft_plans[i].used < g_fft_plans[lru].used) lru = i;
      cudaSetDevice(g_fft_plans[lru].dev);
      cudaDeviceSynchronize();
      cufftDestroy(g_fft_plans[lru].h);
      g_fft_plans.erase(g_fft_plans.begin() + lru);
      cudaSetDevice(ctx->device);
    }
    SharedPlan f{ctx->device, (int)type, side, batch, 0, 0, 0};
    IMC_CUFFT(cufftCreate(&f.h));
    cufftResult r = cufftSetAutoAllocation(f.h, 0);
    int dims[2] = {side, side};
    long long dist_in = (long long)side * side;
    long long dist_out = type == CUFFT_D2Z ? (long long)side * (side / 2 + 1) : dist_in;
    if (r == CUFFT_SUCCESS)
      r = cufftMakePlanMany(f.h, 2, dims, nullptr, 1, (int)dist_in, nullptr, 1, (int)dist_out,
                            type, batch, &f.work);
    if (r != CUFFT_SUCCESS) {
      cufftDestroy(f.h);
      return set_err(ctx, IMCOM_ERR_CUDA, "cuFFT plan %dx%d x%d (type %d): error %d", side, side,
                     batch, (int)type, (int)r);
    }
    g_fft_plans.push_back(f);
    hit = g_fft_plans.size() - 1;
  }
  SharedPlan& f = g_fft_plans[hit];
  f.used = ++g_fft_clock;
  IMC_TRY(ensure_buf(ctx, &ctx->fft_work, ctx->fft_work_bytes, f.work));
  if (f.work) IMC_CUFFT(cufftSetWorkArea(f.h, ctx->fft_work));
  IMC_CUFFT(cufftSetStream(f.h, ctx->stream));
  if (type == CUFFT_Z2Z)
    IMC_CUFFT(cufftExecZ2Z(f.h, (cufftDoubleComplex*)in, (cufftDoubleComplex*)out, dir));
  else
    IMC_CUFFT(cufftExecD2Z(f.h, (cufftDoubleReal*)in, (cufftDoubleComplex*)out));
  return 0;
}
}  // namespace

int fft_z2z(imcom_ctx* ctx, int side, int batch, double2* data, int dir) {
  return fft_exec(ctx, CUFFT_Z2Z, side, batch, data, data, dir);
}

int fft_d2z(imcom_ctx* ctx, int side, int batch, const double* in, double2* out) {
  return fft_exec(ctx, CUFFT_D2Z, side, batch, const_cast<double*>(in), out, 0);
}

void fft_attach() {
  std::lock_guard<std::mutex> lk(g_fft_mu);
  ++g_fft_contexts;
}

void fft_free(imcom_ctx* ctx) {
  {
    std::lock_guard<std::mutex> lk(g_fft_mu);
    if (--g_fft_contexts == 0) {
      // every context's stream has drained (destroy synchronises first)
      std::lock_guard<std::recursive_mutex> lk_alloc(alloc_mutex());
      for (auto& f : g_fft_plans) cufftDestroy(f.h);
      g_fft_plans.clear();
    }
  }
  std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
  if (ctx->fft_work) cudaFree(ctx->fft_work);
  ctx->fft_work = nullptr;
  ctx->fft_work_bytes = 0;
}

int ensure_mat(imcom_ctx* ctx, DMat& M, long long rows, long long cols) {
  long long ld = pad_ld(rows);
  size_t need = (size_t)ld * (size_t)cols * sizeof(double);
  if (M.p && M.ld == ld && M.cols == cols && M.rows == rows) return 0;
  if (M.p && M.cap >= need) {
    M.rows = rows;
    M.cols = cols;
    M.ld = ld;
    return 0;
  }
  std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
  if (M.p) cudaFree(M.p);
  M.p = nullptr;
  M.cap = 0;
  cudaError_t e = cudaMalloc(&M.p, need);
  if (e != cudaSuccess) {
    M.p = nullptr;
    cudaGetLastError();
    return set_err(ctx, IMCOM_ERR_ALLOC, "cudaMalloc(%zu bytes) for %lldx%lld matrix: %s",
                   need, rows, cols, cudaGetErrorString(e));
  }
  M.cap = need;
  M.rows = rows;
  M.cols = cols;
  M.ld = ld;
  return 0;
}

template <class T>
int ensure_vec(imcom_ctx* ctx, T** p, size_t count) {
  const size_t need = count * sizeof(T) + 256;
  size_t& cap = ctx->vec_cap[reinterpret_cast<void**>(p)];
  if (*p && cap >= need) return 0;
  std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
  if (*p) cudaFree(*p);
  *p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void**)p, need);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_err(ctx, IMCOM_ERR_ALLOC, "cudaMalloc(%zu): %s", count * sizeof(T),
                   cudaGetErrorString(e));
  }
  cap = need;
  return 0;
}
template int ensure_vec<double>(imcom_ctx*, double**, size_t);
template int ensure_vec<int>(imcom_ctx*, int**, size_t);
template int ensure_vec<float>(imcom_ctx*, float**, size_t);
template int ensure_vec<double2>(imcom_ctx*, double2**, size_t);
template int ensure_vec<float2>(imcom_ctx*, float2**, size_t);

int upload_mat(imcom_ctx* ctx, DMat& M, const double* host, long long rows,
               long long cols) {
  IMC_TRY(ensure_mat(ctx, M, rows, cols));
  IMC_CUDA(cudaMemcpy2DAsync(M.p, M.ld * sizeof(double), host, rows * sizeof(double),
                             rows * sizeof(double), cols, cudaMemcpyHostToDevice,
                             ctx->stream));
  return 0;
}

int download_mat(imcom_ctx* ctx, const DMat& M, double* host) {
  IMC_CUDA(cudaMemcpy2DAsync(host, M.rows * sizeof(double), M.p, M.ld * sizeof(double),
                             M.rows * sizeof(double), M.cols, cudaMemcpyDeviceToHost,
                             ctx->stream));
  return 0;
}

void stage_begin(imcom_ctx* ctx, Stage s) {
  if (!ctx->ev0[s]) {
    cudaEventCreate(&ctx->ev0[s]);
    cudaEventCreate(&ctx->ev1[s]);
  }
  cudaEventRecord(ctx->ev0[s], ctx->stream);
}

void stage_end(imcom_ctx* ctx, Stage s) {
  cudaEventRecord(ctx->ev1[s], ctx->stream);
  ctx->ev_used[s] = true;
}

int device_sm_count(int d) {
  static int cached[64] = {0};
  if (d >= 0 && d < 64 && cached[d]) return cached[d];
  int v = 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
  if (d >= 0 && d < 64) cached[d] = v;
  return v;
}

// SMs this context sizes its persistent and cooperative grids for: the whole
// device, or the share set with IMCOM_OPT_SM_SHARE (contexts that solve
// independent patches side by side each take a share).
int sm_count(imcom_ctx* ctx) {
  const int v = device_sm_count(ctx->device);
  return (ctx->sm_share > 0 && ctx->sm_share < v) ? ctx->sm_share : v;
}

}  // namespace imcom

using namespace imcom;

static int check_finite(imcom_ctx* ctx, const double* p, long long count, const char* what) {
  if (!p) return 0;
  for (long long k = 0; k < count; ++k)
    if (!std::isfinite(p[k]))
      return set_err(ctx, IMCOM_ERR_NOT_FINITE, "non-finite value in %s at index %lld", what, k);
  return 0;
}

// First index of a non-finite value in a device array (atomicMin into *first,
// which starts at LLONG_MAX).
__global__ void first_nonfinite_kernel(const double* __restrict__ p, long long count,
                                       unsigned long long* first) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x)
    if (!isfinite(p[k])) atomicMin(first, (unsigned long long)k);
}

// Finiteness check of arrays already on the device (large PSF arrays: one
// pass on the GPU instead of a host pass over host memory).
static int check_finite_dev(imcom_ctx* ctx, const double* d, long long count, const char* what) {
  unsigned long long* first = reinterpret_cast<unsigned long long*>(ctx->flags + 28);
  IMC_CUDA(cudaMemsetAsync(first, 0xff, sizeof(unsigned long long), ctx->stream));
  const int blocks = (int)std::min<long long>((count + 255) / 256, 4 * 148);
  first_nonfinite_kernel<<<blocks, 256, 0, ctx->stream>>>(d, count, first);
  IMC_LAUNCH();
  unsigned long long h = 0;
  IMC_CUDA(cudaMemcpyAsync(&h, first, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h != ~0ULL)
    return set_err(ctx, IMCOM_ERR_NOT_FINITE, "non-finite value in %s at index %lld", what,
                   (long long)h);
  return 0;
}

extern "C" {

int imcom_gpu_create(int device, imcom_ctx** out) {
  if (!out) return -2;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return IMCOM_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return -1;
  imcom_ctx* ctx = new imcom_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return IMCOM_ERR_CUDA;
  }
  {
    std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
    if (cudaMalloc(&ctx->flags, 64 * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      cudaStreamDestroy(ctx->stream);
      delete ctx;
      return IMCOM_ERR_ALLOC;
    }
  }
  fft_attach();
  if (cudaMemsetAsync(ctx->flags, 0, 64 * sizeof(int), ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    imcom_gpu_destroy(ctx);
    return IMCOM_ERR_CUDA;
  }
  *out = ctx;
  return 0;
}

int imcom_gpu_destroy(imcom_ctx* ctx) {
  if (!ctx) return 0;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  {
    // released before fft_free, which takes the plan cache's lock first
    std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
    eig_free(ctx);
    split_release(ctx);
    void* ptrs[] = {ctx->x, ctx->y, ctx->X, ctx->Y, ctx->I, ctx->Nd, ctx->exp_i, ctx->G,
                    ctx->Gamma, ctx->Gt, ctx->Gammat, ctx->A.p, ctx->Q.p, ctx->B.p, ctx->P.p,
                    ctx->T.p, ctx->Pt.p, ctx->L, ctx->K, ctx->US, ctx->H, ctx->S, ctx->U,
                    ctx->nev, ctx->flags, ctx->tables, ctx->fftbuf, ctx->mlp.w, ctx->feat, ctx->guess,
                    ctx->gemm_ws, ctx->fb, ctx->train_buf, ctx->band, ctx->jac_buf,
                    ctx->stacks.p, ctx->stack_H.p, ctx->fft_tw, ctx->r2c_tw, ctx->nbr, ctx->band_seg};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
  delete[] ctx->rot;
  fft_free(ctx);
  for (int s = 0; s < ST_N; ++s) {
    if (ctx->ev0[s]) cudaEventDestroy(ctx->ev0[s]);
    if (ctx->ev1[s]) cudaEventDestroy(ctx->ev1[s]);
  }
  for (auto& pair : ctx->tab_ev)
    for (cudaEvent_t e : pair)
      if (e) cudaEventDestroy(e);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return 0;
}

const char* imcom_gpu_last_error(const imcom_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

int imcom_gpu_synchronize(imcom_ctx* ctx) {
  if (!ctx) return -1;
  cudaSetDevice(ctx->device);
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  IMC_CUDA(cudaGetLastError());
  return 0;
}

int imcom_gpu_set_option(imcom_ctx* ctx, int option, long long value) {
  if (!ctx) return -1;
  switch (option) {
    case IMCOM_OPT_EIGENSOLVER:
      if (value != IMCOM_EIGH_DC && value != IMCOM_EIGH_JACOBI && value != IMCOM_EIGH_LIBRARY &&
          value != IMCOM_EIGH_TWOSTAGE)
        return -3;
      ctx->eig_mode = (int)value;
      return 0;
    case IMCOM_OPT_EIGEN_MAXITER:
      if (value < 0) return -3;
      ctx->eig_maxiter = value;
      return 0;
    case IMCOM_OPT_KAPPA_START:
      if (value != 0 && value != 1) return -3;
      ctx->kappa_nonet = (int)value;
      return 0;
    case IMCOM_OPT_DC_MAXITER:
      if (value < 0 || value > 1000000) return -3;
      ctx->dc_maxiter = (int)value;
      return 0;
    case IMCOM_OPT_STALL_TEST:
      if (value < 0 || value > (IMCOM_STALL_SPLIT | IMCOM_STALL_TRIDIAG)) return -3;
      ctx->stall_test = (int)value;
      return 0;
    case IMCOM_OPT_BISECT_KERNEL:
      if (value < IMCOM_BISECT_AUTO || value > IMCOM_BISECT_RESIDENT) return -3;
      ctx->bisect_kernel = (int)value;
      return 0;
    case IMCOM_OPT_SM_SHARE:
      if (value < 0 || value > 1024) return -3;
      ctx->sm_share = (int)value;
      return 0;
    case IMCOM_OPT_TAIL_CTAS:
      if (value != 0 && value != -1 && value != 8 && value != 16) return -3;
      ctx->tail_ctas = (int)value;
      return 0;
    case IMCOM_OPT_KAPPA_FEATURES:
      if (value != 0 && value != 1) return -3;
      ctx->kappa_feat = (int)value;
      return 0;
    case IMCOM_OPT_TABLE_FFT:
      if (value != IMCOM_TABLE_FFT_CUFFT && value != IMCOM_TABLE_FFT_OWN &&
          value != IMCOM_TABLE_FFT_AUTO)
        return -3;
      ctx->table_fft = (int)value;
      return 0;
    case IMCOM_OPT_STACK_KERNEL:
      if (value != IMCOM_STACKS_GEMM && value != IMCOM_STACKS_STREAM && value != IMCOM_STACKS_AUTO)
        return -3;
      ctx->stack_kernel = (int)value;
      return 0;
    case IMCOM_OPT_BISECT_CTAS_PER_SM:
      if (value < 0 || value > 64) return -3;
      ctx->bisect_ctas = (int)value;
      return 0;
    case IMCOM_OPT_PRECISION:
      if (value != IMCOM_PREC_FP64 && value != IMCOM_PREC_SPLIT) return -3;
      ctx->prec = (int)value;
      return 0;
    case IMCOM_OPT_SPLIT_SLICES_P:
    case IMCOM_OPT_SPLIT_SLICES_T:
      if (value < 2 || value > 8) return -3;
      (option == IMCOM_OPT_SPLIT_SLICES_P ? ctx->split_SP : ctx->split_ST) = (int)value;
      return 0;
    case IMCOM_OPT_SPLIT_TOL_US:
    case IMCOM_OPT_SPLIT_TOL_T:
      if (value < 0 || value > 300) return -3;
      (option == IMCOM_OPT_SPLIT_TOL_US ? ctx->split_tol_us : ctx->split_tol_t) =
          std::pow(10.0, -(double)value);
      return 0;
    default:
      return -2;
  }
}

int imcom_gpu_set_inputs(imcom_ctx* ctx, int n, int m, const double* x_i, const double* y_i,
                         const int* exp_i, const double* X_a, const double* Y_a,
                         const double* I_i, const double* Ndiag, double psfxscale,
                         double psfyscale) {
  if (!ctx) return -1;
  if (n <= 0) return -2;
  if (m <= 0) return -3;
  if (!x_i) return -4;
  if (!y_i) return -5;
  if (!exp_i) return -6;
  if (!X_a) return -7;
  if (!Y_a) return -8;
  if (!(psfxscale > 0)) return -11;
  if (!(psfyscale > 0)) return -12;
  for (int i = 0; i < n; ++i)
    if (exp_i[i] < 1) return set_err(ctx, -6, "exp_i(%d) = %d < 1", i + 1, exp_i[i]);
  for (int i = 1; i < n; ++i)
    if (exp_i[i] < exp_i[i - 1])
      return set_err(ctx, -6, "exp_i must be non-decreasing (exposure-major order)");
  IMC_TRY(check_finite(ctx, x_i, n, "x_i"));
  IMC_TRY(check_finite(ctx, y_i, n, "y_i"));
  IMC_TRY(check_finite(ctx, X_a, m, "X_a"));
  IMC_TRY(check_finite(ctx, Y_a, m, "Y_a"));
  IMC_TRY(check_finite(ctx, I_i, n, "I_i"));
  IMC_TRY(check_finite(ctx, Ndiag, n, "Ndiag"));
  cudaSetDevice(ctx->device);
  if (n != ctx->n || m != ctx->m) {
    ctx->have_A = ctx->have_QL = ctx->have_B = ctx->have_P = ctx->have_K = ctx->have_T = false;
  }
  ctx->n = n;
  ctx->m = m;
  ctx->psfx = psfxscale;
  ctx->psfy = psfyscale;
  IMC_TRY(ensure_vec(ctx, &ctx->x, n));
  IMC_TRY(ensure_vec(ctx, &ctx->y, n));
  IMC_TRY(ensure_vec(ctx, &ctx->I, n));
  IMC_TRY(ensure_vec(ctx, &ctx->Nd, n));
  IMC_TRY(ensure_vec(ctx, &ctx->exp_i, n));
  IMC_TRY(ensure_vec(ctx, &ctx->X, m));
  IMC_TRY(ensure_vec(ctx, &ctx->Y, m));
  IMC_TRY(ensure_vec(ctx, &ctx->L, n));
  IMC_TRY(ensure_vec(ctx, &ctx->K, m));
  IMC_TRY(ensure_vec(ctx, &ctx->US, m));
  IMC_TRY(ensure_vec(ctx, &ctx->H, m));
  IMC_TRY(ensure_vec(ctx, &ctx->S, m));
  IMC_TRY(ensure_vec(ctx, &ctx->U, m));
  IMC_TRY(ensure_vec(ctx, &ctx->nev, m));
  ctx->max_exp = 0;
  for (int i = 0; i < n; ++i) ctx->max_exp = exp_i[i] > ctx->max_exp ? exp_i[i] : ctx->max_exp;
  IMC_CUDA(cudaMemcpyAsync(ctx->x, x_i, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(ctx->y, y_i, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(ctx->exp_i, exp_i, n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(ctx->X, X_a, m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(ctx->Y, Y_a, m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  ctx->have_I = I_i != nullptr;
  ctx->nbr_valid = false;  // the neighbour table belongs to the previous inputs
  ctx->have_N = Ndiag != nullptr;
  if (I_i)
    IMC_CUDA(cudaMemcpyAsync(ctx->I, I_i, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (Ndiag)
    IMC_CUDA(cudaMemcpyAsync(ctx->Nd, Ndiag, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int imcom_gpu_set_psfs(imcom_ctx* ctx, int nps, int nexppsf, int psfconst,
                       const double* G_unrot, const double* rotangdeg, const double* Gamma) {
  if (!ctx) return -1;
  if (nps < 2) return -2;
  if (nexppsf < 1) return -3;
  if (psfconst != 0 && psfconst != 1)
    return set_err(ctx, -4, "IMCOM ERROR: PSFCONST must be 1 or 0!");
  if (psfconst == 1 && nexppsf != 1) return -3;
  if (!G_unrot) return -5;
  if (!rotangdeg) return -6;
  if (!Gamma) return -7;
  size_t ps2 = (size_t)nps * nps;
  IMC_TRY(check_finite(ctx, rotangdeg, nexppsf, "rotangdeg"));
  cudaSetDevice(ctx->device);
  ctx->nps = nps;
  ctx->nexppsf = nexppsf;
  ctx->psfconst = psfconst;
  IMC_TRY(ensure_vec(ctx, &ctx->G, ps2 * nexppsf));
  IMC_TRY(ensure_vec(ctx, &ctx->Gamma, ps2));
  IMC_TRY(ensure_vec(ctx, &ctx->Gt, ps2 * nexppsf));
  IMC_TRY(ensure_vec(ctx, &ctx->Gammat, ps2));
  delete[] ctx->rot;
  ctx->rot = new double[nexppsf];
  std::memcpy(ctx->rot, rotangdeg, nexppsf * sizeof(double));
  IMC_CUDA(cudaMemcpyAsync(ctx->G, G_unrot, ps2 * nexppsf * sizeof(double),
                           cudaMemcpyHostToDevice, ctx->stream));
  IMC_CUDA(cudaMemcpyAsync(ctx->Gamma, Gamma, ps2 * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
  ctx->have_psf = false;
  IMC_TRY(check_finite_dev(ctx, ctx->G, (long long)(ps2 * nexppsf), "G_unrot"));
  IMC_TRY(check_finite_dev(ctx, ctx->Gamma, (long long)ps2, "Gamma"));
  ctx->have_psf = true;
  ctx->have_spectra = false;
  return 0;
}

int imcom_gpu_load_A(imcom_ctx* ctx, const double* A) {
  if (!ctx) return -1;
  if (!A) return -2;
  if (ctx->n <= 0) return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_set_inputs has not run");
  cudaSetDevice(ctx->device);
  IMC_TRY(upload_mat(ctx, ctx->A, A, ctx->n, ctx->n));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_A = true;
  return 0;
}

int imcom_gpu_load_QL(imcom_ctx* ctx, const double* Q, const double* L) {
  if (!ctx) return -1;
  if (!Q) return -2;
  if (!L) return -3;
  if (ctx->n <= 0) return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_set_inputs has not run");
  cudaSetDevice(ctx->device);
  IMC_TRY(upload_mat(ctx, ctx->Q, Q, ctx->n, ctx->n));
  IMC_CUDA(cudaMemcpyAsync(ctx->L, L, ctx->n * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_QL = true;
  ctx->sq_P_valid = ctx->sq_T_valid = false;
  return 0;
}

int imcom_gpu_load_B(imcom_ctx* ctx, const double* B) {
  if (!ctx) return -1;
  if (!B) return -2;
  if (ctx->n <= 0) return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_set_inputs has not run");
  cudaSetDevice(ctx->device);
  IMC_TRY(upload_mat(ctx, ctx->B, B, ctx->n, ctx->m));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_B = true;
  return 0;
}

int imcom_gpu_load_P(imcom_ctx* ctx, const double* P) {
  if (!ctx) return -1;
  if (!P) return -2;
  if (ctx->n <= 0) return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_set_inputs has not run");
  cudaSetDevice(ctx->device);
  IMC_TRY(upload_mat(ctx, ctx->P, P, ctx->n, ctx->m));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_P = true;
  ctx->p_split = false;
  return 0;
}

int imcom_gpu_load_T(imcom_ctx* ctx, const double* T) {
  if (!ctx) return -1;
  if (!T) return -2;
  if (ctx->n <= 0) return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_set_inputs has not run");
  cudaSetDevice(ctx->device);
  IMC_TRY(upload_mat(ctx, ctx->T, T, ctx->n, ctx->m));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_T = true;
  return 0;
}

int imcom_gpu_load_K(imcom_ctx* ctx, const double* K) {
  if (!ctx) return -1;
  if (!K) return -2;
  if (ctx->m <= 0) return set_err(ctx, IMCOM_ERR_STATE, "imcom_gpu_set_inputs has not run");
  cudaSetDevice(ctx->device);
  IMC_CUDA(cudaMemcpyAsync(ctx->K, K, ctx->m * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_K = true;
  ctx->have_Pt = false;
  ctx->have_T = false;
  return 0;
}

int imcom_gpu_free_AB(imcom_ctx* ctx) {
  if (!ctx) return -1;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  std::lock_guard<std::recursive_mutex> lk(alloc_mutex());
  if (ctx->A.p) cudaFree(ctx->A.p);
  if (ctx->B.p) cudaFree(ctx->B.p);
  ctx->A = DMat();
  ctx->B = DMat();
  ctx->have_A = ctx->have_B = false;
  return 0;
}

int imcom_gpu_device_buffer(imcom_ctx* ctx, char which, void** dptr, long long* ld) {
  if (!ctx) return -1;
  if (!dptr) return -3;
  long long l = 0;
  void* p = nullptr;
  switch (which) {
    case 'A': p = ctx->A.p; l = ctx->A.ld; break;
    case 'Q': p = ctx->Q.p; l = ctx->Q.ld; break;
    case 'B': p = ctx->B.p; l = ctx->B.ld; break;
    case 'P': p = ctx->P.p; l = ctx->P.ld; break;
    case 'T': p = ctx->T.p; l = ctx->T.ld; break;
    case 'W': p = ctx->Pt.p; l = ctx->Pt.ld; break;
    case 'L': p = ctx->L; l = ctx->n; break;
    case 'K': p = ctx->K; l = ctx->m; break;
    case 'H': p = ctx->H; l = ctx->m; break;
    case 'S': p = ctx->S; l = ctx->m; break;
    case 'U': p = ctx->U; l = ctx->m; break;
    default: return -2;
  }
  *dptr = p;
  if (ld) *ld = l;
  return p ? 0 : set_err(ctx, IMCOM_ERR_STATE, "buffer %c not allocated", which);
}

int imcom_gpu_launch_count(imcom_ctx* ctx, long long* count) {
  if (!ctx) return -1;
  if (!count) return -2;
  *count = (long long)__atomic_load_n(&g_launches, __ATOMIC_RELAXED);
  return 0;
}

int imcom_gpu_get_stream(imcom_ctx* ctx, void** stream) {
  if (!ctx) return -1;
  if (!stream) return -2;
  *stream = (void*)ctx->stream;
  return 0;
}

int imcom_gpu_table_times(imcom_ctx* ctx, double* ms2) {
  if (!ctx) return -1;
  if (!ms2) return -2;
  cudaSetDevice(ctx->device);
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < 2; ++k) {
    float t = 0.f;
    ms2[k] = (ctx->tab_used[k] &&
              cudaEventElapsedTime(&t, ctx->tab_ev[k][0], ctx->tab_ev[k][1]) == cudaSuccess)
                 ? t
                 : 0.0;
  }
  cudaGetLastError();
  return 0;
}

int imcom_gpu_stage_times(imcom_ctx* ctx, double* ms) {
  if (!ctx) return -1;
  if (!ms) return -2;
  cudaSetDevice(ctx->device);
  IMC_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int s = 0; s < ST_N; ++s) {
    float t = 0.f;
    if (ctx->ev_used[s] && cudaEventElapsedTime(&t, ctx->ev0[s], ctx->ev1[s]) == cudaSuccess)
      ms[s] = t;
    else
      ms[s] = 0.0;
  }
  cudaGetLastError();
  return 0;
}

}  // extern "C"
