// Linear transient conduction on the device: the d-form generalized
// trapezoid of linear_nonstat_solv_dform (TRFEL/SRC/npsolvert.cpp:1071-1272).
//
// Reference step (npsolvert.cpp:1146-1230):
//   dd = d + (1 - alpha) dt v                          predictor
//   p  = C dd                                          Cmat->gmxv
//   A  = alpha dt K + C                                scalgm, addgm (same pattern)
//   f  = alpha dt rhs + p                              rhs = trfel_right_hand_side
//   A d = f                                            ssle->solve_system (x starts from d)
//   v  = (d - dd) / dt / alpha
// The v-form of nonstat_solv_vform_comp (npsolvert.cpp:62, one_step_linear
// at 367-480) solves for the rates instead:
//   dd = d + (1 - alpha) dt v;  p = K dd;  f = rhs - p;  A v = f (x starts
//   from v);  d = dd + alpha dt v
// The reference re-integrates K and C every step (npsolvert.cpp:1160,1170);
// for linear materials and a fixed time step their values do not change, so
// here A is formed once on the device and every step is two vector kernels,
// one SpMV with C and one PCG solve, with no host traffic between steps.
#include <cmath>
#include <cstring>
#include <vector>

#include "sgpu_internal.cuh"

namespace sgpu {
int pcg_run(sgpu_matrix m, int64_t ni, double res, double zero, int64_t iv, int crit, int prec, int mode,
            int64_t *ani, double *ares, sgpu_solve_info *info);
int pcg_prepare(sgpu_matrix m, bool mixed);
double *work_x(sgpu_matrix m);
double *work_f(sgpu_matrix m);
}  // namespace sgpu

using namespace sgpu;

namespace {

constexpr int TPB = 256;

inline int blocks_for(int64_t n) {
  int64_t b = (n + TPB - 1) / TPB;
  return (int)(b < 1 ? 1 : (b > 65536 ? 65536 : b));
}

__global__ void k_combine(int64_t nnz, const double *__restrict__ ka, const double *__restrict__ ca, double a,
                          double b, double *__restrict__ out) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
    out[k] = ka[k] * a + ca[k] * b;
}

// dd = d + (1 - alpha) dt v
__global__ void k_predict(int n, const double *__restrict__ d, const double *__restrict__ v, double c,
                          double *__restrict__ dd) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dd[i] = d[i] + c * v[i];
}

// f = alpha dt rhs + p
__global__ void k_rhs(int n, const double *__restrict__ rhs, const double *__restrict__ p, double c,
                      double *__restrict__ f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) f[i] = rhs[i] * c + p[i];
}

// v-form: f = rhs - p
__global__ void k_rhs_v(int n, const double *__restrict__ rhs, const double *__restrict__ p, double *__restrict__ f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) f[i] = rhs[i] - p[i];
}

// v-form: d = dd + alpha dt v
__global__ void k_value(int n, const double *__restrict__ dd, const double *__restrict__ v, double c,
                        double *__restrict__ d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = dd[i] + c * v[i];
}

// v = (d - dd) / dt / alpha
__global__ void k_velocity(int n, const double *__restrict__ d, const double *__restrict__ dd, double dt,
                           double alpha, double *__restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = (d[i] - dd[i]) / dt / alpha;
}

bool same_pattern(sgpu_matrix a, sgpu_matrix b) {
  return a->n == b->n && a->csr.nnz == b->csr.nnz && a->src_negm == b->src_negm;
}

}  // namespace

namespace {
int transient(sgpu_matrix K, sgpu_matrix C, const double *rhs, double *d, double *v, double dt, double alpha,
              int64_t nsteps, int64_t ni, double res, double zero, int64_t iv, int32_t prec, int32_t mode,
              int64_t *step_iterations, sgpu_solve_info *info, bool vform) {
  if (!K || !C || !rhs || !d || !v) return fail(SGPU_BAD_INPUT, "null argument");
  if (!(dt > 0.0) || !(alpha > 0.0) || alpha > 1.0) return fail(SGPU_BAD_INPUT, "need dt > 0 and 0 < alpha <= 1");
  if (nsteps < 0) return fail(SGPU_BAD_INPUT, "negative step count");
  if (prec != SGPU_PREC_JACOBI && prec != SGPU_PREC_AGG) return fail(SGPU_BAD_INPUT, "prec: Jacobi or aggregation");
  if (info) memset(info, 0, sizeof(*info));
  sgpu_matrix A = nullptr;
  // A = alpha dt K + C (scalgm then addgm, GEFEL/gmatrix.cpp:1848/1791)
  SGPU_TRY(sgpu_matrix_combine(K, C, dt * alpha, 1.0, &A));
  const int64_t n = K->n;
  int status = SGPU_OK;
  DevBuf<double> d_d, v_d, dd_d, rhs_d;
  auto cleanup = [&](int st) {
    cudaStream_t s = A->own_stream;
    cudaEvent_t e0 = A->ev0, e1 = A->ev1;
    cudaStreamSynchronize(A->stream);
    delete A;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    return st;
  };
  int st;
  if ((st = d_d.alloc(n)) || (st = v_d.alloc(n)) || (st = dd_d.alloc(n)) || (st = rhs_d.alloc(n)) ||
      (st = pcg_prepare(A, mode == SGPU_MIXED)) || (st = pcg_prepare(C, false)))
    return cleanup(st);
  cudaStream_t s = A->stream;
  cudaStream_t c_stream_saved = C->stream, k_stream_saved = K->stream;
  C->stream = s;  // C's (d-form) or K's (v-form) products run on A's stream for ordering
  K->stream = s;
  cudaMemcpyAsync(d_d.p, d, n * sizeof(double), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(v_d.p, v, n * sizeof(double), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(rhs_d.p, rhs, n * sizeof(double), cudaMemcpyHostToDevice, s);
  const int vb = blocks_for(n);
  int64_t total_its = 0;
  double total_ms = 0.0, last_true = 0.0, setup_ms = 0.0;
  int32_t levels = 0, coarse_n = 0;
  for (int64_t step = 0; step < nsteps; step++) {
    k_predict<<<vb, TPB, 0, s>>>((int)n, d_d.p, v_d.p, (1.0 - alpha) * dt, dd_d.p);
    count_launches(1);
    if (vform) {
      st = spmv64(K, dd_d.p, A->w.p.p, s);  // p = K dd  (A's p buffer as scratch)
      if (st != SGPU_OK) break;
      k_rhs_v<<<vb, TPB, 0, s>>>((int)n, rhs_d.p, A->w.p.p, work_f(A));
      count_launches(1);
      cudaMemcpyAsync(work_x(A), v_d.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    } else {
      st = spmv64(C, dd_d.p, A->w.p.p, s);  // p = C dd
      if (st != SGPU_OK) break;
      k_rhs<<<vb, TPB, 0, s>>>((int)n, rhs_d.p, A->w.p.p, alpha * dt, work_f(A));
      count_launches(1);
      cudaMemcpyAsync(work_x(A), d_d.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    }
    sgpu_solve_info si;
    memset(&si, 0, sizeof(si));
    int64_t ani = -1;
    double ares = 0.0;
    st = pcg_run(A, ni, res, zero, iv, SGPU_CRIT_SCR_PREC, prec, mode, &ani, &ares, &si);
    if (st == SGPU_BAD_INPUT || st == SGPU_CUDA_ERROR) break;
    if (st != SGPU_OK && status == SGPU_OK) status = st;
    st = SGPU_OK;
    if (step_iterations) step_iterations[step] = si.iterations;
    total_its += si.iterations;
    total_ms += si.solve_ms + si.precond_setup_ms;
    setup_ms += si.precond_setup_ms;
    levels = si.precond_levels;
    coarse_n = si.precond_coarse_n;
    last_true = si.true_relres;
    if (vform) {
      cudaMemcpyAsync(v_d.p, work_x(A), n * sizeof(double), cudaMemcpyDeviceToDevice, s);
      k_value<<<vb, TPB, 0, s>>>((int)n, dd_d.p, v_d.p, alpha * dt, d_d.p);
    } else {
      cudaMemcpyAsync(d_d.p, work_x(A), n * sizeof(double), cudaMemcpyDeviceToDevice, s);
      k_velocity<<<vb, TPB, 0, s>>>((int)n, d_d.p, dd_d.p, dt, alpha, v_d.p);
    }
    count_launches(1);
  }
  C->stream = c_stream_saved;
  K->stream = k_stream_saved;
  if (st != SGPU_OK) return cleanup(st);
  cudaMemcpyAsync(d, d_d.p, n * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(v, v_d.p, n * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return cleanup(fail(SGPU_CUDA_ERROR, "transient copy-back failed"));
  if (info) {
    info->iterations = total_its;
    info->solve_ms = total_ms;
    info->true_relres = last_true;
    info->precond_setup_ms = setup_ms;
    info->precond_levels = levels;
    info->precond_coarse_n = coarse_n;
  }
  cleanup(SGPU_OK);
  return status;
}

}  // namespace

extern "C" {

SGPU_API int sgpu_matrix_combine(sgpu_matrix K, sgpu_matrix C, double a, double b, sgpu_matrix *out) {
  if (!K || !C || !out) return fail(SGPU_BAD_INPUT, "null argument");
  if (!same_pattern(K, C)) return fail(SGPU_BAD_INPUT, "matrices do not share one pattern");
  *out = nullptr;
  sgpu_matrix m = new sgpu_matrix_s();
  m->n = K->n;
  m->src_sym = K->src_sym;
  m->src_negm = K->src_negm;
  auto bail = [&](int st) {
    cudaStream_t s = m->own_stream;
    cudaEvent_t e0 = m->ev0, e1 = m->ev1;
    delete m;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    return st;
  };
  if (cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&m->ev0) != cudaSuccess || cudaEventCreate(&m->ev1) != cudaSuccess)
    return bail(fail(SGPU_CUDA_ERROR, "stream/event creation failed"));
  m->stream = m->own_stream;
  cudaStream_t s = m->stream;
  // the two sources must be complete before their arrays are read here
  if (cudaStreamSynchronize(K->stream) != cudaSuccess || cudaStreamSynchronize(C->stream) != cudaSuccess)
    return bail(fail(SGPU_CUDA_ERROR, "synchronising the source matrices failed"));
  const int64_t n = K->n, nnz = K->csr.nnz, negm = K->src_negm;
  int st;
  if ((st = m->src_adr.alloc(n + 1)) || (st = m->src_ci.alloc(negm)) || (st = m->map_lo.alloc(negm)) ||
      (st = m->map_up.alloc(negm)) || (st = m->csr.rowptr.alloc(n + 1)) || (st = m->csr.col.alloc(nnz)) ||
      (st = m->csr.val.alloc(nnz)) || (st = m->csr.diag.alloc(n)))
    return bail(st);
  m->csr.n = (int)n;
  m->csr.nnz = nnz;
  cudaMemcpyAsync(m->src_adr.p, K->src_adr.p, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(m->src_ci.p, K->src_ci.p, negm * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(m->map_lo.p, K->map_lo.p, negm * sizeof(int), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(m->map_up.p, K->map_up.p, negm * sizeof(int), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(m->csr.rowptr.p, K->csr.rowptr.p, (n + 1) * sizeof(int), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(m->csr.col.p, K->csr.col.p, nnz * sizeof(int), cudaMemcpyDeviceToDevice, s);
  k_combine<<<blocks_for(nnz), TPB, 0, s>>>(nnz, K->csr.val.p, C->csr.val.p, a, b, m->csr.val.p);
  count_launches(1);
  if (cudaGetLastError() != cudaSuccess) return bail(fail(SGPU_CUDA_ERROR, "combine kernel failed"));
  m->bsr.nb = -1;
  st = finish_values(m);
  if (st != SGPU_OK) return bail(st);
  if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(SGPU_CUDA_ERROR, "combine failed"));
  *out = m;
  return SGPU_OK;
}

SGPU_API int sgpu_transient_dform(sgpu_matrix K, sgpu_matrix C, const double *rhs, double *d, double *v, double dt,
                                  double alpha, int64_t nsteps, int64_t ni, double res, double zero, int64_t iv,
                                  int32_t prec, int32_t mode, int64_t *step_iterations, sgpu_solve_info *info) {
  return transient(K, C, rhs, d, v, dt, alpha, nsteps, ni, res, zero, iv, prec, mode, step_iterations, info, false);
}

SGPU_API int sgpu_transient_vform(sgpu_matrix K, sgpu_matrix C, const double *rhs, double *d, double *v, double dt,
                                  double alpha, int64_t nsteps, int64_t ni, double res, double zero, int64_t iv,
                                  int32_t prec, int32_t mode, int64_t *step_iterations, sgpu_solve_info *info) {
  return transient(K, C, rhs, d, v, dt, alpha, nsteps, ni, res, zero, iv, prec, mode, step_iterations, info, true);
}

}  // extern "C"
