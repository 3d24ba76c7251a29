// extern "C" entry points of libsifelgpu.so (declared in include/sifelgpu.h).
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "sgpu_internal.cuh"

namespace sgpu {
int pcg_run(sgpu_matrix m, int64_t ni, double res, double zero, int64_t iv, int crit, int prec, int mode,
            int64_t *ani, double *ares, sgpu_solve_info *info);
int pcg_prepare(sgpu_matrix m, bool mixed);
double *work_x(sgpu_matrix m);
double *work_f(sgpu_matrix m);

namespace {
thread_local std::string g_err;
std::atomic<int64_t> g_launches{0};
}  // namespace

void set_error(const std::string &msg) { g_err = msg; }
int fail(int status, const std::string &msg) {
  g_err = msg;
  return status;
}
void count_launches(int64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

}  // namespace sgpu

using namespace sgpu;

namespace {

int create_handle(int64_t n, int32_t sym, int64_t negm, sgpu_matrix *out) {
  if (!out) return fail(SGPU_BAD_INPUT, "null output handle");
  *out = nullptr;
  if (n <= 0) return fail(SGPU_BAD_INPUT, "n must be positive");
  if (negm <= 0) return fail(SGPU_BAD_INPUT, "empty matrix storage");
  sgpu_matrix m = new sgpu_matrix_s();
  m->n = n;
  m->src_sym = sym ? 1 : 0;
  m->src_negm = negm;
  cudaError_t e = cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking);
  m->stream = m->own_stream;
  if (e == cudaSuccess) e = cudaEventCreate(&m->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&m->ev1);
  if (e != cudaSuccess) {
    delete m;
    return fail(SGPU_CUDA_ERROR, std::string("stream/event creation: ") + cudaGetErrorString(e));
  }
  *out = m;
  return SGPU_OK;
}

void destroy_handle(sgpu_matrix m) {
  if (!m) return;
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaStream_t s = m->own_stream;
  cudaEvent_t a = m->ev0, b = m->ev1;
  delete m;  // DevBufs free their memory
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (s) cudaStreamDestroy(s);
}

// upload pattern + values from host GEFEL arrays and build the device forms
// a second stream and two events for the copy of the values, released when
// the upload ends (after its last wait)
struct CopySide {
  cudaStream_t s2 = nullptr;
  cudaEvent_t after_pattern_src = nullptr, after_values = nullptr;
  bool ok = false;
  CopySide() {
    ok = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&after_pattern_src, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&after_values, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) cudaGetLastError();
  }
  ~CopySide() {
    if (s2) {
      cudaStreamSynchronize(s2);
      cudaStreamDestroy(s2);
    }
    if (after_pattern_src) cudaEventDestroy(after_pattern_src);
    if (after_values) cudaEventDestroy(after_values);
  }
};

// The storage arrays to the device and the device formats built from them.
// The values travel on a second stream after the pattern arrays, so that
// their copy (half of the bytes) overlaps the pattern's construction, which
// needs only adr and ci.
int upload(sgpu_matrix m, const int64_t *adr, const int64_t *ci, const double *a, double *setup_ms) {
  cudaStream_t s = m->stream;
  const int64_t n = m->n, negm = m->src_negm;
  SGPU_CUDA(cudaEventRecord(m->ev0, s));
  SGPU_TRY(m->src_adr.alloc(n + 1));
  SGPU_TRY(m->src_ci.alloc(negm));
  DevBuf<double> a_d;
  SGPU_TRY(a_d.alloc(negm));
  CopySide side;
  SGPU_CUDA(cudaMemcpyAsync(m->src_adr.p, adr, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  SGPU_CUDA(cudaMemcpyAsync(m->src_ci.p, ci, negm * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  if (side.ok) {
    SGPU_CUDA(cudaEventRecord(side.after_pattern_src, s));
    SGPU_CUDA(cudaStreamWaitEvent(side.s2, side.after_pattern_src, 0));
    SGPU_CUDA(cudaMemcpyAsync(a_d.p, a, negm * sizeof(double), cudaMemcpyHostToDevice, side.s2));
    SGPU_CUDA(cudaEventRecord(side.after_values, side.s2));
  } else {
    SGPU_CUDA(cudaMemcpyAsync(a_d.p, a, negm * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  SGPU_TRY(matrix_build_from_device_src(m));
  // the 3x3 block form's pattern (the tuned FP64 SpMV and the aggregation
  // cycle use it) while the values are still on their way; its values follow
  // the CSR values in matrix_set_values_device
  SGPU_TRY(ensure_bsr3(m));
  if (side.ok) SGPU_CUDA(cudaStreamWaitEvent(s, side.after_values, 0));
  SGPU_TRY(matrix_set_values_device(m, a_d.p));
  SGPU_CUDA(cudaEventRecord(m->ev1, s));
  SGPU_CUDA(cudaEventSynchronize(m->ev1));
  float ms = 0.f;
  SGPU_CUDA(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
  if (setup_ms) *setup_ms = ms;
  return SGPU_OK;
}

int solve_host(sgpu_matrix m, double *x, const double *y, int64_t ni, double res, double zero, int64_t iv,
               int crit, int prec, int mode, int64_t *ani, double *ares, sgpu_solve_info *info) {
  if (!x || !y) return fail(SGPU_BAD_INPUT, "null vector");
  SGPU_TRY(pcg_prepare(m, mode == SGPU_MIXED));
  cudaStream_t s = m->stream;
  const size_t bytes = (size_t)m->n * sizeof(double);
  SGPU_CUDA(cudaMemcpyAsync(work_f(m), y, bytes, cudaMemcpyHostToDevice, s));
  if (iv != 0) SGPU_CUDA(cudaMemcpyAsync(work_x(m), x, bytes, cudaMemcpyHostToDevice, s));
  int st = pcg_run(m, ni, res, zero, iv, crit, prec, mode, ani, ares, info);
  if (st == SGPU_BAD_INPUT || st == SGPU_CUDA_ERROR) return st;
  SGPU_CUDA(cudaMemcpyAsync(x, work_x(m), bytes, cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  return st;
}

}  // namespace

extern "C" {

const char *sgpu_last_error(void) { return g_err.c_str(); }
const char *sgpu_version(void) { return "sifelgpu 0.1 (sm_100a)"; }
int64_t sgpu_kernel_launches(void) { return g_launches.load(); }

int sgpu_matrix_create(int64_t n, const int64_t *adr, const int64_t *ci, const double *a, int32_t symmetric,
                       sgpu_matrix *out) {
  if (!adr || !ci || !a) return fail(SGPU_BAD_INPUT, "null storage array");
  if (n <= 0) return fail(SGPU_BAD_INPUT, "n must be positive");
  sgpu_matrix m = nullptr;
  SGPU_TRY(create_handle(n, symmetric, adr[n], &m));
  int st = upload(m, adr, ci, a, nullptr);
  if (st != SGPU_OK) {
    destroy_handle(m);
    return st;
  }
  *out = m;
  return SGPU_OK;
}

int sgpu_matrix_update_values(sgpu_matrix m, const double *a) {
  if (!m || !a) return fail(SGPU_BAD_INPUT, "null argument");
  DevBuf<double> a_d;
  SGPU_TRY(a_d.alloc(m->src_negm));
  SGPU_CUDA(cudaMemcpyAsync(a_d.p, a, m->src_negm * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  SGPU_TRY(matrix_set_values_device(m, a_d.p));
  SGPU_CUDA(cudaStreamSynchronize(m->stream));
  return SGPU_OK;
}

int sgpu_matrix_destroy(sgpu_matrix m) {
  destroy_handle(m);
  return SGPU_OK;
}

int sgpu_matrix_info(sgpu_matrix m, int64_t *n, int64_t *nnz_full) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  if (n) *n = m->n;
  if (nnz_full) *nnz_full = m->csr.nnz;
  return SGPU_OK;
}

int sgpu_matrix_download(sgpu_matrix m, int32_t symmetric, int64_t *adr, int64_t *ci, double *a,
                         int64_t *negm) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  // host-side restatement of the storage from the full CSR
  const int n = m->csr.n;
  const int64_t nnz = m->csr.nnz;
  std::vector<int> rp(n + 1), cl(nnz);
  std::vector<double> vl(nnz);
  SGPU_CUDA(cudaMemcpy(rp.data(), m->csr.rowptr.p, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  SGPU_CUDA(cudaMemcpy(cl.data(), m->csr.col.p, nnz * sizeof(int), cudaMemcpyDeviceToHost));
  SGPU_CUDA(cudaMemcpy(vl.data(), m->csr.val.p, nnz * sizeof(double), cudaMemcpyDeviceToHost));
  int64_t k = 0;
  if (adr) adr[0] = 0;
  for (int i = 0; i < n; i++) {
    for (int q = rp[i]; q < rp[i + 1]; q++) {
      if (symmetric && cl[q] > i) continue;
      if (ci) ci[k] = cl[q];
      if (a) a[k] = vl[q];
      k++;
    }
    if (adr) adr[i + 1] = k;
  }
  if (negm) *negm = k;
  return SGPU_OK;
}

int sgpu_matrix_mxv(sgpu_matrix m, const double *x, double *y) {
  if (!m || !x || !y) return fail(SGPU_BAD_INPUT, "null argument");
  SGPU_TRY(pcg_prepare(m, false));
  const size_t bytes = (size_t)m->n * sizeof(double);
  SGPU_CUDA(cudaMemcpyAsync(work_f(m), x, bytes, cudaMemcpyHostToDevice, m->stream));
  SGPU_TRY(spmv64(m, work_f(m), work_x(m), m->stream));
  SGPU_CUDA(cudaMemcpyAsync(y, work_x(m), bytes, cudaMemcpyDeviceToHost, m->stream));
  SGPU_CUDA(cudaStreamSynchronize(m->stream));
  return SGPU_OK;
}

int sgpu_matrix_mxv_d(sgpu_matrix m, const double *x_d, double *y_d) {
  if (!m || !x_d || !y_d) return fail(SGPU_BAD_INPUT, "null argument");
  return spmv64(m, x_d, y_d, m->stream);
}

int sgpu_matrix_set_stream(sgpu_matrix m, void *stream) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  SGPU_CUDA(cudaStreamSynchronize(m->stream));
  m->stream = stream ? (cudaStream_t)stream : m->own_stream;
  return SGPU_OK;
}

int sgpu_matrix_mxv32_d(sgpu_matrix m, const float *x_d, float *y_d) {
  if (!m || !x_d || !y_d) return fail(SGPU_BAD_INPUT, "null argument");
  return spmv32(m, x_d, y_d, m->stream);
}

int sgpu_matrix_spmv_plan(sgpu_matrix m, int32_t precision, double *bytes, int32_t *format, int32_t *variant) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  if (precision != 64 && precision != 32) return fail(SGPU_BAD_INPUT, "precision must be 64 or 32");
  int f = 0, v = 0;
  SGPU_TRY(spmv_plan(m, precision, bytes, &f, &v));
  if (format) *format = f;
  if (variant) *variant = v;
  return SGPU_OK;
}

int sgpu_matrix_set_spmv(sgpu_matrix m, int32_t precision, int32_t format, int32_t variant) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  if (precision != 64 && precision != 32) return fail(SGPU_BAD_INPUT, "precision must be 64 or 32");
  if (format != 0 && format != 2 && format != 3)
    return fail(SGPU_BAD_INPUT, "format must be 0 (CSR), 2 (sliced ELL, FP64) or 3 (BSR3)");
  if (format == 2 && (precision != 64 || variant != 32))
    return fail(SGPU_BAD_INPUT, "sliced ELL is FP64 with variant 32 (a thread per row)");
  if ((format == 0 && variant != 4 && variant != 8 && variant != 16 && variant != 32) ||
      (format == 3 && variant != 8 && variant != 16 && variant != 32 && variant != 132 && variant != 232 &&
       variant != 116 && variant != 216 && variant != 108 && variant != 208))
    return fail(SGPU_BAD_INPUT,
                "variant = lanes per row: 4, 8, 16 or 32 for CSR; 8, 16, 32 (+100/+200: register caps) for BSR3");
  SGPU_TRY(pcg_prepare(m, precision == 32));
  if (precision == 32) {
    if (!m->csr.diag_positive) return fail(SGPU_BAD_INPUT, "scaled operator needs a positive diagonal");
    SGPU_TRY(ensure_fp32(m));
  }
  SGPU_TRY(ensure_bsr3(m));
  if (format == 3 && !m->bsr.valid) return fail(SGPU_BAD_INPUT, "matrix has no 3x3 block-row form");
  if (format == 2) {
    SGPU_TRY(ensure_sell(m));
    if (!m->sell.valid) return fail(SGPU_BAD_INPUT, "rows too uneven for the sliced ELL form");
  }
  SpmvPlan &p = precision == 64 ? m->plan64 : m->plan32;
  p.format = format;
  p.variant = variant;
  p.tuned = true;
  return SGPU_OK;
}

int sgpu_matrix_set_nullspace(sgpu_matrix m, int32_t k, const double *B) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  if (k != 1 && k != 3 && k != 6) return fail(SGPU_BAD_INPUT, "the near-null space has 1, 3 or 6 vectors");
  if (!B) return fail(SGPU_BAD_INPUT, "null near-null space");
  return amg_set_nullspace(m, k, B);
}

int sgpu_matrix_set_rigid_body_modes(sgpu_matrix m, int64_t nn, int32_t ndofn, const double *coords,
                                     const int64_t *cn) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  if (!coords || !cn || nn <= 0) return fail(SGPU_BAD_INPUT, "empty node arrays");
  if (ndofn < 1 || ndofn > 3) return fail(SGPU_BAD_INPUT, "ndofn must be 1, 2 or 3");
  return amg_set_rigid_body_modes(m, nn, ndofn, coords, cn);
}

int sgpu_matrix_pcg_batch_agg(sgpu_matrix m, int32_t nsys, const int64_t *sys_rows, double *x, const double *f,
                              int64_t ni, double res, double zero, int32_t mode, int64_t *ani, double *ares,
                              int32_t *status, int64_t *iterations, sgpu_solve_info *info) {
  (void)zero;
  if (!m || !sys_rows || !x || !f) return fail(SGPU_BAD_INPUT, "null argument");
  if (nsys < 1) return fail(SGPU_BAD_INPUT, "nsys must be positive");
  if (info) memset(info, 0, sizeof(*info));
  return amg_batch_run(m, nsys, sys_rows, x, f, ni, res, mode, ani, ares, status, iterations, info);
}

int sgpu_matrix_precond_clear(sgpu_matrix m) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  amg_values_changed(m);
  return SGPU_OK;
}

int sgpu_matrix_pcg(sgpu_matrix m, double *x, const double *f, int64_t ni, double res, double zero, int64_t iv,
                    int32_t crit, int32_t prec, int32_t mode, int64_t *ani, double *ares, sgpu_solve_info *info) {
  if (!m) return fail(SGPU_BAD_INPUT, "null handle");
  if (info) memset(info, 0, sizeof(*info));
  return solve_host(m, x, f, ni, res, zero, iv, crit, prec, mode, ani, ares, info);
}

int sgpu_matrix_pcg_d(sgpu_matrix m, double *x_d, const double *f_d, int64_t ni, double res, double zero,
                      int64_t iv, int32_t crit, int32_t prec, int32_t mode, int64_t *ani, double *ares,
                      sgpu_solve_info *info) {
  if (!m || !x_d || !f_d) return fail(SGPU_BAD_INPUT, "null argument");
  if (info) memset(info, 0, sizeof(*info));
  SGPU_TRY(pcg_prepare(m, mode == SGPU_MIXED));
  const size_t bytes = (size_t)m->n * sizeof(double);
  cudaStream_t s = m->stream;
  SGPU_CUDA(cudaMemcpyAsync(work_f(m), f_d, bytes, cudaMemcpyDeviceToDevice, s));
  if (iv != 0) SGPU_CUDA(cudaMemcpyAsync(work_x(m), x_d, bytes, cudaMemcpyDeviceToDevice, s));
  int st = pcg_run(m, ni, res, zero, iv, crit, prec, mode, ani, ares, info);
  if (st == SGPU_BAD_INPUT || st == SGPU_CUDA_ERROR) return st;
  SGPU_CUDA(cudaMemcpyAsync(x_d, work_x(m), bytes, cudaMemcpyDeviceToDevice, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  return st;
}

int sgpu_scr_cg_prec(int64_t n, const int64_t *adr, const int64_t *ci, const double *a, double *x,
                     const double *y, int64_t ni, double res, int64_t *ani, double *ares, double zero, int64_t iv,
                     int32_t mode, sgpu_solve_info *info) {
  if (info) memset(info, 0, sizeof(*info));
  if (!adr || !ci || !a || !x || !y) return fail(SGPU_BAD_INPUT, "null argument");
  if (n <= 0) return fail(SGPU_BAD_INPUT, "n must be positive");
  sgpu_matrix m = nullptr;
  SGPU_TRY(create_handle(n, 1, adr[n], &m));
  double setup = 0.0;
  int st = upload(m, adr, ci, a, &setup);
  if (st == SGPU_OK)
    st = solve_host(m, x, y, ni, res, zero, iv, SGPU_CRIT_SCR_PREC, 1, mode, ani, ares, info);
  if (info) info->setup_ms = setup;
  destroy_handle(m);
  return st;
}

int sgpu_cr_cg_prec(int64_t n, const int64_t *adr, const int64_t *ci, const double *a, double *x,
                    const double *y, int64_t ni, double res, int64_t *ani, double *ares, double zero, int64_t iv,
                    int32_t prec, int32_t mode, sgpu_solve_info *info) {
  if (info) memset(info, 0, sizeof(*info));
  if (!adr || !ci || !a || !x || !y) return fail(SGPU_BAD_INPUT, "null argument");
  if (n <= 0) return fail(SGPU_BAD_INPUT, "n must be positive");
  sgpu_matrix m = nullptr;
  SGPU_TRY(create_handle(n, 0, adr[n], &m));
  double setup = 0.0;
  int st = upload(m, adr, ci, a, &setup);
  if (st == SGPU_OK)
    st = solve_host(m, x, y, ni, res, zero, iv, SGPU_CRIT_CR_PREC, prec ? 1 : 0, mode, ani, ares, info);
  if (info) info->setup_ms = setup;
  destroy_handle(m);
  return st;
}

}  // extern "C"
