// Internal declarations shared by the translation units of libsifelgpu.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/sifelgpu.h"

namespace sgpu {

// ---------------------------------------------------------------------------
// error handling: every CUDA call is checked; failures become SGPU_CUDA_ERROR
// with the message kept for sgpu_last_error()
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int status, const std::string &msg);

#define SGPU_CUDA(call)                                                                      \
  do {                                                                                       \
    cudaError_t _e = (call);                                                                 \
    if (_e != cudaSuccess)                                                                   \
      return ::sgpu::fail(SGPU_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

#define SGPU_TRY(expr)           \
  do {                           \
    int _s = (expr);             \
    if (_s != SGPU_OK) return _s; \
  } while (0)

// counts kernel launches issued by this library (graph replays add their nodes)
void count_launches(int64_t k);

constexpr int kNumSMs = 148;

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
// A process-wide cache of device blocks behind DevBuf (sgpu_alloc.cu): a
// released block waits for the device to be idle -- the ordering cudaFree
// gave -- and is kept for the next request of a similar size, so that a
// handle built and destroyed per solve does not pay cudaMalloc / cudaFree
// each time.  *bytes is rounded up to the block actually handed out.
cudaError_t devmem_get(void **p, size_t *bytes);
void devmem_put(void *p, size_t bytes);

template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) devmem_put(p, bytes);
    p = nullptr;
    n = 0;
    bytes = 0;
  }
  int alloc(size_t count) {
    if (count <= n && p) return SGPU_OK;
    release();
    if (count == 0) count = 1;
    size_t b = count * sizeof(T);
    cudaError_t e = devmem_get((void **)&p, &b);
    if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    n = count;
    bytes = b;
    return SGPU_OK;
  }
};

// ---------------------------------------------------------------------------
// device matrix formats
// ---------------------------------------------------------------------------

// Full CSR with int32 indices, FP64 values (and the FP32 Jacobi-scaled copy).
struct Csr {
  int n = 0;
  int64_t nnz = 0;
  DevBuf<int> rowptr, col;
  DevBuf<double> val;
  DevBuf<double> diag;       // a_ii
  DevBuf<float> val32s;      // a_ij / sqrt(a_ii a_jj), FP32 (mixed mode)
  DevBuf<double> dscale;     // 1 / sqrt(a_ii)
  bool have32 = false;
  bool diag_positive = false;
};

// 3x3 block rows (BSR3): node-blocked form of a CSR whose equations come in
// aligned triples sharing their column structure (every 3D elasticity matrix
// whose nodes are either fully free or fully fixed).
struct Bsr3 {
  int nb = 0;          // block rows
  int64_t nblk = 0;    // stored 3x3 blocks
  DevBuf<int> browptr, bcol;
  DevBuf<double> bval;   // nblk * 9, component-major per block row: bval[9*s + comp*nbr + j]
  DevBuf<float> bval32s; // scaled FP32 copy
  DevBuf<int64_t> csr2bsr;  // CSR entry -> position in bval (for value updates)
  bool valid = false;
  bool have32 = false;
  // most blocks in one tile of 32 block rows (the FP32 level-0 products that
  // stream tiles through shared memory); 0 not yet known
  int tile_cap = 0;
};

// SpMV kernel choice for one format/precision, picked by the autotuner.
// Sliced ELL (slices of 32 rows, each padded to its longest row, stored
// column by column: entry k of row 32 q + l at sptr[q] + 32 k + l), FP64 only.
// Thread per row, every load of a warp one contiguous segment; padding
// entries have value 0 and the row's own column.
struct Sell {
  bool examined = false;  // ensure_sell has looked at the pattern
  bool valid = false;     // built (padding within the limit)
  int nslices = 0;
  int64_t nent = 0;       // stored entries, padding included
  DevBuf<int64_t> sptr;   // nslices + 1
  DevBuf<int> scol;
  DevBuf<double> sval;
  DevBuf<int> csr2sell;   // CSR entry -> position in sval
};

struct SpmvPlan {
  int format = 0;   // 0 CSR, 2 sliced ELL (FP64), 3 BSR3
  int variant = 0;  // kernel variant id
  bool tuned = false;
};

// ---------------------------------------------------------------------------
// device-side solver state (one per handle, in Work::scal)
// ---------------------------------------------------------------------------
struct PcgState {
  // configuration
  int64_t ni;
  double res, zero, tol2, delta2;
  int crit, prec;
  // FP64 iteration scalars
  double nory, nom, denom, alpha, beta, rr;
  // mixed iteration scalars
  double ff, rho, rho_prev, rr_ref, kappa2, true_rr, true_rel;
  double sigma;  // scale of the FP32 residual: the first one has unit norm
  int64_t it, it_last_update, refinements;
  // outputs in the reference's conventions
  int64_t ani;
  double ares;
  int ani_set;
  // control
  int done, pause, status;
  double last_dot;
  int64_t loops;  // iterations run by one launch of a device-side loop graph
};

// Per-handle scratch vectors of the iteration.
struct Work {
  DevBuf<double> r, h, d, p, x, f, t;   // FP64 vectors
  DevBuf<float> r32, p32, q32, y32;     // FP32 vectors (mixed)
  DevBuf<double> partials;              // block partial sums
  DevBuf<unsigned> counters;            // last-block tickets
  DevBuf<unsigned char> scal;           // PcgState (see sgpu_pcg.cu)
};

}  // namespace sgpu

struct sgpu_assembly_s;  // element data kept by sgpu_assemble (sgpu_assemble.cu)
void sgpu_free_assembly(sgpu_assembly_s *a);
namespace sgpu {
struct Amg;  // aggregation multilevel preconditioner (sgpu_amg.cu)
void amg_free(Amg *a);
}  // namespace sgpu

struct sgpu_matrix_s {
  int64_t n = 0;
  int32_t src_sym = 0;     // storage the handle was created from
  int64_t src_negm = 0;
  sgpu::DevBuf<int64_t> src_adr, src_ci;  // source pattern (device, int64 as given)
  sgpu::DevBuf<int> map_lo, map_up;       // source entry -> CSR positions
  sgpu::Csr csr;
  sgpu::Bsr3 bsr;
  sgpu::Sell sell;
  sgpu::SpmvPlan plan64, plan32;
  sgpu::Work w;
  cudaStream_t stream = nullptr;      // stream all work of the handle runs on
  cudaStream_t own_stream = nullptr;  // the handle's own (created) stream
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool values_dirty32 = true;
  sgpu_assembly_s *asm_data = nullptr;
  sgpu::Amg *amg = nullptr;  // built on first use of SGPU_PREC_AGG
  ~sgpu_matrix_s() {
    if (asm_data) sgpu_free_assembly(asm_data);
    if (amg) sgpu::amg_free(amg);
  }
};

namespace sgpu {
// sgpu_matrix.cu
int matrix_build_from_device_src(sgpu_matrix m);     // src_* + a (device) -> csr
int matrix_set_values_device(sgpu_matrix m, const double *a_d);
int ensure_fp32(sgpu_matrix m);
int finish_values(sgpu_matrix m);  // diag, derived formats after val changed
int ensure_bsr3(sgpu_matrix m);
int ensure_sell(sgpu_matrix m);
void release_sell(sgpu_matrix m);
// sgpu_spmv.cu
// y = A x (FP64). If dot_out != nullptr also sum_i x_i y_i into a device scalar
// via the block partials of `w`.
int spmv64(sgpu_matrix m, const double *x, double *y, cudaStream_t s);
int spmv_autotune(sgpu_matrix m, int precision);
int spmv32(sgpu_matrix m, const float *x, float *y, cudaStream_t s);
int spmv_plan(sgpu_matrix m, int precision, double *bytes, int *format, int *variant);
// sgpu_amg.cu
void amg_values_changed(sgpu_matrix m);
int amg_set_nullspace(sgpu_matrix m, int k, const double *B_host);
int amg_set_rigid_body_modes(sgpu_matrix m, int64_t nn, int ndofn, const double *coords_h, const int64_t *cn_h);
int amg_pcg_run(sgpu_matrix m, int64_t ni, double res, double zero, int64_t iv, int crit, int mode,
                int64_t *ani, double *ares, sgpu_solve_info *info);
int amg_batch_run(sgpu_matrix m, int nsys, const int64_t *sys_rows, double *x, const double *f, int64_t ni,
                  double res, int mode, int64_t *ani, double *ares, int32_t *status, int64_t *iterations,
                  sgpu_solve_info *info);
}  // namespace sgpu
