// Aggregation multilevel preconditioner: the hierarchy shared by the
// single-vector solve (sgpu_amg.cu) and the many-load-case solve
// (sgpu_amg_multi.cu).
#pragma once

#include <vector>

#include "sgpu_internal.cuh"

namespace sgpu {

// Device buffers of the hierarchy come from the device's stream-ordered
// memory pool (the pool keeps freed memory, so building a hierarchy for a new
// handle -- a batch solved handle after handle -- does not pay for cudaMalloc
// and cudaFree and their device synchronisation).  The stream is the handle's,
// set by the AMG entry points (amg_stream) before any allocation; a buffer is
// freed on the stream it was allocated on, after the work queued there.
extern thread_local cudaStream_t amg_stream;

template <class T>
struct PBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  PBuf() = default;
  PBuf(const PBuf &) = delete;
  PBuf &operator=(const PBuf &) = delete;
  ~PBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  int alloc(size_t count) {
    if (count <= n && p) return SGPU_OK;
    release();
    if (count == 0) count = 1;
    s = amg_stream;
    cudaError_t e = cudaMallocAsync((void **)&p, count * sizeof(T), s);
    if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    n = count;
    return SGPU_OK;
  }
};

template <typename T>
struct LevelVecs {
  PBuf<T> b, x, x2, r, d, d2, res;
  int alloc(size_t n) {
    SGPU_TRY(b.alloc(n));
    SGPU_TRY(x.alloc(n));
    SGPU_TRY(x2.alloc(n));
    SGPU_TRY(r.alloc(n));
    SGPU_TRY(d.alloc(n));
    SGPU_TRY(d2.alloc(n));
    SGPU_TRY(res.alloc(n));
    return SGPU_OK;
  }
};

struct AmgLevel {
  int nb = 0, b = 0, n = 0;
  int64_t nblk = 0;
  int layout = 0;  // 0 owned row-major blocks, 1 handle BSR3, 2 handle CSR
  const int *browptr = nullptr, *bcol = nullptr;
  PBuf<int> own_browptr, own_bcol;
  PBuf<double> val64;  // owned coarse values (FP64), or the level-0 scaled FP64 copy
  PBuf<float> val32;   // owned coarse values (FP32)
  PBuf<double> dinv64;
  PBuf<float> dinv32;
  PBuf<double> dsq64;  // sqrt(dinv): the symmetric scaling of the Lanczos operator
  PBuf<float> dsq32;
  bool unit_diag = false;
  double lmax64 = 0.0, lmax32 = 0.0;
  // transfer to the next level
  int na = 0, k = 0;
  PBuf<int> agg, aggptr, aggnodes;
  PBuf<double> Q64;
  PBuf<float> Q32;
  LevelVecs<double> v64;
  LevelVecs<float> v32;
  // FP32 cycle: values converted, and the slot of this level's smoother
  // bound among the Lanczos runs on the set-up's second stream (-1: none)
  bool val32_ready = false;
  int lz_slot = -1;
};

struct Amg {
  int k0 = 0;             // near-null-space vectors given (0: translations)
  PBuf<double> B0;      // n x k0 as given
  bool built = false;     // hierarchy (FP64 set-up) current
  bool have32 = false;    // FP32 copies current
  bool have64 = false;    // FP64 level-0 scaled copy current
  std::vector<AmgLevel *> lv;
  int nc = 0;             // coarsest (dense) equations
  PBuf<double> M64;
  PBuf<float> M32;
  PBuf<double> cb64, cx64;
  PBuf<float> cb32, cx32;
  // options: Chebyshev degree, coarse-correction weight, smoothing interval
  // [lmax/ratio, 1.1 lmax], largest dense coarsest level, coarse visits per
  // level (1: V-cycle, 2: W-cycle), Lanczos steps of the lmax estimate
  int deg = 1;
  // alpha 1.9: 39 iterations on the 1.01M-DOF cantilever against 41 at 1.7,
  // 33 against 36 on a 362k-DOF plate, 31 against 32 on a 96^3 lognormal
  // conduction cube (all FP32 cycle, true residual 1e-10)
  double ratio = 30.0, alpha = 1.9;
  int coarse_max = 768;
  int dense_max = 4096;  // larger coarsest levels are smoothed, not inverted
  int bottom_deg = 8;    // Chebyshev steps of such a bottom level
  int gamma = 2;       // visits of level 1 per level-0 cycle
  int gamma_deep = 2;  // visits of level l+1 per level-l cycle, l >= 1
  int lanczos_steps = 14;
  // batched independent systems (sgpu_matrix_pcg_batch_agg): the level-0 last
  // smoothing step writes the per-row products z r and z q here
  double *batch_zr = nullptr, *batch_zq = nullptr;
  // level objects by depth, kept when a hierarchy is discarded so that a
  // rebuild of the same matrix reuses their device buffers
  std::vector<AmgLevel *> pool;
  // the level-0 smoother bound of an FP32 cycle, run on a second stream
  // while the aggregation set-up runs on the handle's (amg_build); its
  // workspace stays with the handle
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr;
  bool l0_bound_pending = false;
  bool l0_bound_wanted = false;
  DevBuf<float> lz32;    // 5 vectors of n
  DevBuf<double> lz_ab;  // Lanczos coefficients
  // the coarse smoothing levels' bounds, run on the second stream beside the
  // dense coarsest inverse: 5 vectors of each level, 129 coefficients each
  DevBuf<float> lzc32;
  DevBuf<double> lzc_ab;
  int lzc_levels = 0;
  // Level 0 of the FP32 cycle with half-precision values (3x3 block rows
  // only): every block row padded to a multiple of four blocks (padding:
  // value 0, the row's own column), values component-major per padded row,
  // so that a lane reads one component of four blocks in one 8-byte load.
  // The padded pattern is kept for the handle's life (the pattern of a handle
  // never changes); the values are converted at every FP32 set-up.
  bool want_fp32 = false;  // the set-up under way is for the FP32 cycle
  bool h16_struct = false, h16_vals = false;
  int64_t h16_nblk = 0;     // stored blocks, padding included
  DevBuf<int> h16ptr, h16col;
  DevBuf<uint16_t> h16val;  // IEEE binary16 bit patterns
  ~Amg() {
    for (AmgLevel *l : pool) delete l;
    if (side) {
      cudaStreamSynchronize(side);
      cudaStreamDestroy(side);
    }
    if (fork) cudaEventDestroy(fork);
  }
  void clear() {
    lv.clear();
    built = have32 = have64 = false;
    h16_vals = false;
  }
  AmgLevel *take_level(size_t depth) {
    while (pool.size() <= depth) pool.push_back(new AmgLevel());
    AmgLevel *l = pool[depth];
    l->unit_diag = false;
    l->browptr = l->bcol = nullptr;
    l->val32_ready = false;
    l->lz_slot = -1;
    return l;
  }
};


// Chebyshev smoothing on [lmax/ratio, 1.1 lmax] of D^-1 A: the first step's
// 1/theta and the recurrence coefficients of steps 1..deg-1
struct Cheb {
  double c2_first;             // 1/theta
  double c1[8], c2[8];         // steps 1..deg-1
};

inline Cheb cheb_coeffs(double lmax, double ratio, int deg) {
  Cheb c{};
  const double a = lmax / ratio, b = 1.1 * lmax;
  const double theta = 0.5 * (b + a), delta = 0.5 * (b - a), sigma = theta / delta;
  c.c2_first = 1.0 / theta;
  double rho = 1.0 / sigma;
  for (int k = 1; k < deg && k < 8; k++) {
    const double rn = 1.0 / (2.0 * sigma - rho);
    c.c1[k] = rn * rho;
    c.c2[k] = 2.0 * rn / delta;
    rho = rn;
  }
  return c;
}

template <typename T>
const T *level_vals(const sgpu_matrix m, const AmgLevel &L);
template <>
inline const float *level_vals<float>(const sgpu_matrix m, const AmgLevel &L) {
  if (L.layout == 1) return m->bsr.bval32s.p;
  if (L.layout == 2) return m->csr.val32s.p;
  return L.val32.p;
}
template <>
inline const double *level_vals<double>(const sgpu_matrix m, const AmgLevel &L) {
  return L.val64.p;  // level 0: the scaled FP64 copy; coarse: owned values
}

template <typename T>
const T *level_dinv(const AmgLevel &L);
template <>
inline const float *level_dinv<float>(const AmgLevel &L) { return L.unit_diag ? nullptr : L.dinv32.p; }
template <>
inline const double *level_dinv<double>(const AmgLevel &L) { return L.unit_diag ? nullptr : L.dinv64.p; }

// Builds the hierarchy if the handle has none (set-up in FP64) and the copies
// of the requested cycle precision; set-up device time into *setup_ms.
int amg_ensure(sgpu_matrix m, bool fp32, float *setup_ms);

}  // namespace sgpu
