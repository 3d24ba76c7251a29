// Many load cases with the aggregation preconditioner: every right-hand side
// runs its own flexible CG (FP64: residual, update, alpha, beta, the
// reference's stopping test (r.r)/(f.f) < res per column), all sharing one
// hierarchy and advanced together, so every kernel of the cycle handles all
// columns at once: each level's matrix is read once per sweep for all of
// them (a sparse matrix times a block of vectors), and the launch count of
// one iteration is that of a single solve.
//
// solve_linear_statics (MEFEL/SRC/lssolver.cpp:78-80) solves the load cases
// one after the other; sgpu_matrix_pcg_multi batches them with Jacobi, this
// file with the aggregation cycle (FP32 for SGPU_MIXED, FP64 for SGPU_FP64).
//
// Layout: vectors of one kind are row-major n x RP (RP = 32 * CPL >= nrhs;
// padding columns are zero and marked done), so one warp handles one row
// (block row) and lane l owns columns l, l + 32, ...  Per-column sums are
// reduced deterministically: per block in warp order, then over blocks in
// block order by the last block to finish.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sgpu_amg.cuh"

namespace sgpu {

// sgpu_pcg.cu
int pcg_prepare(sgpu_matrix m, bool mixed);

namespace {

constexpr int TPB = 256;
constexpr int NW = TPB / 32;

struct MCol {  // one load case
  double ff, rr, rho, alpha, beta, ares;
  long long it, it_restart, ani;
  int done, status;
};

struct MState {
  int all_done, active;
  long long ni;
  double res;
};

template <typename T>
struct MVecs {
  T *b, *x, *x2, *r, *d, *d2, *res;
};

// ---------------------------------------------------------------------------
// per-column grid reduction
// ---------------------------------------------------------------------------

// Sums acc[c][q] (column lane + 32 c) over the grid.  Returns true in the
// last block, with the sums in tot[q * RP + col].
template <int NV, int CPL>
__device__ bool col_reduce(const double (&acc)[CPL][NV], double *partials, unsigned *ticket, double *tot) {
  constexpr int RP = 32 * CPL;
  __shared__ double sh[NV][CPL][NW][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++)
#pragma unroll
    for (int c = 0; c < CPL; c++) sh[q][c][wid][lane] = acc[c][q];
  __syncthreads();
  for (int t = threadIdx.x; t < NV * RP; t += blockDim.x) {
    const int q = t / RP, col = t % RP;
    double s = 0.0;
    for (int w = 0; w < NW; w++) s += sh[q][col / 32][w][col % 32];
    partials[((size_t)q * gridDim.x + blockIdx.x) * RP + col] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return false;
  __threadfence();
  for (int t = threadIdx.x; t < NV * RP; t += blockDim.x) {
    const int q = t / RP, col = t % RP;
    double s = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) s += __ldcg(partials + ((size_t)q * gridDim.x + b) * RP + col);
    tot[t] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// all_done when no column is active (run by the last block after a finish)
__device__ void count_active(const MCol *cols, int R, MState *ms) {
  __shared__ int act;
  if (threadIdx.x == 0) act = 0;
  __syncthreads();
  for (int c = threadIdx.x; c < R; c += blockDim.x)
    if (!cols[c].done) atomicAdd(&act, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    ms->active = act;
    if (act == 0) ms->all_done = 1;
  }
}

template <class Op, int CPL>
__device__ __forceinline__ void op_finish(const Op &op, const double (&acc)[CPL][Op::NV > 0 ? Op::NV : 1],
                                          double *partials, unsigned *ticket, MCol *cols, int R, MState *ms) {
  if constexpr (Op::NV > 0) {
    __shared__ double tot[Op::NV * 32 * CPL];
    if (col_reduce<Op::NV, CPL>(acc, partials, ticket, tot)) {
      op.finish(tot, cols, R);
      __syncthreads();
      count_active(cols, R, ms);
    }
  }
}

// ---------------------------------------------------------------------------
// row operators (equation i, column col, y = (A V)[i][col])
// ---------------------------------------------------------------------------
template <typename T>
struct MOpResid {
  static constexpr int NV = 0;
  const T *b;
  T *res;
  int RP;
  __device__ void row(int i, int col, T y, double *) const {
    const size_t k = (size_t)i * RP + col;
    res[k] = b[k] - y;
  }
  __device__ void finish(const double *, MCol *, int) const {}
};

// Chebyshev step fused with the product (as OpCheb of the single solve)
template <typename T, bool FIRST, bool OUTER>
struct MOpCheb {
  static constexpr int NV = OUTER ? 2 : 0;
  const T *b, *x_in;
  T *x, *r;
  const T *d_in;
  T *d_out;
  const T *dinv;
  T c1, c2;
  int last, RP;
  // outer coupling (level 0): z = S x, per-column r.z and q.z
  const double *dscale, *r64, *q64;
  __device__ void row(int i, int col, T y, double *acc) const {
    const size_t k = (size_t)i * RP + col;
    const T di_ = dinv ? dinv[i] : T(1);
    T ri, di, xi;
    if (FIRST) {
      ri = di_ * (b[k] - y);
      di = c2 * ri;
      xi = x_in[k] + di;
    } else {
      ri = r[k] - di_ * y;
      di = c1 * d_in[k] + c2 * ri;
      xi = x[k] + di;
    }
    x[k] = xi;
    if (!last) {
      r[k] = ri;
      d_out[k] = di;
    }
    if constexpr (OUTER) {
      const double z = dscale[i] * (double)xi;
      acc[0] += z * r64[k];
      acc[1] += z * q64[k];
    }
  }
  __device__ void finish(const double *tot, MCol *cols, int R) const {
    if constexpr (OUTER) {
      for (int c = threadIdx.x; c < R; c += blockDim.x) {
        MCol &mc = cols[c];
        if (mc.done) continue;
        const double rz = tot[c], zq = tot[RP + c];
        if (!(rz > 0.0) || !isfinite(zq)) {  // the preconditioner is SPD
          mc.done = 1;
          mc.status = SGPU_BREAKDOWN;
          continue;
        }
        // Polak-Ribiere: z_new.(r_new - r_old) / rho_old with r_new - r_old = -alpha q
        mc.beta = mc.it > mc.it_restart ? -mc.alpha * zq / mc.rho : 0.0;
        mc.rho = rz;
      }
    }
  }
};

// outer FP64 product q = K p, per-column p.q and alpha = rho / p.q
struct MOpAlpha {
  static constexpr int NV = 1;
  const double *p;
  double *q;
  int RP;
  __device__ void row(int i, int col, double y, double *acc) const {
    const size_t k = (size_t)i * RP + col;
    q[k] = y;
    acc[0] += p[k] * y;
  }
  __device__ void finish(const double *tot, MCol *cols, int R) const {
    for (int c = threadIdx.x; c < R; c += blockDim.x) {
      MCol &mc = cols[c];
      if (mc.done) {
        mc.alpha = 0.0;
        continue;
      }
      const double pq = tot[c];
      if (!(pq > 0.0)) {
        mc.done = 1;
        mc.status = SGPU_BREAKDOWN;
        mc.alpha = 0.0;
        continue;
      }
      mc.alpha = mc.rho / pq;
    }
  }
};

struct MOpStore {  // q = K x (start of the recurrence)
  static constexpr int NV = 0;
  double *q;
  int RP;
  __device__ void row(int i, int col, double y, double *) const { q[(size_t)i * RP + col] = y; }
  __device__ void finish(const double *, MCol *, int) const {}
};

// ---------------------------------------------------------------------------
// products of a level matrix with a block of vectors
// ---------------------------------------------------------------------------

// 3x3 block rows with component-major values (the handle's BSR3); VT values,
// T vectors
template <typename VT, typename T, int CPL, class Op>
__global__ void __launch_bounds__(TPB) k_mspmm_bsr3(int nb, const int *__restrict__ browptr,
                                                    const int *__restrict__ bcol, const VT *__restrict__ bval,
                                                    const T *__restrict__ X, Op op, MCol *cols, int R, MState *ms,
                                                    double *partials, unsigned *ticket) {
  if (ms->all_done) return;
  constexpr int RP = 32 * CPL;
  constexpr int NVX = Op::NV > 0 ? Op::NV : 1;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double acc[CPL][NVX] = {};
  for (int br = warp; br < nb; br += nw) {
    const int s = __ldg(browptr + br), nbr = __ldg(browptr + br + 1) - s;
    const VT *bv = bval + 9ll * s;
    T y[3][CPL];
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int c = 0; c < CPL; c++) y[q][c] = 0;
#pragma unroll 2
    for (int j = 0; j < nbr; j++) {
      const int col = __ldg(bcol + s + j);
      T v[9];
#pragma unroll
      for (int q = 0; q < 9; q++) v[q] = (T)__ldg(bv + q * nbr + j);  // same address in every lane
      const T *x0 = X + (size_t)(3 * col) * RP + lane;
#pragma unroll
      for (int c = 0; c < CPL; c++) {
        const T a0 = __ldg(x0 + 32 * c), a1 = __ldg(x0 + RP + 32 * c), a2 = __ldg(x0 + 2 * RP + 32 * c);
        y[0][c] += v[0] * a0 + v[1] * a1 + v[2] * a2;
        y[1][c] += v[3] * a0 + v[4] * a1 + v[5] * a2;
        y[2][c] += v[6] * a0 + v[7] * a1 + v[8] * a2;
      }
    }
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int c = 0; c < CPL; c++) op.row(3 * br + q, lane + 32 * c, y[q][c], acc[c]);
  }
  op_finish<Op, CPL>(op, acc, partials, ticket, cols, R, ms);
}

// scalar CSR (warp per row)
template <typename VT, typename T, int CPL, class Op>
__global__ void __launch_bounds__(TPB) k_mspmm_csr(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                                                   const VT *__restrict__ val, const T *__restrict__ X, Op op,
                                                   MCol *cols, int R, MState *ms, double *partials,
                                                   unsigned *ticket) {
  if (ms->all_done) return;
  constexpr int RP = 32 * CPL;
  constexpr int NVX = Op::NV > 0 ? Op::NV : 1;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double acc[CPL][NVX] = {};
  for (int i = warp; i < n; i += nw) {
    T y[CPL];
#pragma unroll
    for (int c = 0; c < CPL; c++) y[c] = 0;
#pragma unroll 4
    for (int k = __ldg(rowptr + i); k < __ldg(rowptr + i + 1); k++) {
      const T a = (T)__ldg(val + k);
      const T *x = X + (size_t)__ldg(col + k) * RP + lane;
#pragma unroll
      for (int c = 0; c < CPL; c++) y[c] += a * __ldg(x + 32 * c);
    }
#pragma unroll
    for (int c = 0; c < CPL; c++) op.row(i, lane + 32 * c, y[c], acc[c]);
  }
  op_finish<Op, CPL>(op, acc, partials, ticket, cols, R, ms);
}

// Loads a B x B row-major block (16-byte aligned: the value array is from
// cudaMalloc and every block is B*B*sizeof(T) bytes, a multiple of 16 for
// B = 6) with 16-byte loads; other sizes element by element.
template <typename T, int B>
__device__ __forceinline__ void load_block(const T *__restrict__ a, T (&v)[B * B]) {
  constexpr int NB = B * B * (int)sizeof(T);
  if constexpr (NB % 16 == 0) {
    constexpr int PER = 16 / (int)sizeof(T);
    const float4 *a4 = reinterpret_cast<const float4 *>(a);
#pragma unroll
    for (int t = 0; t < NB / 16; t++) {
      const float4 w = __ldg(a4 + t);
      const T *wt = reinterpret_cast<const T *>(&w);
#pragma unroll
      for (int u = 0; u < PER; u++) v[t * PER + u] = wt[u];
    }
  } else {
#pragma unroll
    for (int t = 0; t < B * B; t++) v[t] = __ldg(a + t);
  }
}

// B x B row-major blocks (coarse levels).  A coarse level has few block rows,
// so each is split over SPLIT warps of a CTA (each takes every SPLIT-th
// block); the partial sums meet in shared memory and the first warp of the
// group applies the row operator.
template <typename T, int B, int CPL, class Op>
__global__ void __launch_bounds__(TPB) k_mspmm_bsrb(int nb, const int *__restrict__ browptr,
                                                    const int *__restrict__ bcol, const T *__restrict__ bval,
                                                    const T *__restrict__ X, Op op, MCol *cols, int R, MState *ms,
                                                    double *partials, unsigned *ticket) {
  if (ms->all_done) return;
  constexpr int RP = 32 * CPL, SPLIT = 4, GROUPS = NW / SPLIT;
  constexpr int NVX = Op::NV > 0 ? Op::NV : 1;
  __shared__ T part[GROUPS][SPLIT][B][RP];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int grp = wid / SPLIT, sub = wid % SPLIT;
  double acc[CPL][NVX] = {};
  for (int base = blockIdx.x * GROUPS; base < nb; base += gridDim.x * GROUPS) {
    const int br = base + grp;
    T y[B][CPL];
#pragma unroll
    for (int q = 0; q < B; q++)
#pragma unroll
      for (int c = 0; c < CPL; c++) y[q][c] = 0;
    if (br < nb) {
#pragma unroll 2
      for (int k = __ldg(browptr + br) + sub; k < __ldg(browptr + br + 1); k += SPLIT) {
        const int col = __ldg(bcol + k);
        T a[B * B];
        load_block<T, B>(bval + (size_t)k * B * B, a);
        const T *x0 = X + (size_t)(B * col) * RP + lane;
#pragma unroll
        for (int c = 0; c < CPL; c++) {
          T xv[B];
#pragma unroll
          for (int q = 0; q < B; q++) xv[q] = __ldg(x0 + (size_t)q * RP + 32 * c);
#pragma unroll
          for (int r = 0; r < B; r++) {
            T s = 0;
#pragma unroll
            for (int q = 0; q < B; q++) s += a[r * B + q] * xv[q];
            y[r][c] += s;
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < B; q++)
#pragma unroll
      for (int c = 0; c < CPL; c++) part[grp][sub][q][lane + 32 * c] = y[q][c];
    __syncthreads();
    if (sub == 0 && br < nb) {
#pragma unroll
      for (int q = 0; q < B; q++)
#pragma unroll
        for (int c = 0; c < CPL; c++) {
          T t = part[grp][0][q][lane + 32 * c];
#pragma unroll
          for (int w = 1; w < SPLIT; w++) t += part[grp][w][q][lane + 32 * c];
          op.row(B * br + q, lane + 32 * c, t, acc[c]);
        }
    }
    __syncthreads();
  }
  op_finish<Op, CPL>(op, acc, partials, ticket, cols, R, ms);
}

// ---------------------------------------------------------------------------
// transfers, coarsest solve
// ---------------------------------------------------------------------------

// B_c = Q^T Res: one warp per coarse equation (aggregate G, component q),
// lanes over columns, rows of the aggregate summed in order; with START the
// coarse smoothing starts from x = 0 (r = D^-1 b, d = x = c2 r)
template <typename T, int B, int K, int CPL, bool START>
__global__ void __launch_bounds__(TPB) k_mrestrict(int na, const int *__restrict__ aggptr,
                                                   const int *__restrict__ aggnodes, const T *__restrict__ Q,
                                                   const T *__restrict__ res, T *__restrict__ bc, T *__restrict__ rc,
                                                   T *__restrict__ dc, T *__restrict__ xc,
                                                   const T *__restrict__ dinvc, T c2, const MState *ms) {
  if (ms->all_done) return;
  constexpr int RP = 32 * CPL;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int p = warp; p < na * K; p += nw) {
    const int G = p / K, q = p % K;
    T acc[CPL];
#pragma unroll
    for (int c = 0; c < CPL; c++) acc[c] = 0;
    const int t0 = __ldg(aggptr + G), t1 = __ldg(aggptr + G + 1);
#pragma unroll 2
    for (int t = t0; t < t1; t++) {
      const int i = __ldg(aggnodes + t);
#pragma unroll
      for (int e = 0; e < B; e++) {
        const T qv = __ldg(Q + ((size_t)B * i + e) * K + q);
        const T *rr = res + ((size_t)B * i + e) * RP + lane;
#pragma unroll
        for (int c = 0; c < CPL; c++) acc[c] += qv * rr[32 * c];
      }
    }
#pragma unroll
    for (int c = 0; c < CPL; c++) {
      const size_t k = (size_t)p * RP + lane + 32 * c;
      bc[k] = acc[c];
      if (START) {
        const T ri = dinvc[p] * acc[c];
        rc[k] = ri;
        dc[k] = c2 * ri;
        xc[k] = c2 * ri;
      }
    }
  }
}

// X += alpha Q X_c (warp per equation)
template <typename T, int B, int K, int CPL>
__global__ void __launch_bounds__(TPB) k_mprolong(int n, const int *__restrict__ agg, const T *__restrict__ Q,
                                                  const T *__restrict__ xc, T *__restrict__ x, T alpha,
                                                  const MState *ms) {
  if (ms->all_done) return;
  constexpr int RP = 32 * CPL;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int p = warp; p < n; p += nw) {
    const int G = __ldg(agg + p / B);
    const T *qr = Q + (size_t)p * K;
    T qv[K];
#pragma unroll
    for (int q = 0; q < K; q++) qv[q] = __ldg(qr + q);
#pragma unroll
    for (int c = 0; c < CPL; c++) {
      T s = 0;
#pragma unroll
      for (int q = 0; q < K; q++) s += qv[q] * __ldg(xc + (size_t)(K * G + q) * RP + lane + 32 * c);
      x[(size_t)p * RP + lane + 32 * c] += alpha * s;
    }
  }
}

// X_c = M^-1 B_c, a small dense product tiled through shared memory: a CTA
// owns 32 rows of M (4 per warp), stages 32 columns of M and the matching 32
// rows of B_c per step; lanes own the right-hand sides
template <typename T, int CPL>
__global__ void __launch_bounds__(TPB) k_mdense(int nc, const T *__restrict__ M, const T *__restrict__ b,
                                                T *__restrict__ x, const MState *ms) {
  if (ms->all_done) return;
  constexpr int RP = 32 * CPL, TR = 32, TJ = 32;
  __shared__ T ms_[TR][TJ + 1];
  __shared__ T bs[TJ][RP];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i0 = blockIdx.x * TR; i0 < nc; i0 += gridDim.x * TR) {
    T s[4][CPL];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < CPL; c++) s[r][c] = 0;
    for (int j0 = 0; j0 < nc; j0 += TJ) {
      for (int t = threadIdx.x; t < TR * TJ; t += blockDim.x) {
        const int r = t / TJ, j = t % TJ;
        ms_[r][j] = (i0 + r < nc && j0 + j < nc) ? M[(size_t)(i0 + r) * nc + j0 + j] : T(0);
      }
      for (int t = threadIdx.x; t < TJ * RP; t += blockDim.x) {
        const int j = t / RP, c = t % RP;
        bs[j][c] = (j0 + j < nc) ? b[(size_t)(j0 + j) * RP + c] : T(0);
      }
      __syncthreads();
#pragma unroll 8
      for (int j = 0; j < TJ; j++) {
        T bv[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) bv[c] = bs[j][lane + 32 * c];
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const T a = ms_[4 * wid + r][j];
#pragma unroll
          for (int c = 0; c < CPL; c++) s[r][c] += a * bv[c];
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int i = i0 + 4 * wid + r;
      if (i < nc) {
#pragma unroll
        for (int c = 0; c < CPL; c++) x[(size_t)i * RP + lane + 32 * c] = s[r][c];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// flexible CG vector kernels (FP64), warp per equation, lanes over columns
// ---------------------------------------------------------------------------

// R = F - Q (Q = K X); per-column f.f and r.r; level-0 right-hand side S r
// and the first smoothing step from zero; every column restarts its recurrence
template <typename T, int CPL>
__global__ void __launch_bounds__(TPB) k_mfcg_init(int n, const double *__restrict__ F, const double *__restrict__ Q,
                                                   double *__restrict__ Rv, const double *__restrict__ dscale,
                                                   T *__restrict__ b0, T *__restrict__ r0, T *__restrict__ d0,
                                                   T *__restrict__ x0, T c2, MCol *cols, int R, MState *ms,
                                                   double *partials, unsigned *ticket) {
  constexpr int RP = 32 * CPL;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double acc[CPL][2] = {};
  for (int i = warp; i < n; i += nw) {
    const double si = dscale[i];
#pragma unroll
    for (int c = 0; c < CPL; c++) {
      const size_t k = (size_t)i * RP + lane + 32 * c;
      const double fi = F[k], ri = fi - Q[k];
      Rv[k] = ri;
      acc[c][0] += fi * fi;
      acc[c][1] += ri * ri;
      const T bi = (T)(si * ri);
      b0[k] = bi;
      r0[k] = bi;
      d0[k] = c2 * bi;
      x0[k] = c2 * bi;
    }
  }
  __shared__ double tot[2 * RP];
  if (col_reduce<2, CPL>(acc, partials, ticket, tot)) {
    for (int c = threadIdx.x; c < R; c += blockDim.x) {
      MCol &mc = cols[c];
      mc.it_restart = mc.it;
      mc.beta = 0.0;
      if (mc.done) continue;
      mc.ff = tot[c];
      mc.rr = tot[RP + c];
      if (mc.ff < 1e-300) {
        mc.done = 1;
        mc.status = SGPU_ZERO_RHS;
      } else if (mc.rr < ms->res * mc.ff) {
        mc.done = 1;
        mc.ani = mc.it;
        mc.ares = mc.rr / mc.ff;
      }
    }
    __syncthreads();
    count_active(cols, R, ms);
  }
}

// X += alpha P; R -= alpha Q; per-column r.r and the stopping test; the
// next cycle's level-0 right-hand side and first smoothing step
template <typename T, int CPL>
__global__ void __launch_bounds__(TPB) k_mfcg_update(int n, double *__restrict__ X, double *__restrict__ Rv,
                                                     const double *__restrict__ P, const double *__restrict__ Q,
                                                     const double *__restrict__ dscale, T *__restrict__ b0,
                                                     T *__restrict__ r0, T *__restrict__ d0, T *__restrict__ x0, T c2,
                                                     MCol *cols, int R, MState *ms, double *partials,
                                                     unsigned *ticket) {
  if (ms->all_done) return;
  constexpr int RP = 32 * CPL;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double al[CPL];
#pragma unroll
  for (int c = 0; c < CPL; c++) {
    const int col = lane + 32 * c;
    al[c] = col < R ? cols[col].alpha : 0.0;
  }
  double acc[CPL][1] = {};
  for (int i = warp; i < n; i += nw) {
    const double si = dscale[i];
#pragma unroll
    for (int c = 0; c < CPL; c++) {
      const size_t k = (size_t)i * RP + lane + 32 * c;
      X[k] += al[c] * P[k];
      const double ri = Rv[k] - al[c] * Q[k];
      Rv[k] = ri;
      acc[c][0] += ri * ri;
      const T bi = (T)(si * ri);
      b0[k] = bi;
      r0[k] = bi;
      d0[k] = c2 * bi;
      x0[k] = c2 * bi;
    }
  }
  __shared__ double tot[RP];
  if (col_reduce<1, CPL>(acc, partials, ticket, tot)) {
    for (int c = threadIdx.x; c < R; c += blockDim.x) {
      MCol &mc = cols[c];
      if (mc.done) continue;
      mc.it += 1;
      mc.rr = tot[c];
      if (mc.rr < ms->res * mc.ff) {  // (r.r)/(f.f) < res, symcomprow::cg_prec's test
        mc.done = 1;
        mc.ani = mc.it;
        mc.ares = mc.rr / mc.ff;
      } else if (mc.it >= ms->ni) {
        mc.done = 1;
        mc.status = SGPU_NOT_CONVERGED;
      }
    }
    __syncthreads();
    count_active(cols, R, ms);
  }
}

// P = S x0 + beta P for the active columns
template <typename T, int CPL>
__global__ void __launch_bounds__(TPB) k_mfcg_dir(int n, double *__restrict__ P, const T *__restrict__ x0,
                                                  const double *__restrict__ dscale, const MCol *cols, int R,
                                                  const MState *ms) {
  if (ms->all_done) return;
  constexpr int RP = 32 * CPL;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double be[CPL];
  bool live[CPL];
#pragma unroll
  for (int c = 0; c < CPL; c++) {
    const int col = lane + 32 * c;
    live[c] = col < R && !cols[col].done;
    be[c] = live[c] ? cols[col].beta : 0.0;
  }
  for (int i = warp; i < n; i += nw) {
    const double si = dscale[i];
#pragma unroll
    for (int c = 0; c < CPL; c++) {
      if (!live[c]) continue;
      const size_t k = (size_t)i * RP + lane + 32 * c;
      P[k] = si * (double)x0[k] + be[c] * P[k];
    }
  }
}

// host layout (R column blocks of n) <-> device row-major n x RP
__global__ void k_to_rows(int n, int R, int RP, const double *__restrict__ cols, double *__restrict__ rows) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)n * RP;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t / RP), c = (int)(t % RP);
    rows[t] = c < R ? cols[(size_t)c * n + i] : 0.0;
  }
}

__global__ void k_to_cols(int n, int R, int RP, const double *__restrict__ rows, double *__restrict__ cols) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)n * R;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(t / n), i = (int)(t % n);
    cols[t] = rows[(size_t)i * RP + c];
  }
}

int grid_warps(int64_t warps) {
  int64_t g = (warps * 32 + TPB - 1) / TPB;
  if (g < 1) g = 1;
  if (g > 8 * kNumSMs) g = 8 * kNumSMs;
  return (int)g;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

template <class T>
struct Buf {  // stream-ordered device buffer of one call
  T *p = nullptr;
  cudaStream_t s = nullptr;
  explicit Buf(cudaStream_t st) : s(st) {}
  Buf(const Buf &) = delete;
  Buf &operator=(const Buf &) = delete;
  ~Buf() {
    if (p) cudaFreeAsync(p, s);
  }
  int alloc(size_t n) {
    cudaError_t e = cudaMallocAsync((void **)&p, (n ? n : 1) * sizeof(T), s);
    if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    return SGPU_OK;
  }
};

template <typename T>
const T *qm(const AmgLevel &L);
template <>
const float *qm<float>(const AmgLevel &L) { return L.Q32.p; }
template <>
const double *qm<double>(const AmgLevel &L) { return L.Q64.p; }

template <typename T, int CPL>
struct Multi {
  sgpu_matrix m;
  Amg *A;
  int R, n;
  cudaStream_t s;
  MCol *cols;
  MState *ms;
  double *partials;
  unsigned *tickets;
  double *X, *Rv, *P, *Q, *F;
  std::vector<MVecs<T>> lv;  // per smoothing level
  T *cb, *cx;                // coarsest
  std::vector<Cheb> ch;

  static constexpr int RP = 32 * CPL;

  template <class Op>
  int level_product(int l, const T *v, const Op &op, int slot) {
    const AmgLevel &L = *A->lv[l];
    const T *val = level_vals<T>(m, L);
    const int g = grid_warps(L.nb);
    const int gb = (int)std::min<int64_t>(((int64_t)L.nb + 1) / 2, 8 * kNumSMs);  // 2 block rows per CTA
    unsigned *tk = tickets + slot;
    if (L.layout == 1)
      k_mspmm_bsr3<T, T, CPL, Op><<<g, TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, cols, R, ms, partials, tk);
    else if (L.layout == 2)
      k_mspmm_csr<T, T, CPL, Op><<<g, TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, cols, R, ms, partials, tk);
    else if constexpr (Op::NV > 0)  // (operators with column sums run on level 0 only)
      return fail(SGPU_BAD_INPUT, "reduction on a coarse level");
    else if (L.b == 6)
      k_mspmm_bsrb<T, 6, CPL, Op><<<gb, TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, cols, R, ms, partials, tk);
    else if (L.b == 3)
      k_mspmm_bsrb<T, 3, CPL, Op><<<gb, TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, cols, R, ms, partials, tk);
    else if (L.b == 1)
      k_mspmm_bsrb<T, 1, CPL, Op><<<gb, TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, cols, R, ms, partials, tk);
    else
      return fail(SGPU_BAD_INPUT, "unsupported coarse block size");
    count_launches(1);
    SGPU_CUDA(cudaGetLastError());
    return SGPU_OK;
  }

  // the outer FP64 product with the handle's FP64 matrix (unscaled K)
  template <class Op>
  int outer_product(const double *v, const Op &op, int slot) {
    const int g = grid_warps(m->bsr.valid ? m->bsr.nb : m->n);
    unsigned *tk = tickets + slot;
    if (m->bsr.valid)
      k_mspmm_bsr3<double, double, CPL, Op><<<g, TPB, 0, s>>>(m->bsr.nb, m->bsr.browptr.p, m->bsr.bcol.p,
                                                              m->bsr.bval.p, v, op, cols, R, ms, partials, tk);
    else
      k_mspmm_csr<double, double, CPL, Op><<<g, TPB, 0, s>>>(n, m->csr.rowptr.p, m->csr.col.p, m->csr.val.p, v, op,
                                                             cols, R, ms, partials, tk);
    count_launches(1);
    SGPU_CUDA(cudaGetLastError());
    return SGPU_OK;
  }

  template <int B, int K>
  void restrict_bk(const AmgLevel &L, const T *res, T *bc, T *rc, T *dc, T *xc, const T *dinvc, T c2, bool start) {
    const int g = grid_warps((int64_t)L.na * K);
    if (start)
      k_mrestrict<T, B, K, CPL, true><<<g, TPB, 0, s>>>(L.na, L.aggptr.p, L.aggnodes.p, qm<T>(L), res, bc, rc, dc, xc,
                                                        dinvc, c2, ms);
    else
      k_mrestrict<T, B, K, CPL, false><<<g, TPB, 0, s>>>(L.na, L.aggptr.p, L.aggnodes.p, qm<T>(L), res, bc, rc, dc,
                                                         xc, dinvc, c2, ms);
  }

  int restrict_level(int l, const T *res, T *bc, T *rc, T *dc, T *xc, const T *dinvc, T c2, bool start) {
    const AmgLevel &L = *A->lv[l];
    const int B = L.b, K = L.k;
    if (B == 3 && K == 6) restrict_bk<3, 6>(L, res, bc, rc, dc, xc, dinvc, c2, start);
    else if (B == 6 && K == 6) restrict_bk<6, 6>(L, res, bc, rc, dc, xc, dinvc, c2, start);
    else if (B == 1 && K == 1) restrict_bk<1, 1>(L, res, bc, rc, dc, xc, dinvc, c2, start);
    else if (B == 1 && K == 3) restrict_bk<1, 3>(L, res, bc, rc, dc, xc, dinvc, c2, start);
    else if (B == 3 && K == 3) restrict_bk<3, 3>(L, res, bc, rc, dc, xc, dinvc, c2, start);
    else if (B == 1 && K == 6) restrict_bk<1, 6>(L, res, bc, rc, dc, xc, dinvc, c2, start);
    else return fail(SGPU_BAD_INPUT, "unsupported block size / near-null-space size");
    count_launches(1);
    SGPU_CUDA(cudaGetLastError());
    return SGPU_OK;
  }

  int prolong_level(int l, const T *xc, T *x) {
    const AmgLevel &L = *A->lv[l];
    const int B = L.b, K = L.k, g = grid_warps(L.n);
    const T al = (T)A->alpha;
    if (B == 3 && K == 6) k_mprolong<T, 3, 6, CPL><<<g, TPB, 0, s>>>(L.n, L.agg.p, qm<T>(L), xc, x, al, ms);
    else if (B == 6 && K == 6) k_mprolong<T, 6, 6, CPL><<<g, TPB, 0, s>>>(L.n, L.agg.p, qm<T>(L), xc, x, al, ms);
    else if (B == 1 && K == 1) k_mprolong<T, 1, 1, CPL><<<g, TPB, 0, s>>>(L.n, L.agg.p, qm<T>(L), xc, x, al, ms);
    else if (B == 1 && K == 3) k_mprolong<T, 1, 3, CPL><<<g, TPB, 0, s>>>(L.n, L.agg.p, qm<T>(L), xc, x, al, ms);
    else if (B == 3 && K == 3) k_mprolong<T, 3, 3, CPL><<<g, TPB, 0, s>>>(L.n, L.agg.p, qm<T>(L), xc, x, al, ms);
    else if (B == 1 && K == 6) k_mprolong<T, 1, 6, CPL><<<g, TPB, 0, s>>>(L.n, L.agg.p, qm<T>(L), xc, x, al, ms);
    else return fail(SGPU_BAD_INPUT, "unsupported block size / near-null-space size");
    count_launches(1);
    SGPU_CUDA(cudaGetLastError());
    return SGPU_OK;
  }

  // remaining smoothing steps (1..deg-1) from x and the current direction
  int cheb_steps(int l, T *x, T **din, T **dout, bool outer) {
    const AmgLevel &L = *A->lv[l];
    MVecs<T> &V = lv[l];
    const int deg = A->deg;
    for (int k = 1; k < deg; k++) {
      const bool last = (k == deg - 1);
      if (outer && last) {
        MOpCheb<T, false, true> op{V.b, nullptr, x, V.r, *din, *dout, level_dinv<T>(L), (T)ch[l].c1[k],
                                   (T)ch[l].c2[k], 1, RP, m->csr.dscale.p, Rv, Q};
        SGPU_TRY(level_product(l, *din, op, 6));
      } else {
        MOpCheb<T, false, false> op{V.b, nullptr, x, V.r, *din, *dout, level_dinv<T>(L), (T)ch[l].c1[k],
                                    (T)ch[l].c2[k], last ? 1 : 0, RP, nullptr, nullptr, nullptr};
        SGPU_TRY(level_product(l, *din, op, 0));
      }
      std::swap(*din, *dout);
    }
    return SGPU_OK;
  }

  // one cycle on level l (as cycle() of the single solve); result in xcur[l]
  int cycle(int l, bool zero_init, std::vector<T *> &xcur) {
    const int nl = (int)A->lv.size();
    const int deg = A->deg;
    if (l == nl) {
      const T *M = sizeof(T) == 4 ? (const T *)A->M32.p : (const T *)A->M64.p;
      k_mdense<T, CPL><<<(A->nc + 31) / 32, TPB, 0, s>>>(A->nc, M, cb, cx, ms);
      count_launches(1);
      xcur[l] = cx;
      return SGPU_OK;
    }
    const AmgLevel &L = *A->lv[l];
    MVecs<T> &V = lv[l];
    if (l == nl - 1 && A->nc == 0) {  // bottom level without a dense inverse (as the single solve)
      const Cheb cb = cheb_coeffs(sizeof(T) == 4 ? L.lmax32 : L.lmax64, A->ratio, A->bottom_deg);
      T *xp = V.x;
      if (!zero_init) {
        T *from = xcur[l], *to = (from == V.x) ? V.x2 : V.x;
        MOpCheb<T, true, false> op{V.b, from, to, V.r, nullptr, V.d, level_dinv<T>(L), (T)0, (T)cb.c2_first, 0, RP,
                                   nullptr, nullptr, nullptr};
        SGPU_TRY(level_product(l, from, op, 0));
        xp = to;
      }
      T *din = V.d, *dout = V.d2;
      for (int k = 1; k < A->bottom_deg; k++) {
        const bool last = (k == A->bottom_deg - 1);
        MOpCheb<T, false, false> op{V.b, nullptr, xp, V.r, din, dout, level_dinv<T>(L), (T)cb.c1[k], (T)cb.c2[k],
                                    last ? 1 : 0, RP, nullptr, nullptr, nullptr};
        SGPU_TRY(level_product(l, din, op, 0));
        std::swap(din, dout);
      }
      xcur[l] = xp;
      return SGPU_OK;
    }
    T *xp;
    if (zero_init) {
      xp = V.x;
    } else {
      T *from = xcur[l], *to = (from == V.x) ? V.x2 : V.x;
      MOpCheb<T, true, false> op{V.b, from, to, V.r, nullptr, V.d, level_dinv<T>(L), (T)0, (T)ch[l].c2_first,
                                 deg == 1 ? 1 : 0, RP, nullptr, nullptr, nullptr};
      SGPU_TRY(level_product(l, from, op, 0));
      xp = to;
    }
    {
      T *din = V.d, *dout = V.d2;
      SGPU_TRY(cheb_steps(l, xp, &din, &dout, false));
    }
    {
      MOpResid<T> op{V.b, V.res, RP};
      SGPU_TRY(level_product(l, xp, op, 0));
    }
    if (l + 1 < nl) {
      const AmgLevel &C = *A->lv[l + 1];
      MVecs<T> &W = lv[l + 1];
      SGPU_TRY(restrict_level(l, V.res, W.b, W.r, W.d, W.x, level_dinv<T>(C), (T)ch[l + 1].c2_first, true));
      const int visits = l == 0 ? A->gamma : A->gamma_deep;
      for (int v = 0; v < visits; v++) SGPU_TRY(cycle(l + 1, v == 0, xcur));
    } else {
      SGPU_TRY(restrict_level(l, V.res, cb, nullptr, nullptr, nullptr, nullptr, (T)0, false));
      SGPU_TRY(cycle(l + 1, true, xcur));
    }
    SGPU_TRY(prolong_level(l, xcur[l + 1], xp));
    const bool outer = (l == 0);
    T *to = (xp == V.x) ? V.x2 : V.x;
    if (outer && deg == 1) {
      MOpCheb<T, true, true> op{V.b, xp, to, V.r, nullptr, V.d, level_dinv<T>(L), (T)0, (T)ch[l].c2_first, 1, RP,
                                m->csr.dscale.p, Rv, Q};
      SGPU_TRY(level_product(l, xp, op, 6));
    } else {
      MOpCheb<T, true, false> op{V.b, xp, to, V.r, nullptr, V.d, level_dinv<T>(L), (T)0, (T)ch[l].c2_first,
                                 deg == 1 ? 1 : 0, RP, nullptr, nullptr, nullptr};
      SGPU_TRY(level_product(l, xp, op, 0));
    }
    {
      T *din = V.d, *dout = V.d2;
      SGPU_TRY(cheb_steps(l, to, &din, &dout, outer));
    }
    xcur[l] = to;
    return SGPU_OK;
  }

  // cycle, then P = S x0 + beta P
  int cycle_dir() {
    std::vector<T *> xcur(A->lv.size() + 1, nullptr);
    SGPU_TRY(cycle(0, true, xcur));
    k_mfcg_dir<T, CPL><<<grid_warps(n), TPB, 0, s>>>(n, P, xcur[0], m->csr.dscale.p, cols, R, ms);
    count_launches(1);
    return SGPU_OK;
  }

  T c2_level0() const { return (T)ch[0].c2_first; }

  int start() {  // R = F - K X, a cycle, P = S x0
    MOpStore op{Q, RP};
    SGPU_TRY(outer_product(X, op, 0));
    MVecs<T> &V = lv[0];
    k_mfcg_init<T, CPL><<<grid_warps(n), TPB, 0, s>>>(n, F, Q, Rv, m->csr.dscale.p, V.b, V.r, V.d, V.x, c2_level0(),
                                                      cols, R, ms, partials, tickets + 2);
    count_launches(1);
    return cycle_dir();
  }

  int iteration() {
    MOpAlpha op{P, Q, RP};
    SGPU_TRY(outer_product(P, op, 1));
    MVecs<T> &V = lv[0];
    k_mfcg_update<T, CPL><<<grid_warps(n), TPB, 0, s>>>(n, X, Rv, P, Q, m->csr.dscale.p, V.b, V.r, V.d, V.x,
                                                        c2_level0(), cols, R, ms, partials, tickets + 2);
    count_launches(1);
    return cycle_dir();
  }
};

template <typename T, int CPL>
int run_multi(sgpu_matrix m, int R, double *Xh, const double *Fh, int64_t ni, double res, int64_t iv, int64_t *ani,
              double *ares, int32_t *status, sgpu_solve_info *info, float setup_ms) {
  constexpr int RP = 32 * CPL;
  cudaStream_t s = m->stream;
  Amg &A = *m->amg;
  const int n = (int)m->n;
  const int nl = (int)A.lv.size();
  Multi<T, CPL> M;
  M.m = m;
  M.A = &A;
  M.R = R;
  M.n = n;
  M.s = s;
  Buf<MCol> cols(s);
  Buf<MState> ms(s);
  Buf<double> partials(s), X(s), Rv(s), P(s), Q(s), F(s), stage(s);
  Buf<unsigned> tickets(s);
  SGPU_TRY(cols.alloc(R));
  SGPU_TRY(ms.alloc(1));
  SGPU_TRY(partials.alloc((size_t)2 * RP * 8 * kNumSMs));
  SGPU_TRY(tickets.alloc(8));
  for (Buf<double> *b : {&X, &Rv, &P, &Q, &F}) SGPU_TRY(b->alloc((size_t)n * RP));
  SGPU_TRY(stage.alloc((size_t)n * R));
  std::vector<Buf<T> *> owned;
  auto cleanup = [&]() {
    for (Buf<T> *b : owned) delete b;
  };
  auto vec = [&](size_t cnt) -> T * {
    Buf<T> *b = new Buf<T>(s);
    owned.push_back(b);
    return b->alloc(cnt) == SGPU_OK ? b->p : nullptr;
  };
  M.lv.resize(nl);
  for (int l = 0; l < nl; l++) {
    const size_t cnt = (size_t)A.lv[l]->n * RP;
    MVecs<T> &V = M.lv[l];
    V.b = vec(cnt), V.x = vec(cnt), V.x2 = vec(cnt), V.r = vec(cnt), V.d = vec(cnt), V.d2 = vec(cnt),
    V.res = vec(cnt);
    if (!V.b || !V.x || !V.x2 || !V.r || !V.d || !V.d2 || !V.res) {
      cleanup();
      return SGPU_CUDA_ERROR;
    }
  }
  M.cb = vec((size_t)std::max(A.nc, 1) * RP);
  M.cx = vec((size_t)std::max(A.nc, 1) * RP);
  if (!M.cb || !M.cx) {
    cleanup();
    return SGPU_CUDA_ERROR;
  }
  M.ch.resize(nl);
  for (int l = 0; l < nl; l++) M.ch[l] = cheb_coeffs(sizeof(T) == 4 ? A.lv[l]->lmax32 : A.lv[l]->lmax64, A.ratio, A.deg);
  M.cols = cols.p;
  M.ms = ms.p;
  M.partials = partials.p;
  M.tickets = tickets.p;
  M.X = X.p, M.Rv = Rv.p, M.P = P.p, M.Q = Q.p, M.F = F.p;
  // state and inputs
  std::vector<MCol> hc(R);
  for (auto &c : hc) { memset(&c, 0, sizeof(c)); c.ani = -1; }
  MState hm{};
  hm.ni = ni;
  hm.res = res;
  int rc = SGPU_OK;
  const int g = grid_warps((int64_t)n * RP / 32 + 1);
  auto go = [&]() -> int {
    SGPU_CUDA(cudaMemsetAsync(tickets.p, 0, 8 * sizeof(unsigned), s));
    SGPU_CUDA(cudaMemcpyAsync(cols.p, hc.data(), R * sizeof(MCol), cudaMemcpyHostToDevice, s));
    SGPU_CUDA(cudaMemcpyAsync(ms.p, &hm, sizeof(MState), cudaMemcpyHostToDevice, s));
    SGPU_CUDA(cudaMemcpyAsync(stage.p, Fh, (size_t)n * R * sizeof(double), cudaMemcpyHostToDevice, s));
    k_to_rows<<<g, TPB, 0, s>>>(n, R, RP, stage.p, F.p);
    if (iv) {
      SGPU_CUDA(cudaMemcpyAsync(stage.p, Xh, (size_t)n * R * sizeof(double), cudaMemcpyHostToDevice, s));
      k_to_rows<<<g, TPB, 0, s>>>(n, R, RP, stage.p, X.p);
    } else {
      SGPU_CUDA(cudaMemsetAsync(X.p, 0, (size_t)n * RP * sizeof(double), s));
    }
    // padding columns of P must be finite (they are read by the product)
    SGPU_CUDA(cudaMemsetAsync(P.p, 0, (size_t)n * RP * sizeof(double), s));
    count_launches(iv ? 2 : 1);
    SGPU_CUDA(cudaEventRecord(m->ev0, s));
    SGPU_TRY(M.start());
    // iterations in graphs of 8; the host reads the small state between them
    cudaGraph_t graph;
    cudaGraphExec_t exec = nullptr;
    const int64_t before = sgpu_kernel_launches();
    SGPU_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    int crc = SGPU_OK;
    for (int k = 0; k < 8 && crc == SGPU_OK; k++) crc = M.iteration();
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (crc != SGPU_OK) return crc;
    if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    const int64_t nodes = sgpu_kernel_launches() - before;
    count_launches(-nodes);
    int lrc = SGPU_OK;
    for (int64_t it = 0;; it += 8) {
      MState cur{};
      SGPU_CUDA(cudaMemcpyAsync(&cur, ms.p, sizeof(MState), cudaMemcpyDeviceToHost, s));
      SGPU_CUDA(cudaStreamSynchronize(s));
      if (cur.all_done || it > ni + 8) break;
      e = cudaGraphLaunch(exec, s);
      if (e != cudaSuccess) { lrc = fail(SGPU_CUDA_ERROR, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e)); break; }
      count_launches(nodes);
    }
    cudaGraphExecDestroy(exec);
    SGPU_CUDA(cudaEventRecord(m->ev1, s));
    return lrc;
  };
  rc = go();
  if (rc == SGPU_OK) {
    k_to_cols<<<g, TPB, 0, s>>>(n, R, RP, X.p, stage.p);
    count_launches(1);
    cudaMemcpyAsync(Xh, stage.p, (size_t)n * R * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hc.data(), cols.p, R * sizeof(MCol), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = fail(SGPU_CUDA_ERROR, "copy-back failed");
  }
  float solve_ms = 0.f;
  if (rc == SGPU_OK) cudaEventElapsedTime(&solve_ms, m->ev0, m->ev1);
  cudaStreamSynchronize(s);
  cleanup();
  if (rc != SGPU_OK) return rc;
  int first_bad = SGPU_OK;
  long long maxit = 0;
  for (int c = 0; c < R; c++) {
    const MCol &mc = hc[c];
    if (status) status[c] = mc.status;
    if (mc.status == SGPU_OK && mc.done && mc.ani >= 0) {
      if (ani) ani[c] = mc.ani;
      if (ares) ares[c] = mc.ares;
    }
    if (mc.status != SGPU_OK && first_bad == SGPU_OK) first_bad = mc.status;
    maxit = std::max(maxit, mc.it);
  }
  if (info) {
    info->iterations = maxit;
    info->solve_ms = solve_ms;
    info->precond_setup_ms = setup_ms;
    info->precond_levels = nl + 1;
    info->precond_coarse_n = A.nc;
  }
  return first_bad;
}

}  // namespace
}  // namespace sgpu

using namespace sgpu;

extern "C" SGPU_API int sgpu_matrix_pcg_multi_agg(sgpu_matrix m, int32_t nrhs, double *X, const double *F, int64_t ni,
                                                  double res, double zero, int64_t iv, int32_t mode, int64_t *ani,
                                                  double *ares, int32_t *status, sgpu_solve_info *info) {
  (void)zero;
  if (!m || !X || !F) return fail(SGPU_BAD_INPUT, "null argument");
  if (nrhs < 1 || nrhs > 128) return fail(SGPU_BAD_INPUT, "nrhs must be 1..128");
  if (info) memset(info, 0, sizeof(*info));
  if (!m->csr.diag_positive)
    return fail(SGPU_BAD_INPUT, "the aggregation preconditioner needs a positive diagonal (Jacobi scaling)");
  SGPU_TRY(pcg_prepare(m, false));
  if (!m->plan64.tuned) SGPU_TRY(spmv_autotune(m, 64));
  const bool fp32 = (mode == SGPU_MIXED);
  if (fp32 && !m->plan32.tuned) SGPU_TRY(spmv_autotune(m, 32));
  float setup_ms = 0.f;
  SGPU_TRY(amg_ensure(m, fp32, &setup_ms));
  if (nrhs <= 32)
    return fp32 ? run_multi<float, 1>(m, nrhs, X, F, ni, res, iv, ani, ares, status, info, setup_ms)
                : run_multi<double, 1>(m, nrhs, X, F, ni, res, iv, ani, ares, status, info, setup_ms);
  if (nrhs <= 64)
    return fp32 ? run_multi<float, 2>(m, nrhs, X, F, ni, res, iv, ani, ares, status, info, setup_ms)
                : run_multi<double, 2>(m, nrhs, X, F, ni, res, iv, ani, ares, status, info, setup_ms);
  return fp32 ? run_multi<float, 4>(m, nrhs, X, F, ni, res, iv, ani, ares, status, info, setup_ms)
              : run_multi<double, 4>(m, nrhs, X, F, ni, res, iv, ani, ares, status, info, setup_ms);
}
