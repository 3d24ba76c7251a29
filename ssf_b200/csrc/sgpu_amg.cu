// Aggregation multilevel preconditioner (SGPU_PREC_AGG) and the flexible CG
// around it.
//
// GEFEL's own aggregation preconditioner is the BOSS aggregator
// (GEFEL/aggregator.cpp; precondtype boss = 101, GEFEL/galias.h:103, set up by
// precond::initiation, GEFEL/precond.cpp:136-139): node aggregates
// (aggregator::prepare_tlnagr, aggregator.cpp:220), a tentative prolongator
// made of the rigid-body modes restricted to each aggregate
// (gener_rbm_1/gener_rbm_2, aggregator.cpp:638-700), the coarse matrix
// P^T A P (coarse_matrix, aggregator.cpp:708) and, as the preconditioner
// itself, a symmetric multiplicative Schwarz sweep over the aggregates with
// exact local solves (aggregator::boss, aggregator.cpp:1275; the coarse
// correction of that routine is commented out).  The sweep is sequential over
// the aggregates and runs one global SpMV per aggregate, so it has no useful
// GPU form.  This file keeps the ingredients -- aggregates, a near-null-space
// tentative prolongator, the Galerkin coarse matrix -- and applies them as a
// multilevel V-cycle:
//
// set-up, on the device in FP64, once per matrix values:
//   * aggregation: a distance-2 maximal independent set of the node graph
//     (Luby-style rounds over packed (state, hash, index) keys) gives the
//     roots; a root takes its neighbours, every other node joins an
//     aggregated neighbour;
//   * tentative prolongator: per aggregate, a thin QR (modified Gram-Schmidt,
//     two passes) of the near-null-space rows: Q (b x k per node) and R (the
//     coarse near-null space);
//   * Galerkin product A_c = Q^T A Q: every stored block (i, j) adds
//     Q_i^T A_ij Q_j to the coarse block (agg i, agg j); the blocks are radix
//     sorted by that key and each run is summed by one warp in a fixed order,
//     so the coarse matrices are deterministic;
//   * smoother bound: power iteration on D^-1 A for each level;
//   * coarsest level: dense inverse, Gauss-Jordan in one CTA.
// application (FP32 for SGPU_MIXED, FP64 for SGPU_FP64): one V-cycle with
// Chebyshev smoothing of degree `deg` on [lmax/ratio, 1.1 lmax] of D^-1 A,
// the SpMV and the Chebyshev update fused in one kernel; level 0 is the
// Jacobi-scaled matrix S K S (unit diagonal) the mixed Jacobi form uses too.
//
// The outer iteration is CG in FP64 on K with the Polak-Ribiere beta
// (flexible CG: the FP32 preconditioner is not exactly the same linear map at
// every call); the residual, the solution update, alpha and beta are FP64.
#include <cooperative_groups.h>
#include <cuda_fp16.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "sgpu_amg.cuh"

namespace sgpu {

// sgpu_pcg.cu
int pcg_prepare(sgpu_matrix m, bool mixed);
int spmv64_flex(sgpu_matrix m, const double *x, double *y, cudaStream_t s);
PcgState *pcg_state(sgpu_matrix m);

namespace {

constexpr int TPB = 256;

// ---------------------------------------------------------------------------
// deterministic reductions (one partial per block, the last block sums them)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][TPB / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q]);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) sh[q][wid] = v[q];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = warp_sum(lane < (int)(blockDim.x >> 5) ? sh[q][lane] : 0.0);
  }
}

template <int NV>
__device__ __forceinline__ bool reduce_grid(double (&v)[NV], double *partials, unsigned *ticket,
                                            double (&tot)[NV]) {
  __shared__ bool am_last;
  block_sum<NV>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) partials[(size_t)q * gridDim.x + blockIdx.x] = v[q];
    __threadfence();
    am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double s[NV];
#pragma unroll
  for (int q = 0; q < NV; q++) s[q] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NV; q++) s[q] += __ldcg(partials + (size_t)q * gridDim.x + b);
  }
  block_sum<NV>(s);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) tot[q] = s[q];
    *ticket = 0u;
  }
  return threadIdx.x == 0;
}

// Sums the row contributions of an operator with NV > 0 over the grid and lets
// the last block finish.
template <class Op>
__device__ __forceinline__ void op_reduce(const Op &op, double (&acc)[Op::NV > 0 ? Op::NV : 1], PcgState *st,
                                          double *partials, unsigned *ticket) {
  if constexpr (Op::NV > 0) {
    double tot[Op::NV];
    if (reduce_grid<Op::NV>(acc, partials, ticket, tot)) op.finish(st, tot);
  }
}

// A product that is never fused into a following add: the kernels that must
// give the same bits whichever launch form runs them (the separate level
// kernels and the fused coarse tail) round these products the same way.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// ---------------------------------------------------------------------------
// row operators: what a level SpMV does with y_i = (A v)_i
// ---------------------------------------------------------------------------
template <typename T>
struct OpResid {  // res = b - A x
  static constexpr int NV = 0;
  const T *b;
  T *res;
  __device__ void row(int i, T y, double *) const { res[i] = b[i] - y; }
  __device__ static void finish(PcgState *, const double *) {}
};

// Lanczos step on M = D^-1/2 A D^-1/2 (the SpMV input is u = D^-1/2 w_j,
// unnormalised; v_j = w_j / beta_j): y = M v_j and alpha_j = y . v_j
template <typename T>
struct OpLanczos {
  static constexpr int NV = 1;
  const T *dsq;
  const T *wj;
  const double *beta_j;
  T *y;
  double *alpha_out;
  __device__ void row(int i, T ay, double *acc) const {
    const double ib = 1.0 / *beta_j;
    const double yi = (dsq ? (double)dsq[i] : 1.0) * (double)ay * ib;
    y[i] = (T)yi;
    acc[0] += yi * (double)wj[i] * ib;
  }
  __device__ void finish(PcgState *, const double *tot) const { *alpha_out = tot[0]; }
};

// Chebyshev smoothing step fused with its SpMV.
//   FIRST (SpMV of x_in): r = D^-1 (b - A x_in); d = c2 r; x = x_in + d
//   else  (SpMV of d_in): r = r - D^-1 A d_in;   d = c1 d_in + c2 r; x += d
// The last step of a smoothing pass writes x only.  OUTER (level 0, last
// step of the V-cycle) also forms z = S x in FP64 and the two dot products of
// the flexible CG, r.z and q.z, whose last block sets rho and beta.
template <typename T, bool FIRST, bool OUTER>
struct OpCheb {
  static constexpr int NV = OUTER ? 2 : 0;
  const T *b;
  const T *x_in;
  T *x;
  T *r;
  const T *d_in;
  T *d_out;
  const T *dinv;
  T c1, c2;
  int last;
  // outer coupling (level 0): z = S x is formed on the fly for r.z and q.z
  // (k_fcg_dir forms it again from x)
  const double *dscale, *r64, *q64;
  double *unused;
  __device__ void row(int i, T y, double *acc) const {
    const T di_ = dinv ? dinv[i] : T(1);
    T ri, di, xi;
    if (FIRST) {
      ri = di_ * (b[i] - y);
      di = mul_rn(c2, ri);
      xi = x_in[i] + di;
    } else {
      ri = r[i] - di_ * y;
      di = c1 * d_in[i] + c2 * ri;
      xi = x[i] + di;
    }
    x[i] = xi;
    if (!last) {
      r[i] = ri;
      d_out[i] = di;
    }
    if constexpr (OUTER) {
      const double z = dscale[i] * (double)xi;
      acc[0] += z * r64[i];
      acc[1] += z * q64[i];
    }
  }
  __device__ static void finish(PcgState *st, const double *tot) {
    const double rz = tot[0], zq = tot[1];
    if (!(rz > 0.0) || !isfinite(zq)) {  // the preconditioner is SPD: r.z <= 0 is a breakdown
      if (st->status == 0) st->status = SGPU_BREAKDOWN;
      st->done = 1;
      return;
    }
    // Polak-Ribiere: beta = z_new.(r_new - r_old) / (r_old.z_old), r_new - r_old = -alpha q
    st->beta = st->it > st->it_last_update ? -st->alpha * zq / st->rho : 0.0;
    st->rho_prev = st->rho;
    st->rho = rz;
  }
};

// The same last step for many independent systems solved together: the
// products z_i r_i and z_i q_i are written per row and summed per system
// afterwards (k_bseg_*), since every system has its own scalars.
template <typename T, bool FIRST>
struct OpChebRows {
  static constexpr int NV = 0;
  const T *b, *x_in;
  T *x;
  const T *r, *d_in, *dinv;
  T c1, c2;
  const double *dscale, *r64, *q64;
  double *zr, *zq;
  __device__ void row(int i, T y, double *) const {
    const T di_ = dinv ? dinv[i] : T(1);
    T xi;
    if (FIRST) xi = x_in[i] + c2 * (di_ * (b[i] - y));
    else xi = x[i] + c1 * d_in[i] + c2 * (r[i] - di_ * y);
    x[i] = xi;
    const double z = dscale[i] * (double)xi;
    zr[i] = z * r64[i];
    zq[i] = z * q64[i];
  }
  __device__ static void finish(PcgState *, const double *) {}
};

// q = K p with the products p_i q_i (batched systems)
struct OpStorePQ {
  static constexpr int NV = 0;
  const double *p;
  double *q, *prod;
  __device__ void row(int i, double y, double *) const {
    q[i] = y;
    prod[i] = p[i] * y;
  }
  __device__ static void finish(PcgState *, const double *) {}
};

// ---------------------------------------------------------------------------
// level SpMV kernels: y = A v with a row operator.  Every kernel returns at
// once when the solve has stopped (graph chunks past convergence are empty).
// ---------------------------------------------------------------------------

// level 0 in 3x3 block rows, values component-major per block row (as the
// handle keeps them): LPR lanes per block row
// (6 resident blocks per SM for FP32 -- 40 registers; 4 for FP64, whose
// operators with the outer coupling need more registers)
template <typename T, int LPR, class Op, int UNR = 2>
__global__ void __launch_bounds__(TPB, sizeof(T) == 8 ? 4 : (UNR > 2 ? 4 : 6))
    k_lv_bsr3(int nb, const int *__restrict__ browptr, const int *__restrict__ bcol, const T *__restrict__ bval,
              const T *__restrict__ v, Op op, PcgState *st, double *partials, unsigned *ticket) {
  if (st->done) return;
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, g = lane / LPR, sub = lane % LPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double acc[Op::NV > 0 ? Op::NV : 1] = {};
  for (int base = warp * RPW; base < nb; base += nwarps * RPW) {
    const int br = base + g;
    int s = 0, nbr = 0;
    if (br < nb) { s = __ldg(browptr + br); nbr = __ldg(browptr + br + 1) - s; }
    const T *bv = bval + 9ll * s;
    T y0 = 0, y1 = 0, y2 = 0;
    int j = sub;
    if constexpr (UNR == 4) {
      // four blocks of the row in flight per lane: twice the loads of the
      // two-block loop before the first x gather depends on them
      for (; j + 3 * LPR < nbr; j += 4 * LPR) {
        int c[4];
        T a[4][9];
#pragma unroll
        for (int u = 0; u < 4; u++) c[u] = __ldcs(bcol + s + j + u * LPR);
#pragma unroll
        for (int q = 0; q < 9; q++)
#pragma unroll
          for (int u = 0; u < 4; u++) a[u][q] = __ldcs(bv + q * nbr + j + u * LPR);
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const T x0 = __ldg(v + 3 * c[u]), x1 = __ldg(v + 3 * c[u] + 1), x2 = __ldg(v + 3 * c[u] + 2);
          y0 += a[u][0] * x0 + a[u][1] * x1 + a[u][2] * x2;
          y1 += a[u][3] * x0 + a[u][4] * x1 + a[u][5] * x2;
          y2 += a[u][6] * x0 + a[u][7] * x1 + a[u][8] * x2;
        }
      }
    }
    for (; j + LPR < nbr; j += 2 * LPR) {
      const int j2 = j + LPR;
      const int c = __ldcs(bcol + s + j), c2 = __ldcs(bcol + s + j2);
      T a[9], w[9];
#pragma unroll
      for (int q = 0; q < 9; q++) { a[q] = __ldcs(bv + q * nbr + j); w[q] = __ldcs(bv + q * nbr + j2); }
      const T x0 = __ldg(v + 3 * c), x1 = __ldg(v + 3 * c + 1), x2 = __ldg(v + 3 * c + 2);
      const T z0 = __ldg(v + 3 * c2), z1 = __ldg(v + 3 * c2 + 1), z2 = __ldg(v + 3 * c2 + 2);
      y0 += a[0] * x0 + a[1] * x1 + a[2] * x2 + w[0] * z0 + w[1] * z1 + w[2] * z2;
      y1 += a[3] * x0 + a[4] * x1 + a[5] * x2 + w[3] * z0 + w[4] * z1 + w[5] * z2;
      y2 += a[6] * x0 + a[7] * x1 + a[8] * x2 + w[6] * z0 + w[7] * z1 + w[8] * z2;
    }
    if (j < nbr) {
      const int c = __ldcs(bcol + s + j);
      T a[9];
#pragma unroll
      for (int q = 0; q < 9; q++) a[q] = __ldcs(bv + q * nbr + j);
      const T x0 = __ldg(v + 3 * c), x1 = __ldg(v + 3 * c + 1), x2 = __ldg(v + 3 * c + 2);
      y0 += a[0] * x0 + a[1] * x1 + a[2] * x2;
      y1 += a[3] * x0 + a[4] * x1 + a[5] * x2;
      y2 += a[6] * x0 + a[7] * x1 + a[8] * x2;
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      y0 += __shfl_xor_sync(0xffffffffu, y0, o, LPR);
      y1 += __shfl_xor_sync(0xffffffffu, y1, o, LPR);
      y2 += __shfl_xor_sync(0xffffffffu, y2, o, LPR);
    }
    if (sub < 3 && br < nb) op.row(3 * br + sub, sub == 0 ? y0 : (sub == 1 ? y1 : y2), acc);
  }
  op_reduce<Op>(op, acc, st, partials, ticket);
}

// ----- level 0 of the FP32 cycle with half-precision values -----
// The scaled level-0 matrix S K S has a unit diagonal and |a_ij| <= 1 (an SPD
// matrix has a_ij^2 <= a_ii a_jj), so binary16 holds its entries with a
// relative rounding of 2^-11 and no overflow; entries below 2^-14 lose
// relative precision (absolutely at most 2^-25 against the unit diagonal).
// The cycle is a preconditioner of a flexible CG whose residual and update
// stay FP64, so this rounding changes the preconditioner slightly, never the
// answer, and halves the bytes of the two level-0 products of every cycle.
// Arithmetic and the vectors stay FP32.
//
// Layout: block row br holds blocks [hptr[br], hptr[br+1]) of the padded
// arrays, a multiple of four; value (comp, j) of the row at
// hval[9 hptr[br] + comp len + j].  A lane takes four consecutive blocks: one
// 16-byte load of their columns and nine 8-byte loads of their components.
__device__ __forceinline__ float2 h2f(unsigned bits) {
  __half2 h;
  memcpy(&h, &bits, sizeof(h));
  return __half22float2(h);
}

template <int LPR, int UNR, class Op>
__global__ void __launch_bounds__(TPB, UNR == 2 ? 4 : 6)
    k_lv_h16(int nb, const int *__restrict__ hptr, const int *__restrict__ hcol, const uint16_t *__restrict__ hval,
             const float *__restrict__ v, Op op, PcgState *st, double *partials, unsigned *ticket) {
  if (st->done) return;
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, g = lane / LPR, sub = lane % LPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double acc[Op::NV > 0 ? Op::NV : 1] = {};
  for (int base = warp * RPW; base < nb; base += nwarps * RPW) {
    const int br = base + g;
    int s = 0, len = 0;
    if (br < nb) { s = __ldg(hptr + br); len = __ldg(hptr + br + 1) - s; }
    const uint16_t *bv = hval + 9ll * s;
    float y0 = 0.f, y1 = 0.f, y2 = 0.f;
    for (int j = 4 * sub; j < len; j += 4 * LPR * UNR) {
      int4 c[UNR];
      uint2 a[UNR][9];
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        const int ju = j + 4 * LPR * u;
        if (ju < len) {
          c[u] = __ldcs(reinterpret_cast<const int4 *>(hcol + s + ju));
#pragma unroll
          for (int q = 0; q < 9; q++) a[u][q] = __ldcs(reinterpret_cast<const uint2 *>(bv + q * len + ju));
        } else {
          c[u] = make_int4(0, 0, 0, 0);
#pragma unroll
          for (int q = 0; q < 9; q++) a[u][q] = make_uint2(0u, 0u);
        }
      }
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        if (j + 4 * LPR * u >= len) continue;
        const int cols[4] = {c[u].x, c[u].y, c[u].z, c[u].w};
#pragma unroll
        for (int h = 0; h < 2; h++) {  // blocks 2h, 2h+1 of the four
          float2 w[9];
#pragma unroll
          for (int q = 0; q < 9; q++) w[q] = h2f(h == 0 ? a[u][q].x : a[u][q].y);
          const int ca = cols[2 * h], cb = cols[2 * h + 1];
          const float xa0 = __ldg(v + 3 * ca), xa1 = __ldg(v + 3 * ca + 1), xa2 = __ldg(v + 3 * ca + 2);
          const float xb0 = __ldg(v + 3 * cb), xb1 = __ldg(v + 3 * cb + 1), xb2 = __ldg(v + 3 * cb + 2);
          y0 += w[0].x * xa0 + w[1].x * xa1 + w[2].x * xa2 + w[0].y * xb0 + w[1].y * xb1 + w[2].y * xb2;
          y1 += w[3].x * xa0 + w[4].x * xa1 + w[5].x * xa2 + w[3].y * xb0 + w[4].y * xb1 + w[5].y * xb2;
          y2 += w[6].x * xa0 + w[7].x * xa1 + w[8].x * xa2 + w[6].y * xb0 + w[7].y * xb1 + w[8].y * xb2;
        }
      }
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      y0 += __shfl_xor_sync(0xffffffffu, y0, o, LPR);
      y1 += __shfl_xor_sync(0xffffffffu, y1, o, LPR);
      y2 += __shfl_xor_sync(0xffffffffu, y2, o, LPR);
    }
    if (sub < 3 && br < nb) op.row(3 * br + sub, sub == 0 ? y0 : (sub == 1 ? y1 : y2), acc);
  }
  op_reduce<Op>(op, acc, st, partials, ticket);
}

// padded row lengths (multiples of four blocks)
__global__ void k_h16_len(int nb, const int *__restrict__ browptr, int *__restrict__ len) {
  for (int br = blockIdx.x * blockDim.x + threadIdx.x; br < nb; br += gridDim.x * blockDim.x)
    len[br] = (browptr[br + 1] - browptr[br] + 3) & ~3;
}

// padded columns: one warp per block row
__global__ void k_h16_cols(int nb, const int *__restrict__ browptr, const int *__restrict__ bcol,
                           const int *__restrict__ hptr, int *__restrict__ hcol) {
  const int lane = threadIdx.x & 31;
  for (int br = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; br < nb; br += (gridDim.x * blockDim.x) >> 5) {
    const int s = browptr[br], len = browptr[br + 1] - s;
    const int hs = hptr[br], hlen = hptr[br + 1] - hs;
    for (int j = lane; j < hlen; j += 32) hcol[hs + j] = j < len ? bcol[s + j] : br;
  }
}

// padded binary16 values from the scaled FP32 values (round to nearest even):
// one warp per block row, over its (component, block) pairs
__global__ void k_h16_vals(int nb, const int *__restrict__ browptr, const float *__restrict__ b32,
                           const int *__restrict__ hptr, uint16_t *__restrict__ hval) {
  const int lane = threadIdx.x & 31;
  for (int br = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; br < nb; br += (gridDim.x * blockDim.x) >> 5) {
    const int s = browptr[br], len = browptr[br + 1] - s;
    const int hs = hptr[br], hlen = hptr[br + 1] - hs;
    for (int q = 0; q < 9; q++)
      for (int j = lane; j < hlen; j += 32) {
        const __half h = __float2half_rn(j < len ? b32[9ll * s + (int64_t)q * len + j] : 0.f);
        uint16_t bits;
        memcpy(&bits, &h, sizeof(bits));
        hval[9ll * hs + (int64_t)q * hlen + j] = bits;
      }
  }
}

// ----- level 0 in FP32 BSR3, streamed through shared memory by bulk copies -----
// A tile is kLvTileRows consecutive block rows.  Its values (component-major
// per row) and column indices are two contiguous byte ranges, so one bulk
// copy each (cp.async.bulk, completion on an mbarrier) brings the tile into a
// stage buffer; kLvStages tiles are in flight per CTA while the oldest is
// multiplied, whatever the registers and occupancy of the arithmetic.  The
// copies start at the 16-byte boundary at or below a range's first byte and
// end at the one at or above its last (the arrays carry 16 bytes of slack).
// Every wait is bounded by time; one that runs out sets SGPU_CUDA_ERROR in
// the solver state, waits (bounded) for the copies still in flight and ends
// the kernel.
constexpr int kLvTileRows = 32;  // 8 lanes per block row, 256 threads
constexpr int kLvStages = 3;
constexpr uint64_t kLvWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// waits for phase `parity` of *bar to complete; false after kLvWaitNs
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_test(bar, parity))
    if (global_ns() - t0 > kLvWaitNs) return false;
  return true;
}

// global -> this CTA's shared memory, completion counted on *bar (both
// addresses 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

struct LvTile {
  int vbytes, cbytes;  // a stage's value and column buffers
  __host__ __device__ static LvTile of(int cap_blocks) {
    return LvTile{(36 * cap_blocks + 32 + 15) & ~15, (4 * cap_blocks + 32 + 15) & ~15};
  }
  __host__ __device__ int stage_bytes() const { return vbytes + cbytes; }
  __host__ __device__ size_t smem_bytes() const { return (size_t)kLvStages * stage_bytes() + kLvStages * 8; }
};

template <class Op>
__global__ void __launch_bounds__(TPB) k_lv_bsr3_tma(int nb, int cap_blocks, const int *__restrict__ browptr,
                                                     const int *__restrict__ bcol, const float *__restrict__ bval,
                                                     const float *__restrict__ v, Op op, PcgState *st,
                                                     double *partials, unsigned *ticket) {
  static_assert(TPB == kLvTileRows * 8, "one 8-lane group per block row of a tile");
  if (st->done) return;
  extern __shared__ __align__(128) unsigned char lv_sm[];
  const LvTile lt = LvTile::of(cap_blocks);
  const int sb = lt.stage_bytes();
  uint64_t *bar = reinterpret_cast<uint64_t *>(lv_sm + (size_t)kLvStages * sb);
  const int tid = threadIdx.x, g = tid >> 3, sub = tid & 7;
  const int ntiles = (nb + kLvTileRows - 1) / kLvTileRows;
  auto issue = [&](int t, int q) {
    const int r0 = t * kLvTileRows, r1 = min(nb, r0 + kLvTileRows);
    const int64_t b0 = __ldg(browptr + r0), b1 = __ldg(browptr + r1);
    const int64_t vs = (36 * b0) & ~15ll, ve = (36 * b1 + 15) & ~15ll;
    const int64_t cs = (4 * b0) & ~15ll, ce = (4 * b1 + 15) & ~15ll;
    unsigned char *dst = lv_sm + (size_t)q * sb;
    mbar_expect_tx(&bar[q], (unsigned)((ve - vs) + (ce - cs)));
    if (ve > vs) bulk_g2s(dst, reinterpret_cast<const unsigned char *>(bval) + vs, (unsigned)(ve - vs), &bar[q]);
    if (ce > cs)
      bulk_g2s(dst + lt.vbytes, reinterpret_cast<const unsigned char *>(bcol) + cs, (unsigned)(ce - cs), &bar[q]);
  };
  if (tid == 0) {
    for (int q = 0; q < kLvStages; q++) mbar_init(&bar[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int q = 0; q < kLvStages; q++) {
      const int t = blockIdx.x + q * gridDim.x;
      if (t < ntiles) issue(t, q);
    }
  double acc[Op::NV > 0 ? Op::NV : 1] = {};
  int k = 0;
  bool failed = false;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, k++) {
    const int q = k % kLvStages;
    const unsigned par = (unsigned)(k / kLvStages) & 1u;
    if (__syncthreads_or(!mbar_wait_bounded(&bar[q], par))) {
      failed = true;
      break;
    }
    const int r0 = t * kLvTileRows, br = r0 + g;
    const int b0 = __ldg(browptr + r0);
    const float *sv = reinterpret_cast<const float *>(lv_sm + (size_t)q * sb) + (((36ll * b0) & 15) >> 2);
    const int *sc = reinterpret_cast<const int *>(lv_sm + (size_t)q * sb + lt.vbytes) + (((4ll * b0) & 15) >> 2);
    float y0 = 0.f, y1 = 0.f, y2 = 0.f;
    if (br < nb) {
      const int s = __ldg(browptr + br), nbr = __ldg(browptr + br + 1) - s;
      const float *a = sv + 9 * (s - b0);
      const int *cc = sc + (s - b0);
#pragma unroll 4
      for (int j = sub; j < nbr; j += 8) {
        const int c = cc[j];
        const float x0 = __ldg(v + 3 * c), x1 = __ldg(v + 3 * c + 1), x2 = __ldg(v + 3 * c + 2);
        y0 += a[j] * x0 + a[nbr + j] * x1 + a[2 * nbr + j] * x2;
        y1 += a[3 * nbr + j] * x0 + a[4 * nbr + j] * x1 + a[5 * nbr + j] * x2;
        y2 += a[6 * nbr + j] * x0 + a[7 * nbr + j] * x1 + a[8 * nbr + j] * x2;
      }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      y0 += __shfl_xor_sync(0xffffffffu, y0, o, 8);
      y1 += __shfl_xor_sync(0xffffffffu, y1, o, 8);
      y2 += __shfl_xor_sync(0xffffffffu, y2, o, 8);
    }
    if (sub < 3 && br < nb) op.row(3 * br + sub, sub == 0 ? y0 : (sub == 1 ? y1 : y2), acc);
    __syncthreads();  // stage q is read: the tile kLvStages ahead may overwrite it
    if (tid == 0 && t + kLvStages * (int)gridDim.x < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(t + kLvStages * gridDim.x, q);
    }
  }
  if (failed && tid == 0) {
    // the copies issued and not yet seen complete: tiles k .. k + kLvStages - 1
    for (int d = 0; d < kLvStages; d++) {
      const int t = blockIdx.x + (k + d) * gridDim.x;
      if (t >= ntiles) break;
      mbar_wait_bounded(&bar[(k + d) % kLvStages], (unsigned)((k + d) / kLvStages) & 1u);
    }
    atomicCAS(&st->status, 0, (int)SGPU_CUDA_ERROR);
    st->done = 1;
  }
  // the grid reduction runs in any case, so that its ticket returns to zero
  op_reduce<Op>(op, acc, st, partials, ticket);
}

// level 0 in scalar CSR: L lanes per row
template <typename T, int L, class Op>
__global__ void __launch_bounds__(TPB) k_lv_csr(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                                                const T *__restrict__ val, const T *__restrict__ v, Op op,
                                                PcgState *st, double *partials, unsigned *ticket) {
  if (st->done) return;
  constexpr int GPW = 32 / L;
  const int lane = threadIdx.x & 31, g = lane / L, sub = lane % L;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double acc[Op::NV > 0 ? Op::NV : 1] = {};
  for (int base = warp * GPW; base < n; base += nwarps * GPW) {
    const int i = base + g;
    int b = 0, e = 0;
    if (i < n) { b = __ldg(rowptr + i); e = __ldg(rowptr + i + 1); }
    T s = 0;
    for (int k = b + sub; k < e; k += L) s += __ldcs(val + k) * __ldg(v + __ldcs(col + k));
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, L);
    if (sub == 0 && i < n) op.row(i, s, acc);
  }
  op_reduce<Op>(op, acc, st, partials, ticket);
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

// coarse levels: B x B blocks stored row-major, one warp per block row
template <typename T, int B, class Op>
__global__ void __launch_bounds__(TPB) k_lv_bsrb(int nb, const int *__restrict__ browptr,
                                                 const int *__restrict__ bcol, const T *__restrict__ bval,
                                                 const T *__restrict__ v, Op op, PcgState *st, double *partials,
                                                 unsigned *ticket) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double acc[Op::NV > 0 ? Op::NV : 1] = {};
  for (int br = warp; br < nb; br += nwarps) {
    const int s = __ldg(browptr + br), e = __ldg(browptr + br + 1);
    T y[B];
#pragma unroll
    for (int c = 0; c < B; c++) y[c] = 0;
    for (int k = s + lane; k < e; k += 32) {
      const int c = __ldg(bcol + k);
      T a[B * B];
      load_block<T, B>(bval + (size_t)k * B * B, a);
      T xv[B];
#pragma unroll
      for (int q = 0; q < B; q++) xv[q] = __ldg(v + B * c + q);
#pragma unroll
      for (int r = 0; r < B; r++) {
#pragma unroll
        for (int q = 0; q < B; q++) y[r] += a[r * B + q] * xv[q];
      }
    }
#pragma unroll
    for (int r = 0; r < B; r++) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) y[r] += __shfl_xor_sync(0xffffffffu, y[r], o);
    }
    if (lane < B) {
      T yv = y[0];
#pragma unroll
      for (int r = 1; r < B; r++)
        if (lane == r) yv = y[r];
      op.row(B * br + lane, yv, acc);
    }
  }
  op_reduce<Op>(op, acc, st, partials, ticket);
}

// ---------------------------------------------------------------------------
// transfer kernels
// ---------------------------------------------------------------------------

// b_c = Q^T res over each aggregate (one warp per aggregate).  With START the
// coarse level's smoothing starts here from x = 0: r = D^-1 b, d = x = c2 r.
template <typename T, int B, int K, bool START>
__global__ void __launch_bounds__(TPB) k_restrict(int na, const int *__restrict__ aggptr,
                                                  const int *__restrict__ aggnodes, const T *__restrict__ Q,
                                                  const T *__restrict__ res, T *__restrict__ bc, T *__restrict__ rc,
                                                  T *__restrict__ dc, T *__restrict__ xc, const T *__restrict__ dinvc,
                                                  T c2, const PcgState *st) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int G = warp; G < na; G += nwarps) {
    const int s = __ldg(aggptr + G), e = __ldg(aggptr + G + 1);
    T acc[K];
#pragma unroll
    for (int q = 0; q < K; q++) acc[q] = 0;
    for (int t = s + lane; t < e; t += 32) {
      const int i = __ldg(aggnodes + t);
#pragma unroll
      for (int c = 0; c < B; c++) {
        const T rv = res[B * i + c];
        const T *qr = Q + ((size_t)B * i + c) * K;
#pragma unroll
        for (int q = 0; q < K; q++) acc[q] += __ldg(qr + q) * rv;
      }
    }
#pragma unroll
    for (int q = 0; q < K; q++) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    }
    if (lane < K) {
      T v = acc[0];
#pragma unroll
      for (int q = 1; q < K; q++)
        if (lane == q) v = acc[q];
      const int p = K * G + lane;
      bc[p] = v;
      if (START) {
        const T ri = dinvc[p] * v;
        rc[p] = ri;
        dc[p] = c2 * ri;
        xc[p] = c2 * ri;
      }
    }
  }
}

// x += alpha Q x_c (one thread per equation)
template <typename T, int B, int K>
__global__ void __launch_bounds__(TPB) k_prolong(int n, const int *__restrict__ agg, const T *__restrict__ Q,
                                                 const T *__restrict__ xc, T *__restrict__ x, T alpha,
                                                 const PcgState *st) {
  if (st->done) return;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int G = __ldg(agg + p / B);
    const T *qr = Q + (size_t)p * K;
    T s = 0;
#pragma unroll
    for (int q = 0; q < K; q++) s += __ldg(qr + q) * __ldg(xc + K * G + q);
    x[p] = x[p] + mul_rn(alpha, s);
  }
}

// x_c = M^-1 b_c with the dense inverse of the coarsest level (warp per row)
template <typename T>
__global__ void __launch_bounds__(TPB) k_dense_mv(int nc, const T *__restrict__ M, const T *__restrict__ b,
                                                  T *__restrict__ x, const PcgState *st) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < nc; i += nwarps) {
    const T *row = M + (size_t)i * nc;
    T s = 0;
    for (int j = lane; j < nc; j += 32) s += __ldg(row + j) * __ldg(b + j);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) x[i] = s;
  }
}

// ---------------------------------------------------------------------------
// the coarse tail of the cycle in one launch
//
// The last smoothed level (a few thousand equations) and the dense coarsest
// level below it are visited gamma times per visit of the level above, each
// visit a chain of small dependent steps (smoothing, residual, restriction,
// dense solve, prolongation, smoothing) that as separate launches cost a
// launch latency each while doing a microsecond of work.  Here one thread-
// block cluster runs all the visits of one coarse correction: the cluster's
// CTAs split every step's rows, and a cluster barrier (release/acquire at
// cluster scope, no spinning) separates the steps.  Every row is computed
// with the same loop and summation order as the separate kernels above
// (k_lv_bsrb, k_restrict, k_dense_mv, k_prolong), so both forms give the same
// bits.  Vectors written inside the launch are read through L2 (ld.global.cg),
// never through the non-coherent read-only path.
// ---------------------------------------------------------------------------
constexpr int kTailThreads = 512;

template <typename T>
struct TailArgs {
  int nb;                                       // block rows of the level
  const int *browptr, *bcol;
  const T *val, *dinv;                          // B x B row-major blocks; D^-1 (NULL: unit diagonal)
  const T *b;                                   // the level's right-hand side
  T *x, *x2, *res;                              // x holds the first smoothing step (from the restriction)
  int na;                                       // aggregates of the level = dense rows / K
  const int *aggptr, *aggnodes, *agg;
  const T *Q;                                   // n x K tentative prolongator
  int nc;                                       // dense coarsest equations
  const T *M;                                   // its inverse, nc x nc row-major
  T *cb, *cx;
  T c2, alpha;                                  // first Chebyshev coefficient, coarse-correction weight
  int visits;
  const PcgState *st;
};

// (A v) of block row br, the lanes' partial sums reduced as k_lv_bsrb does;
// lane r < B returns y_r
template <typename T, int B>
__device__ __forceinline__ T tail_bsrb_row(const TailArgs<T> &a, int br, int lane, const T *v) {
  const int s = __ldg(a.browptr + br), e = __ldg(a.browptr + br + 1);
  T y[B];
#pragma unroll
  for (int c = 0; c < B; c++) y[c] = 0;
  for (int k = s + lane; k < e; k += 32) {
    const int c = __ldg(a.bcol + k);
    T blk[B * B];
    load_block<T, B>(a.val + (size_t)k * B * B, blk);
    T xv[B];
#pragma unroll
    for (int q = 0; q < B; q++) xv[q] = __ldcg(v + B * c + q);
#pragma unroll
    for (int r = 0; r < B; r++) {
#pragma unroll
      for (int q = 0; q < B; q++) y[r] += blk[r * B + q] * xv[q];
    }
  }
#pragma unroll
  for (int r = 0; r < B; r++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) y[r] += __shfl_xor_sync(0xffffffffu, y[r], o);
  }
  T yv = y[0];
#pragma unroll
  for (int r = 1; r < B; r++)
    if (lane == r) yv = y[r];
  return yv;
}

// to = from + c2 D^-1 (b - A from)   (a first Chebyshev step, OpCheb FIRST)
template <typename T, int B>
__device__ __forceinline__ void tail_smooth(const TailArgs<T> &a, int gw, int nw, int lane, const T *from, T *to) {
  for (int br = gw; br < a.nb; br += nw) {
    const T y = tail_bsrb_row<T, B>(a, br, lane, from);
    if (lane < B) {
      const int i = B * br + lane;
      const T di_ = a.dinv ? __ldg(a.dinv + i) : T(1);
      const T ri = di_ * (__ldg(a.b + i) - y);
      const T di = mul_rn(a.c2, ri);
      to[i] = __ldcg(from + i) + di;
    }
  }
}

template <typename T, int B, int K>
__global__ void __launch_bounds__(kTailThreads) k_coarse_tail(TailArgs<T> a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  if (a.st->done) return;  // the same for every CTA: nothing writes the state during the launch
  const int lane = threadIdx.x & 31;
  const int wpc = kTailThreads / 32;
  const int gw = (int)cluster.block_rank() * wpc + (threadIdx.x >> 5);
  const int nw = (int)cluster.num_blocks() * wpc;
  const int gt = (int)cluster.block_rank() * kTailThreads + threadIdx.x;
  const int nt = (int)cluster.num_blocks() * kTailThreads;
  T *xp = a.x;
  for (int v = 0; v < a.visits; v++) {
    if (v > 0) {  // pre-smoothing from the previous visit's result
      T *to = (xp == a.x) ? a.x2 : a.x;
      tail_smooth<T, B>(a, gw, nw, lane, xp, to);
      xp = to;
      cluster.sync();
    }
    // residual
    for (int br = gw; br < a.nb; br += nw) {
      const T y = tail_bsrb_row<T, B>(a, br, lane, xp);
      if (lane < B) a.res[B * br + lane] = __ldg(a.b + B * br + lane) - y;
    }
    cluster.sync();
    // restriction to the dense level: cb = Q^T res per aggregate
    for (int G = gw; G < a.na; G += nw) {
      const int s = __ldg(a.aggptr + G), e = __ldg(a.aggptr + G + 1);
      T acc[K];
#pragma unroll
      for (int q = 0; q < K; q++) acc[q] = 0;
      for (int t = s + lane; t < e; t += 32) {
        const int i = __ldg(a.aggnodes + t);
#pragma unroll
        for (int c = 0; c < B; c++) {
          const T rv = __ldcg(a.res + B * i + c);
          const T *qr = a.Q + ((size_t)B * i + c) * K;
#pragma unroll
          for (int q = 0; q < K; q++) acc[q] += __ldg(qr + q) * rv;
        }
      }
#pragma unroll
      for (int q = 0; q < K; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
      }
      if (lane < K) {
        T vq = acc[0];
#pragma unroll
        for (int q = 1; q < K; q++)
          if (lane == q) vq = acc[q];
        a.cb[K * G + lane] = vq;
      }
    }
    cluster.sync();
    // dense coarsest solve: cx = M cb
    for (int i = gw; i < a.nc; i += nw) {
      const T *row = a.M + (size_t)i * a.nc;
      T sum = 0;
      for (int j = lane; j < a.nc; j += 32) sum += __ldg(row + j) * __ldcg(a.cb + j);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (lane == 0) a.cx[i] = sum;
    }
    cluster.sync();
    // prolongation: xp += alpha Q cx
    for (int p = gt; p < B * a.nb; p += nt) {
      const int G = __ldg(a.agg + p / B);
      const T *qr = a.Q + (size_t)p * K;
      T sum = 0;
#pragma unroll
      for (int q = 0; q < K; q++) sum += __ldg(qr + q) * __ldcg(a.cx + K * G + q);
      xp[p] = __ldcg(xp + p) + mul_rn(a.alpha, sum);
    }
    cluster.sync();
    // post-smoothing
    {
      T *to = (xp == a.x) ? a.x2 : a.x;
      tail_smooth<T, B>(a, gw, nw, lane, xp, to);
      xp = to;
    }
    cluster.sync();
  }
}

// ---------------------------------------------------------------------------
// flexible CG kernels (FP64) and the start of the level-0 smoothing
// ---------------------------------------------------------------------------

// r = f - K x0 (q holds K x0); f.f and r.r; level-0 right-hand side S r and
// the first Chebyshev step from zero (unit diagonal: r0 = b0, d0 = x0 = c2 b0)
template <typename T>
__global__ void __launch_bounds__(TPB) k_fcg_init(int n, const double *__restrict__ f, const double *__restrict__ q,
                                                  double *__restrict__ r, const double *__restrict__ dscale,
                                                  T *__restrict__ b0, T *__restrict__ r0, T *__restrict__ d0,
                                                  T *__restrict__ x0, T c2, PcgState *st, double *partials,
                                                  unsigned *ticket) {
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double fi = f[i], ri = fi - q[i];
    r[i] = ri;
    v[0] += fi * fi;
    v[1] += ri * ri;
    const T bi = (T)(dscale[i] * ri);
    b0[i] = bi;
    r0[i] = bi;
    d0[i] = c2 * bi;
    x0[i] = c2 * bi;
  }
  double t[2];
  if (reduce_grid<2>(v, partials, ticket, t)) {
    st->nory = t[0];
    st->ff = t[0];
    st->rr = t[1];
    st->it_last_update = st->it;  // the next V-cycle starts the recurrence: beta = 0
    st->beta = 0.0;
    const bool conv = st->crit == SGPU_CRIT_SCR_PREC ? t[1] < st->res * t[0] : t[1] < st->tol2 * t[0];
    if (t[0] < st->zero) {  // zero right-hand side: x = 0 is the solution
      st->status = SGPU_ZERO_RHS;
      st->done = 1;
    } else if (conv) {
      st->ani = st->it;
      st->ares = t[1] / t[0];
      st->ani_set = 1;
      st->done = 1;
    }
  }
}

// x += alpha p; r -= alpha q; r.r and the stopping test; then the level-0
// right-hand side of the next V-cycle and its first Chebyshev step
template <typename T>
__global__ void __launch_bounds__(TPB) k_fcg_update(int n, double *__restrict__ x, double *__restrict__ r,
                                                    const double *__restrict__ p, const double *__restrict__ q,
                                                    const double *__restrict__ dscale, T *__restrict__ b0,
                                                    T *__restrict__ r0, T *__restrict__ d0, T *__restrict__ x0, T c2,
                                                    PcgState *st, double *partials, unsigned *ticket) {
  if (st->done) return;
  const double alpha = st->alpha;
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * q[i];
    r[i] = ri;
    v[0] += ri * ri;
    const T bi = (T)(dscale[i] * ri);
    b0[i] = bi;
    r0[i] = bi;
    d0[i] = c2 * bi;
    x0[i] = c2 * bi;
  }
  double t[1];
  if (reduce_grid<1>(v, partials, ticket, t)) {
    st->it += 1;
    st->rr = t[0];
    const double ff = st->nory;
    bool conv;
    if (st->crit == SGPU_CRIT_SCR_PREC) conv = t[0] < st->res * ff;       // (r.r)/(f.f) < res
    else conv = t[0] < st->tol2 * ff;                                      // sqrt((r.r)/(f.f)) < res
    if (conv) {
      st->ani = st->it;
      st->ares = t[0] / ff;
      st->ani_set = 1;
      st->done = 1;
    } else if (st->it >= st->ni) {
      st->status = SGPU_NOT_CONVERGED;
      st->done = 1;
    }
  }
}

// p = z + beta p with z = S x0 (x0: the V-cycle's level-0 result)
template <typename T>
__global__ void __launch_bounds__(TPB) k_fcg_dir(int n, double *__restrict__ p, const T *__restrict__ x0,
                                                 const double *__restrict__ dscale, const PcgState *st) {
  if (st->done) return;
  const double beta = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = dscale[i] * (double)x0[i] + beta * p[i];
}

// r = f - q (restart of the recurrence on the true residual); r.r
__global__ void __launch_bounds__(TPB) k_fcg_true(int n, const double *__restrict__ f, const double *__restrict__ q,
                                                  PcgState *st, double *partials, unsigned *ticket) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = f[i] - q[i];
    v[0] += ri * ri;
  }
  double t[1];
  if (reduce_grid<1>(v, partials, ticket, t)) {
    st->true_rr = t[0];
    st->true_rel = st->nory > 0 ? sqrt(t[0] / st->nory) : 0.0;
  }
}

// ---------------------------------------------------------------------------
// many independent systems (diagonal blocks of one matrix), each with its own
// flexible CG scalars: rows carry products, one warp per system sums them in
// row order (deterministic), then updates that system's state
// ---------------------------------------------------------------------------
struct BSys {
  double ff, rr, rho, alpha, beta, ares;
  long long it, it_restart, ani;
  int done, status;
};

__device__ __forceinline__ double seg_sum(const double *__restrict__ v, long long r0, long long r1) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (long long i = r0 + lane; i < r1; i += 32) s += v[i];
  return warp_sum(s);
}

// start of every system's recurrence: f.f and r.r
__global__ void k_bseg_init(int nsys, const long long *__restrict__ sysptr, const double *__restrict__ pff,
                            const double *__restrict__ prr, BSys *sys, double res) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int k = warp; k < nsys; k += nw) {
    const double ff = seg_sum(pff, sysptr[k], sysptr[k + 1]);
    const double rr = seg_sum(prr, sysptr[k], sysptr[k + 1]);
    if (lane == 0) {
      BSys &b = sys[k];
      b.it_restart = b.it;
      b.beta = 0.0;
      if (b.done) continue;
      b.ff = ff;
      b.rr = rr;
      if (ff < 1e-300) {
        b.done = 1;
        b.status = SGPU_ZERO_RHS;
      } else if (rr < res * ff) {
        b.done = 1;
        b.ani = b.it;
        b.ares = rr / ff;
      }
    }
  }
}

__global__ void k_bseg_alpha(int nsys, const long long *__restrict__ sysptr, const double *__restrict__ ppq,
                             BSys *sys) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int k = warp; k < nsys; k += nw) {
    if (sys[k].done) {
      if (lane == 0) sys[k].alpha = 0.0;
      continue;
    }
    const double pq = seg_sum(ppq, sysptr[k], sysptr[k + 1]);
    if (lane == 0) {
      BSys &b = sys[k];
      if (!(pq > 0.0)) {
        b.done = 1;
        b.status = SGPU_BREAKDOWN;
        b.alpha = 0.0;
      } else {
        b.alpha = b.rho / pq;
      }
    }
  }
}

__global__ void k_bseg_rr(int nsys, const long long *__restrict__ sysptr, const double *__restrict__ prr, BSys *sys,
                          long long ni, double res) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int k = warp; k < nsys; k += nw) {
    if (sys[k].done) continue;
    const double rr = seg_sum(prr, sysptr[k], sysptr[k + 1]);
    if (lane == 0) {
      BSys &b = sys[k];
      b.it += 1;
      b.rr = rr;
      if (rr < res * b.ff) {  // (r.r)/(f.f) < res per system, symcomprow::cg_prec's test
        b.done = 1;
        b.ani = b.it;
        b.ares = rr / b.ff;
      } else if (b.it >= ni) {
        b.done = 1;
        b.status = SGPU_NOT_CONVERGED;
      }
    }
  }
}

__global__ void k_bseg_beta(int nsys, const long long *__restrict__ sysptr, const double *__restrict__ pzr,
                            const double *__restrict__ pzq, BSys *sys) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int k = warp; k < nsys; k += nw) {
    if (sys[k].done) continue;
    const double rz = seg_sum(pzr, sysptr[k], sysptr[k + 1]);
    const double zq = seg_sum(pzq, sysptr[k], sysptr[k + 1]);
    if (lane == 0) {
      BSys &b = sys[k];
      if (!(rz > 0.0) || !isfinite(zq)) {
        b.done = 1;
        b.status = SGPU_BREAKDOWN;
      } else {
        b.beta = b.it > b.it_restart ? -b.alpha * zq / b.rho : 0.0;
        b.rho = rz;
      }
    }
  }
}

// the solve stops (every kernel returns at once) when no system is active
__global__ void k_bcount(int nsys, const BSys *sys, PcgState *st) {
  __shared__ int act;
  if (threadIdx.x == 0) act = 0;
  __syncthreads();
  int c = 0;
  for (int k = threadIdx.x; k < nsys; k += blockDim.x) c += sys[k].done ? 0 : 1;
  if (c) atomicAdd(&act, c);
  __syncthreads();
  if (threadIdx.x == 0 && act == 0) st->done = 1;
}

// r = f - q (q = K x0), the products f_i^2 and r_i^2, level-0 right-hand side
template <typename T>
__global__ void __launch_bounds__(TPB) k_b_init_rows(int n, const double *__restrict__ f, const double *__restrict__ q,
                                                     double *__restrict__ r, const double *__restrict__ dscale,
                                                     T *__restrict__ b0, T *__restrict__ r0, T *__restrict__ d0,
                                                     T *__restrict__ x0, T c2, double *__restrict__ pff,
                                                     double *__restrict__ prr) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double fi = f[i], ri = fi - q[i];
    r[i] = ri;
    pff[i] = fi * fi;
    prr[i] = ri * ri;
    const T bi = (T)(dscale[i] * ri);
    b0[i] = bi;
    r0[i] = bi;
    d0[i] = c2 * bi;
    x0[i] = c2 * bi;
  }
}

template <typename T>
__global__ void __launch_bounds__(TPB) k_b_update(int n, const int *__restrict__ rowsys, const BSys *sys,
                                                  double *__restrict__ x, double *__restrict__ r,
                                                  const double *__restrict__ p, const double *__restrict__ q,
                                                  const double *__restrict__ dscale, T *__restrict__ b0,
                                                  T *__restrict__ r0, T *__restrict__ d0, T *__restrict__ x0, T c2,
                                                  double *__restrict__ prr, const PcgState *st) {
  if (st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double al = sys[rowsys[i]].alpha;
    x[i] += al * p[i];
    const double ri = r[i] - al * q[i];
    r[i] = ri;
    prr[i] = ri * ri;
    const T bi = (T)(dscale[i] * ri);
    b0[i] = bi;
    r0[i] = bi;
    d0[i] = c2 * bi;
    x0[i] = c2 * bi;
  }
}

template <typename T>
__global__ void __launch_bounds__(TPB) k_b_dir(int n, const int *__restrict__ rowsys, const BSys *sys,
                                               double *__restrict__ p, const T *__restrict__ x0,
                                               const double *__restrict__ dscale, const PcgState *st) {
  if (st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const BSys &b = sys[rowsys[i]];
    if (b.done) continue;
    p[i] = dscale[i] * (double)x0[i] + b.beta * p[i];
  }
}

__global__ void k_b_rowsys(int nsys, const long long *__restrict__ sysptr, int *__restrict__ rowsys) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (int k = warp; k < nsys; k += nw)
    for (long long i = sysptr[k] + lane; i < sysptr[k + 1]; i += 32) rowsys[i] = k;
}

// ---------------------------------------------------------------------------
// set-up kernels
// ---------------------------------------------------------------------------

// FP64 values of a level for the set-up.  layout 1: the handle's BSR3
// (component-major per block row, unscaled), 2: the handle's CSR (unscaled),
// 0: an owned coarse level (row-major B x B blocks, already scaled).
struct LevelView {
  int layout;
  const int *browptr, *bcol;
  const double *val;
  const double *dscale;
  template <int B>
  __device__ __forceinline__ double get(int i, int e, int c) const {
    if (layout == 1) {
      const int s = browptr[i], nbr = browptr[i + 1] - s;
      const int j = bcol[e];
      return val[9ll * s + (int64_t)c * nbr + (e - s)] * dscale[3 * i + c / 3] * dscale[3 * j + c % 3];
    }
    if (layout == 2) return val[e] * dscale[i] * dscale[bcol[e]];
    return val[(size_t)e * B * B + c];
  }
};

__global__ void k_block_rows(int nb, const int *__restrict__ browptr, int *__restrict__ rowid) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    for (int e = browptr[i]; e < browptr[i + 1]; e++) rowid[e] = i;
}

// level-0 scaled FP64 copy for the FP64 V-cycle (same layout as the source);
// one warp per (block) row, lanes over its entries
__global__ void k_scale_level0(int nb, int layout, const int *__restrict__ browptr, const int *__restrict__ bcol,
                               const double *__restrict__ val, const double *__restrict__ dscale,
                               double *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < nb; i += nwarps) {
    const int s = browptr[i], e = browptr[i + 1];
    if (layout == 2) {
      const double si = dscale[i];
      for (int k = s + lane; k < e; k += 32) out[k] = val[k] * si * dscale[bcol[k]];
    } else {
      const int nbr = e - s;
      for (int j = lane; j < nbr; j += 32) {
        const int c = bcol[s + j];
        for (int comp = 0; comp < 9; comp++) {
          const int64_t pos = 9ll * s + (int64_t)comp * nbr + j;
          out[pos] = val[pos] * dscale[3 * i + comp / 3] * dscale[3 * c + comp % 3];
        }
      }
    }
  }
}

__device__ __forceinline__ uint32_t mix32(uint32_t x) {  // integer hash (xorshift-multiply)
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// MIS-2 keys: state in the top 2 bits (0 out, 1 undecided, 2 in), then a
// hash of the index, then the index (ties impossible)
__device__ __forceinline__ uint64_t mis_key(uint32_t state, uint32_t i) {
  return ((uint64_t)state << 62) | ((uint64_t)(mix32(i * 2654435761u + 12345u) >> 2) << 32) | i;
}

// cand == nullptr: every node is a candidate
__global__ void k_mis_init(int nb, const int *__restrict__ cand, uint64_t *__restrict__ t) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    t[i] = mis_key(cand == nullptr || cand[i] ? 1 : 0, i);
}

// max of the keys over the closed neighbourhood; with `agg`, only over the
// subgraph of the nodes not yet aggregated (agg < 0)
// (go: the undecided count the previous round left; 0 = nothing to do)
__global__ void k_mis_max(int nb, const int *__restrict__ browptr, const int *__restrict__ bcol,
                          const int *__restrict__ agg, const uint64_t *__restrict__ in, uint64_t *__restrict__ out,
                          const int *go) {
  if (*go == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    uint64_t m = in[i];
    for (int e = browptr[i]; e < browptr[i + 1]; e++) {
      const int j = bcol[e];
      if (agg == nullptr || agg[j] < 0) m = max(m, in[j]);
    }
    out[i] = m;
  }
}

// The same maximum with LPR lanes per node (coalesced column reads, the
// neighbours' keys gathered in parallel, a shuffle maximum).  DECIDE: the
// second pass of a round, which also makes the round's decision for its
// nodes (k_mis_decide's rule, with m2 = the maximum it just formed), so a
// round is two launches.  The keys and their maxima are those of the
// thread-per-node form, so the independent set is the same.
template <int LPR, bool DECIDE>
__global__ void k_mis_max_w(int nb, const int *__restrict__ browptr, const int *__restrict__ bcol,
                            const int *__restrict__ agg, const uint64_t *__restrict__ in, uint64_t *__restrict__ out,
                            const int *go, uint64_t *__restrict__ t, int *__restrict__ undecided,
                            int *__restrict__ settled) {
  if (*go == 0) return;
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, g = lane / LPR, sub = lane % LPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  int cnt = 0;
  for (int base = warp * RPW; base < nb; base += nwarps * RPW) {
    const int i = base + g;
    uint64_t m = 0;
    // nodes that take no part: an aggregated node (second phase: no node
    // reads its maximum, it has nothing to decide); in the deciding pass, a
    // node already decided (its maximum feeds nothing else); in the first
    // pass, a settled node: one whose closed neighbourhood had no undecided
    // node at an earlier round (decisions are final, so no undecided node
    // will read its maximum again)
    uint64_t ti = 0;
    bool on_i = i < nb && (agg == nullptr || __ldg(agg + i) < 0);
    if (DECIDE && on_i) {
      ti = t[i];
      on_i = (ti >> 62) == 1;
    }
    if (!DECIDE && on_i) on_i = settled[i] == 0;
    int open = 0;  // first pass: an undecided node in the closed neighbourhood
    if (on_i) {
      if (sub == 0) {
        m = in[i];
        open = (m >> 62) == 1;
      }
      const int re = browptr[i + 1];
      // four neighbours per lane in flight: their columns first, then their
      // keys (and aggregate marks)
      for (int e0 = browptr[i] + sub; e0 < re; e0 += 4 * LPR) {
        int js[4];
#pragma unroll
        for (int u = 0; u < 4; u++) js[u] = e0 + u * LPR < re ? __ldg(bcol + e0 + u * LPR) : -1;
        uint64_t kv[4];
        bool on[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          kv[u] = js[u] >= 0 ? in[js[u]] : 0;
          on[u] = js[u] >= 0 && (agg == nullptr || __ldg(agg + js[u]) < 0);
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (on[u]) {
            m = max(m, kv[u]);
            if (!DECIDE) open |= (kv[u] >> 62) == 1;
          }
      }
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) m = max(m, (uint64_t)__shfl_xor_sync(0xffffffffu, (unsigned long long)m, o, LPR));
    if (!DECIDE) {
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) open |= __shfl_xor_sync(0xffffffffu, open, o, LPR);
    }
    if (on_i && sub == 0) {
      if (!DECIDE) {
        out[i] = m;
        if (!open) settled[i] = 1;
      } else {  // ti undecided
        if (m == ti) t[i] = mis_key(2, i);
        else if ((m >> 62) == 2) t[i] = ti & ~(3ull << 62);
        else cnt++;
      }
    }
  }
  if (DECIDE) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(undecided, cnt);
  }
}

// The whole independent-set loop of a small graph in one launch: one
// thread-block cluster runs the rounds of k_mis_max / k_mis_decide (the
// same keys, maxima and decisions, so the same set), a cluster barrier (a
// hardware barrier, no spinning) between the passes of a round, and stops
// after the round that leaves no node undecided or after kMisRounds rounds
// (*rounds_out: the rounds run; cnt[r + 1]: the nodes round r left
// undecided, cnt zeroed by the caller).  Small graphs (the coarse levels)
// otherwise pay a launch per pass and a host read per group of rounds for a
// microsecond of work each.
constexpr int kMisRounds = 200;
constexpr int kMisClusterThreads = 1024;

__global__ void __launch_bounds__(kMisClusterThreads)
    k_mis2_cluster(int nb, const int *__restrict__ browptr, const int *__restrict__ bcol,
                   const int *__restrict__ agg, const int *__restrict__ cand, uint64_t *__restrict__ t,
                   uint64_t *__restrict__ m1, int *__restrict__ cnt, int *__restrict__ rounds_out) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int nth = (int)(cl.num_blocks() * blockDim.x);
  const int tid = (int)(cl.block_rank() * blockDim.x + threadIdx.x);
  __shared__ int bsum;
  for (int i = tid; i < nb; i += nth) t[i] = mis_key(cand == nullptr || cand[i] ? 1 : 0, i);
  cl.sync();
  int r = 0;
  bool done = false;
  for (; r < kMisRounds; r++) {
    for (int i = tid; i < nb; i += nth) {
      uint64_t m = t[i];
      for (int e = browptr[i]; e < browptr[i + 1]; e++) {
        const int j = bcol[e];
        if (agg == nullptr || agg[j] < 0) m = max(m, t[j]);
      }
      m1[i] = m;
    }
    cl.sync();
    if (threadIdx.x == 0) bsum = 0;
    __syncthreads();
    int c = 0;
    for (int i = tid; i < nb; i += nth) {
      uint64_t m = m1[i];
      for (int e = browptr[i]; e < browptr[i + 1]; e++) {
        const int j = bcol[e];
        if (agg == nullptr || agg[j] < 0) m = max(m, m1[j]);
      }
      const uint64_t ti = t[i];
      if ((ti >> 62) == 1) {
        if (m == ti) t[i] = mis_key(2, i);
        else if ((m >> 62) == 2) t[i] = ti & ~(3ull << 62);
        else c++;
      }
    }
    if (c) atomicAdd(&bsum, c);
    __syncthreads();
    if (threadIdx.x == 0 && bsum) atomicAdd(cnt + r + 1, bsum);
    cl.sync();
    if (__ldcg(cnt + r + 1) == 0) {
      r++;
      done = true;
      break;
    }
  }
  if (tid == 0) *rounds_out = done ? r : -1;
}

// second-phase candidates: unaggregated nodes with at least `min_free`
// unaggregated neighbours
__global__ void k_mis_cand(int nb, const int *__restrict__ browptr, const int *__restrict__ bcol,
                           const int *__restrict__ agg, int min_free, int *__restrict__ cand) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    int c = 0;
    if (agg[i] < 0)
      for (int e = browptr[i]; e < browptr[i + 1]; e++) c += (bcol[e] != i && agg[bcol[e]] < 0);
    cand[i] = (agg[i] < 0 && c >= min_free) ? 1 : 0;
  }
}

__global__ void k_mis_decide(int nb, uint64_t *__restrict__ t, const uint64_t *__restrict__ m2, const int *go,
                             int *__restrict__ undecided) {
  if (*go == 0) return;
  int cnt = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    const uint64_t ti = t[i];
    if ((ti >> 62) != 1) continue;
    const uint64_t mi = m2[i];
    if (mi == ti) t[i] = mis_key(2, i);
    else if ((mi >> 62) == 2) t[i] = ti & ~(3ull << 62);
    else cnt++;
  }
  if (cnt) atomicAdd(undecided, cnt);
}

__global__ void k_root_flags(int nb, const uint64_t *__restrict__ t, int *__restrict__ flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    flag[i] = (t[i] >> 62) == 2 ? 1 : 0;
}

// an unaggregated root starts aggregate base + rootid; an unaggregated node
// next to a root joins it (the roots are >= 3 apart: at most one is adjacent)
__global__ void k_attach_roots(int nb, const int *__restrict__ browptr, const int *__restrict__ bcol,
                               const uint64_t *__restrict__ t, const int *__restrict__ rootid,
                               const int *__restrict__ base_d, int *__restrict__ agg) {
  const int base = base_d ? *base_d : 0;  // aggregates numbered by earlier passes
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    if (agg[i] >= 0) continue;
    int a = -1;
    if ((t[i] >> 62) == 2) {
      a = base + rootid[i];
    } else {
      for (int e = browptr[i]; e < browptr[i + 1]; e++) {
        const int j = bcol[e];
        if ((t[j] >> 62) == 2) { a = base + rootid[j]; break; }
      }
    }
    agg[i] = a;
  }
}

// *total = (base_d ? *base_d : 0) + the roots of the exclusive scan `rootid`
// of `flag` (one thread)
__global__ void k_root_total(int nb, const int *__restrict__ rootid, const int *__restrict__ flag,
                             const int *__restrict__ base_d, int *__restrict__ total) {
  *total = (base_d ? *base_d : 0) + rootid[nb - 1] + flag[nb - 1];
}

__global__ void k_attach2(int nb, const int *__restrict__ browptr, const int *__restrict__ bcol,
                          const int *__restrict__ agg1, int *__restrict__ agg, int *__restrict__ lost) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    int a = agg1[i];
    if (a < 0) {
      for (int e = browptr[i]; e < browptr[i + 1]; e++) {
        const int j = bcol[e];
        if (agg1[j] >= 0) { a = agg1[j]; break; }
      }
      if (a < 0) atomicAdd(lost, 1);
    }
    agg[i] = a;
  }
}

__global__ void k_iota(int n, int *__restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// aggptr from the nodes sorted by aggregate
__global__ void k_agg_ptr(int nb, int na, const int *__restrict__ sorted_agg, int *__restrict__ aggptr) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += gridDim.x * blockDim.x) {
    const int a = sorted_agg[t];
    if (t == 0 || sorted_agg[t - 1] != a) aggptr[a] = t;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) aggptr[na] = nb;
}

// level-0 near-null space, Jacobi-scaled and equation-major: B0[p][q] = B[p + q n] / S_p
// (k0 = 0: one constant per equation of a node, translations)
__global__ void k_nullspace0(int n, int b, int k0, const double *__restrict__ B, const double *__restrict__ dscale,
                             double *__restrict__ out, int K) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const double sp = 1.0 / dscale[p];
    for (int q = 0; q < K; q++)
      out[(size_t)p * K + q] = (k0 > 0 ? B[p + (size_t)q * n] : (p % b == q ? 1.0 : 0.0)) * sp;
  }
}

// Thin QR of the near-null-space rows of each aggregate (one warp per
// aggregate): modified Gram-Schmidt with a second orthogonalisation pass; a
// column that (numerically) depends on the previous ones becomes zero.
// Q (per equation K values) replaces the rows; R is the coarse near-null space.
constexpr int kTentRows = 4;  // rows per lane of an aggregate QR held in registers (128 rows)

template <int B, int K>
__global__ void __launch_bounds__(TPB) k_tentative(int na, const int *__restrict__ aggptr,
                                                   const int *__restrict__ aggnodes, const double *__restrict__ Bl,
                                                   double *__restrict__ Q, double *__restrict__ Bnext) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int G = warp; G < na; G += nwarps) {
    const int s = __ldg(aggptr + G), e = __ldg(aggptr + G + 1);
    const int rows = (e - s) * B;
    auto eq = [&](int r) { return B * __ldg(aggnodes + s + r / B) + r % B; };
    if (rows <= 32 * kTentRows) {
      // the aggregate's rows in registers (lane: rows lane, lane + 32, ...):
      // the same sweeps, sums and order as below, without the round trips
      // through memory
      double v[kTentRows][K];
      int pr[kTentRows];
#pragma unroll
      for (int u = 0; u < kTentRows; u++) {
        const int r = lane + 32 * u;
        pr[u] = r < rows ? eq(r) : -1;
#pragma unroll
        for (int q = 0; q < K; q++) v[u][q] = pr[u] >= 0 ? Bl[(size_t)pr[u] * K + q] : 0.0;
      }
      double R[K][K];
#pragma unroll
      for (int a = 0; a < K; a++)
#pragma unroll
        for (int c = 0; c < K; c++) R[a][c] = 0.0;
      bool live[K];
#pragma unroll
      for (int q = 0; q < K; q++) {
        double o2 = 0.0;
#pragma unroll
        for (int u = 0; u < kTentRows; u++) o2 += v[u][q] * v[u][q];
        o2 = warp_sum(o2);
        for (int pass = 0; pass < 2; pass++) {
#pragma unroll
          for (int pp = 0; pp < q; pp++) {
            if (!live[pp]) continue;
            double dt = 0.0;
#pragma unroll
            for (int u = 0; u < kTentRows; u++) dt += v[u][pp] * v[u][q];
            dt = warp_sum(dt);
            R[pp][q] += dt;
#pragma unroll
            for (int u = 0; u < kTentRows; u++) v[u][q] -= dt * v[u][pp];
          }
        }
        double n2 = 0.0;
#pragma unroll
        for (int u = 0; u < kTentRows; u++) n2 += v[u][q] * v[u][q];
        n2 = warp_sum(n2);
        const double nrm = sqrt(n2);
        live[q] = nrm > 1e-10 * sqrt(o2) && nrm > 0.0;
        R[q][q] = live[q] ? nrm : 0.0;
        const double inv = live[q] ? 1.0 / nrm : 0.0;
#pragma unroll
        for (int u = 0; u < kTentRows; u++) v[u][q] *= inv;
      }
#pragma unroll
      for (int u = 0; u < kTentRows; u++)
        if (pr[u] >= 0) {
#pragma unroll
          for (int q = 0; q < K; q++) Q[(size_t)pr[u] * K + q] = v[u][q];
        }
      if (lane < K) {
#pragma unroll
        for (int a = 0; a < K; a++)
          if (lane == a) {
#pragma unroll
            for (int c = 0; c < K; c++) Bnext[((size_t)G * K + a) * K + c] = live[a] ? R[a][c] : 0.0;
          }
      }
      continue;
    }
    for (int r = lane; r < rows; r += 32) {
      const int p = eq(r);
#pragma unroll
      for (int q = 0; q < K; q++) Q[(size_t)p * K + q] = Bl[(size_t)p * K + q];
    }
    __syncwarp();
    double R[K][K];
#pragma unroll
    for (int a = 0; a < K; a++)
#pragma unroll
      for (int c = 0; c < K; c++) R[a][c] = 0.0;
    bool live[K];
#pragma unroll
    for (int q = 0; q < K; q++) {
      double o2 = 0.0;
      for (int r = lane; r < rows; r += 32) { const double v = Q[(size_t)eq(r) * K + q]; o2 += v * v; }
      o2 = warp_sum(o2);
      for (int pass = 0; pass < 2; pass++) {
#pragma unroll
        for (int pp = 0; pp < q; pp++) {
          if (!live[pp]) continue;
          double dt = 0.0;
          for (int r = lane; r < rows; r += 32) {
            const size_t p = (size_t)eq(r) * K;
            dt += Q[p + pp] * Q[p + q];
          }
          dt = warp_sum(dt);
          R[pp][q] += dt;
          for (int r = lane; r < rows; r += 32) {
            const size_t p = (size_t)eq(r) * K;
            Q[p + q] -= dt * Q[p + pp];
          }
          __syncwarp();
        }
      }
      double n2 = 0.0;
      for (int r = lane; r < rows; r += 32) { const double v = Q[(size_t)eq(r) * K + q]; n2 += v * v; }
      n2 = warp_sum(n2);
      const double nrm = sqrt(n2);
      live[q] = nrm > 1e-10 * sqrt(o2) && nrm > 0.0;
      R[q][q] = live[q] ? nrm : 0.0;
      const double inv = live[q] ? 1.0 / nrm : 0.0;
      for (int r = lane; r < rows; r += 32) Q[(size_t)eq(r) * K + q] *= inv;
      __syncwarp();
    }
    if (lane < K) {
#pragma unroll
      for (int a = 0; a < K; a++)
        if (lane == a) {
#pragma unroll
          for (int c = 0; c < K; c++) Bnext[((size_t)G * K + a) * K + c] = live[a] ? R[a][c] : 0.0;
        }
    }
  }
}

__global__ void k_gal_keys(int64_t nblk, const int *__restrict__ rowid, const int *__restrict__ bcol,
                           const int *__restrict__ agg, uint64_t *__restrict__ keys, int *__restrict__ idx) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nblk; e += (int64_t)gridDim.x * blockDim.x) {
    keys[e] = ((uint64_t)(uint32_t)agg[rowid[e]] << 32) | (uint32_t)agg[bcol[e]];
    idx[e] = (int)e;
  }
}

// coarse pattern from the sorted unique keys: block r is (G, H) = key >> 32, key
__global__ void k_gal_pattern(int nruns, int na, const uint64_t *__restrict__ ukeys, int *__restrict__ browptr,
                              int *__restrict__ bcol) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nruns; r += gridDim.x * blockDim.x) {
    const uint64_t k = ukeys[r];
    const int G = (int)(k >> 32);
    bcol[r] = (int)(k & 0xffffffffu);
    if (r == 0 || (int)(ukeys[r - 1] >> 32) != G) browptr[G] = r;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) browptr[na] = nruns;
}

// A_c(G,H) = sum over the run of Q_i^T A_ij Q_j (one warp per run)
template <int B, int K>
__global__ void __launch_bounds__(128) k_galerkin(int nruns, const int *__restrict__ runoff,
                                                  const int *__restrict__ eidx, const int *__restrict__ rowid,
                                                  LevelView A, const double *__restrict__ Q, double *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r = warp; r < nruns; r += nwarps) {
    double acc[K * K];
#pragma unroll
    for (int t = 0; t < K * K; t++) acc[t] = 0.0;
    for (int t = runoff[r] + lane; t < runoff[r + 1]; t += 32) {
      const int e = eidx[t];
      const int i = rowid[e], j = A.bcol[e];
      double a[B * B];
#pragma unroll
      for (int c = 0; c < B * B; c++) a[c] = A.get<B>(i, e, c);
      const double *Qi = Q + (size_t)i * B * K, *Qj = Q + (size_t)j * B * K;
#pragma unroll
      for (int q2 = 0; q2 < K; q2++) {
        double tcol[B];
#pragma unroll
        for (int c = 0; c < B; c++) {
          double s = 0.0;
#pragma unroll
          for (int c2 = 0; c2 < B; c2++) s += a[c * B + c2] * Qj[c2 * K + q2];
          tcol[c] = s;
        }
#pragma unroll
        for (int q1 = 0; q1 < K; q1++) {
          double s = 0.0;
#pragma unroll
          for (int c = 0; c < B; c++) s += Qi[c * K + q1] * tcol[c];
          acc[q1 * K + q2] += s;
        }
      }
    }
#pragma unroll
    for (int t = 0; t < K * K; t++) acc[t] = warp_sum(acc[t]);
#pragma unroll
    for (int t = 0; t < K * K; t++)
      if ((t & 31) == lane) out[(size_t)r * K * K + t] = acc[t];
  }
}

// ----- Galerkin product without a global sort -------------------------------
// One warp per aggregate G builds coarse row G directly: the aggregates H
// that the rows of G's nodes reach (a hash set in shared memory, then ranked
// into ascending order) and A_c(G,H) = sum over i in G and the entries (i,j)
// of row i with agg[j] = H of Q_i^T A_ij Q_j.  The sum runs over G's nodes
// in aggregate order and each row's entries in column order, so every run
// gives the same bits.  A coarse row of more than kGalCap blocks makes the
// count pass raise a flag and the level takes the sort-based path above.
constexpr int kGalCap = 64;
constexpr int kGalHash = 128;
constexpr int kGalWarps = 2;

struct GalTable {
  int key[kGalHash];  // aggregate H, or -1
  int pos[kGalHash];  // H's position in the ascending coarse row
  int list[kGalCap];  // the coarse row's columns, ascending
};

__device__ __forceinline__ unsigned gal_hash(int h) { return ((unsigned)h * 2654435761u) >> 25; }

// G's coarse columns into T; returns their number, or -1 above kGalCap
__device__ int gal_table(int G, const int *__restrict__ aggptr, const int *__restrict__ aggnodes,
                         const int *__restrict__ browptr, const int *__restrict__ bcol, const int *__restrict__ agg,
                         GalTable &T) {
  const int lane = threadIdx.x & 31;
  for (int h = lane; h < kGalHash; h += 32) T.key[h] = -1;
  __syncwarp();
  int n = 0;
  for (int a = aggptr[G]; a < aggptr[G + 1] && n <= kGalCap; a++) {
    const int i = aggnodes[a];
    const int re = browptr[i + 1];
    for (int t0 = browptr[i]; t0 < re && n <= kGalCap; t0 += 32) {
      const int e = t0 + lane;
      bool fresh = false;
      if (e < re) {
        const int H = agg[bcol[e]];
        unsigned h = gal_hash(H);
        // a full table (kGalHash > kGalCap keys) already means overflow
        for (int p = 0; p < kGalHash; p++) {
          const int k = atomicCAS(&T.key[h], -1, H);
          if (k == -1) { fresh = true; break; }
          if (k == H) break;
          h = (h + 1) & (kGalHash - 1);
        }
      }
      n += __popc(__ballot_sync(0xffffffffu, fresh));
      __syncwarp();
    }
  }
  if (n > kGalCap) return -1;
  for (int h = lane; h < kGalHash; h += 32) {
    const int k = T.key[h];
    if (k >= 0) {
      int r = 0;
      for (int q = 0; q < kGalHash; q++) {
        const int o = T.key[q];
        r += (o >= 0 && o < k);
      }
      T.pos[h] = r;
      T.list[r] = k;
    }
  }
  __syncwarp();
  return n;
}

__device__ __forceinline__ int gal_find(const GalTable &T, int H) {
  unsigned h = gal_hash(H);
  for (int p = 0; p < kGalHash; p++) {
    const int k = T.key[h];
    if (k == H) return T.pos[h];
    if (k < 0) return -1;
    h = (h + 1) & (kGalHash - 1);
  }
  return -1;
}

// blocks per coarse row -> cnt[G] and the row's columns, ascending, ->
// lists[G * kGalCap ...]; *over = 1 when a row exceeds kGalCap
__global__ void __launch_bounds__(32 * kGalWarps)
    k_gal_count(int na, const int *__restrict__ aggptr, const int *__restrict__ aggnodes,
                const int *__restrict__ browptr, const int *__restrict__ bcol, const int *__restrict__ agg,
                int *__restrict__ cnt, int *__restrict__ lists, int *__restrict__ over, int *__restrict__ maxn) {
  __shared__ GalTable tab[kGalWarps];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int G = blockIdx.x * kGalWarps + w; G < na; G += gridDim.x * kGalWarps) {
    const int n = gal_table(G, aggptr, aggnodes, browptr, bcol, agg, tab[w]);
    if (lane == 0) {
      cnt[G] = n < 0 ? 0 : n;
      if (n < 0) atomicOr(over, 1);
      else atomicMax(maxn, n);
    }
    for (int t = lane; t < n; t += 32) lists[(size_t)G * kGalCap + t] = tab[w].list[t];
    __syncwarp();
  }
}

// warps per aggregate in k_gal_values
constexpr int kGalCtaWarps = 4;

template <int K>
constexpr size_t gal_shared_bytes() {
  // per CTA: the accumulators [kGalCap][K*K], a staging area per warp with an
  // odd stride in doubles (32 lanes' stores hit distinct banks), the staged
  // entries' positions and counts, the table
  return ((size_t)kGalCap * K * K + (size_t)kGalCtaWarps * 32 * (K * K | 1)) * sizeof(double) +
         kGalCtaWarps * 33 * sizeof(int) + sizeof(GalTable);
}

// Coarse row G's values, one CTA per aggregate (columns from the count pass).
// The CTA's warps take the aggregate's nodes in turn (warp w: nodes w, w + 4,
// ...), one chunk of up to 32 entries of a row per round: each lane forms the
// product Q_i^T A_ij Q_j of its entry and stages it.  Then K*K threads, one
// per value, add the staged products of warps 0..3, rows in entry order, into
// the accumulators (a run of entries into one block summed first).  The
// order of every sum is fixed by the data, so every run gives the same bits.
template <int B, int K>
__global__ void __launch_bounds__(32 * kGalCtaWarps, 3)
    k_gal_values(int na, const int *__restrict__ aggptr, const int *__restrict__ aggnodes,
                 const int *__restrict__ agg, LevelView A, const double *__restrict__ Q,
                 const int *__restrict__ lists, const int *__restrict__ cbrowptr, int *__restrict__ cbcol,
                 double *__restrict__ out) {
  constexpr int KK = K * K, SS = KK | 1, W = kGalCtaWarps, BK = B * K;
  extern __shared__ double gal_sh[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double *acc = gal_sh;                         // [kGalCap][KK]
  double *stages = acc + kGalCap * KK;          // [W][32][SS]
  double *stage = stages + w * 32 * SS;         // this warp's
  int *spos = reinterpret_cast<int *>(stages + W * 32 * SS);  // [W][32]
  int *srows = spos + W * 32;                                  // [W]
  GalTable &T = *reinterpret_cast<GalTable *>(srows + W + (W & 1));
  for (int G = blockIdx.x; G < na; G += gridDim.x) {
    const int base = cbrowptr[G], n = cbrowptr[G + 1] - base;
    // the table of the row's columns: key -> position in the ascending list
    for (int h = threadIdx.x; h < kGalHash; h += blockDim.x) T.key[h] = -1;
    for (int t = threadIdx.x; t < n * KK; t += blockDim.x) acc[t] = 0.0;
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const int H = __ldg(lists + (size_t)G * kGalCap + t);
      T.list[t] = H;
      unsigned h = gal_hash(H);
      for (int p = 0; p < kGalHash; p++) {  // n <= kGalCap < kGalHash keys: a free slot exists
        if (atomicCAS(&T.key[h], -1, H) == -1) {
          T.pos[h] = t;
          break;
        }
        h = (h + 1) & (kGalHash - 1);
      }
    }
    __syncthreads();
    const int a_end = aggptr[G];
    int a = a_end + w;  // this warp's current node
    const int a_last = aggptr[G + 1];
    int i = 0, rs = 0, re = 0, t0 = 0;
    if (a < a_last) {
      i = __ldg(aggnodes + a);
      rs = __ldg(A.browptr + i);
      re = __ldg(A.browptr + i + 1);
      t0 = rs;
    }
    while (__syncthreads_or(a < a_last)) {
      int p = -1, rows = 0;
      if (a < a_last) {
        const int e = t0 + lane;
        const bool live = e < re;
        rows = min(32, re - t0);
        double prod[KK];
#pragma unroll
        for (int t = 0; t < KK; t++) prod[t] = 0.0;
        if (live) {
          const int j = __ldg(A.bcol + e);
          p = gal_find(T, __ldg(agg + j));
          double av[B * B];
          if (A.layout == 0) {
#pragma unroll
            for (int c = 0; c < B * B; c++) av[c] = __ldg(A.val + (size_t)e * B * B + c);
          } else {
            double di[B], dj[B];
#pragma unroll
            for (int c = 0; c < B; c++) {
              di[c] = __ldg(A.dscale + (size_t)B * i + c);
              dj[c] = __ldg(A.dscale + (size_t)B * j + c);
            }
            const int nbr = re - rs;
#pragma unroll
            for (int c = 0; c < B * B; c++) {
              // layout 1: the row's blocks component-major; layout 2 (B = 1): CSR
              const double v = A.layout == 1 ? __ldg(A.val + 9ll * rs + (int64_t)c * nbr + (e - rs))
                                             : __ldg(A.val + e);
              av[c] = v * di[c / B] * dj[c % B];
            }
          }
          double qj[BK], qi[BK];
          if constexpr (BK % 2 == 0) {  // a node's Q rows are 16-byte aligned (BK * 8 bytes each, BK even)
            const double2 *Qj2 = reinterpret_cast<const double2 *>(Q + (size_t)j * BK);
            const double2 *Qi2 = reinterpret_cast<const double2 *>(Q + (size_t)i * BK);
#pragma unroll
            for (int c = 0; c < BK / 2; c++) {
              const double2 u = __ldg(Qj2 + c), z = __ldg(Qi2 + c);
              qj[2 * c] = u.x;
              qj[2 * c + 1] = u.y;
              qi[2 * c] = z.x;
              qi[2 * c + 1] = z.y;
            }
          } else {
#pragma unroll
            for (int c = 0; c < BK; c++) {
              qj[c] = __ldg(Q + (size_t)j * BK + c);
              qi[c] = __ldg(Q + (size_t)i * BK + c);
            }
          }
#pragma unroll
          for (int q2 = 0; q2 < K; q2++) {
            double tcol[B];
#pragma unroll
            for (int c = 0; c < B; c++) {
              double sacc = 0.0;
#pragma unroll
              for (int c2 = 0; c2 < B; c2++) sacc += av[c * B + c2] * qj[c2 * K + q2];
              tcol[c] = sacc;
            }
#pragma unroll
            for (int q1 = 0; q1 < K; q1++) {
              double sacc = 0.0;
#pragma unroll
              for (int c = 0; c < B; c++) sacc += qi[c * K + q1] * tcol[c];
              prod[q1 * K + q2] = sacc;
            }
          }
        }
#pragma unroll
        for (int t = 0; t < KK; t++) stage[lane * SS + t] = prod[t];
        // next chunk of this row, or this warp's next node
        t0 += 32;
        if (t0 >= re) {
          a += W;
          if (a < a_last) {
            i = __ldg(aggnodes + a);
            rs = __ldg(A.browptr + i);
            re = __ldg(A.browptr + i + 1);
            t0 = rs;
          }
        }
      }
      spos[w * 32 + lane] = p;
      if (lane == 0) srows[w] = rows;
      __syncthreads();
      // one thread per value: the staged rows of warps 0..W-1 in order; a
      // stage's values and positions are loaded before its walk, so that only
      // the adds at the end of a run wait on shared memory
      for (int v = threadIdx.x; v < KK; v += blockDim.x) {
        int cur = -1;
        double run = 0.0;
#pragma unroll 1
        for (int ws = 0; ws < W; ws++) {
          const int nr = srows[ws];
          const double *sg = stages + ws * 32 * SS + v;
          const int *sp = spos + ws * 32;
          double sv[32];
          int pq[32];
#pragma unroll
          for (int r = 0; r < 32; r++) {
            sv[r] = r < nr ? sg[r * SS] : 0.0;
            pq[r] = r < nr ? sp[r] : -1;
          }
#pragma unroll
          for (int r = 0; r < 32; r++) {
            if (r < nr) {
              if (pq[r] != cur) {
                if (cur >= 0) acc[cur * KK + v] += run;
                run = 0.0;
                cur = pq[r];
              }
              run += sv[r];
            }
          }
        }
        if (cur >= 0) acc[cur * KK + v] += run;
      }
      // (the loop condition's barrier orders these adds before the next staging)
    }
    for (int t = threadIdx.x; t < n; t += blockDim.x) cbcol[base + t] = T.list[t];
    for (int t = threadIdx.x; t < n * KK; t += blockDim.x) out[(size_t)base * KK + t] = acc[t];
    __syncthreads();
  }
}

// Coarse row G's values with warp-private accumulators (the default when no
// coarse row has more than kGal2Cap blocks).  One CTA per aggregate; warp w
// takes the aggregate's nodes w, w + 4, ... and a node's row in chunks of 32
// entries.  Each lane forms T_ij = A_ij Q_j (B x K) for its entry and stages
// it; the lanes of a chunk whose entries fall into one coarse block (one
// aggregate H of j) form a group, and the group's lowest lane sums the group
// in lane order and adds Q_i^T (that sum) into the warp's own accumulator of
// block (G, H).  The four warps' accumulators are added in warp order at the
// end.  Every sum has an order fixed by the data (nodes, entries, warps), so
// every run gives the same bits; no thread walks another's products, which
// the staging form above does with K*K threads over all 128 lanes' stages.
constexpr int kGal2Cap = 40;  // blocks per coarse row
constexpr int kGal2Warps = 4;
constexpr int kGal2Nodes = 128;  // an aggregate's nodes and rows read ahead into shared memory

// cap: the longest coarse row of the level (<= kGal2Cap), the accumulators'
// blocks per warp (fewer blocks, more CTAs per SM)
template <int B, int K>
constexpr size_t gal2_shared_bytes(int cap) {
  // [W][cap][K*K] accumulators, [W][32][B*K | 1] staging, [W][B*K] the
  // current node's Q rows, the table
  return ((size_t)kGal2Warps * cap * K * K + (size_t)kGal2Warps * 32 * ((B * K) | 1) +
          (size_t)kGal2Warps * B * K) * sizeof(double) + sizeof(GalTable) +
         (3 * kGal2Nodes + 64 * kGal2Warps) * sizeof(int);
}

// One chunk of the row walk of k_gal_values2: node k of the aggregate (i,
// its row [rs, re)), entries t0 .. t0 + 31; fresh: the node's first chunk.
struct GalChunk {
  int k, i, rs, re, t0;
  bool fresh;
};

// The groups of one staged chunk (the lanes whose entries fall into one
// coarse block): each group's sum in lane order into its leader's stage row,
// then Q_i^T (that sum) added into the warp's accumulator of the block.
template <int B, int K>
__device__ __forceinline__ void gal2_groups(int lane, bool ok, int p, double *stage, int *gpos, int *gmask,
                                            const double *qi, double *acc) {
  constexpr int KK = K * K, BK = B * K, SS = BK | 1;
  const unsigned grp = __match_any_sync(0xffffffffu, ok ? p : -2 - lane);
  const bool leader = ok && __ffs(grp) - 1 == lane;
  const unsigned lmask = __ballot_sync(0xffffffffu, leader);
  const int ng = __popc(lmask);
  if (leader) {  // the groups in leader-lane order
    const int g = __popc(lmask & ((1u << lane) - 1u));
    gpos[g] = p;
    gmask[g] = (int)grp;
  }
  __syncwarp();
  // the group sums, work item (group, component) over all lanes: the
  // members in lane order, the sum stored in the leader's stage row (only
  // this item reads or writes that column of the group's rows)
  for (int t = lane; t < ng * BK; t += 32) {
    const int g = t / BK, x = t - g * BK;
    const unsigned gm = (unsigned)gmask[g];
    double sm = 0.0;
    for (unsigned mm = gm; mm; mm &= mm - 1) sm += stage[(__ffs(mm) - 1) * SS + x];
    stage[(__ffs(gm) - 1) * SS + x] = sm;
  }
  __syncwarp();
  // Q_i^T (group sum) into the warp's accumulator, work item (group, entry)
  for (int t = lane; t < ng * KK; t += 32) {
    const int g = t / KK, v = t - g * KK, q1 = v / K, q2 = v - q1 * K;
    const double *sg = stage + (__ffs((unsigned)gmask[g]) - 1) * SS;
    double o = 0.0;
#pragma unroll
    for (int c = 0; c < B; c++) o += qi[c * K + q1] * sg[c * K + q2];
    acc[(size_t)gpos[g] * KK + v] += o;
  }
  __syncwarp();
}

template <int B, int K>
__global__ void __launch_bounds__(32 * kGal2Warps)
    k_gal_values2(int na, const int *__restrict__ aggptr, const int *__restrict__ aggnodes,
                  const int *__restrict__ agg, LevelView A, const double *__restrict__ Q,
                  const int *__restrict__ lists, const int *__restrict__ cbrowptr, int *__restrict__ cbcol,
                  double *__restrict__ out, int cap, bool pipe) {
  constexpr int KK = K * K, BK = B * K, SS = BK | 1, W = kGal2Warps;
  extern __shared__ double gal2_sh[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double *accs = gal2_sh;                            // [W][cap][KK]
  double *stages = accs + (size_t)W * cap * KK;      // [W][32][SS]
  double *qis = stages + (size_t)W * 32 * SS;        // [W][BK]
  GalTable &T = *reinterpret_cast<GalTable *>(qis + (size_t)W * BK);
  int *pnode = reinterpret_cast<int *>(&T + 1);  // [kGal2Nodes] the aggregate's nodes
  int *prs = pnode + kGal2Nodes, *pre = prs + kGal2Nodes;  // their rows' ranges
  int *gpos = pre + kGal2Nodes + 64 * w, *gmask = gpos + 32;  // this warp's groups of a chunk
  double *acc = accs + (size_t)w * cap * KK;
  double *stage = stages + (size_t)w * 32 * SS;
  double *qi = qis + (size_t)w * BK;
  for (int G = blockIdx.x; G < na; G += gridDim.x) {
    const int base = cbrowptr[G], n = cbrowptr[G + 1] - base;
    // the aggregate's nodes, then their row ranges, read ahead (two waits
    // per aggregate instead of two per node)
    const int a0 = aggptr[G], an = aggptr[G + 1] - a0;
    const bool ahead = an <= kGal2Nodes;
    if (ahead)
      for (int t = threadIdx.x; t < an; t += blockDim.x) pnode[t] = __ldg(aggnodes + a0 + t);
    for (int h = threadIdx.x; h < kGalHash; h += blockDim.x) T.key[h] = -1;
    for (int t = threadIdx.x; t < W * n * KK; t += blockDim.x) {
      const int ww = t / (n * KK);
      accs[(size_t)ww * cap * KK + (t - ww * n * KK)] = 0.0;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const int H = __ldg(lists + (size_t)G * kGalCap + t);
      T.list[t] = H;
      unsigned h = gal_hash(H);
      for (int p = 0; p < kGalHash; p++) {  // n <= cap < kGalHash keys: a free slot exists
        if (atomicCAS(&T.key[h], -1, H) == -1) {
          T.pos[h] = t;
          break;
        }
        h = (h + 1) & (kGalHash - 1);
      }
    }
    if (ahead)
      for (int t = threadIdx.x; t < an; t += blockDim.x) {
        const int i = pnode[t];
        prs[t] = __ldg(A.browptr + i);
        pre[t] = __ldg(A.browptr + i + 1);
      }
    __syncthreads();
    // the plain walk: a node's chunks one after another
    auto walk_plain = [&]() {
      for (int k = w; k < an; k += W) {
        const int i = ahead ? pnode[k] : __ldg(aggnodes + a0 + k);
        const int rs = ahead ? prs[k] : __ldg(A.browptr + i), re = ahead ? pre[k] : __ldg(A.browptr + i + 1);
        for (int c = lane; c < BK; c += 32) qi[c] = __ldg(Q + (size_t)i * BK + c);
        double di[B];
#pragma unroll
        for (int c = 0; c < B; c++) di[c] = A.layout == 0 ? 1.0 : __ldg(A.dscale + (size_t)B * i + c);
        __syncwarp();
        for (int t0 = rs; t0 < re; t0 += 32) {
          const int e = t0 + lane;
          const bool live = e < re;
          int p = -1;
          if (live) {
            const int j = __ldg(A.bcol + e);
            p = gal_find(T, __ldg(agg + j));
            double av[B * B];
            if (A.layout == 0) {
#pragma unroll
              for (int c = 0; c < B * B; c++) av[c] = __ldg(A.val + (size_t)e * B * B + c);
            } else {
              double dj[B];
#pragma unroll
              for (int c = 0; c < B; c++) dj[c] = __ldg(A.dscale + (size_t)B * j + c);
              const int nbr = re - rs;
#pragma unroll
              for (int c = 0; c < B * B; c++) {
                // layout 1: the row's blocks component-major; layout 2 (B = 1): CSR
                const double v = A.layout == 1 ? __ldg(A.val + 9ll * rs + (int64_t)c * nbr + (e - rs))
                                               : __ldg(A.val + e);
                av[c] = v * di[c / B] * dj[c % B];
              }
            }
#pragma unroll
            for (int q2 = 0; q2 < K; q2++) {
              double qj[B];
#pragma unroll
              for (int c2 = 0; c2 < B; c2++) qj[c2] = __ldg(Q + (size_t)j * BK + c2 * K + q2);
#pragma unroll
              for (int c = 0; c < B; c++) {
                double sacc = 0.0;
#pragma unroll
                for (int c2 = 0; c2 < B; c2++) sacc += av[c * B + c2] * qj[c2];
                stage[lane * SS + c * K + q2] = sacc;
              }
            }
          }
          __syncwarp();
          gal2_groups<B, K>(lane, live && p >= 0, p, stage, gpos, gmask, qi, acc);
        }
      }
    };
    if constexpr (B > 3) {
      walk_plain();
    } else if (!pipe) {
      walk_plain();
    } else {
      // The same walk software-pipelined (B <= 3, where one chunk's loads fit
      // in registers): the chunks in the same order and the same arithmetic,
      // so the same bits, but the global loads of the next chunk (its values,
      // the aggregates, scalings and Q rows of its columns) are in flight
      // while this chunk's groups are summed in shared memory, and the
      // columns of the chunk after that one a step earlier still.
      auto node_at = [&](GalChunk &c) {
        if (c.k >= an) return;
        c.i = ahead ? pnode[c.k] : __ldg(aggnodes + a0 + c.k);
        c.rs = ahead ? prs[c.k] : __ldg(A.browptr + c.i);
        c.re = ahead ? pre[c.k] : __ldg(A.browptr + c.i + 1);
        c.t0 = c.rs;
        c.fresh = true;
      };
      auto advance = [&](GalChunk &c) {
        if (c.t0 + 32 < c.re) {
          c.t0 += 32;
          c.fresh = false;
        } else {
          c.k += W;
          node_at(c);
        }
      };
      auto column = [&](const GalChunk &c) {
        const int e = c.t0 + lane;
        return c.k < an && e < c.re ? __ldg(A.bcol + e) : -1;
      };
      // one chunk's loads: its column's aggregate, the values, both
      // scalings, Q_j, and (first chunk of a node) lane x's entry of Q_i
      int rH = -1;
      double rav[B * B], rdi[B], rdj[B], rq[BK], rqi = 0.0;
      auto fetch = [&](const GalChunk &c, int j) {
        if (c.k >= an) return;
        const int e = c.t0 + lane;
#pragma unroll
        for (int x = 0; x < B; x++) rdi[x] = A.layout == 0 ? 1.0 : __ldg(A.dscale + (size_t)B * c.i + x);
        if (c.fresh && lane < BK) rqi = __ldg(Q + (size_t)c.i * BK + lane);
        if (j >= 0) {
          rH = __ldg(agg + j);
          if (A.layout == 0) {
#pragma unroll
            for (int x = 0; x < B * B; x++) rav[x] = __ldg(A.val + (size_t)e * B * B + x);
          } else {
            const int nbr = c.re - c.rs;
#pragma unroll
            for (int x = 0; x < B; x++) rdj[x] = __ldg(A.dscale + (size_t)B * j + x);
#pragma unroll
            for (int x = 0; x < B * B; x++)
              rav[x] = A.layout == 1 ? __ldg(A.val + 9ll * c.rs + (int64_t)x * nbr + (e - c.rs)) : __ldg(A.val + e);
          }
#pragma unroll
          for (int x = 0; x < BK; x++) rq[x] = __ldg(Q + (size_t)j * BK + x);
        }
      };
      GalChunk cur{w, 0, 0, 0, 0, true};
      node_at(cur);
      int cj = column(cur);
      fetch(cur, cj);
      GalChunk nx = cur;
      advance(nx);
      int nj = column(nx);
      while (cur.k < an) {
        // this chunk: stage T_ij = A_ij Q_j, the node's Q_i rows on its first chunk
        const bool live = cj >= 0;
        int p = -1;
        if (cur.fresh && lane < BK) qi[lane] = rqi;
        if (live) {
          p = gal_find(T, rH);
          double av[B * B];
#pragma unroll
          for (int x = 0; x < B * B; x++) av[x] = A.layout == 0 ? rav[x] : rav[x] * rdi[x / B] * rdj[x % B];
#pragma unroll
          for (int q2 = 0; q2 < K; q2++) {
#pragma unroll
            for (int c = 0; c < B; c++) {
              double sacc = 0.0;
#pragma unroll
              for (int c2 = 0; c2 < B; c2++) sacc += av[c * B + c2] * rq[c2 * K + q2];
              stage[lane * SS + c * K + q2] = sacc;
            }
          }
        }
        __syncwarp();
        // the next chunk's loads, and the columns of the one after it
        fetch(nx, nj);
        GalChunk nn = nx;
        advance(nn);
        const int nnj = column(nn);
        gal2_groups<B, K>(lane, live && p >= 0, p, stage, gpos, gmask, qi, acc);
        cur = nx;
        cj = nj;
        nx = nn;
        nj = nnj;
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n * KK; t += blockDim.x) {
      double v = accs[t];
#pragma unroll
      for (int ww = 1; ww < W; ww++) v += accs[(size_t)ww * cap * KK + t];
      out[(size_t)base * KK + t] = v;
    }
    for (int t = threadIdx.x; t < n; t += blockDim.x) cbcol[base + t] = T.list[t];
    __syncthreads();
  }
}

// 1/diag of a coarse level (0 for a zero diagonal: an equation that a
// dependent near-null-space column left empty stays 0)
__global__ void k_coarse_dinv(int na, int K, const int *__restrict__ browptr, const int *__restrict__ bcol,
                              const double *__restrict__ val, double *__restrict__ dinv64, float *__restrict__ dinv32) {
  for (int G = blockIdx.x * blockDim.x + threadIdx.x; G < na; G += gridDim.x * blockDim.x) {
    int rd = -1;
    for (int e = browptr[G]; e < browptr[G + 1]; e++)
      if (bcol[e] == G) { rd = e; break; }
    for (int q = 0; q < K; q++) {
      const double d = rd >= 0 ? val[(size_t)rd * K * K + q * K + q] : 0.0;
      const double iv = d > 0.0 ? 1.0 / d : 0.0;
      dinv64[G * K + q] = iv;
      dinv32[G * K + q] = (float)iv;
    }
  }
}

// the coarsest level's blocks into the dense matrix: a warp per block row,
// its lanes over the row's values in storage order (coalesced reads)
__global__ void k_dense_fill(int nb, int K, int nc, const int *__restrict__ browptr, const int *__restrict__ bcol,
                             const double *__restrict__ val, double *__restrict__ M) {
  const int lane = threadIdx.x & 31, KK = K * K;
  for (int G = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; G < nb; G += (gridDim.x * blockDim.x) >> 5) {
    const int rs = browptr[G], cnt = (browptr[G + 1] - rs) * KK;
    for (int t = lane; t < cnt; t += 32) {
      const int e = rs + t / KK, v = t % KK, a = v / K, c = v - a * K;
      M[(size_t)(G * K + a) * nc + bcol[e] * K + c] = val[(size_t)rs * KK + t];
    }
  }
}

// Blocked Gauss-Jordan inverse (pivot blocks of 32, no pivoting: the matrix
// is SPD, so every diagonal block of the successive Schur complements is):
// for the block K of rows/columns [k0, k0 + bs):
//   P = A[K,K]^-1                                   (k_bgj_diag, one CTA)
//   A[K,j] = P A[K,j]              for j not in K   (k_bgj_rowpanel)
//   A[i,j] -= A[i,K] A[K,j]        for i, j not in K (k_bgj_update, tiled)
//   A[i,K] = -A[i,K] P, A[K,K] = P for i not in K   (k_bgj_colpanel)
constexpr int GJB = 32;

// one CTA, a thread per entry; every step reads the previous step's matrix
// and writes the other copy, so a step needs one barrier
__global__ void __launch_bounds__(GJB *GJB) k_bgj_diag(int n, int k0, int bs, const double *__restrict__ A,
                                                       double *__restrict__ P) {
  __shared__ double d[2][GJB][GJB + 1];
  const int r = threadIdx.x / GJB, c = threadIdx.x % GJB;
  d[0][r][c] = (r < bs && c < bs) ? A[(size_t)(k0 + r) * n + k0 + c] : (r == c ? 1.0 : 0.0);
  __syncthreads();
  for (int k = 0; k < GJB; k++) {
    const double(*o)[GJB + 1] = d[k & 1];
    const double piv = 1.0 / o[k][k];
    const double colr = o[r][k];
    double v = o[r][c];
    if (r == k) v = (c == k) ? piv : v * piv;
    else v = (c == k) ? -colr * piv : v - colr * o[k][c] * piv;
    d[(k + 1) & 1][r][c] = v;
    __syncthreads();
  }
  P[r * GJB + c] = d[GJB & 1][r][c];
}

// A[K, j] = P A[K, j] for the columns j outside K: a CTA per 32 columns, the
// columns' K rows staged first (each CTA reads and writes only its columns)
__global__ void __launch_bounds__(TPB) k_bgj_rowpanel(int n, int k0, int bs, const double *__restrict__ P,
                                                      double *__restrict__ A) {
  __shared__ double ps[GJB][GJB + 1];
  __shared__ double vt[GJB][GJB + 1];  // vt[k][jj] = A[k0 + k, j0 + jj]
  const int j0 = blockIdx.x * GJB;
  for (int t = threadIdx.x; t < GJB * GJB; t += blockDim.x) {
    const int k = t / GJB, jj = t % GJB, j = j0 + jj;
    ps[k][jj] = P[t];
    vt[k][jj] = (k < bs && j < n) ? A[(size_t)(k0 + k) * n + j] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < GJB * GJB; t += blockDim.x) {
    const int r = t / GJB, jj = t % GJB, j = j0 + jj;
    if (r >= bs || j >= n || (j >= k0 && j < k0 + bs)) continue;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < GJB; k++) s += ps[r][k] * vt[k][jj];
    A[(size_t)(k0 + r) * n + j] = s;
  }
}

// A[i,j] -= A[i,K] A[K,j] on 32 x 32 tiles (rows and columns of K skipped)
__global__ void __launch_bounds__(TPB) k_bgj_update(int n, int k0, int bs, double *__restrict__ A) {
  constexpr int TI = 32, TJ = 32;
  __shared__ double ak[TI][GJB + 1];  // A[i, K]
  __shared__ double kb[GJB][TJ];      // A[K, j]
  const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
  for (int t = threadIdx.x; t < TI * GJB; t += blockDim.x) {
    const int r = t / GJB, k = t % GJB, i = i0 + r;
    ak[r][k] = (i < n && k < bs) ? A[(size_t)i * n + k0 + k] : 0.0;
  }
  for (int t = threadIdx.x; t < GJB * TJ; t += blockDim.x) {
    const int k = t / TJ, c = t % TJ, j = j0 + c;
    kb[k][c] = (j < n && k < bs) ? A[(size_t)(k0 + k) * n + j] : 0.0;
  }
  __syncthreads();
  // 256 threads, 4 elements each: thread (ty, tx) owns rows ty + 16 a and
  // columns tx + 16 b (a, b < 2); every element's sum over k in order
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[2][2];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++) acc[a][b] = 0.0;
#pragma unroll 8
  for (int k = 0; k < GJB; k++) {
    double av[2], bv[2];
#pragma unroll
    for (int a = 0; a < 2; a++) av[a] = ak[ty + 16 * a][k];
#pragma unroll
    for (int b = 0; b < 2; b++) bv[b] = kb[k][tx + 16 * b];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 2; b++) acc[a][b] += av[a] * bv[b];
  }
#pragma unroll
  for (int a = 0; a < 2; a++) {
    const int i = i0 + ty + 16 * a;
    if (i >= n || (i >= k0 && i < k0 + bs)) continue;
#pragma unroll
    for (int b = 0; b < 2; b++) {
      const int j = j0 + tx + 16 * b;
      if (j >= n || (j >= k0 && j < k0 + bs)) continue;
      A[(size_t)i * n + j] -= acc[a][b];
    }
  }
}

// A[i, K] = -A[i, K] P for the rows i outside K, A[K, K] = P: a CTA per 32
// rows, the rows' K columns staged first
__global__ void __launch_bounds__(TPB) k_bgj_colpanel(int n, int k0, int bs, const double *__restrict__ P,
                                                      double *__restrict__ A) {
  __shared__ double ps[GJB][GJB + 1];
  __shared__ double vt[GJB][GJB + 1];  // vt[ii][k] = A[i0 + ii, k0 + k]
  const int i0 = blockIdx.x * GJB;
  for (int t = threadIdx.x; t < GJB * GJB; t += blockDim.x) {
    const int ii = t / GJB, k = t % GJB, i = i0 + ii;
    ps[ii][k] = P[t];
    vt[ii][k] = (i < n && k < bs) ? A[(size_t)i * n + k0 + k] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < GJB * GJB; t += blockDim.x) {
    const int ii = t / GJB, c = t % GJB, i = i0 + ii;
    if (i >= n || c >= bs) continue;
    if (i >= k0 && i < k0 + bs) {
      A[(size_t)i * n + k0 + c] = ps[i - k0][c];
      continue;
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < GJB; k++) s += vt[ii][k] * ps[k][c];
    A[(size_t)i * n + k0 + c] = -s;
  }
}

// The blocked Gauss-Jordan inverse above in one thread-block-cluster launch:
// the four steps of every pivot block (diagonal inverse by CTA 0, row panel,
// rank-32 update of 64 x 64 tiles, column panel) spread over the cluster's
// CTAs with a cluster barrier (a hardware barrier, no spinning) between them,
// instead of four launches per pivot block.  The matrix (8 n^2 bytes, L2
// resident for the coarsest levels here) is read through L2 (ld.global.cg)
// since the launch itself rewrites it.  Every entry is computed with the
// expressions and summation order of k_bgj_diag / _rowpanel / _update /
// _colpanel.
__global__ void __launch_bounds__(TPB) k_bgj_cluster(int n, double *__restrict__ A, double *__restrict__ Pbuf) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), ncta = (int)cl.num_blocks();
  const int tid = threadIdx.x;
  constexpr int TI = 64, TJ = 64;
  __shared__ double ps[GJB][GJB];
  __shared__ double buf[TI * (GJB + 1) + GJB * TJ];  // update tiles; the diagonal block in CTA 0
  __shared__ double colv[GJB];
  double(*ak)[GJB + 1] = reinterpret_cast<double(*)[GJB + 1]>(buf);
  double(*kb)[TJ] = reinterpret_cast<double(*)[TJ]>(buf + TI * (GJB + 1));
  double(*d)[GJB + 1] = reinterpret_cast<double(*)[GJB + 1]>(buf);
  const int ntj = (n + TJ - 1) / TJ, ntiles = ntj * ((n + TI - 1) / TI);
  for (int k0 = 0; k0 < n; k0 += GJB) {
    const int bs = min(GJB, n - k0);
    if (rank == 0) {  // P = A[K,K]^-1, each thread four entries (rows r0, r0 + 8, ...)
      const int c = tid % GJB, r0 = tid / GJB;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = r0 + 8 * q;
        d[r][c] = (r < bs && c < bs) ? __ldcg(A + (size_t)(k0 + r) * n + k0 + c) : (r == c ? 1.0 : 0.0);
      }
      __syncthreads();
      for (int k = 0; k < GJB; k++) {
        const double piv = 1.0 / d[k][k];
        if (c == 0) {
#pragma unroll
          for (int q = 0; q < 4; q++) colv[r0 + 8 * q] = d[r0 + 8 * q][k];
        }
        __syncthreads();
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int r = r0 + 8 * q;
          double x = d[r][c];
          if (r == k) x = (c == k) ? piv : x * piv;
          else x = (c == k) ? -colv[r] * piv : x - colv[r] * d[k][c] * piv;
          v[q] = x;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; q++) d[r0 + 8 * q][c] = v[q];
        __syncthreads();
      }
#pragma unroll
      for (int q = 0; q < 4; q++) Pbuf[(r0 + 8 * q) * GJB + c] = d[r0 + 8 * q][c];
    }
    cl.sync();
    for (int t = tid; t < GJB * GJB; t += blockDim.x) ps[t / GJB][t % GJB] = __ldcg(Pbuf + t);
    __syncthreads();
    // row panel: A[K, j] = P A[K, j], j outside K
    for (int j = rank * blockDim.x + tid; j < n; j += ncta * blockDim.x) {
      if (j >= k0 && j < k0 + bs) continue;
      double v[GJB];
#pragma unroll
      for (int k = 0; k < GJB; k++) v[k] = k < bs ? __ldcg(A + (size_t)(k0 + k) * n + j) : 0.0;
      for (int r = 0; r < bs; r++) {
        double sm = 0.0;
#pragma unroll
        for (int k = 0; k < GJB; k++) sm += ps[r][k] * v[k];
        A[(size_t)(k0 + r) * n + j] = sm;
      }
    }
    cl.sync();
    // A[i,j] -= A[i,K] A[K,j] on 64 x 64 tiles, rows and columns of K skipped
    for (int tile = rank; tile < ntiles; tile += ncta) {
      const int i0 = (tile / ntj) * TI, j0 = (tile % ntj) * TJ;
      for (int t = tid; t < TI * GJB; t += blockDim.x) {
        const int r = t / GJB, k = t % GJB, i = i0 + r;
        ak[r][k] = (i < n && k < bs) ? __ldcg(A + (size_t)i * n + k0 + k) : 0.0;
      }
      for (int t = tid; t < GJB * TJ; t += blockDim.x) {
        const int k = t / TJ, c = t % TJ, j = j0 + c;
        kb[k][c] = (j < n && k < bs) ? __ldcg(A + (size_t)(k0 + k) * n + j) : 0.0;
      }
      __syncthreads();
      const int tx = tid % 16, ty = tid / 16;
      double acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
#pragma unroll 8
      for (int k = 0; k < GJB; k++) {
        double av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; a++) av[a] = ak[ty + 16 * a][k];
#pragma unroll
        for (int b = 0; b < 4; b++) bv[b] = kb[k][tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 4; b++) acc[a][b] += av[a] * bv[b];
      }
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int i = i0 + ty + 16 * a;
        if (i >= n || (i >= k0 && i < k0 + bs)) continue;
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int j = j0 + tx + 16 * b;
          if (j >= n || (j >= k0 && j < k0 + bs)) continue;
          A[(size_t)i * n + j] = __ldcg(A + (size_t)i * n + j) - acc[a][b];
        }
      }
      __syncthreads();
    }
    cl.sync();
    // column panel: A[i, K] = -A[i, K] P outside K, P itself on K
    for (int i = rank * blockDim.x + tid; i < n; i += ncta * blockDim.x) {
      if (i >= k0 && i < k0 + bs) {
        for (int c = 0; c < bs; c++) A[(size_t)i * n + k0 + c] = ps[i - k0][c];
        continue;
      }
      double v[GJB];
#pragma unroll
      for (int k = 0; k < GJB; k++) v[k] = k < bs ? __ldcg(A + (size_t)i * n + k0 + k) : 0.0;
      for (int c = 0; c < bs; c++) {
        double sm = 0.0;
#pragma unroll
        for (int k = 0; k < GJB; k++) sm += v[k] * ps[k][c];
        A[(size_t)i * n + k0 + c] = -sm;
      }
    }
    cl.sync();
  }
}

// an equation with a zero diagonal (a near-null-space column dropped by the
// QR leaves a zero row and column) gets the identity
__global__ void k_unit_empty_diag(int n, double *__restrict__ a) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    if (!(a[(size_t)p * n + p] > 0.0)) a[(size_t)p * n + p] = 1.0;
}

// w_{j+1} = y - alpha_j v_j - beta_j v_{j-1} (v = w / beta), u = D^-1/2 w_{j+1},
// beta_{j+1} = |w_{j+1}|.  ab holds alpha_0..alpha_63 then beta_0..beta_64.
// The first call (wj == nullptr) takes y as the start vector.
template <typename T>
__global__ void __launch_bounds__(TPB) k_lanczos_w(int n, const T *__restrict__ y, const T *__restrict__ wj,
                                                   const T *__restrict__ wprev, const T *__restrict__ dsq,
                                                   const double *__restrict__ ab, int j, T *__restrict__ wnext,
                                                   T *__restrict__ u, double *partials, unsigned *ticket,
                                                   double *beta_out) {
  double a = 0.0, bj = 1.0, bp = 1.0;
  if (wj) {
    a = ab[j];
    bj = ab[64 + j];
    if (wprev) bp = ab[64 + j - 1];
  }
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double w = (double)y[i];
    if (wj) {
      w -= a * (double)wj[i] / bj;
      if (wprev) w -= bj * (double)wprev[i] / bp;
    }
    wnext[i] = (T)w;
    u[i] = (T)((dsq ? (double)dsq[i] : 1.0) * w);
    v[0] += w * w;
  }
  double t[1];
  if (reduce_grid<1>(v, partials, ticket, t)) *beta_out = sqrt(t[0]);
}

__global__ void k_sqrt_vec(int n, const double *__restrict__ dinv, float *__restrict__ d32,
                           double *__restrict__ d64) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = sqrt(dinv[i]);
    d32[i] = (float)v;
    d64[i] = v;
  }
}

__global__ void k_to32(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

template <typename T>
__global__ void k_rand_vec(int n, T *__restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = (T)((double)(mix32(i + 777u) >> 8) * (2.0 / 16777216.0) - 1.0);
}

int grid_for(int64_t work, int per_block = TPB) {
  int64_t g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > 8 * kNumSMs) g = 8 * kNumSMs;
  return (int)g;
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

thread_local cudaStream_t amg_stream = nullptr;

void amg_free(Amg *a) { delete a; }

void amg_values_changed(sgpu_matrix m) {
  if (m->amg) m->amg->clear();
}

namespace {
// the rigid-body motions of node i in its equations, B column after column
// (B[eq + q n], the layout of sgpu_matrix_set_nullspace): the translations,
// then the rotations about z, x, y of the centred coordinates (the vectors
// aggregator::gener_rbm_1/2, GEFEL/aggregator.cpp:638-700, builds per
// aggregate); plane problems: 2 translations and the rotation; scalar
// problems: the constant
__global__ void k_rigid_body_modes(int64_t nn, int ndofn, int k, const double *__restrict__ xyz,
                                   const int64_t *__restrict__ cn, double cx, double cy, double cz,
                                   double *__restrict__ B, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const double x = xyz[3 * i] - cx, y = xyz[3 * i + 1] - cy, z = xyz[3 * i + 2] - cz;
  for (int c = 0; c < ndofn; c++) {
    const int64_t eq = cn[i * ndofn + c];
    if (eq <= 0 || eq > n) continue;
    double *b = B + (eq - 1);
    if (ndofn == 1) {
      b[0] = 1.0;
    } else if (ndofn == 2) {
      b[0] = c == 0 ? 1.0 : 0.0;
      b[n] = c == 1 ? 1.0 : 0.0;
      b[2 * n] = c == 0 ? -y : x;
    } else {
      b[0] = c == 0 ? 1.0 : 0.0;
      b[n] = c == 1 ? 1.0 : 0.0;
      b[2 * n] = c == 2 ? 1.0 : 0.0;
      b[3 * n] = c == 0 ? -y : (c == 1 ? x : 0.0);  // about z
      b[4 * n] = c == 1 ? -z : (c == 2 ? y : 0.0);  // about x
      b[5 * n] = c == 0 ? z : (c == 2 ? -x : 0.0);  // about y
    }
  }
}
}  // namespace

int amg_set_rigid_body_modes(sgpu_matrix m, int64_t nn, int ndofn, const double *coords_h, const int64_t *cn_h) {
  amg_stream = m->stream;
  if (!m->amg) m->amg = new Amg();
  Amg &A = *m->amg;
  A.clear();
  const int k = ndofn == 1 ? 1 : (ndofn == 2 ? 3 : 6);
  A.k0 = k;
  double c[3] = {0.0, 0.0, 0.0};
  for (int64_t i = 0; i < nn; i++)
    for (int q = 0; q < 3; q++) c[q] += coords_h[3 * i + q];
  for (int q = 0; q < 3; q++) c[q] /= (double)nn;
  SGPU_TRY(A.B0.alloc((size_t)m->n * k));
  PBuf<double> xyz;
  PBuf<int64_t> cn;
  SGPU_TRY(xyz.alloc((size_t)nn * 3));
  SGPU_TRY(cn.alloc((size_t)nn * ndofn));
  SGPU_CUDA(cudaMemcpyAsync(xyz.p, coords_h, (size_t)nn * 3 * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  SGPU_CUDA(cudaMemcpyAsync(cn.p, cn_h, (size_t)nn * ndofn * sizeof(int64_t), cudaMemcpyHostToDevice, m->stream));
  SGPU_CUDA(cudaMemsetAsync(A.B0.p, 0, (size_t)m->n * k * sizeof(double), m->stream));
  k_rigid_body_modes<<<(unsigned)((nn + 255) / 256), 256, 0, m->stream>>>(nn, ndofn, k, xyz.p, cn.p, c[0], c[1],
                                                                           c[2], A.B0.p, m->n);
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  SGPU_CUDA(cudaStreamSynchronize(m->stream));
  return SGPU_OK;
}

int amg_set_nullspace(sgpu_matrix m, int k, const double *B_host) {
  amg_stream = m->stream;
  if (!m->amg) m->amg = new Amg();
  Amg &A = *m->amg;
  A.clear();
  A.k0 = k;
  SGPU_TRY(A.B0.alloc((size_t)m->n * k));
  SGPU_CUDA(cudaMemcpyAsync(A.B0.p, B_host, (size_t)m->n * k * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  SGPU_CUDA(cudaStreamSynchronize(m->stream));
  return SGPU_OK;
}

namespace {

// Set-up temporaries: stream-ordered allocations from the device's memory
// pool (the pool keeps freed memory, so repeated set-ups do not pay for
// cudaMalloc / cudaFree and their device synchronisation).
void keep_pool_memory() {
  static bool done = false;
  if (done) return;
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done = true;
}

template <class T>
struct TmpBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  explicit TmpBuf(cudaStream_t st) : s(st) {}
  TmpBuf(const TmpBuf &) = delete;
  TmpBuf &operator=(const TmpBuf &) = delete;
  ~TmpBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  int alloc(size_t count) {
    if (count <= n && p) return SGPU_OK;
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocAsync((void **)&p, count * sizeof(T), s);
    if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    n = count;
    return SGPU_OK;
  }
};

struct CubTmp {
  TmpBuf<unsigned char> buf;
  explicit CubTmp(cudaStream_t s) : buf(s) {}
  int ensure(size_t bytes) { return buf.alloc(bytes); }
};

int read_int(const int *d, cudaStream_t s, int *out) {
  SGPU_CUDA(cudaMemcpyAsync(out, d, sizeof(int), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  return SGPU_OK;
}

// Distance-2 maximal independent set over the candidate nodes (all nodes, or
// with `agg` the candidates among the unaggregated ones, on their subgraph):
// on return the roots have state 2 in t.
// cluster size for k_mis2_cluster: 16 where the device schedules it, else 8,
// 0 when neither (the rounds then run as separate launches)
int mis_cluster_size() {
  static std::atomic<int> cached{-1};
  int c = cached.load();
  if (c >= 0) return c;
  c = 0;
  if (cudaFuncSetAttribute(k_mis2_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    cudaGetLastError();
  for (int cs : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kMisClusterThreads);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_mis2_cluster, &cfg) == cudaSuccess && nclusters >= 1) {
      c = cs;
      break;
    }
    cudaGetLastError();
  }
  cached.store(c);
  return c;
}

// Graphs of at most kMisClusterDefault nodes run their independent-set
// rounds in one cluster launch (on the 1.01M-DOF cantilever that is the
// 945-node level 2: set-up 5.08-5.11 ms against 5.17-5.19 ms with a launch
// per pass); the larger graphs' rounds run as separate launches over the
// whole GPU (with the cluster for the 14,586-node level 1 as well, 5.11 ms;
// up to kMisClusterNodes, 0.02-0.07 ms slower than launches)
constexpr int kMisClusterDefault = 2048;
constexpr int kMisClusterNodes = 32768;

int mis2(const AmgLevel &L, const int *cand, const int *agg, TmpBuf<uint64_t> &t, cudaStream_t s) {
  const int nb = L.nb, g = grid_for(nb);
  {
    // graphs of at most kMisClusterDefault nodes; SGPU_MIS=cluster:N (at
    // most N nodes), cluster (kMisClusterNodes), rounds (none)
    const char *me = getenv("SGPU_MIS");
    int most = kMisClusterDefault;
    if (me && !strncmp(me, "cluster", 7)) most = me[7] == ':' ? atoi(me + 8) : kMisClusterNodes;
    else if (me) most = 0;
    const int cs = nb <= std::min(most, kMisClusterNodes) ? mis_cluster_size() : 0;
    if (cs > 0) {
      TmpBuf<uint64_t> m1(s);
      TmpBuf<int> cnt(s);
      SGPU_TRY(m1.alloc(nb));
      SGPU_TRY(cnt.alloc(kMisRounds + 2));
      SGPU_CUDA(cudaMemsetAsync(cnt.p, 0, (kMisRounds + 2) * sizeof(int), s));
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(cs);
      cfg.blockDim = dim3(kMisClusterThreads);
      cfg.stream = s;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = cs;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int *rounds_d = cnt.p + kMisRounds + 1;
      SGPU_CUDA(cudaLaunchKernelEx(&cfg, k_mis2_cluster, nb, L.browptr, L.bcol, agg, cand, t.p, m1.p, cnt.p,
                                   rounds_d));
      count_launches(1);
      int rounds = 0;
      SGPU_TRY(read_int(rounds_d, s, &rounds));
      if (rounds < 0) return fail(SGPU_CUDA_ERROR, "aggregation: independent-set rounds did not finish");
      return SGPU_OK;
    }
  }
  // 8 lanes per node (SGPU_MIS=thread: a thread per node and a separate
  // decision pass); the same rounds and the same set either way
  const char *mis_env = getenv("SGPU_MIS");
  const bool warp_rows = !(mis_env && !strcmp(mis_env, "thread"));
  const int gw = grid_for((int64_t)nb * 8);
  constexpr int kMaxRounds = 200, kGroup = 16;  // rounds enqueued per host read of the count
  TmpBuf<uint64_t> m1(s), m2(s);
  TmpBuf<int> cnt(s), settled(s);
  SGPU_TRY(m1.alloc(nb));
  SGPU_TRY(m2.alloc(nb));
  SGPU_TRY(settled.alloc(nb));
  SGPU_CUDA(cudaMemsetAsync(settled.p, 0, (size_t)nb * sizeof(int), s));
  // cnt[r]: the nodes round r left undecided; cnt[0] a non-zero start.  A
  // round whose predecessor left none returns at once, so the host enqueues
  // kGroup rounds and reads the count once per group.
  SGPU_TRY(cnt.alloc(kMaxRounds + 1));
  SGPU_CUDA(cudaMemsetAsync(cnt.p, 0, (kMaxRounds + 1) * sizeof(int), s));
  SGPU_CUDA(cudaMemsetAsync(cnt.p, 0x01, sizeof(int), s));
  k_mis_init<<<g, TPB, 0, s>>>(nb, cand, t.p);
  count_launches(1);
  int undecided = nb, rounds = 0;
  while (undecided > 0) {
    if (rounds + kGroup > kMaxRounds) return fail(SGPU_CUDA_ERROR, "aggregation: independent-set rounds did not finish");
    for (int k = 0; k < kGroup; k++, rounds++) {
      const int *go = cnt.p + rounds;
      if (warp_rows) {
        k_mis_max_w<8, false><<<gw, TPB, 0, s>>>(nb, L.browptr, L.bcol, agg, t.p, m1.p, go, nullptr, nullptr,
                                                  settled.p);
        k_mis_max_w<8, true><<<gw, TPB, 0, s>>>(nb, L.browptr, L.bcol, agg, m1.p, nullptr, go, t.p,
                                                 cnt.p + rounds + 1, nullptr);
        count_launches(2);
      } else {
        k_mis_max<<<g, TPB, 0, s>>>(nb, L.browptr, L.bcol, agg, t.p, m1.p, go);
        k_mis_max<<<g, TPB, 0, s>>>(nb, L.browptr, L.bcol, agg, m1.p, m2.p, go);
        k_mis_decide<<<g, TPB, 0, s>>>(nb, t.p, m2.p, go, cnt.p + rounds + 1);
        count_launches(3);
      }
    }
    SGPU_CUDA(cudaGetLastError());
    SGPU_TRY(read_int(cnt.p + rounds, s, &undecided));
  }
  if (getenv("SGPU_AMG_VERBOSE")) {  // the rounds that had work
    std::vector<int> hc((size_t)rounds + 1);
    SGPU_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, hc.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    SGPU_CUDA(cudaStreamSynchronize(s));
    int used = 0;
    while (used < rounds && hc[used] != 0) used++;
    fprintf(stderr, "amg independent set: %d nodes, %d rounds (%d launched)\n", nb, used, rounds);
  }
  return SGPU_OK;
}

// numbers the roots of t after `base` and attaches their unaggregated
// neighbours; returns the number of new aggregates
int take_roots(const AmgLevel &L, const TmpBuf<uint64_t> &t, const int *base_d, int *agg, cudaStream_t s,
               CubTmp &tmp, int *total_d) {
  const int nb = L.nb, g = grid_for(nb);
  TmpBuf<int> flag(s), rootid(s);
  SGPU_TRY(flag.alloc(nb));
  SGPU_TRY(rootid.alloc(nb));
  k_root_flags<<<g, TPB, 0, s>>>(nb, t.p, flag.p);
  count_launches(1);
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, flag.p, rootid.p, nb, s);
  SGPU_TRY(tmp.ensure(bytes));
  SGPU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.buf.p, bytes, flag.p, rootid.p, nb, s));
  k_root_total<<<1, 1, 0, s>>>(nb, rootid.p, flag.p, base_d, total_d);
  k_attach_roots<<<g, TPB, 0, s>>>(nb, L.browptr, L.bcol, t.p, rootid.p, base_d, agg);
  count_launches(2);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

// Aggregation of a level's node graph -> L.agg, L.aggptr, L.aggnodes, L.na.
//   phase 1: MIS-2 roots over all nodes; a root takes its neighbours;
//   phase 2: MIS-2 roots among the left-over nodes that still have at least
//            4 left-over neighbours, on the left-over subgraph; same rule;
//   phase 3: every node still left joins an aggregated neighbour.
// Phase 2 keeps the aggregates near the size of a node's neighbourhood (a
// random MIS-2 alone leaves many distance-2 nodes, which then swell the
// aggregates and weaken the coarse levels).
int aggregate(AmgLevel &L, cudaStream_t s, CubTmp &tmp) {
  const int nb = L.nb, g = grid_for(nb);
  TmpBuf<uint64_t> t(s);
  TmpBuf<int> agg1(s), cand(s), cnt(s);
  SGPU_TRY(t.alloc(nb));
  SGPU_TRY(agg1.alloc(nb));
  SGPU_TRY(cand.alloc(nb));
  // cnt: aggregates after the first pass, after the second, nodes left over;
  // the counts stay on the device until the one read after the last pass
  SGPU_TRY(cnt.alloc(3));
  SGPU_CUDA(cudaMemsetAsync(cnt.p, 0, 3 * sizeof(int), s));
  SGPU_CUDA(cudaMemsetAsync(agg1.p, 0xff, (size_t)nb * sizeof(int), s));  // -1: unaggregated
  SGPU_TRY(mis2(L, nullptr, nullptr, t, s));
  SGPU_TRY(take_roots(L, t, nullptr, agg1.p, s, tmp, cnt.p));
  // second-pass candidates: left-over nodes with at least 4 left-over
  // neighbours (2, 3, 5, 6 or 8 measured: 40-43 iterations against 39 on the
  // 1.01M-DOF cantilever)
  k_mis_cand<<<g, TPB, 0, s>>>(nb, L.browptr, L.bcol, agg1.p, 4, cand.p);
  count_launches(1);
  SGPU_TRY(mis2(L, cand.p, agg1.p, t, s));
  SGPU_TRY(take_roots(L, t, cnt.p, agg1.p, s, tmp, cnt.p + 1));
  SGPU_TRY(L.agg.alloc(nb));
  k_attach2<<<g, TPB, 0, s>>>(nb, L.browptr, L.bcol, agg1.p, L.agg.p, cnt.p + 2);
  count_launches(1);
  int hc[2] = {0, 0};
  SGPU_CUDA(cudaMemcpyAsync(hc, cnt.p + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  L.na = hc[0];
  const int lost = hc[1];
  if (lost) return fail(SGPU_CUDA_ERROR, "aggregation left " + std::to_string(lost) + " nodes unassigned");
  // node lists per aggregate
  TmpBuf<int> keys_out(s), ids(s);
  SGPU_TRY(keys_out.alloc(nb));
  SGPU_TRY(ids.alloc(nb));
  SGPU_TRY(L.aggnodes.alloc(nb));
  SGPU_TRY(L.aggptr.alloc((size_t)L.na + 1));
  k_iota<<<g, TPB, 0, s>>>(nb, ids.p);
  count_launches(1);
  int end_bit = 1;
  while ((1ll << end_bit) <= L.na) end_bit++;
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, L.agg.p, keys_out.p, ids.p, L.aggnodes.p, nb, 0, end_bit, s);
  SGPU_TRY(tmp.ensure(bytes));
  SGPU_CUDA(cub::DeviceRadixSort::SortPairs(tmp.buf.p, bytes, L.agg.p, keys_out.p, ids.p, L.aggnodes.p, nb, 0,
                                            end_bit, s));
  k_agg_ptr<<<g, TPB, 0, s>>>(nb, L.na, keys_out.p, L.aggptr.p);
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

template <int B, int K>
void launch_tentative(AmgLevel &L, const double *Bl, double *Bnext, cudaStream_t s) {
  k_tentative<B, K><<<grid_for((int64_t)L.na * 32), TPB, 0, s>>>(L.na, L.aggptr.p, L.aggnodes.p, Bl, L.Q64.p, Bnext);
}

template <int B, int K>
void launch_galerkin(int nruns, const int *runoff, const int *eidx, const int *rowid, const LevelView &A,
                     const double *Q, double *out, cudaStream_t s) {
  k_galerkin<B, K><<<grid_for((int64_t)nruns * 32, 128), 128, 0, s>>>(nruns, runoff, eidx, rowid, A, Q, out);
}

bool bk_supported(int B, int K) {
  return (B == 3 && K == 6) || (B == 6 && K == 6) || (B == 1 && K == 1) || (B == 1 && K == 3) ||
         (B == 3 && K == 3) || (B == 1 && K == 6);
}

int tentative(AmgLevel &L, int K, const double *Bl, double *Bnext, cudaStream_t s) {
  SGPU_TRY(L.Q64.alloc((size_t)L.n * K));
  const int B = L.b;
  if (B == 3 && K == 6) launch_tentative<3, 6>(L, Bl, Bnext, s);
  else if (B == 6 && K == 6) launch_tentative<6, 6>(L, Bl, Bnext, s);
  else if (B == 1 && K == 1) launch_tentative<1, 1>(L, Bl, Bnext, s);
  else if (B == 1 && K == 3) launch_tentative<1, 3>(L, Bl, Bnext, s);
  else if (B == 3 && K == 3) launch_tentative<3, 3>(L, Bl, Bnext, s);
  else if (B == 1 && K == 6) launch_tentative<1, 6>(L, Bl, Bnext, s);
  else return fail(SGPU_BAD_INPUT, "unsupported block size / near-null-space size");
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

// SGPU_GALERKIN=plain: the row walk of k_gal_values2 without its software
// pipelining (the same sums in the same order: a check of the pipelined walk)
bool gal_pipelined() {
  const char *g = getenv("SGPU_GALERKIN");
  return !(g && !strcmp(g, "plain"));
}

template <int B, int K>
int launch_gal_values(const AmgLevel &L, const LevelView &view, const int *lists, AmgLevel &C, cudaStream_t s,
                      bool private_acc, int max_row) {
  if (private_acc) {
    const int cap = std::max(1, std::min(max_row, kGal2Cap));
    const size_t sm2 = gal2_shared_bytes<B, K>(cap);
    SGPU_CUDA(cudaFuncSetAttribute(k_gal_values2<B, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)gal2_shared_bytes<B, K>(kGal2Cap)));
    const int grid = (int)std::min<int64_t>(L.na, 64ll * kNumSMs);
    k_gal_values2<B, K><<<grid, 32 * kGal2Warps, sm2, s>>>(L.na, L.aggptr.p, L.aggnodes.p, L.agg.p, view, L.Q64.p,
                                                           lists, C.own_browptr.p, C.own_bcol.p, C.val64.p, cap,
                                                           gal_pipelined());
    count_launches(1);
    return SGPU_OK;
  }
  constexpr size_t sm = gal_shared_bytes<K>();
  SGPU_CUDA(cudaFuncSetAttribute(k_gal_values<B, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int grid = (int)std::min<int64_t>(L.na, 64ll * kNumSMs);
  k_gal_values<B, K><<<grid, 32 * kGalCtaWarps, sm, s>>>(L.na, L.aggptr.p, L.aggnodes.p, L.agg.p, view, L.Q64.p,
                                                          lists, C.own_browptr.p, C.own_bcol.p, C.val64.p);
  count_launches(1);
  return SGPU_OK;
}

// 1/diag and its square root for a new coarse level
int coarse_diagonals(AmgLevel &C, int K, cudaStream_t s) {
  SGPU_TRY(C.dinv64.alloc(C.n));
  SGPU_TRY(C.dinv32.alloc(C.n));
  k_coarse_dinv<<<grid_for(C.nb), TPB, 0, s>>>(C.nb, K, C.browptr, C.bcol, C.val64.p, C.dinv64.p, C.dinv32.p);
  SGPU_TRY(C.dsq64.alloc(C.n));
  SGPU_TRY(C.dsq32.alloc(C.n));
  k_sqrt_vec<<<grid_for(C.n), TPB, 0, s>>>(C.n, C.dinv64.p, C.dsq32.p, C.dsq64.p);
  count_launches(2);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

// Galerkin product by aggregate rows (k_gal_count, a scan, k_gal_values);
// *done stays false when a coarse row exceeds kGalCap blocks
// SGPU_GALERKIN=staged: the by-rows Galerkin product through the staging
// kernel (k_gal_values) even where the warp-private accumulators fit
bool gal_staged_forced() {
  const char *g = getenv("SGPU_GALERKIN");
  return g && !strcmp(g, "staged");
}

int galerkin_direct(AmgLevel &L, const LevelView &view, AmgLevel &C, int K, cudaStream_t s, CubTmp &tmp,
                    bool *done) {
  *done = false;
  const int na = L.na;
  TmpBuf<int> cnt(s), lists(s);
  SGPU_TRY(cnt.alloc((size_t)na + 2));
  SGPU_TRY(lists.alloc((size_t)na * kGalCap));
  // cnt[na] is the overflow flag (the exclusive scan's last output leaves it
  // out), cnt[na + 1] the longest coarse row
  SGPU_CUDA(cudaMemsetAsync(cnt.p + na, 0, 2 * sizeof(int), s));
  const int grid = (int)std::min<int64_t>(((int64_t)na + kGalWarps - 1) / kGalWarps, 64ll * kNumSMs);
  k_gal_count<<<grid, 32 * kGalWarps, 0, s>>>(na, L.aggptr.p, L.aggnodes.p, L.browptr, L.bcol, L.agg.p, cnt.p,
                                               lists.p, cnt.p + na, cnt.p + na + 1);
  count_launches(1);
  SGPU_TRY(C.own_browptr.alloc((size_t)na + 1));
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt.p, C.own_browptr.p, na + 1, s);
  SGPU_TRY(tmp.ensure(bytes));
  SGPU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.buf.p, bytes, cnt.p, C.own_browptr.p, na + 1, s));
  int hv[3] = {0, 0, 0};
  SGPU_CUDA(cudaMemcpyAsync(&hv[0], C.own_browptr.p + na, sizeof(int), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaMemcpyAsync(&hv[1], cnt.p + na, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  if (hv[1]) return SGPU_OK;
  const bool private_acc = hv[2] <= kGal2Cap && !gal_staged_forced();
  C.nb = na;
  C.b = K;
  C.n = na * K;
  C.nblk = hv[0];
  C.layout = 0;
  SGPU_TRY(C.own_bcol.alloc((size_t)hv[0]));
  SGPU_TRY(C.val64.alloc((size_t)hv[0] * K * K));
  C.browptr = C.own_browptr.p;
  C.bcol = C.own_bcol.p;
  const int B = L.b;
  if (B == 3 && K == 6) SGPU_TRY((launch_gal_values<3, 6>(L, view, lists.p, C, s, private_acc, hv[2])));
  else if (B == 6 && K == 6) SGPU_TRY((launch_gal_values<6, 6>(L, view, lists.p, C, s, private_acc, hv[2])));
  else if (B == 1 && K == 1) SGPU_TRY((launch_gal_values<1, 1>(L, view, lists.p, C, s, private_acc, hv[2])));
  else if (B == 1 && K == 3) SGPU_TRY((launch_gal_values<1, 3>(L, view, lists.p, C, s, private_acc, hv[2])));
  else if (B == 3 && K == 3) SGPU_TRY((launch_gal_values<3, 3>(L, view, lists.p, C, s, private_acc, hv[2])));
  else if (B == 1 && K == 6) SGPU_TRY((launch_gal_values<1, 6>(L, view, lists.p, C, s, private_acc, hv[2])));
  else return fail(SGPU_BAD_INPUT, "unsupported block size / near-null-space size");
  SGPU_CUDA(cudaGetLastError());
  *done = true;
  return SGPU_OK;
}

// Galerkin product of level L into a new coarse level C (owned, block size K):
// by aggregate rows, or (SGPU_GALERKIN=sort, or a coarse row above kGalCap
// blocks) by a global sort of the fine blocks' (G, H) keys
int galerkin(AmgLevel &L, const LevelView &view, AmgLevel &C, int K, cudaStream_t s, CubTmp &tmp, bool *by_rows) {
  const char *gm = getenv("SGPU_GALERKIN");
  *by_rows = false;
  if (!(gm && !strcmp(gm, "sort"))) {
    SGPU_TRY(galerkin_direct(L, view, C, K, s, tmp, by_rows));
    if (*by_rows) return coarse_diagonals(C, K, s);
  }
  const int64_t nblk = L.nblk;
  if (nblk >= (int64_t)INT32_MAX) return fail(SGPU_BAD_INPUT, "too many blocks for the aggregation set-up");
  const int nbk = (int)nblk;
  TmpBuf<int> rowid(s), idx(s), sidx(s), counts(s), runoff(s), nruns_d(s);
  TmpBuf<uint64_t> keys(s), skeys(s), ukeys(s);
  SGPU_TRY(rowid.alloc(nblk));
  SGPU_TRY(idx.alloc(nblk));
  SGPU_TRY(sidx.alloc(nblk));
  SGPU_TRY(keys.alloc(nblk));
  SGPU_TRY(skeys.alloc(nblk));
  k_block_rows<<<grid_for(L.nb), TPB, 0, s>>>(L.nb, L.browptr, rowid.p);
  k_gal_keys<<<grid_for(nblk), TPB, 0, s>>>(nblk, rowid.p, L.bcol, L.agg.p, keys.p, idx.p);
  count_launches(2);
  int abits = 1;
  while ((1ll << abits) <= L.na) abits++;
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.p, skeys.p, idx.p, sidx.p, nbk, 0, 32 + abits, s);
  SGPU_TRY(tmp.ensure(bytes));
  SGPU_CUDA(cub::DeviceRadixSort::SortPairs(tmp.buf.p, bytes, keys.p, skeys.p, idx.p, sidx.p, nbk, 0, 32 + abits, s));
  keys.release();
  idx.release();
  SGPU_TRY(ukeys.alloc(nblk));
  SGPU_TRY(counts.alloc(nblk + 1));
  SGPU_TRY(nruns_d.alloc(1));
  bytes = 0;
  cub::DeviceRunLengthEncode::Encode(nullptr, bytes, skeys.p, ukeys.p, counts.p, nruns_d.p, nbk, s);
  SGPU_TRY(tmp.ensure(bytes));
  SGPU_CUDA(cub::DeviceRunLengthEncode::Encode(tmp.buf.p, bytes, skeys.p, ukeys.p, counts.p, nruns_d.p, nbk, s));
  int nruns = 0;
  SGPU_TRY(read_int(nruns_d.p, s, &nruns));
  SGPU_TRY(runoff.alloc((size_t)nruns + 1));
  SGPU_CUDA(cudaMemsetAsync(counts.p + nruns, 0, sizeof(int), s));
  bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, counts.p, runoff.p, nruns + 1, s);
  SGPU_TRY(tmp.ensure(bytes));
  SGPU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.buf.p, bytes, counts.p, runoff.p, nruns + 1, s));
  // coarse level
  C.nb = L.na;
  C.b = K;
  C.n = L.na * K;
  C.nblk = nruns;
  C.layout = 0;
  SGPU_TRY(C.own_browptr.alloc((size_t)C.nb + 1));
  SGPU_TRY(C.own_bcol.alloc(nruns));
  SGPU_TRY(C.val64.alloc((size_t)nruns * K * K));
  C.browptr = C.own_browptr.p;
  C.bcol = C.own_bcol.p;
  k_gal_pattern<<<grid_for(nruns), TPB, 0, s>>>(nruns, C.nb, ukeys.p, C.own_browptr.p, C.own_bcol.p);
  count_launches(1);
  const int B = L.b;
  if (B == 3 && K == 6) launch_galerkin<3, 6>(nruns, runoff.p, sidx.p, rowid.p, view, L.Q64.p, C.val64.p, s);
  else if (B == 6 && K == 6) launch_galerkin<6, 6>(nruns, runoff.p, sidx.p, rowid.p, view, L.Q64.p, C.val64.p, s);
  else if (B == 1 && K == 1) launch_galerkin<1, 1>(nruns, runoff.p, sidx.p, rowid.p, view, L.Q64.p, C.val64.p, s);
  else if (B == 1 && K == 3) launch_galerkin<1, 3>(nruns, runoff.p, sidx.p, rowid.p, view, L.Q64.p, C.val64.p, s);
  else if (B == 3 && K == 3) launch_galerkin<3, 3>(nruns, runoff.p, sidx.p, rowid.p, view, L.Q64.p, C.val64.p, s);
  else if (B == 1 && K == 6) launch_galerkin<1, 6>(nruns, runoff.p, sidx.p, rowid.p, view, L.Q64.p, C.val64.p, s);
  else return fail(SGPU_BAD_INPUT, "unsupported block size / near-null-space size");
  count_launches(1);
  return coarse_diagonals(C, K, s);
}

// ----- level SpMV dispatch --------------------------------------------------

// grids of the FP32 smoother-bound products are halved (set by
// lanczos_enqueue): on the set-up's second stream the other half of the GPU
// stays free for the aggregation rounds that run beside them
thread_local int g_grid_div = 1;

// resident blocks of a kernel, queried once and cached (no query inside a capture)
template <class K>
int resident_grid(K kern, int64_t warps_needed) {
  static std::mutex mu;
  static std::unordered_map<const void *, int> cache;
  int nb = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find((const void *)kern);
    if (it != cache.end()) {
      nb = it->second;
    } else {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, TPB, 0);
      cache[(const void *)kern] = nb;
    }
  }
  int64_t g = (int64_t)kNumSMs * (nb > 0 ? nb : 4) / g_grid_div;
  const int64_t need = (warps_needed * 32 + TPB - 1) / TPB;
  if (g > need) g = need;
  if (g > 8192) g = 8192;
  return (int)(g < 1 ? 1 : g);
}

// blocks in flight per lane of the FP32 level-0 products with 8 lanes per
// block row: 4 (the default: 1.6 ms less solve time on the 1.01M-DOF
// cantilever than 2), or 2 with SGPU_LV0_UNROLL=2
int level0_unroll() {
  static const int u = [] {
    const char *e = getenv("SGPU_LV0_UNROLL");
    return (e && atoi(e) == 2) ? 2 : 4;
  }();
  return u;
}

// SGPU_LV0_TMA=1: the FP32 level-0 products stream tiles through shared
// memory (k_lv_bsr3_tma).  Not the default: on the 1.01M-DOF cantilever the
// solve takes 25.4 ms with it against 24.3 ms with the register kernel (its
// CTAs wait on each tile's x gathers and row updates between barriers; the
// register kernel's 32 independent warps per SM hide that latency better).
// Read at every launch, so a process can compare both.
bool level0_tma_enabled() {
  const char *e = getenv("SGPU_LV0_TMA");
  return e && !strcmp(e, "1");
}

__global__ void k_tile_blocks(int nb, const int *__restrict__ browptr, int *__restrict__ cap) {
  const int ntiles = (nb + kLvTileRows - 1) / kLvTileRows;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const int r0 = t * kLvTileRows, r1 = min(nb, r0 + kLvTileRows);
    atomicMax(cap, browptr[r1] - browptr[r0]);
  }
}

// the most blocks in a tile of the level-0 BSR3 (once per pattern; set-up
// only, never inside a capture)
int level0_tile_plan(sgpu_matrix m, cudaStream_t s) {
  Bsr3 &b = m->bsr;
  if (!b.valid || b.tile_cap != 0) return SGPU_OK;
  TmpBuf<int> cap(s);
  SGPU_TRY(cap.alloc(1));
  SGPU_CUDA(cudaMemsetAsync(cap.p, 0, sizeof(int), s));
  k_tile_blocks<<<grid_for((b.nb + kLvTileRows - 1) / kLvTileRows), TPB, 0, s>>>(b.nb, b.browptr.p, cap.p);
  count_launches(1);
  int c = 0;
  SGPU_TRY(read_int(cap.p, s, &c));
  // a stage set must fit the shared memory of one CTA
  b.tile_cap = (c > 0 && LvTile::of(c).smem_bytes() <= 200 * 1024) ? c : -1;
  return SGPU_OK;
}

// launches the streamed level-0 kernel; false when it cannot run here (no
// plan, or its shared-memory attribute not yet set while the stream captures)
template <class Op>
bool launch_level0_tma(sgpu_matrix m, const AmgLevel &L, const float *v, const Op &op, cudaStream_t s,
                       unsigned *ticket) {
  const int cap = m->bsr.tile_cap;
  if (cap <= 0 || !level0_tma_enabled()) return false;
  static int ready = 0, per_sm = 0;  // per instantiation: attribute set, resident CTAs per SM
  const size_t smem = LvTile::of(cap).smem_bytes();
  static size_t ready_smem = 0;
  auto kern = k_lv_bsr3_tma<Op>;
  if (!ready || ready_smem < smem) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TPB, smem);
    if (per_sm < 1) return false;
    ready = 1;
    ready_smem = smem;
  }
  const int ntiles = (L.nb + kLvTileRows - 1) / kLvTileRows;
  const int grid = std::max(1, std::min(ntiles, kNumSMs * per_sm));
  kern<<<grid, TPB, smem, s>>>(L.nb, cap, L.browptr, L.bcol, m->bsr.bval32s.p, v, op, pcg_state(m),
                               m->w.partials.p, ticket);
  return true;
}

// Half-precision level-0 values for the FP32 cycle: on unless SGPU_LV0_H16=0
// (read at every use, so a process can compare both forms).
bool level0_h16_enabled() {
  const char *e = getenv("SGPU_LV0_H16");
  return !(e && !strcmp(e, "0"));
}

// lanes per block row and four-block groups in flight per lane of k_lv_h16:
// SGPU_LV0_H16_SHAPE = "lanes,groups" (4 or 8 lanes, 1 or 2 groups)
void level0_h16_shape(int *lanes, int *groups) {
  *lanes = 8;
  *groups = 1;
  if (const char *e = getenv("SGPU_LV0_H16_SHAPE")) {
    int l = 0, u = 0;
    if (sscanf(e, "%d,%d", &l, &u) == 2 && (l == 4 || l == 8) && (u == 1 || u == 2)) {
      *lanes = l;
      *groups = u;
    }
  }
}

// The padded pattern (once per handle) and the binary16 values (once per
// FP32 set-up) of level 0; stream-ordered on s, never inside a capture.
// The padded pattern (once per handle) on s, then the values on vs (none
// when vs is null): the set-up converts them on its second stream, beside
// the aggregation, after a fork that follows the pattern.
int ensure_level0_h16(sgpu_matrix m, cudaStream_t s, cudaStream_t vs) {
  Amg &A = *m->amg;
  Bsr3 &b = m->bsr;
  if (!b.valid || !b.have32 || !level0_h16_enabled()) return SGPU_OK;
  if (!A.h16_struct) {
    const int nb = b.nb;
    TmpBuf<int> len(s);
    SGPU_TRY(len.alloc((size_t)nb + 1));
    k_h16_len<<<grid_for(nb), TPB, 0, s>>>(nb, b.browptr.p, len.p);
    SGPU_CUDA(cudaMemsetAsync(len.p + nb, 0, sizeof(int), s));
    SGPU_TRY(A.h16ptr.alloc((size_t)nb + 1));
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, len.p, A.h16ptr.p, nb + 1, s);
    TmpBuf<unsigned char> t(s);
    SGPU_TRY(t.alloc(tmp));
    cub::DeviceScan::ExclusiveSum(t.p, tmp, len.p, A.h16ptr.p, nb + 1, s);
    int total = 0;
    SGPU_TRY(read_int(A.h16ptr.p + nb, s, &total));
    A.h16_nblk = total;
    SGPU_TRY(A.h16col.alloc((size_t)total));
    SGPU_TRY(A.h16val.alloc((size_t)total * 9));
    k_h16_cols<<<grid_for((int64_t)nb * 32), TPB, 0, s>>>(nb, b.browptr.p, b.bcol.p, A.h16ptr.p, A.h16col.p);
    count_launches(2);
    SGPU_CUDA(cudaGetLastError());
    A.h16_struct = true;
  }
  if (!A.h16_vals) {
    if (!vs) return SGPU_OK;  // the pattern only
    k_h16_vals<<<grid_for((int64_t)b.nb * 32), TPB, 0, vs>>>(b.nb, b.browptr.p, b.bval32s.p, A.h16ptr.p,
                                                              A.h16val.p);
    count_launches(1);
    SGPU_CUDA(cudaGetLastError());
    A.h16_vals = true;
  }
  return SGPU_OK;
}

// launches the half-precision level-0 product; false when its values are not
// there (another level-0 form runs)
template <class Op>
bool launch_level0_h16(sgpu_matrix m, const AmgLevel &L, const float *v, const Op &op, cudaStream_t s,
                       unsigned *ticket) {
  const Amg &A = *m->amg;
  if (!A.h16_vals || !level0_h16_enabled()) return false;
  int lanes = 8, groups = 1;
  level0_h16_shape(&lanes, &groups);
  PcgState *st = pcg_state(m);
  double *part = m->w.partials.p;
  if (lanes == 4 && groups == 2) {
    auto k = k_lv_h16<4, 2, Op>;
    k<<<resident_grid(k, (L.nb + 7) / 8), TPB, 0, s>>>(L.nb, A.h16ptr.p, A.h16col.p, A.h16val.p, v, op, st, part,
                                                     ticket);
  } else if (lanes == 4) {
    auto k = k_lv_h16<4, 1, Op>;
    k<<<resident_grid(k, (L.nb + 7) / 8), TPB, 0, s>>>(L.nb, A.h16ptr.p, A.h16col.p, A.h16val.p, v, op, st, part,
                                                     ticket);
  } else if (groups == 2) {
    auto k = k_lv_h16<8, 2, Op>;
    k<<<resident_grid(k, (L.nb + 3) / 4), TPB, 0, s>>>(L.nb, A.h16ptr.p, A.h16col.p, A.h16val.p, v, op, st, part,
                                                     ticket);
  } else {
    auto k = k_lv_h16<8, 1, Op>;
    k<<<resident_grid(k, (L.nb + 3) / 4), TPB, 0, s>>>(L.nb, A.h16ptr.p, A.h16col.p, A.h16val.p, v, op, st, part,
                                                     ticket);
  }
  return true;
}

// the level-0 lanes per row follow the tuned SpMV of the same precision
int level0_lanes(const sgpu_matrix m, bool fp32) {
  const SpmvPlan &p = fp32 ? m->plan32 : m->plan64;
  int v = p.variant % 100;
  if (v != 4 && v != 8 && v != 16 && v != 32) v = 8;
  return v;
}

template <typename T, class Op>
int launch_level(sgpu_matrix m, const AmgLevel &L, const T *v, const Op &op, cudaStream_t s, int slot) {
  PcgState *st = pcg_state(m);
  double *part = m->w.partials.p;
  unsigned *tk = m->w.counters.p + slot;
  const T *val = level_vals<T>(m, L);
  if (L.layout == 1) {
    const int lanes = level0_lanes(m, sizeof(T) == 4);
    bool streamed = false;
    if constexpr (sizeof(T) == 4) {
      streamed = launch_level0_h16<Op>(m, L, v, op, s, tk);
      if (!streamed) streamed = launch_level0_tma<Op>(m, L, v, op, s, tk);
    }
    if (streamed) {
    } else if (sizeof(T) == 4 && lanes == 8 && level0_unroll() == 4) {
      auto k = k_lv_bsr3<T, 8, Op, 4>;
      k<<<resident_grid(k, (L.nb + 3) / 4), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk);
    } else if (lanes == 32) {
      auto k = k_lv_bsr3<T, 32, Op>;
      k<<<resident_grid(k, L.nb), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk);
    } else if (lanes == 16) {
      auto k = k_lv_bsr3<T, 16, Op>;
      k<<<resident_grid(k, (L.nb + 1) / 2), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk);
    } else {
      auto k = k_lv_bsr3<T, 8, Op>;
      k<<<resident_grid(k, (L.nb + 3) / 4), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk);
    }
  } else if (L.layout == 2) {
    const int lanes = level0_lanes(m, sizeof(T) == 4);
    if (lanes == 32) {
      auto k = k_lv_csr<T, 32, Op>;
      k<<<resident_grid(k, L.nb), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk);
    } else if (lanes == 16) {
      auto k = k_lv_csr<T, 16, Op>;
      k<<<resident_grid(k, (L.nb + 1) / 2), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk);
    } else if (lanes == 4) {
      auto k = k_lv_csr<T, 4, Op>;
      k<<<resident_grid(k, (L.nb + 7) / 8), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk);
    } else {
      auto k = k_lv_csr<T, 8, Op>;
      k<<<resident_grid(k, (L.nb + 3) / 4), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk);
    }
  } else {
    switch (L.b) {
      case 1: { auto k = k_lv_bsrb<T, 1, Op>;
        k<<<resident_grid(k, L.nb), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk); break; }
      case 3: { auto k = k_lv_bsrb<T, 3, Op>;
        k<<<resident_grid(k, L.nb), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk); break; }
      case 6: { auto k = k_lv_bsrb<T, 6, Op>;
        k<<<resident_grid(k, L.nb), TPB, 0, s>>>(L.nb, L.browptr, L.bcol, val, v, op, st, part, tk); break; }
      default:
        return fail(SGPU_BAD_INPUT, "unsupported coarse block size");
    }
  }
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}


template <typename T>
const T *level_dsq(const AmgLevel &L);
template <>
const float *level_dsq<float>(const AmgLevel &L) { return L.unit_diag ? nullptr : L.dsq32.p; }
template <>
const double *level_dsq<double>(const AmgLevel &L) { return L.unit_diag ? nullptr : L.dsq64.p; }

// largest eigenvalue of the symmetric tridiagonal matrix (a on the diagonal,
// b[1..k-1] below it) by bisection on Sturm counts
double tridiag_lmax(const std::vector<double> &a, const std::vector<double> &b) {
  const int k = (int)a.size();
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < k; i++) {
    const double r = (i > 0 ? fabs(b[i]) : 0.0) + (i + 1 < k ? fabs(b[i + 1]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  auto below = [&](double x) {  // number of eigenvalues < x
    int c = 0;
    double q = a[0] - x;
    if (q < 0) c++;
    for (int i = 1; i < k; i++) {
      if (q == 0.0) q = 1e-300;
      q = a[i] - x - b[i] * b[i] / q;
      if (q < 0) c++;
    }
    return c;
  };
  for (int it = 0; it < 200 && hi - lo > 1e-12 * std::max(1.0, fabs(hi)); it++) {
    const double mid = 0.5 * (lo + hi);
    if (below(mid) >= k) hi = mid;  // every eigenvalue is below mid
    else lo = mid;
  }
  return hi;
}

// Enqueues `steps` Lanczos steps on M = D^-1/2 A D^-1/2 on stream s; the
// coefficients land in ab[0..steps) (alpha) and ab[64..] (beta).  w0..w2, u,
// y: work vectors of L.n.
template <typename T>
int lanczos_enqueue(sgpu_matrix m, const AmgLevel &L, cudaStream_t s, int steps, T *w0, T *w1, T *w2, T *u, T *y,
                    double *ab) {
  T *w[3] = {w0, w1, w2};
  const T *dsq = level_dsq<T>(L);
  Work &wk = m->w;
  // FP32 bounds (the ones the set-up runs on its second stream) with half
  // grids, on either stream, so that the overlapped and the serial set-up
  // sum every product in the same order; restored on every return
  struct GridDiv {
    explicit GridDiv(int d) { g_grid_div = d; }
    ~GridDiv() { g_grid_div = 1; }
  } grid_div(sizeof(T) == 4 ? 2 : 1);
  const int g = grid_for(L.n);
  k_rand_vec<T><<<g, TPB, 0, s>>>(L.n, y);
  k_lanczos_w<T><<<g, TPB, 0, s>>>(L.n, y, nullptr, nullptr, dsq, ab, 0, w[0], u, wk.partials.p,
                                   wk.counters.p + 7, ab + 64);
  count_launches(2);
  for (int j = 0; j < steps; j++) {
    OpLanczos<T> op{dsq, w[j % 3], ab + 64 + j, y, ab + j};
    SGPU_TRY(launch_level<T>(m, L, u, op, s, 5));
    k_lanczos_w<T><<<g, TPB, 0, s>>>(L.n, y, w[j % 3], j > 0 ? w[(j + 2) % 3] : nullptr, dsq, ab, j,
                                     w[(j + 1) % 3], u, wk.partials.p, wk.counters.p + 7, ab + 64 + j + 1);
    count_launches(1);
  }
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

int lanczos_finish(const std::vector<double> &h, int steps, double *lmax);

// lmax of D^-1 A (= that of the symmetric D^-1/2 A D^-1/2) by `steps`
// Lanczos steps; the host reads the coefficients once at the end
template <typename T>
int lanczos_lmax(sgpu_matrix m, const AmgLevel &L, cudaStream_t s, int steps, double *lmax) {
  steps = std::max(2, std::min(steps, 63));
  TmpBuf<T> w0(s), w1(s), w2(s), u(s), y(s);
  TmpBuf<double> ab(s);
  SGPU_TRY(w0.alloc(L.n));
  SGPU_TRY(w1.alloc(L.n));
  SGPU_TRY(w2.alloc(L.n));
  SGPU_TRY(u.alloc(L.n));
  SGPU_TRY(y.alloc(L.n));
  SGPU_TRY(ab.alloc(129));
  SGPU_TRY(lanczos_enqueue<T>(m, L, s, steps, w0.p, w1.p, w2.p, u.p, y.p, ab.p));
  std::vector<double> h(129);
  SGPU_CUDA(cudaMemcpyAsync(h.data(), ab.p, 129 * sizeof(double), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  return lanczos_finish(h, steps, lmax);
}

// the largest eigenvalue of the Lanczos tridiagonal matrix of h
int lanczos_finish(const std::vector<double> &h, int steps, double *lmax) {
  std::vector<double> a(h.begin(), h.begin() + steps), b(steps, 0.0);
  for (int j = 1; j < steps; j++) b[j] = h[64 + j];
  for (int j = 0; j < steps; j++)
    if (!std::isfinite(a[j]) || !std::isfinite(b[j])) return fail(SGPU_BAD_INPUT, "smoother bound: Lanczos failed");
  *lmax = tridiag_lmax(a, b);
  if (!(*lmax > 0.0)) return fail(SGPU_BAD_INPUT, "smoother bound: non-positive estimate");
  return SGPU_OK;
}

const char *env_or(const char *name) { return getenv(name); }

// Host-side phase timer of the set-up (SGPU_AMG_VERBOSE only: it synchronises).
struct PhaseClock {
  bool on;
  cudaStream_t s;
  std::chrono::steady_clock::time_point t0;
  explicit PhaseClock(cudaStream_t st) : on(getenv("SGPU_AMG_VERBOSE") != nullptr), s(st) {
    if (on) { cudaStreamSynchronize(s); t0 = std::chrono::steady_clock::now(); }
  }
  void mark(const char *what) {
    if (!on) return;
    cudaStreamSynchronize(s);
    auto t1 = std::chrono::steady_clock::now();
    fprintf(stderr, "amg set-up %-28s %8.3f ms\n", what, std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  }
};

// The FP32 cycle's smoother bounds of the coarse smoothing levels: their
// values converted here, their Lanczos steps queued on the set-up's second
// stream after the level-0 bound, so that they run beside the dense coarsest
// inverse (both are chains of small launches).  amg_prepare_precision reads
// the coefficients.  The same kernels on the same data as lanczos_lmax, so
// the same bounds.
int coarse_bounds_enqueue(sgpu_matrix m, cudaStream_t s) {
  Amg &A = *m->amg;
  const AmgLevel *Cl = A.lv.back();
  const bool dense = Cl->n <= A.dense_max;  // the dense coarsest level is not a smoothing level
  const size_t last = dense ? A.lv.size() - 1 : A.lv.size();
  size_t need = 0;
  int cnt = 0;
  for (size_t l = 1; l < last; l++) {
    if (A.lv[l]->layout != 0) continue;
    need += 5 * (size_t)A.lv[l]->n;
    cnt++;
  }
  A.lzc_levels = 0;
  if (cnt == 0) return SGPU_OK;
  SGPU_TRY(A.lzc32.alloc(need));
  SGPU_TRY(A.lzc_ab.alloc((size_t)129 * cnt));
  for (size_t l = 1; l < last; l++) {
    AmgLevel &L = *A.lv[l];
    if (L.layout != 0) continue;
    SGPU_TRY(L.val32.alloc((size_t)L.nblk * L.b * L.b));
    k_to32<<<grid_for((int64_t)L.nblk * L.b * L.b), TPB, 0, s>>>((int64_t)L.nblk * L.b * L.b, L.val64.p, L.val32.p);
    count_launches(1);
    L.val32_ready = true;
  }
  SGPU_CUDA(cudaEventRecord(A.fork, s));
  SGPU_CUDA(cudaStreamWaitEvent(A.side, A.fork, 0));
  const int steps = std::max(2, std::min(A.lanczos_steps, 63));
  float *z = A.lzc32.p;
  int slot = 0;
  for (size_t l = 1; l < last; l++) {
    AmgLevel &L = *A.lv[l];
    if (L.layout != 0) continue;
    const size_t n = (size_t)L.n;
    SGPU_TRY(lanczos_enqueue<float>(m, L, A.side, steps, z, z + n, z + 2 * n, z + 3 * n, z + 4 * n,
                                    A.lzc_ab.p + (size_t)129 * slot));
    L.lz_slot = slot++;
    z += 5 * n;
  }
  A.lzc_levels = slot;
  return SGPU_OK;
}

// cluster size for k_bgj_cluster (SGPU_GJ=cluster): 16 where the device
// schedules it, else 8; 0 runs the four launches per pivot block, the
// default: on the 1.01M-DOF cantilever the cluster launch took 1.34 ms
// against 0.99 ms, since its 16 CTAs wait for SMs that the smoother bounds
// on the second stream hold, where the separate launches interleave with them
int gj_cluster_size() {
  const char *e = getenv("SGPU_GJ");
  if (!(e && !strcmp(e, "cluster"))) return 0;
  static std::atomic<int> cached{-1};
  int c = cached.load();
  if (c >= 0) return c;
  c = 0;
  if (cudaFuncSetAttribute(k_bgj_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    cudaGetLastError();
  for (int cs : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(TPB);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_bgj_cluster, &cfg) == cudaSuccess && nclusters >= 1) {
      c = cs;
      break;
    }
    cudaGetLastError();
  }
  cached.store(c);
  return c;
}

// Builds the hierarchy (FP64 set-up).
int amg_build(sgpu_matrix m) {
  Amg &A = *m->amg;
  cudaStream_t s = m->stream;
  A.clear();
  // "deg,alpha,ratio,coarse_max,gamma,lanczos,gamma_deep,dense_max" (tuning runs)
  if (const char *o = env_or("SGPU_AMG")) {
    int deg = A.deg, cmax = A.coarse_max, gam = A.gamma, pw = A.lanczos_steps, gd = A.gamma_deep, dm = A.dense_max;
    double al = A.alpha, ra = A.ratio;
    if (sscanf(o, "%d,%lf,%lf,%d,%d,%d,%d,%d", &deg, &al, &ra, &cmax, &gam, &pw, &gd, &dm) >= 1) {
      A.dense_max = std::max(0, std::min(dm, 4096));
      A.gamma_deep = std::max(1, std::min(gd, 2));
      A.deg = std::max(1, std::min(deg, 6));
      A.alpha = al;
      A.ratio = ra;
      A.coarse_max = std::max(16, std::min(cmax, 4096));
      A.gamma = std::max(1, std::min(gam, 2));
      A.lanczos_steps = std::max(4, std::min(pw, 63));
    }
  }
  SGPU_TRY(ensure_bsr3(m));
  SGPU_TRY(ensure_fp32(m));  // scaled FP32 level 0 and S = diag^-1/2
  SGPU_TRY(level0_tile_plan(m, s));
  // the binary16 level 0 before the level-0 bound below reads it: its
  // values on the second stream when the bound runs there
  if (A.want_fp32) SGPU_TRY(ensure_level0_h16(m, s, A.l0_bound_wanted ? nullptr : s));
  const int n = (int)m->n;
  keep_pool_memory();
  CubTmp tmp(s);
  PhaseClock clk(s);
  // level 0
  AmgLevel *L0 = A.take_level(0);
  A.lv.push_back(L0);
  if (m->bsr.valid) {
    L0->layout = 1;
    L0->b = 3;
    L0->nb = m->bsr.nb;
    L0->browptr = m->bsr.browptr.p;
    L0->bcol = m->bsr.bcol.p;
    L0->nblk = m->bsr.nblk;
  } else {
    L0->layout = 2;
    L0->b = 1;
    L0->nb = n;
    L0->browptr = m->csr.rowptr.p;
    L0->bcol = m->csr.col.p;
    L0->nblk = m->csr.nnz;
  }
  L0->n = n;
  L0->unit_diag = true;
  if (A.l0_bound_wanted) {
    // the FP32 cycle's level-0 smoother bound needs only the scaled level 0
    // (its binary16 values, converted first on the same stream): its
    // Lanczos steps (bandwidth-bound SpMVs) run on a second stream while
    // the aggregation (latency-bound rounds with host reads) runs here;
    // amg_prepare_precision collects it.  Neither touches the other's
    // buffers (the set-up kernels use no reduction partials).
    if (!A.side) SGPU_CUDA(cudaStreamCreateWithFlags(&A.side, cudaStreamNonBlocking));
    if (!A.fork) SGPU_CUDA(cudaEventCreateWithFlags(&A.fork, cudaEventDisableTiming));
    SGPU_TRY(A.lz32.alloc((size_t)5 * n));
    SGPU_TRY(A.lz_ab.alloc(129));
    SGPU_CUDA(cudaEventRecord(A.fork, s));
    SGPU_CUDA(cudaStreamWaitEvent(A.side, A.fork, 0));
    SGPU_TRY(ensure_level0_h16(m, s, A.side));
    float *z = A.lz32.p;
    SGPU_TRY(lanczos_enqueue<float>(m, *L0, A.side, std::max(2, std::min(A.lanczos_steps, 63)), z, z + n, z + 2 * n,
                                    z + 3 * (size_t)n, z + 4 * (size_t)n, A.lz_ab.p));
    A.l0_bound_pending = true;
  }
  const int K = A.k0 > 0 ? A.k0 : L0->b;
  TmpBuf<double> Bcur(s), Bnext(s);
  SGPU_TRY(Bcur.alloc((size_t)n * K));
  k_nullspace0<<<grid_for(n), TPB, 0, s>>>(n, L0->b, A.k0, A.B0.p, m->csr.dscale.p, Bcur.p, K);
  count_launches(1);
  // coarsen
  for (int level = 0; level < 12; level++) {
    AmgLevel &L = *A.lv.back();
    if (!bk_supported(L.b, K)) return fail(SGPU_BAD_INPUT, "unsupported block size / near-null-space size");
    SGPU_TRY(aggregate(L, s, tmp));
    clk.mark("aggregation");
    L.k = K;
    SGPU_TRY(Bnext.alloc((size_t)L.na * K * K));
    SGPU_TRY(tentative(L, K, Bcur.p, Bnext.p, s));
    clk.mark("tentative prolongator");
    AmgLevel *C = A.take_level(A.lv.size());
    A.lv.push_back(C);
    LevelView view{L.layout, L.browptr, L.bcol,
                   L.layout == 1 ? m->bsr.bval.p : (L.layout == 2 ? m->csr.val.p : L.val64.p), m->csr.dscale.p};
    bool by_rows = false;
    SGPU_TRY(galerkin(L, view, *C, K, s, tmp, &by_rows));
    clk.mark(by_rows ? "galerkin product (rows)" : "galerkin product (sort)");
    std::swap(Bcur.p, Bnext.p);
    std::swap(Bcur.n, Bnext.n);
    // stop when the next level is small enough for the dense solve, or when
    // aggregation no longer reduces the size
    if (C->n <= A.coarse_max || C->nb * 10 > L.nb * 8) break;
  }
  if (A.l0_bound_pending) SGPU_TRY(coarse_bounds_enqueue(m, s));
  AmgLevel *Cl = A.lv.back();
  if (Cl->n > A.dense_max) {
    // The coarsening stalled above the dense limit (many small independent
    // components, e.g. a batch of systems, each down to one or a few
    // aggregates): the last level stays a smoothing level and its "solve" is
    // `bottom_deg` Chebyshev steps, which the flexible outer CG tolerates.
    Cl->na = 0;
    Cl->k = 0;
    A.nc = 0;
    A.built = true;
    clk.mark("bottom level (smoothed, no dense inverse)");
    return SGPU_OK;
  }
  // coarsest: dense inverse
  A.nc = Cl->n;
  SGPU_TRY(A.M64.alloc((size_t)A.nc * A.nc));
  SGPU_CUDA(cudaMemsetAsync(A.M64.p, 0, (size_t)A.nc * A.nc * sizeof(double), s));
  k_dense_fill<<<grid_for((int64_t)Cl->nb * 32), TPB, 0, s>>>(Cl->nb, Cl->b, A.nc, Cl->browptr, Cl->bcol,
                                                               Cl->val64.p, A.M64.p);
  k_unit_empty_diag<<<grid_for(A.nc), TPB, 0, s>>>(A.nc, A.M64.p);
  const int gj_cs = gj_cluster_size();
  if (gj_cs > 0) {
    TmpBuf<double> P(s);
    SGPU_TRY(P.alloc(GJB * GJB));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(gj_cs);
    cfg.blockDim = dim3(TPB);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = gj_cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    SGPU_CUDA(cudaLaunchKernelEx(&cfg, k_bgj_cluster, A.nc, A.M64.p, P.p));
    count_launches(3);  // with k_dense_fill and k_unit_empty_diag
  } else {
    TmpBuf<double> P(s);
    SGPU_TRY(P.alloc(GJB * GJB));
    const int nc = A.nc;
    const int nt = (nc + GJB - 1) / GJB;  // 32-wide panels and tiles
    const dim3 tiles(nt, nt);
    for (int k0 = 0; k0 < nc; k0 += GJB) {
      const int bs = std::min(GJB, nc - k0);
      k_bgj_diag<<<1, GJB * GJB, 0, s>>>(nc, k0, bs, A.M64.p, P.p);
      k_bgj_rowpanel<<<nt, TPB, 0, s>>>(nc, k0, bs, P.p, A.M64.p);
      k_bgj_update<<<tiles, TPB, 0, s>>>(nc, k0, bs, A.M64.p);
      k_bgj_colpanel<<<nt, TPB, 0, s>>>(nc, k0, bs, P.p, A.M64.p);
    }
    count_launches(2 + 4 * ((nc + GJB - 1) / GJB));
  }
  SGPU_CUDA(cudaGetLastError());
  clk.mark("dense coarsest inverse");
  // the dense level is not a smoothing level
  A.lv.pop_back();  // (its object stays in the pool)
  A.built = true;
  if (getenv("SGPU_AMG_VERBOSE")) {
    for (size_t l = 0; l < A.lv.size(); l++) {
      const AmgLevel &L = *A.lv[l];
      fprintf(stderr, "amg level %zu: n %d nb %d b %d blocks %lld -> aggregates %d (k %d)\n", l, L.n, L.nb, L.b,
              (long long)L.nblk, L.na, L.k);
    }
    fprintf(stderr, "amg coarsest: %d equations\n", A.nc);
  }
  return SGPU_OK;
}

int amg_prepare_precision(sgpu_matrix m, bool fp32) {
  Amg &A = *m->amg;
  cudaStream_t s = m->stream;
  PhaseClock clk(s);
  if (fp32 && !A.have32) {
    SGPU_TRY(ensure_level0_h16(m, s, s));
    std::vector<double> hc;  // the coarse levels' Lanczos coefficients from the second stream
    for (size_t l = 0; l < A.lv.size(); l++) {
      AmgLevel &L = *A.lv[l];
      SGPU_TRY(L.v32.alloc(L.n));
      if (L.k > 0) {
        SGPU_TRY(L.Q32.alloc((size_t)L.n * L.k));
        k_to32<<<grid_for((int64_t)L.n * L.k), TPB, 0, s>>>((int64_t)L.n * L.k, L.Q64.p, L.Q32.p);
        count_launches(1);
      }
      if (L.layout == 0 && !L.val32_ready) {
        SGPU_TRY(L.val32.alloc((size_t)L.nblk * L.b * L.b));
        k_to32<<<grid_for((int64_t)L.nblk * L.b * L.b), TPB, 0, s>>>((int64_t)L.nblk * L.b * L.b, L.val64.p,
                                                                     L.val32.p);
        count_launches(1);
      }
      clk.mark("fp32 copies");
      if (l == 0 && A.l0_bound_pending) {
        A.l0_bound_pending = false;
        std::vector<double> h(129);
        SGPU_CUDA(cudaMemcpyAsync(h.data(), A.lz_ab.p, 129 * sizeof(double), cudaMemcpyDeviceToHost, A.side));
        if (A.lzc_levels > 0) {
          hc.resize((size_t)129 * A.lzc_levels);
          SGPU_CUDA(cudaMemcpyAsync(hc.data(), A.lzc_ab.p, hc.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                    A.side));
        }
        SGPU_CUDA(cudaStreamSynchronize(A.side));
        SGPU_TRY(lanczos_finish(h, std::max(2, std::min(A.lanczos_steps, 63)), &L.lmax32));
      } else if (L.lz_slot >= 0 && (size_t)(L.lz_slot + 1) * 129 <= hc.size()) {
        const std::vector<double> h(hc.begin() + (size_t)129 * L.lz_slot, hc.begin() + (size_t)129 * (L.lz_slot + 1));
        SGPU_TRY(lanczos_finish(h, std::max(2, std::min(A.lanczos_steps, 63)), &L.lmax32));
      } else {
        SGPU_TRY(lanczos_lmax<float>(m, L, s, A.lanczos_steps, &L.lmax32));
      }
      clk.mark("Lanczos bound");
      if (getenv("SGPU_AMG_VERBOSE")) fprintf(stderr, "amg level %zu: lmax (fp32) %.6g\n", l, L.lmax32);
    }
    if (A.nc > 0) {
      SGPU_TRY(A.M32.alloc((size_t)A.nc * A.nc));
      k_to32<<<grid_for((int64_t)A.nc * A.nc), TPB, 0, s>>>((int64_t)A.nc * A.nc, A.M64.p, A.M32.p);
      count_launches(1);
      SGPU_TRY(A.cb32.alloc(A.nc));
      SGPU_TRY(A.cx32.alloc(A.nc));
    }
    SGPU_CUDA(cudaGetLastError());
    A.have32 = true;
  }
  if (!fp32 && !A.have64) {
    for (size_t l = 0; l < A.lv.size(); l++) {
      AmgLevel &L = *A.lv[l];
      SGPU_TRY(L.v64.alloc(L.n));
      if (L.layout != 0) {
        SGPU_TRY(L.val64.alloc(L.layout == 1 ? (size_t)L.nblk * 9 : (size_t)L.nblk));
        k_scale_level0<<<grid_for((int64_t)L.nb * 32), TPB, 0, s>>>(L.nb, L.layout, L.browptr, L.bcol,
                                                      L.layout == 1 ? m->bsr.bval.p : m->csr.val.p,
                                                      m->csr.dscale.p, L.val64.p);
        count_launches(1);
      }
      clk.mark("fp64 scaled level 0");
      SGPU_TRY(lanczos_lmax<double>(m, L, s, A.lanczos_steps, &L.lmax64));
      clk.mark("Lanczos bound");
      if (getenv("SGPU_AMG_VERBOSE")) fprintf(stderr, "amg level %zu: lmax (fp64) %.6g\n", l, L.lmax64);
    }
    SGPU_TRY(A.cb64.alloc(A.nc));
    SGPU_TRY(A.cx64.alloc(A.nc));
    SGPU_CUDA(cudaGetLastError());
    A.have64 = true;
  }
  return SGPU_OK;
}

// ----- the V-cycle ------------------------------------------------------------

template <typename T>
LevelVecs<T> &vecs(AmgLevel &L);
template <>
LevelVecs<float> &vecs<float>(AmgLevel &L) { return L.v32; }
template <>
LevelVecs<double> &vecs<double>(AmgLevel &L) { return L.v64; }
template <typename T>
const T *qmat(const AmgLevel &L);
template <>
const float *qmat<float>(const AmgLevel &L) { return L.Q32.p; }
template <>
const double *qmat<double>(const AmgLevel &L) { return L.Q64.p; }

template <typename T, int B, int K>
void launch_restrict(const AmgLevel &L, const T *res, T *bc, T *rc, T *dc, T *xc, const T *dinvc, T c2, bool start,
                     const PcgState *st, cudaStream_t s) {
  const int g = grid_for((int64_t)L.na * 32);
  if (start)
    k_restrict<T, B, K, true><<<g, TPB, 0, s>>>(L.na, L.aggptr.p, L.aggnodes.p, qmat<T>(L), res, bc, rc, dc, xc,
                                                 dinvc, c2, st);
  else
    k_restrict<T, B, K, false><<<g, TPB, 0, s>>>(L.na, L.aggptr.p, L.aggnodes.p, qmat<T>(L), res, bc, rc, dc, xc,
                                                  dinvc, c2, st);
}

template <typename T>
int restrict_level(const AmgLevel &L, const T *res, T *bc, T *rc, T *dc, T *xc, const T *dinvc, T c2, bool start,
                   const PcgState *st, cudaStream_t s) {
  const int B = L.b, K = L.k;
  if (B == 3 && K == 6) launch_restrict<T, 3, 6>(L, res, bc, rc, dc, xc, dinvc, c2, start, st, s);
  else if (B == 6 && K == 6) launch_restrict<T, 6, 6>(L, res, bc, rc, dc, xc, dinvc, c2, start, st, s);
  else if (B == 1 && K == 1) launch_restrict<T, 1, 1>(L, res, bc, rc, dc, xc, dinvc, c2, start, st, s);
  else if (B == 1 && K == 3) launch_restrict<T, 1, 3>(L, res, bc, rc, dc, xc, dinvc, c2, start, st, s);
  else if (B == 3 && K == 3) launch_restrict<T, 3, 3>(L, res, bc, rc, dc, xc, dinvc, c2, start, st, s);
  else if (B == 1 && K == 6) launch_restrict<T, 1, 6>(L, res, bc, rc, dc, xc, dinvc, c2, start, st, s);
  else return fail(SGPU_BAD_INPUT, "unsupported block size / near-null-space size");
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

template <typename T>
int prolong_level(const AmgLevel &L, const T *xc, T *x, T alpha, const PcgState *st, cudaStream_t s) {
  const int B = L.b, K = L.k, g = grid_for(L.n);
  if (B == 3 && K == 6) k_prolong<T, 3, 6><<<g, TPB, 0, s>>>(L.n, L.agg.p, qmat<T>(L), xc, x, alpha, st);
  else if (B == 6 && K == 6) k_prolong<T, 6, 6><<<g, TPB, 0, s>>>(L.n, L.agg.p, qmat<T>(L), xc, x, alpha, st);
  else if (B == 1 && K == 1) k_prolong<T, 1, 1><<<g, TPB, 0, s>>>(L.n, L.agg.p, qmat<T>(L), xc, x, alpha, st);
  else if (B == 1 && K == 3) k_prolong<T, 1, 3><<<g, TPB, 0, s>>>(L.n, L.agg.p, qmat<T>(L), xc, x, alpha, st);
  else if (B == 3 && K == 3) k_prolong<T, 3, 3><<<g, TPB, 0, s>>>(L.n, L.agg.p, qmat<T>(L), xc, x, alpha, st);
  else if (B == 1 && K == 6) k_prolong<T, 1, 6><<<g, TPB, 0, s>>>(L.n, L.agg.p, qmat<T>(L), xc, x, alpha, st);
  else return fail(SGPU_BAD_INPUT, "unsupported block size / near-null-space size");
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

// One smoothing pass after the first step (the first step from x = 0 is
// fused into whatever produced b).  `x` is the current iterate, `din` the
// current direction; on return x holds the smoothed iterate.
template <typename T>
int cheb_steps(sgpu_matrix m, AmgLevel &L, const Cheb &c, int deg, T *x, T **din, T **dout, bool outer,
               cudaStream_t s) {
  LevelVecs<T> &V = vecs<T>(L);
  Work &w = m->w;
  for (int k = 1; k < deg; k++) {
    const bool last = (k == deg - 1);
    if (outer && last && m->amg->batch_zr) {
      OpChebRows<T, false> op{V.b.p, nullptr, x, V.r.p, *din, level_dinv<T>(L), (T)c.c1[k], (T)c.c2[k],
                              m->csr.dscale.p, w.r.p, w.p.p, m->amg->batch_zr, m->amg->batch_zq};
      SGPU_TRY(launch_level<T>(m, L, *din, op, s, 0));
    } else if (outer && last) {
      OpCheb<T, false, true> op{V.b.p, nullptr, x, V.r.p, *din, *dout, level_dinv<T>(L), (T)c.c1[k], (T)c.c2[k], 1,
                                m->csr.dscale.p, w.r.p, w.p.p, w.h.p};
      SGPU_TRY(launch_level<T>(m, L, *din, op, s, 6));
    } else {
      OpCheb<T, false, false> op{V.b.p, nullptr, x, V.r.p, *din, *dout, level_dinv<T>(L), (T)c.c1[k], (T)c.c2[k],
                                 last ? 1 : 0, nullptr, nullptr, nullptr, nullptr};
      SGPU_TRY(launch_level<T>(m, L, *din, op, s, 0));
    }
    std::swap(*din, *dout);
  }
  return SGPU_OK;
}

// ----- the fused coarse tail (k_coarse_tail) ----------------------------------

constexpr int kTailMaxN = 24576;  // larger last levels keep the full-GPU kernels

// cluster size k_coarse_tail<T, B, K> runs with on this device: 16 CTAs when
// the device schedules such a cluster, else 8, else 0 (not used).  Asked once
// per process, on the first cycle (which runs before any graph capture).
template <typename T, int B, int K>
int tail_cluster_size() {
  static std::atomic<int> cached{-1};
  int c = cached.load();
  if (c >= 0) return c;
  auto kern = k_coarse_tail<T, B, K>;
  c = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) cudaGetLastError();
  for (int cs : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kTailThreads);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) == cudaSuccess && nclusters >= 1) {
      c = cs;
      break;
    }
    cudaGetLastError();
  }
  cached.store(c);
  return c;
}

template <typename T, int B, int K>
int launch_tail_bk(const TailArgs<T> &a, cudaStream_t s, bool *launched) {
  *launched = false;
  const int cs = tail_cluster_size<T, B, K>();
  if (cs == 0) return SGPU_OK;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(kTailThreads);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  SGPU_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_tail<T, B, K>, a));
  count_launches(1);
  *launched = true;
  return SGPU_OK;
}

// Runs all `visits` cycles of level C (the last smoothed level, with the
// dense coarsest below it) in one cluster launch when the block and
// near-null-space sizes have an instantiation; *launched tells the caller
// whether it has to run the separate kernels instead.
template <typename T>
int launch_tail(const TailArgs<T> &a, int B, int K, cudaStream_t s, bool *launched) {
  *launched = false;
  if (B == 6 && K == 6) return launch_tail_bk<T, 6, 6>(a, s, launched);
  if (B == 3 && K == 3) return launch_tail_bk<T, 3, 3>(a, s, launched);
  if (B == 1 && K == 1) return launch_tail_bk<T, 1, 1>(a, s, launched);
  return SGPU_OK;
}

// The fused tail runs with SGPU_AMG_TAIL=1 (read at every cycle build, so
// that a process can compare both forms).  It is not the default: on the
// 1.01M-DOF cantilever the 16 SMs of one cluster read the coarse level more
// slowly than the separate full-GPU kernels pay in launch latency (28.3 ms
// against 26.1 ms of solve).
bool tail_enabled() {
  const char *e = getenv("SGPU_AMG_TAIL");
  return e && e[0] == '1';
}

// One cycle on level l (l = number of smoothing levels: the dense coarsest).
// With zero_init the first smoothing step from x = 0 was fused into whatever
// produced b (k_fcg_update / k_fcg_init for level 0, the restriction for the
// coarser levels); otherwise the cycle starts from xcur[l].  Each level
// visits the next one `gamma` times (1: V-cycle, 2: W-cycle).  The level-0
// post-smoothing's last step forms z = S x with r.z and q.z (OpCheb OUTER).
template <typename T>
int cycle(sgpu_matrix m, int l, bool zero_init, const std::vector<Cheb> &ch, std::vector<T *> &xcur, cudaStream_t s) {
  Amg &A = *m->amg;
  const int nl = (int)A.lv.size();
  const int deg = A.deg;
  PcgState *st = pcg_state(m);
  Work &w = m->w;
  if (l == nl) {
    const T *M = sizeof(T) == 4 ? (const T *)A.M32.p : (const T *)A.M64.p;
    T *cb = sizeof(T) == 4 ? (T *)A.cb32.p : (T *)A.cb64.p;
    T *cx = sizeof(T) == 4 ? (T *)A.cx32.p : (T *)A.cx64.p;
    k_dense_mv<T><<<grid_for((int64_t)A.nc * 32), TPB, 0, s>>>(A.nc, M, cb, cx, st);
    count_launches(1);
    xcur[l] = cx;
    return SGPU_OK;
  }
  AmgLevel &L = *A.lv[l];
  LevelVecs<T> &V = vecs<T>(L);
  if (l == nl - 1 && A.nc == 0) {
    // bottom level without a dense inverse: bottom_deg Chebyshev steps
    const Cheb cb = cheb_coeffs(sizeof(T) == 4 ? L.lmax32 : L.lmax64, A.ratio, A.bottom_deg);
    T *xp = V.x.p;
    if (!zero_init) {
      T *from = xcur[l], *to = (from == V.x.p) ? V.x2.p : V.x.p;
      OpCheb<T, true, false> op{V.b.p, from, to, V.r.p, nullptr, V.d.p, level_dinv<T>(L), (T)0, (T)cb.c2_first, 0,
                                nullptr, nullptr, nullptr, nullptr};
      SGPU_TRY(launch_level<T>(m, L, from, op, s, 0));
      xp = to;
    }
    T *din = V.d.p, *dout = V.d2.p;
    SGPU_TRY(cheb_steps<T>(m, L, cb, A.bottom_deg, xp, &din, &dout, false, s));
    xcur[l] = xp;
    return SGPU_OK;
  }
  T *xp;
  // pre-smoothing
  if (zero_init) {
    xp = V.x.p;
  } else {
    T *from = xcur[l], *to = (from == V.x.p) ? V.x2.p : V.x.p;
    OpCheb<T, true, false> op{V.b.p, from, to, V.r.p, nullptr, V.d.p, level_dinv<T>(L), (T)0, (T)ch[l].c2_first,
                              deg == 1 ? 1 : 0, nullptr, nullptr, nullptr, nullptr};
    SGPU_TRY(launch_level<T>(m, L, from, op, s, 0));
    xp = to;
  }
  {
    T *din = V.d.p, *dout = V.d2.p;
    SGPU_TRY(cheb_steps<T>(m, L, ch[l], deg, xp, &din, &dout, false, s));
  }
  // residual and restriction
  {
    OpResid<T> op{V.b.p, V.res.p};
    SGPU_TRY(launch_level<T>(m, L, xp, op, s, 0));
  }
  if (l + 1 < nl) {
    AmgLevel &C = *A.lv[l + 1];
    LevelVecs<T> &W = vecs<T>(C);
    SGPU_TRY(restrict_level<T>(L, V.res.p, W.b.p, W.r.p, W.d.p, W.x.p, level_dinv<T>(C), (T)ch[l + 1].c2_first, true,
                               st, s));
    // coarse correction
    const int visits = l == 0 ? A.gamma : A.gamma_deep;
    bool fused = false;
    if (l + 1 == nl - 1 && A.nc > 0 && A.deg == 1 && C.layout == 0 && C.n <= kTailMaxN && tail_enabled()) {
      TailArgs<T> ta{C.nb, C.browptr, C.bcol, level_vals<T>(m, C), level_dinv<T>(C), W.b.p, W.x.p, W.x2.p,
                     W.res.p, C.na, C.aggptr.p, C.aggnodes.p, C.agg.p, qmat<T>(C), A.nc,
                     sizeof(T) == 4 ? (const T *)A.M32.p : (const T *)A.M64.p,
                     sizeof(T) == 4 ? (T *)A.cb32.p : (T *)A.cb64.p, sizeof(T) == 4 ? (T *)A.cx32.p : (T *)A.cx64.p,
                     (T)ch[l + 1].c2_first, (T)A.alpha, visits, st};
      SGPU_TRY(launch_tail<T>(ta, C.b, C.k, s, &fused));
      if (fused) xcur[l + 1] = W.x2.p;
    }
    if (!fused)
      for (int v = 0; v < visits; v++) SGPU_TRY(cycle<T>(m, l + 1, v == 0, ch, xcur, s));
    SGPU_TRY(prolong_level<T>(L, xcur[l + 1], xp, (T)A.alpha, st, s));
  } else {
    T *cb = sizeof(T) == 4 ? (T *)A.cb32.p : (T *)A.cb64.p;
    SGPU_TRY(restrict_level<T>(L, V.res.p, cb, nullptr, nullptr, nullptr, nullptr, (T)0, false, st, s));
    SGPU_TRY(cycle<T>(m, l + 1, true, ch, xcur, s));
    SGPU_TRY(prolong_level<T>(L, xcur[l + 1], xp, (T)A.alpha, st, s));
  }
  // post-smoothing: first step from x (SpMV of x, result in the other buffer)
  const bool outer = (l == 0);
  T *to = (xp == V.x.p) ? V.x2.p : V.x.p;
  if (outer && deg == 1 && A.batch_zr) {
    OpChebRows<T, true> op{V.b.p, xp, to, nullptr, nullptr, level_dinv<T>(L), (T)0, (T)ch[l].c2_first,
                           m->csr.dscale.p, w.r.p, w.p.p, A.batch_zr, A.batch_zq};
    SGPU_TRY(launch_level<T>(m, L, xp, op, s, 0));
  } else if (outer && deg == 1) {
    OpCheb<T, true, true> op{V.b.p, xp, to, V.r.p, nullptr, V.d.p, level_dinv<T>(L), (T)0, (T)ch[l].c2_first, 1,
                             m->csr.dscale.p, w.r.p, w.p.p, w.h.p};
    SGPU_TRY(launch_level<T>(m, L, xp, op, s, 6));
  } else {
    OpCheb<T, true, false> op{V.b.p, xp, to, V.r.p, nullptr, V.d.p, level_dinv<T>(L), (T)0, (T)ch[l].c2_first,
                              deg == 1 ? 1 : 0, nullptr, nullptr, nullptr, nullptr};
    SGPU_TRY(launch_level<T>(m, L, xp, op, s, 0));
  }
  {
    T *din = V.d.p, *dout = V.d2.p;
    SGPU_TRY(cheb_steps<T>(m, L, ch[l], deg, to, &din, &dout, outer, s));
  }
  xcur[l] = to;
  return SGPU_OK;
}

// One preconditioner application followed by p = S x0 + beta p.
template <typename T>
int vcycle_dir(sgpu_matrix m, cudaStream_t s) {
  Amg &A = *m->amg;
  const int nl = (int)A.lv.size();
  std::vector<Cheb> ch(nl);
  for (int l = 0; l < nl; l++)
    ch[l] = cheb_coeffs(sizeof(T) == 4 ? A.lv[l]->lmax32 : A.lv[l]->lmax64, A.ratio, A.deg);
  std::vector<T *> xcur(nl + 1, nullptr);
  SGPU_TRY(cycle<T>(m, 0, true, ch, xcur, s));
  k_fcg_dir<T><<<grid_for(m->n), TPB, 0, s>>>((int)m->n, m->w.d.p, xcur[0], m->csr.dscale.p, pcg_state(m));
  count_launches(1);
  return SGPU_OK;
}

template <typename T>
int fcg_update(sgpu_matrix m, cudaStream_t s) {
  Amg &A = *m->amg;
  AmgLevel &L0 = *A.lv[0];
  LevelVecs<T> &V = vecs<T>(L0);
  Work &w = m->w;
  const double l0 = sizeof(T) == 4 ? L0.lmax32 : L0.lmax64;
  const T c2 = (T)cheb_coeffs(l0, A.ratio, A.deg).c2_first;
  k_fcg_update<T><<<grid_for(m->n), TPB, 0, s>>>((int)m->n, w.x.p, w.r.p, w.d.p, w.p.p, m->csr.dscale.p, V.b.p,
                                                  V.r.p, V.d.p, V.x.p, c2, pcg_state(m), w.partials.p,
                                                  w.counters.p + 2);
  count_launches(1);
  return SGPU_OK;
}

template <typename T>
int fcg_init(sgpu_matrix m, cudaStream_t s) {
  Amg &A = *m->amg;
  AmgLevel &L0 = *A.lv[0];
  LevelVecs<T> &V = vecs<T>(L0);
  Work &w = m->w;
  const double l0 = sizeof(T) == 4 ? L0.lmax32 : L0.lmax64;
  const T c2 = (T)cheb_coeffs(l0, A.ratio, A.deg).c2_first;
  k_fcg_init<T><<<grid_for(m->n), TPB, 0, s>>>((int)m->n, w.f.p, w.p.p, w.r.p, m->csr.dscale.p, V.b.p, V.r.p, V.d.p,
                                                V.x.p, c2, pcg_state(m), w.partials.p, w.counters.p + 2);
  count_launches(1);
  return SGPU_OK;
}

int read_st(sgpu_matrix m, PcgState *h) {
  SGPU_CUDA(cudaMemcpyAsync(h, pcg_state(m), sizeof(PcgState), cudaMemcpyDeviceToHost, m->stream));
  SGPU_CUDA(cudaStreamSynchronize(m->stream));
  return SGPU_OK;
}

int write_st(sgpu_matrix m, const PcgState *h) {
  SGPU_CUDA(cudaMemcpyAsync(pcg_state(m), h, sizeof(PcgState), cudaMemcpyHostToDevice, m->stream));
  SGPU_CUDA(cudaStreamSynchronize(m->stream));
  return SGPU_OK;
}

template <typename T>
int capture_chunk(sgpu_matrix m, int iters, cudaGraphExec_t *exec, int64_t *nodes) {
  cudaStream_t s = m->stream;
  Work &w = m->w;
  const int64_t before = sgpu_kernel_launches();
  cudaGraph_t g;
  SGPU_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  int rc = SGPU_OK;
  for (int it = 0; it < iters && rc == SGPU_OK; it++) {
    rc = spmv64_flex(m, w.d.p, w.p.p, s);
    if (rc == SGPU_OK) rc = fcg_update<T>(m, s);
    if (rc == SGPU_OK) rc = vcycle_dir<T>(m, s);
  }
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc != SGPU_OK) return rc;
  if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  *nodes = sgpu_kernel_launches() - before;
  count_launches(-*nodes);  // captured launches run (and are counted) at each replay
  return SGPU_OK;
}

// The loop body's last kernel: run the body again while the iteration has
// not stopped and the launch's iteration cap is not reached.
__global__ void k_fcg_continue(cudaGraphConditionalHandle h, PcgState *st, int64_t cap) {
  const int64_t c = ++st->loops;
  cudaGraphSetConditional(h, (!st->done && c < cap) ? 1u : 0u);
}

// The flexible CG's iterations as one graph: a conditional WHILE node whose
// body is one iteration (FP64 SpMV, update, V-cycle and direction) and
// k_fcg_continue, which ends the loop when the solver's state says done (the
// stopping test, a breakdown or ni iterations) or after `cap` iterations of
// one launch, whichever comes first.  The host waits once per launch.
// Returns SGPU_OK with *exec == nullptr when the runtime offers no
// conditional nodes (the caller then uses capture_chunk).
template <typename T>
int capture_loop(sgpu_matrix m, int64_t cap, cudaGraphExec_t *exec, int64_t *nodes) {
  cudaStream_t s = m->stream;
  Work &w = m->w;
  *exec = nullptr;
  cudaGraph_t g = nullptr;
  SGPU_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return SGPU_OK;
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, g, nullptr, 0, &cp) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return SGPU_OK;
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  const int64_t before = sgpu_kernel_launches();
  cudaError_t e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(SGPU_CUDA_ERROR, std::string("cudaStreamBeginCaptureToGraph: ") + cudaGetErrorString(e));
  }
  int rc = spmv64_flex(m, w.d.p, w.p.p, s);
  if (rc == SGPU_OK) rc = fcg_update<T>(m, s);
  if (rc == SGPU_OK) rc = vcycle_dir<T>(m, s);
  if (rc == SGPU_OK) {
    k_fcg_continue<<<1, 1, 0, s>>>(h, pcg_state(m), cap);
    count_launches(1);
  }
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(s, &captured);
  if (rc != SGPU_OK) {
    cudaGraphDestroy(g);
    return rc;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  *nodes = sgpu_kernel_launches() - before;  // kernels of one iteration
  count_launches(-*nodes);
  if (e != cudaSuccess) {  // a body the runtime does not take: the caller captures chunks
    cudaGetLastError();
    *exec = nullptr;
    if (getenv("SGPU_AMG_VERBOSE"))
      fprintf(stderr, "amg: no device-side loop graph (%s); chunks of iterations\n", cudaGetErrorString(e));
  }
  return SGPU_OK;
}

// r = f - K x with a fresh V-cycle and p = z: (re)start of the recurrence
template <typename T>
int fcg_start(sgpu_matrix m, cudaStream_t s) {
  Work &w = m->w;
  SGPU_TRY(spmv64(m, w.x.p, w.p.p, s));
  SGPU_TRY(fcg_init<T>(m, s));
  return vcycle_dir<T>(m, s);
}

template <typename T>
int fcg_solve(sgpu_matrix m, int64_t ni, double res, double zero, int64_t iv, int crit, PcgState *hs) {
  cudaStream_t s = m->stream;
  Work &w = m->w;
  const int n = (int)m->n;
  PcgState init{};
  init.ni = ni;
  init.res = res;
  init.zero = zero;
  init.tol2 = res * res;
  init.crit = crit;
  init.prec = SGPU_PREC_AGG;
  SGPU_TRY(write_st(m, &init));
  if (iv == 0) SGPU_CUDA(cudaMemsetAsync(w.x.p, 0, (size_t)n * sizeof(double), s));
  SGPU_TRY(fcg_start<T>(m, s));
  SGPU_TRY(read_st(m, hs));
  if (hs->done) return SGPU_OK;
  const int chunk = 8;
  cudaGraphExec_t exec = nullptr;
  int64_t nodes = 0;
  PhaseClock clk(s);
  // the device-side loop (SGPU_FCG_LOOP=chunk: graphs of `chunk` iterations
  // and a host test between them)
  const char *lm = getenv("SGPU_FCG_LOOP");
  bool loop = !(lm && !strcmp(lm, "chunk"));
  if (loop) {
    // at most the remaining iterations (plus one) per launch
    SGPU_TRY(capture_loop<T>(m, std::max<int64_t>(2, ni - hs->it + 1), &exec, &nodes));
    loop = exec != nullptr;
  }
  if (!loop) SGPU_TRY(capture_chunk<T>(m, chunk, &exec, &nodes));
  clk.mark(loop ? "graph capture + instantiate (loop)" : "graph capture + instantiate");
  int rc = SGPU_OK;
  int restarts = 0;
  for (;;) {
    if (loop) SGPU_CUDA(cudaMemsetAsync(&pcg_state(m)->loops, 0, sizeof(int64_t), s));
    cudaError_t e = cudaGraphLaunch(exec, s);
    if (e != cudaSuccess) { rc = fail(SGPU_CUDA_ERROR, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e)); break; }
    rc = read_st(m, hs);
    if (rc != SGPU_OK) break;
    count_launches(loop ? nodes * hs->loops : nodes);
    if (!hs->done) continue;
    // converged on the recurrence: with SGPU_CRIT_TRUE the true residual must
    // agree, else the recurrence restarts from it (at most four times; a
    // threshold still unmet then is reported as not reached)
    if (crit != SGPU_CRIT_TRUE || hs->status != 0) break;
    rc = spmv64(m, w.x.p, w.p.p, s);
    if (rc != SGPU_OK) break;
    k_fcg_true<<<grid_for(n), TPB, 0, s>>>(n, w.f.p, w.p.p, pcg_state(m), w.partials.p, w.counters.p + 3);
    count_launches(1);
    rc = read_st(m, hs);
    if (rc != SGPU_OK || hs->true_rel < res) break;
    if (restarts >= 4 || hs->it >= ni) {
      PcgState t = *hs;
      t.status = SGPU_NOT_CONVERGED;
      t.ani_set = 0;
      rc = write_st(m, &t);
      *hs = t;
      break;
    }
    restarts++;
    PcgState t = *hs;
    t.done = 0;
    t.ani_set = 0;
    rc = write_st(m, &t);
    if (rc == SGPU_OK) rc = fcg_start<T>(m, s);
    if (rc != SGPU_OK) break;
  }
  cudaGraphExecDestroy(exec);
  return rc;
}

}  // namespace

int amg_ensure(sgpu_matrix m, bool fp32, float *setup_ms) {
  cudaStream_t s = m->stream;
  amg_stream = s;
  if (!m->amg) m->amg = new Amg();
  Amg &A = *m->amg;
  SGPU_CUDA(cudaEventRecord(m->ev0, s));
  {
    PcgState zero_st{};
    SGPU_TRY(write_st(m, &zero_st));  // set-up kernels run with a live state
  }
  A.l0_bound_wanted = fp32 && !A.built && !getenv("SGPU_AMG_SERIAL_BOUND");
  A.want_fp32 = fp32;
  if (!A.built) {
    const int rc = amg_build(m);
    if (rc != SGPU_OK) {
      if (A.side) cudaStreamSynchronize(A.side);
      A.l0_bound_pending = false;
      return rc;
    }
  }
  A.l0_bound_wanted = false;
  SGPU_TRY(amg_prepare_precision(m, fp32));
  SGPU_CUDA(cudaEventRecord(m->ev1, s));
  SGPU_CUDA(cudaEventSynchronize(m->ev1));
  *setup_ms = 0.f;
  SGPU_CUDA(cudaEventElapsedTime(setup_ms, m->ev0, m->ev1));
  return SGPU_OK;
}

int amg_pcg_run(sgpu_matrix m, int64_t ni, double res, double zero, int64_t iv, int crit, int mode, int64_t *ani,
                double *ares, sgpu_solve_info *info) {
  cudaStream_t s = m->stream;
  if (!m->csr.diag_positive)
    return fail(SGPU_BAD_INPUT, "the aggregation preconditioner needs a positive diagonal (Jacobi scaling)");
  SGPU_TRY(pcg_prepare(m, false));
  if (!m->plan64.tuned) SGPU_TRY(spmv_autotune(m, 64));
  const bool fp32 = (mode == SGPU_MIXED);
  if (fp32 && !m->plan32.tuned) SGPU_TRY(spmv_autotune(m, 32));
  float setup_ms = 0.f;
  SGPU_TRY(amg_ensure(m, fp32, &setup_ms));
  Amg &A = *m->amg;
  PcgState hs{};
  SGPU_CUDA(cudaEventRecord(m->ev0, s));
  int rc = fp32 ? fcg_solve<float>(m, ni, res, zero, iv, crit, &hs) : fcg_solve<double>(m, ni, res, zero, iv, crit, &hs);
  SGPU_CUDA(cudaEventRecord(m->ev1, s));
  if (rc != SGPU_OK) return rc;
  SGPU_CUDA(cudaEventSynchronize(m->ev1));
  float solve_ms = 0.f;
  SGPU_CUDA(cudaEventElapsedTime(&solve_ms, m->ev0, m->ev1));
  // true FP64 residual of the returned x: the solve's own last check when it
  // stopped on the true residual (x has not changed since), else formed here
  PcgState fin{};
  if (crit == SGPU_CRIT_TRUE && hs.status == 0 && hs.true_rel > 0.0 && hs.true_rel < res) {
    fin = hs;
  } else {
    Work &w = m->w;
    SGPU_TRY(spmv64(m, w.x.p, w.p.p, s));
    k_fcg_true<<<grid_for(m->n), TPB, 0, s>>>((int)m->n, w.f.p, w.p.p, pcg_state(m), w.partials.p,
                                              w.counters.p + 3);
    count_launches(1);
    SGPU_TRY(read_st(m, &fin));
  }
  if (hs.ani_set && hs.status == 0) {
    if (ani) *ani = hs.ani;
    if (ares) *ares = hs.ares;
  }
  if (info) {
    info->iterations = hs.it;
    info->refinements = 0;
    info->rh_over_ff = hs.rho / (hs.nory > 0 ? hs.nory : 1.0);
    info->crit_value = crit == SGPU_CRIT_SCR_PREC ? hs.rr / (hs.nory > 0 ? hs.nory : 1.0)
                                                  : sqrt(hs.rr / (hs.nory > 0 ? hs.nory : 1.0));
    info->true_relres = fin.true_rel;
    info->solve_ms = solve_ms;
    info->precond_setup_ms = setup_ms;
    info->precond_levels = (int32_t)A.lv.size() + 1;
    info->precond_coarse_n = A.nc;
    info->spmv_format = m->plan64.format;
    info->spmv_variant = m->plan64.variant;
    info->spmv_bytes = 0.0;
  }
  return hs.status;
}


// ---------------------------------------------------------------------------
// many independent systems with the aggregation preconditioner
// ---------------------------------------------------------------------------
namespace {

template <typename T>
int batch_cycle_dir(sgpu_matrix m, const int *rowsys, const BSys *sys, cudaStream_t s) {
  Amg &A = *m->amg;
  const int nl = (int)A.lv.size();
  std::vector<Cheb> ch(nl);
  for (int l = 0; l < nl; l++)
    ch[l] = cheb_coeffs(sizeof(T) == 4 ? A.lv[l]->lmax32 : A.lv[l]->lmax64, A.ratio, A.deg);
  std::vector<T *> xcur(nl + 1, nullptr);
  SGPU_TRY(cycle<T>(m, 0, true, ch, xcur, s));
  k_b_dir<T><<<grid_for(m->n), TPB, 0, s>>>((int)m->n, rowsys, sys, m->w.d.p, xcur[0], m->csr.dscale.p, pcg_state(m));
  count_launches(1);
  return SGPU_OK;
}

// the outer FP64 product q = K p with the products p_i q_i
int batch_spmv64(sgpu_matrix m, const double *p, double *q, double *prod, cudaStream_t s) {
  PcgState *st = pcg_state(m);
  OpStorePQ op{p, q, prod};
  if (m->bsr.valid) {
    auto k = k_lv_bsr3<double, 32, OpStorePQ>;
    k<<<resident_grid(k, m->bsr.nb), TPB, 0, s>>>(m->bsr.nb, m->bsr.browptr.p, m->bsr.bcol.p, m->bsr.bval.p, p, op,
                                                  st, m->w.partials.p, m->w.counters.p);
  } else {
    auto k = k_lv_csr<double, 8, OpStorePQ>;
    k<<<resident_grid(k, (m->n + 3) / 4), TPB, 0, s>>>((int)m->n, m->csr.rowptr.p, m->csr.col.p, m->csr.val.p, p, op,
                                                        st, m->w.partials.p, m->w.counters.p);
  }
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

template <typename T>
int batch_solve(sgpu_matrix m, int nsys, const long long *sysptr, const int *rowsys, BSys *sys, double *pff,
                double *prr, double *ppq, int64_t ni, double res, PcgState *hs) {
  cudaStream_t s = m->stream;
  Work &w = m->w;
  Amg &A = *m->amg;
  const int n = (int)m->n;
  const int g = grid_for(n);
  const int gs = grid_for((int64_t)nsys * 32);
  AmgLevel &L0 = *A.lv[0];
  LevelVecs<T> &V = vecs<T>(L0);
  const T c2 = (T)cheb_coeffs(sizeof(T) == 4 ? L0.lmax32 : L0.lmax64, A.ratio, A.deg).c2_first;
  PcgState init{};
  SGPU_TRY(write_st(m, &init));
  // start: x = 0, r = f
  SGPU_CUDA(cudaMemsetAsync(w.x.p, 0, (size_t)n * sizeof(double), s));
  SGPU_CUDA(cudaMemsetAsync(w.p.p, 0, (size_t)n * sizeof(double), s));
  SGPU_CUDA(cudaMemsetAsync(w.d.p, 0, (size_t)n * sizeof(double), s));
  k_b_init_rows<T><<<g, TPB, 0, s>>>(n, w.f.p, w.p.p, w.r.p, m->csr.dscale.p, V.b.p, V.r.p, V.d.p, V.x.p, c2, pff,
                                     prr);
  k_bseg_init<<<gs, TPB, 0, s>>>(nsys, sysptr, pff, prr, sys, res);
  k_bcount<<<1, TPB, 0, s>>>(nsys, sys, pcg_state(m));
  count_launches(3);
  SGPU_TRY(batch_cycle_dir<T>(m, rowsys, sys, s));
  k_bseg_beta<<<gs, TPB, 0, s>>>(nsys, sysptr, A.batch_zr, A.batch_zq, sys);
  count_launches(1);
  // (k_b_dir ran before the first beta: p = S x0, beta = 0 at a start)
  cudaGraph_t graph;
  cudaGraphExec_t exec = nullptr;
  const int64_t before = sgpu_kernel_launches();
  SGPU_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  int rc = SGPU_OK;
  for (int it = 0; it < 8 && rc == SGPU_OK; it++) {
    rc = batch_spmv64(m, w.d.p, w.p.p, ppq, s);
    if (rc != SGPU_OK) break;
    k_bseg_alpha<<<gs, TPB, 0, s>>>(nsys, sysptr, ppq, sys);
    k_b_update<T><<<g, TPB, 0, s>>>(n, rowsys, sys, w.x.p, w.r.p, w.d.p, w.p.p, m->csr.dscale.p, V.b.p, V.r.p, V.d.p,
                                    V.x.p, c2, prr, pcg_state(m));
    k_bseg_rr<<<gs, TPB, 0, s>>>(nsys, sysptr, prr, sys, (long long)ni, res);
    k_bcount<<<1, TPB, 0, s>>>(nsys, sys, pcg_state(m));
    count_launches(4);
    // the new residual's preconditioned direction: cycle, beta, then p
    Amg &Ar = *m->amg;
    const int nl = (int)Ar.lv.size();
    std::vector<Cheb> ch(nl);
    for (int l = 0; l < nl; l++)
      ch[l] = cheb_coeffs(sizeof(T) == 4 ? Ar.lv[l]->lmax32 : Ar.lv[l]->lmax64, Ar.ratio, Ar.deg);
    std::vector<T *> xcur(nl + 1, nullptr);
    rc = cycle<T>(m, 0, true, ch, xcur, s);
    if (rc != SGPU_OK) break;
    k_bseg_beta<<<gs, TPB, 0, s>>>(nsys, sysptr, A.batch_zr, A.batch_zq, sys);
    k_b_dir<T><<<g, TPB, 0, s>>>(n, rowsys, sys, w.d.p, xcur[0], m->csr.dscale.p, pcg_state(m));
    count_launches(2);
  }
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (rc != SGPU_OK) return rc;
  if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  const int64_t nodes = sgpu_kernel_launches() - before;
  count_launches(-nodes);
  for (int64_t it = 0;; it += 8) {
    SGPU_TRY(read_st(m, hs));
    if (hs->done || it > ni + 8) break;
    e = cudaGraphLaunch(exec, s);
    if (e != cudaSuccess) { rc = fail(SGPU_CUDA_ERROR, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e)); break; }
    count_launches(nodes);
  }
  cudaGraphExecDestroy(exec);
  return rc;
}

}  // namespace

int amg_batch_run(sgpu_matrix m, int nsys, const int64_t *sys_rows, double *x, const double *f, int64_t ni,
                  double res, int mode, int64_t *ani, double *ares, int32_t *status, int64_t *iterations,
                  sgpu_solve_info *info) {
  cudaStream_t s = m->stream;
  const int64_t n = m->n;
  std::vector<long long> ptr(nsys + 1, 0);
  for (int k = 0; k < nsys; k++) {
    if (sys_rows[k] <= 0) return fail(SGPU_BAD_INPUT, "every system needs at least one equation");
    ptr[k + 1] = ptr[k] + sys_rows[k];
  }
  if (ptr[nsys] != n) return fail(SGPU_BAD_INPUT, "system sizes do not add up to the matrix size");
  if (!m->csr.diag_positive)
    return fail(SGPU_BAD_INPUT, "the aggregation preconditioner needs a positive diagonal (Jacobi scaling)");
  SGPU_TRY(pcg_prepare(m, false));
  if (!m->plan64.tuned) SGPU_TRY(spmv_autotune(m, 64));
  const bool fp32 = (mode == SGPU_MIXED);
  if (fp32 && !m->plan32.tuned) SGPU_TRY(spmv_autotune(m, 32));
  float setup_ms = 0.f;
  SGPU_TRY(amg_ensure(m, fp32, &setup_ms));
  Amg &A = *m->amg;
  TmpBuf<long long> sysptr(s);
  TmpBuf<int> rowsys(s);
  TmpBuf<BSys> sys(s);
  TmpBuf<double> pff(s), prr(s), ppq(s), pzr(s), pzq(s);
  SGPU_TRY(sysptr.alloc(nsys + 1));
  SGPU_TRY(rowsys.alloc(n));
  SGPU_TRY(sys.alloc(nsys));
  for (TmpBuf<double> *b : {&pff, &prr, &ppq, &pzr, &pzq}) SGPU_TRY(b->alloc(n));
  SGPU_CUDA(cudaMemcpyAsync(sysptr.p, ptr.data(), (nsys + 1) * sizeof(long long), cudaMemcpyHostToDevice, s));
  std::vector<BSys> hsys(nsys);
  for (auto &b : hsys) { memset(&b, 0, sizeof(b)); b.ani = -1; }
  SGPU_CUDA(cudaMemcpyAsync(sys.p, hsys.data(), nsys * sizeof(BSys), cudaMemcpyHostToDevice, s));
  SGPU_CUDA(cudaMemcpyAsync(m->w.f.p, f, n * sizeof(double), cudaMemcpyHostToDevice, s));
  k_b_rowsys<<<grid_for((int64_t)nsys * 32), TPB, 0, s>>>(nsys, sysptr.p, rowsys.p);
  count_launches(1);
  A.batch_zr = pzr.p;
  A.batch_zq = pzq.p;
  SGPU_CUDA(cudaEventRecord(m->ev0, s));
  PcgState hs{};
  int rc = fp32 ? batch_solve<float>(m, nsys, sysptr.p, rowsys.p, sys.p, pff.p, prr.p, ppq.p, ni, res, &hs)
                : batch_solve<double>(m, nsys, sysptr.p, rowsys.p, sys.p, pff.p, prr.p, ppq.p, ni, res, &hs);
  A.batch_zr = A.batch_zq = nullptr;
  SGPU_CUDA(cudaEventRecord(m->ev1, s));
  if (rc != SGPU_OK) return rc;
  SGPU_CUDA(cudaMemcpyAsync(x, m->w.x.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaMemcpyAsync(hsys.data(), sys.p, nsys * sizeof(BSys), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  float solve_ms = 0.f;
  SGPU_CUDA(cudaEventElapsedTime(&solve_ms, m->ev0, m->ev1));
  int first_bad = SGPU_OK;
  long long maxit = 0;
  for (int k = 0; k < nsys; k++) {
    const BSys &b = hsys[k];
    if (status) status[k] = b.status;
    if (iterations) iterations[k] = b.it;
    if (b.status == SGPU_OK && b.done && b.ani >= 0) {
      if (ani) ani[k] = b.ani;
      if (ares) ares[k] = b.ares;
    }
    if (b.status != SGPU_OK && first_bad == SGPU_OK) first_bad = b.status;
    maxit = std::max(maxit, b.it);
  }
  if (info) {
    info->iterations = maxit;
    info->solve_ms = solve_ms;
    info->precond_setup_ms = setup_ms;
    info->precond_levels = (int32_t)A.lv.size() + 1;
    info->precond_coarse_n = A.nc;
  }
  return first_bad;
}

}  // namespace sgpu
