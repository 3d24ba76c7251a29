// Many load cases at once: batched Jacobi-PCG with a sparse matrix times a
// block of vectors (SpMM).
//
// solve_linear_statics (MEFEL/SRC/lssolver.cpp:78-80) solves the nlc load
// cases one after the other, each a full symcomprow::cg_prec.  Here all R
// right-hand sides iterate together: one SpMM per iteration reads the matrix
// once for all of them (the matrix bytes are shared, the vector blocks are
// L2-resident gathers), and every column keeps its own CG scalars, stopping
// test and (ani, ares) exactly as R independent reference solves would.
//
// Layout: the R vectors of one kind are stored row-major (n x RP, RP = R
// rounded up to a multiple of 32), so the R values of one equation are
// contiguous: a warp reading one equation's row of X reads 8*RP consecutive
// bytes.  Host arrays keep the reference's layout (R column blocks of n,
// lhsrhs.cpp:72-74) and are transposed on upload/download.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sgpu_internal.cuh"

using namespace sgpu;

namespace {

constexpr int TPB = 256;

struct ColState {
  double nory, nom, denom, alpha, beta, rr, ares;
  long long ani;
  int done, status, ani_set, pad;
};

// Y = A X on BSR3 (warp per block row; lane owns columns lane, lane+32, ...)
template <int CPL>  // columns per lane: RP = 32 * CPL
__global__ void __launch_bounds__(TPB) k_spmm_bsr3(int nb, const int *__restrict__ browptr,
                                                   const int *__restrict__ bcol, const double *__restrict__ bval,
                                                   const double *__restrict__ X, double *__restrict__ Y) {
  constexpr int RP = 32 * CPL;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int br = warp; br < nb; br += nw) {
    const int s = browptr[br], nbr = browptr[br + 1] - s;
    const double *bv = bval + 9ll * s;
    double y[3][CPL];
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int c = 0; c < CPL; c++) y[q][c] = 0.0;
    for (int j = 0; j < nbr; j++) {
      const int col = __ldg(bcol + s + j);
      double v[9];
#pragma unroll
      for (int q = 0; q < 9; q++) v[q] = __ldg(bv + q * nbr + j);  // same address in every lane
      const double *x0 = X + (size_t)(3 * col) * RP + lane;
#pragma unroll
      for (int c = 0; c < CPL; c++) {
        const double a0 = __ldg(x0 + 32 * c), a1 = __ldg(x0 + RP + 32 * c), a2 = __ldg(x0 + 2 * RP + 32 * c);
        y[0][c] += v[0] * a0 + v[1] * a1 + v[2] * a2;
        y[1][c] += v[3] * a0 + v[4] * a1 + v[5] * a2;
        y[2][c] += v[6] * a0 + v[7] * a1 + v[8] * a2;
      }
    }
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int c = 0; c < CPL; c++) Y[(size_t)(3 * br + q) * RP + lane + 32 * c] = y[q][c];
  }
}

// Y = A X on CSR (warp per row)
template <int CPL>
__global__ void __launch_bounds__(TPB) k_spmm_csr(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                                                  const double *__restrict__ val, const double *__restrict__ X,
                                                  double *__restrict__ Y) {
  constexpr int RP = 32 * CPL;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < n; i += nw) {
    double y[CPL];
#pragma unroll
    for (int c = 0; c < CPL; c++) y[c] = 0.0;
    for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
      const double a = __ldg(val + k);
      const double *x = X + (size_t)__ldg(col + k) * RP + lane;
#pragma unroll
      for (int c = 0; c < CPL; c++) y[c] += a * __ldg(x + 32 * c);
    }
#pragma unroll
    for (int c = 0; c < CPL; c++) Y[(size_t)i * RP + lane + 32 * c] = y[c];
  }
}

// per-column sums over the rows: thread (rg, c) of a block adds rows
// rg, rg + rows_per_step, ...; the block's partial sums go to partials, the
// last block sums them in block order
__device__ bool col_reduce(double *v, int nv, int RP, double *sh, double *partials, unsigned *ticket,
                           double *tot) {
  // v: nv values of this thread's column; sh: nv * TPB doubles
  const int t = threadIdx.x, c = t % RP;
  for (int q = 0; q < nv; q++) sh[q * TPB + t] = v[q];
  __syncthreads();
  __shared__ bool last;
  if (t < RP) {
    for (int q = 0; q < nv; q++) {
      double s = 0.0;
      for (int k = c; k < TPB; k += RP) s += sh[q * TPB + k];
      partials[((size_t)q * gridDim.x + blockIdx.x) * RP + c] = s;
    }
  }
  __threadfence();
  __syncthreads();
  if (t == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return false;
  __threadfence();
  if (t < RP) {
    for (int q = 0; q < nv; q++) {
      double s = 0.0;
      for (int b = 0; b < (int)gridDim.x; b++) s += __ldcg(partials + ((size_t)q * gridDim.x + b) * RP + c);
      tot[q * RP + c] = s;
    }
  }
  __syncthreads();
  if (t == 0) *ticket = 0u;
  return true;
}

// init: R = F - P; H = R/diag; D = H; per column f.f and r.h
__global__ void __launch_bounds__(TPB) k_mpcg_init(int n, int R, int RP, const double *__restrict__ F,
                                                   const double *__restrict__ P, const double *__restrict__ diag,
                                                   double *__restrict__ Rv, double *__restrict__ H,
                                                   double *__restrict__ D, ColState *cs, double *partials,
                                                   unsigned *ticket, double zero, long long ni) {
  __shared__ double sh[2 * TPB];
  __shared__ double tot[2 * 128];
  const int t = threadIdx.x, c = t % RP, rg = t / RP, rps = TPB / RP;
  double v[2] = {0.0, 0.0};
  for (long long i = (long long)blockIdx.x * rps + rg; i < n; i += (long long)gridDim.x * rps) {
    const size_t k = (size_t)i * RP + c;
    const double f = F[k], r = f - P[k], h = r / diag[i];
    Rv[k] = r;
    H[k] = h;
    D[k] = h;
    v[0] += f * f;
    v[1] += r * h;
  }
  if (col_reduce(v, 2, RP, sh, partials, ticket, tot) && t < R) {
    ColState s = {};
    s.nory = tot[c];
    s.nom = tot[RP + c];
    s.ani = -1;
    if (s.nory < zero) {  // scr.cpp:1117-1120
      s.status = SGPU_ZERO_RHS;
      s.ares = s.nory;
      s.ani = 0;
      s.ani_set = 1;
    }
    if (ni <= 0) s.done = 1;
    cs[c] = s;
  }
}

// per column: denom = d.p -> alpha (breakdown test), from the SpMM output P
__global__ void __launch_bounds__(TPB) k_mpcg_alpha(int n, int R, int RP, const double *__restrict__ D,
                                                    const double *__restrict__ P, ColState *cs, double *partials,
                                                    unsigned *ticket, double zero, long long it) {
  __shared__ double sh[TPB];
  __shared__ double tot[128];
  const int t = threadIdx.x, c = t % RP, rg = t / RP, rps = TPB / RP;
  double v[1] = {0.0};
  for (long long i = (long long)blockIdx.x * rps + rg; i < n; i += (long long)gridDim.x * rps) {
    const size_t k = (size_t)i * RP + c;
    v[0] += D[k] * P[k];
  }
  if (col_reduce(v, 1, RP, sh, partials, ticket, tot) && t < R) {
    ColState &s = cs[c];
    if (s.done) return;
    s.denom = tot[c];
    if (fabs(tot[c]) < zero) {  // scr.cpp:1146-1151
      s.ani = it;
      s.ares = s.nom;
      s.ani_set = 1;
      if (s.status == 0) s.status = SGPU_BREAKDOWN;
      s.done = 1;
      s.alpha = 0.0;
    } else {
      s.alpha = s.nom / tot[c];
    }
  }
}

// per column: x += alpha d; r -= alpha p; h = r/diag; r.r, r.h -> beta, stop
__global__ void __launch_bounds__(TPB) k_mpcg_update(int n, int R, int RP, double *__restrict__ X,
                                                     double *__restrict__ Rv, double *__restrict__ H,
                                                     const double *__restrict__ D, const double *__restrict__ P,
                                                     const double *__restrict__ diag, ColState *cs, double *partials,
                                                     unsigned *ticket, double res, long long it, long long ni,
                                                     int *alldone) {
  __shared__ double sh[2 * TPB];
  __shared__ double tot[2 * 128];
  const int t = threadIdx.x, c = t % RP, rg = t / RP, rps = TPB / RP;
  const bool live = c < R && !cs[c].done;
  const double alpha = live ? cs[c].alpha : 0.0;
  double v[2] = {0.0, 0.0};
  for (long long i = (long long)blockIdx.x * rps + rg; i < n; i += (long long)gridDim.x * rps) {
    const size_t k = (size_t)i * RP + c;
    if (live) {
      X[k] += alpha * D[k];
      const double r = Rv[k] - alpha * P[k];
      const double h = r / diag[i];
      Rv[k] = r;
      H[k] = h;
      v[0] += r * r;
      v[1] += r * h;
    }
  }
  if (col_reduce(v, 2, RP, sh, partials, ticket, tot)) {
    if (t < R) {
      ColState &s = cs[c];
      if (!s.done) {
        const double rr = tot[c], nom = tot[RP + c];
        s.rr = rr;
        s.beta = nom / s.nom;
        s.nom = nom;
        if (fabs(rr / s.nory) < res) {  // scr.cpp:1188
          s.ani = it;
          s.ares = nom / s.nory;
          s.ani_set = 1;
          s.done = 1;
        } else if (it + 1 >= ni) {
          s.done = 1;
          if (s.status == 0) s.status = SGPU_NOT_CONVERGED;
        }
      }
    }
    __syncthreads();
    if (t == 0) {
      int all = 1;
      for (int k = 0; k < R; k++) all &= cs[k].done;
      *alldone = all;
    }
  }
}

// per column: d = beta d + h
__global__ void __launch_bounds__(TPB) k_mpcg_dir(int n, int R, int RP, double *__restrict__ D,
                                                  const double *__restrict__ H, const ColState *cs) {
  const int t = threadIdx.x, c = t % RP, rg = t / RP, rps = TPB / RP;
  if (c >= R || cs[c].done) return;
  const double beta = cs[c].beta;
  for (long long i = (long long)blockIdx.x * rps + rg; i < n; i += (long long)gridDim.x * rps) {
    const size_t k = (size_t)i * RP + c;
    D[k] = beta * D[k] + H[k];
  }
}

__global__ void k_pack(int n, int R, int RP, const double *__restrict__ src_cols, double *__restrict__ dst) {
  // src: R column blocks of n (host layout), dst: n x RP row-major, pad = 0
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (size_t)n * RP;
       k += (size_t)gridDim.x * blockDim.x) {
    const size_t i = k / RP;
    const int c = (int)(k % RP);
    dst[k] = c < R ? src_cols[(size_t)c * n + i] : 0.0;
  }
}

__global__ void k_unpack(int n, int R, int RP, const double *__restrict__ src, double *__restrict__ dst_cols) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (size_t)n * R;
       k += (size_t)gridDim.x * blockDim.x) {
    const size_t c = k / n, i = k % n;
    dst_cols[k] = src[i * RP + c];
  }
}

int spmm(sgpu_matrix m, int CPL, const double *X, double *Y, cudaStream_t s) {
  const int grid = kNumSMs * 8;
  if (m->bsr.valid) {
    switch (CPL) {
      case 1: k_spmm_bsr3<1><<<grid, TPB, 0, s>>>(m->bsr.nb, m->bsr.browptr.p, m->bsr.bcol.p, m->bsr.bval.p, X, Y); break;
      case 2: k_spmm_bsr3<2><<<grid, TPB, 0, s>>>(m->bsr.nb, m->bsr.browptr.p, m->bsr.bcol.p, m->bsr.bval.p, X, Y); break;
      default: k_spmm_bsr3<4><<<grid, TPB, 0, s>>>(m->bsr.nb, m->bsr.browptr.p, m->bsr.bcol.p, m->bsr.bval.p, X, Y); break;
    }
  } else {
    const Csr &c = m->csr;
    switch (CPL) {
      case 1: k_spmm_csr<1><<<grid, TPB, 0, s>>>(c.n, c.rowptr.p, c.col.p, c.val.p, X, Y); break;
      case 2: k_spmm_csr<2><<<grid, TPB, 0, s>>>(c.n, c.rowptr.p, c.col.p, c.val.p, X, Y); break;
      default: k_spmm_csr<4><<<grid, TPB, 0, s>>>(c.n, c.rowptr.p, c.col.p, c.val.p, X, Y); break;
    }
  }
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

}  // namespace

extern "C" SGPU_API int sgpu_matrix_pcg_multi(sgpu_matrix m, int32_t nrhs, double *X, const double *F, int64_t ni,
                                              double res, double zero, int64_t iv, int64_t *ani, double *ares,
                                              int32_t *status, sgpu_solve_info *info) {
  if (!m || !X || !F) return fail(SGPU_BAD_INPUT, "null argument");
  if (nrhs <= 0 || nrhs > 128) return fail(SGPU_BAD_INPUT, "nrhs must be 1..128");
  if (!m->csr.diag_positive) return fail(SGPU_BAD_INPUT, "Jacobi preconditioner needs a positive diagonal");
  if (info) memset(info, 0, sizeof(*info));
  SGPU_TRY(ensure_bsr3(m));
  // columns per lane 1, 2 or 4: RP divides the 256 threads of a block
  const int n = (int)m->n, R = nrhs, CPL = R <= 32 ? 1 : (R <= 64 ? 2 : 4), RP = 32 * CPL;
  cudaStream_t s = m->stream;
  DevBuf<double> Xd, Fd, Pd, Rd, Hd, Dd, part, hostcols;
  DevBuf<ColState> cs;
  DevBuf<unsigned> tk;
  DevBuf<int> alldone;
  const size_t nn = (size_t)n * RP;
  const int vgrid = kNumSMs * 4;
  SGPU_TRY(Xd.alloc(nn));
  SGPU_TRY(Fd.alloc(nn));
  SGPU_TRY(Pd.alloc(nn));
  SGPU_TRY(Rd.alloc(nn));
  SGPU_TRY(Hd.alloc(nn));
  SGPU_TRY(Dd.alloc(nn));
  SGPU_TRY(part.alloc((size_t)2 * vgrid * RP));
  SGPU_TRY(hostcols.alloc((size_t)n * R));
  SGPU_TRY(cs.alloc(RP));
  SGPU_TRY(tk.alloc(4));
  SGPU_TRY(alldone.alloc(1));
  SGPU_CUDA(cudaMemsetAsync(tk.p, 0, 4 * sizeof(unsigned), s));
  SGPU_CUDA(cudaMemsetAsync(cs.p, 0, RP * sizeof(ColState), s));
  SGPU_CUDA(cudaEventRecord(m->ev0, s));
  // upload (host column blocks -> row-major blocks)
  SGPU_CUDA(cudaMemcpyAsync(hostcols.p, F, (size_t)n * R * sizeof(double), cudaMemcpyHostToDevice, s));
  k_pack<<<kNumSMs * 8, TPB, 0, s>>>(n, R, RP, hostcols.p, Fd.p);
  if (iv) {
    SGPU_CUDA(cudaMemcpyAsync(hostcols.p, X, (size_t)n * R * sizeof(double), cudaMemcpyHostToDevice, s));
    k_pack<<<kNumSMs * 8, TPB, 0, s>>>(n, R, RP, hostcols.p, Xd.p);
  } else {
    SGPU_CUDA(cudaMemsetAsync(Xd.p, 0, nn * sizeof(double), s));
  }
  count_launches(iv ? 2 : 1);
  SGPU_TRY(spmm(m, CPL, Xd.p, Pd.p, s));
  k_mpcg_init<<<vgrid, TPB, 0, s>>>(n, R, RP, Fd.p, Pd.p, m->csr.diag.p, Rd.p, Hd.p, Dd.p, cs.p, part.p, tk.p, zero,
                                    (long long)ni);
  count_launches(1);
  int64_t it = 0;
  int done = 0;
  while (it < ni && !done) {
    const int64_t chunk_end = std::min<int64_t>(it + 16, ni);
    for (; it < chunk_end; it++) {
      SGPU_TRY(spmm(m, CPL, Dd.p, Pd.p, s));
      k_mpcg_alpha<<<vgrid, TPB, 0, s>>>(n, R, RP, Dd.p, Pd.p, cs.p, part.p, tk.p + 1, zero, (long long)it);
      k_mpcg_update<<<vgrid, TPB, 0, s>>>(n, R, RP, Xd.p, Rd.p, Hd.p, Dd.p, Pd.p, m->csr.diag.p, cs.p, part.p,
                                          tk.p + 2, res, (long long)it, (long long)ni, alldone.p);
      k_mpcg_dir<<<vgrid, TPB, 0, s>>>(n, R, RP, Dd.p, Hd.p, cs.p);
      count_launches(3);
    }
    SGPU_CUDA(cudaMemcpyAsync(&done, alldone.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SGPU_CUDA(cudaStreamSynchronize(s));
  }
  SGPU_CUDA(cudaEventRecord(m->ev1, s));
  k_unpack<<<kNumSMs * 8, TPB, 0, s>>>(n, R, RP, Xd.p, hostcols.p);
  count_launches(1);
  SGPU_CUDA(cudaMemcpyAsync(X, hostcols.p, (size_t)n * R * sizeof(double), cudaMemcpyDeviceToHost, s));
  std::vector<ColState> h(RP);
  SGPU_CUDA(cudaMemcpyAsync(h.data(), cs.p, RP * sizeof(ColState), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  SGPU_CUDA(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
  int worst = SGPU_OK;
  for (int c = 0; c < R; c++) {
    int st = h[c].status;
    if (!h[c].done && st == SGPU_OK) st = SGPU_NOT_CONVERGED;
    if (status) status[c] = st;
    if (h[c].ani_set) {
      if (ani) ani[c] = h[c].ani;
      if (ares) ares[c] = h[c].ares;
    }
    if (st != SGPU_OK && worst == SGPU_OK) worst = st;
  }
  if (info) {
    info->iterations = it;
    info->solve_ms = ms;
    info->spmv_format = m->bsr.valid ? 3 : 0;
    info->spmv_bytes = m->bsr.valid ? (double)m->bsr.nblk * 76.0 + 2.0 * nn * 8.0
                                    : (double)m->csr.nnz * 12.0 + 2.0 * nn * 8.0;
  }
  return worst;
}
