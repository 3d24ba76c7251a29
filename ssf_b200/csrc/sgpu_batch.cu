// Many independent systems of uneven size: batched Jacobi-PCG over a
// block-diagonal matrix, as one persistent launch (the default) or as a
// graph of segmented launches per iteration.
//
// The uneven batch (hundreds of plane-stress plates of different sizes, each
// its own symcomprow::cg_prec in the reference, GEFEL/scr.cpp:1093) is held
// as ONE block-diagonal CSR whose diagonal blocks are the systems; every
// system keeps its own CG scalars, stopping test and (ani, ares).
//
// Work is cut into segments: a segment is a run of at most S consecutive rows
// of one system.  One CTA handles one segment at a time (grid-stride over the
// segment table); its warps cover the rows.  A segment writes one partial sum;
// the last segment of a system to finish (per-system atomic ticket, no
// waiting) adds the system's partials in segment order (deterministic) and
// updates that system's scalars.  Systems that have converged cost one flag
// read per segment from then on.  S and the lanes per CSR row are picked by a
// short autotuning run on the batch itself.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sgpu_internal.cuh"

using namespace sgpu;

namespace sgpu {
int pcg_prepare(sgpu_matrix m, bool mixed);
}

namespace {

constexpr int TPB = 256;

struct SysState {
  double nory, nom, denom, alpha, beta, rr, ares;
  long long ani, it;
  int done, status, ani_set, pad;
};

struct Seg {
  int sys, row0, row1, idx;  // idx: position of the segment within its system
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][TPB / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) sh[q][w] = v[q];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = warp_sum(lane < TPB / 32 ? sh[q][lane] : 0.0);
  }
}

// writes the segment's partials; returns true in thread 0 of the CTA that
// completes the system, with the system totals in tot
template <int NV>
__device__ bool seg_reduce(double (&v)[NV], const Seg &sg, const int *__restrict__ sys_seg0,
                           const int *__restrict__ sys_nseg, double *partials, int nseg_total,
                           unsigned *tickets, double (&tot)[NV]) {
  block_sum<NV>(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    const int k = sys_seg0[sg.sys] + sg.idx;
#pragma unroll
    for (int q = 0; q < NV; q++) partials[(size_t)q * nseg_total + k] = v[q];
    __threadfence();
    last = (atomicAdd(tickets + sg.sys, 1u) == (unsigned)sys_nseg[sg.sys] - 1u);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return false;
  __threadfence();
  const int k0 = sys_seg0[sg.sys], ns = sys_nseg[sg.sys];
#pragma unroll
  for (int q = 0; q < NV; q++) {
    double s = 0.0;
    for (int k = 0; k < ns; k++) s += __ldcg(partials + (size_t)q * nseg_total + k0 + k);
    tot[q] = s;
  }
  tickets[sg.sys] = 0u;
  return true;
}

// rows of a segment, L lanes per row; returns the row's value in sub-lane 0
template <int L>
__device__ __forceinline__ double row_dot(int i, const int *__restrict__ rowptr, const int *__restrict__ col,
                                          const double *__restrict__ val, const double *__restrict__ x, int sub) {
  double s = 0.0;
  const int b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
#pragma unroll 4
  for (int k = b + sub; k < e; k += L) s += __ldcs(val + k) * __ldg(x + __ldcs(col + k));
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, L);
  return s;
}

// p = A v on the rows of every live segment; with DOT, d.p per system -> alpha
template <int L, bool DOT>
__global__ void __launch_bounds__(TPB) k_bspmv(int nsegs, const Seg *__restrict__ segs, const int *__restrict__ rowptr,
                                               const int *__restrict__ col, const double *__restrict__ val,
                                               const double *__restrict__ v, double *__restrict__ y, SysState *st,
                                               const int *__restrict__ sys_seg0, const int *__restrict__ sys_nseg,
                                               double *partials, unsigned *tickets, double zero) {
  constexpr int GPW = 32 / L;
  const int lane = threadIdx.x & 31, g = lane / L, sub = lane % L, w = threadIdx.x >> 5;
  __shared__ int skip;
  for (int si = blockIdx.x; si < nsegs; si += gridDim.x) {
    const Seg sg = segs[si];
    if (DOT) {  // one read of the flag for the whole CTA
      if (threadIdx.x == 0) skip = st[sg.sys].done;
      __syncthreads();
      const int sk = skip;
      __syncthreads();
      if (sk) continue;
    }
    double acc = 0.0;
    for (int base = sg.row0 + w * GPW; base < sg.row1; base += (TPB / 32) * GPW) {
      const int i = base + g;
      const int ii = i < sg.row1 ? i : sg.row1 - 1;  // every lane shuffles
      const double s = row_dot<L>(ii, rowptr, col, val, v, sub);
      if (sub == 0 && i < sg.row1) {
        y[i] = s;
        acc += v[i] * s;
      }
    }
    if (DOT) {
      double vv[1] = {acc}, tot[1];
      if (seg_reduce<1>(vv, sg, sys_seg0, sys_nseg, partials, nsegs, tickets, tot)) {
        SysState &s = st[sg.sys];
        s.denom = tot[0];
        if (fabs(tot[0]) < zero) {  // scr.cpp:1146-1151
          s.ani = s.it;
          s.ares = s.nom;
          s.ani_set = 1;
          if (s.status == 0) s.status = SGPU_BREAKDOWN;
          s.done = 1;
        } else {
          s.alpha = s.nom / tot[0];
        }
      }
      __syncthreads();
    }
  }
}

// r = f - p; h = r/diag; d = h; per system f.f, r.h
__global__ void __launch_bounds__(TPB) k_binit(int nsegs, const Seg *__restrict__ segs, const double *__restrict__ f,
                                               const double *__restrict__ p, const double *__restrict__ diag,
                                               double *__restrict__ r, double *__restrict__ h, double *__restrict__ d,
                                               SysState *st, const int *__restrict__ sys_seg0,
                                               const int *__restrict__ sys_nseg, double *partials, unsigned *tickets,
                                               double zero, long long ni) {
  for (int si = blockIdx.x; si < nsegs; si += gridDim.x) {
    const Seg sg = segs[si];
    double v[2] = {0.0, 0.0};
    for (int i = sg.row0 + threadIdx.x; i < sg.row1; i += TPB) {
      const double fi = f[i], ri = fi - p[i], hi = ri / diag[i];
      r[i] = ri;
      h[i] = hi;
      d[i] = hi;
      v[0] += fi * fi;
      v[1] += ri * hi;
    }
    double tot[2];
    if (seg_reduce<2>(v, sg, sys_seg0, sys_nseg, partials, nsegs, tickets, tot)) {
      SysState s = {};
      s.nory = tot[0];
      s.nom = tot[1];
      s.ani = -1;
      if (tot[0] < zero) {  // scr.cpp:1117-1120
        s.status = SGPU_ZERO_RHS;
        s.ares = tot[0];
        s.ani = 0;
        s.ani_set = 1;
      }
      if (ni <= 0) s.done = 1;
      st[sg.sys] = s;
    }
    __syncthreads();
  }
}

// x += alpha d; r -= alpha p; h = r/diag; per system r.r, r.h -> beta, stop
__global__ void __launch_bounds__(TPB) k_bupdate(int nsegs, const Seg *__restrict__ segs, double *__restrict__ x,
                                                 double *__restrict__ r, double *__restrict__ h,
                                                 const double *__restrict__ d, const double *__restrict__ p,
                                                 const double *__restrict__ diag, SysState *st,
                                                 const int *__restrict__ sys_seg0, const int *__restrict__ sys_nseg,
                                                 double *partials, unsigned *tickets, double res, long long ni,
                                                 int *live_count) {
  __shared__ int skip;
  __shared__ double alpha_s;
  for (int si = blockIdx.x; si < nsegs; si += gridDim.x) {
    const Seg sg = segs[si];
    if (threadIdx.x == 0) {
      skip = st[sg.sys].done;
      alpha_s = st[sg.sys].alpha;
    }
    __syncthreads();
    const int sk = skip;
    const double alpha = alpha_s;
    __syncthreads();
    if (sk) continue;
    double v[2] = {0.0, 0.0};
    for (int i = sg.row0 + threadIdx.x; i < sg.row1; i += TPB) {
      x[i] += alpha * d[i];
      const double ri = r[i] - alpha * p[i], hi = ri / diag[i];
      r[i] = ri;
      h[i] = hi;
      v[0] += ri * ri;
      v[1] += ri * hi;
    }
    double tot[2];
    if (seg_reduce<2>(v, sg, sys_seg0, sys_nseg, partials, nsegs, tickets, tot)) {
      SysState &s = st[sg.sys];
      s.rr = tot[0];
      s.beta = tot[1] / s.nom;
      s.nom = tot[1];
      const long long it = s.it;
      s.it = it + 1;
      if (fabs(tot[0] / s.nory) < res) {  // scr.cpp:1188
        s.ani = it;
        s.ares = tot[1] / s.nory;
        s.ani_set = 1;
        s.done = 1;
      } else if (it + 1 >= ni) {
        s.done = 1;
        if (s.status == 0) s.status = SGPU_NOT_CONVERGED;
      }
      if (s.done) atomicSub(live_count, 1);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(TPB) k_bdir(int nsegs, const Seg *__restrict__ segs, double *__restrict__ d,
                                              const double *__restrict__ h, const SysState *st) {
  for (int si = blockIdx.x; si < nsegs; si += gridDim.x) {
    const Seg sg = segs[si];
    if (st[sg.sys].done) continue;
    const double beta = st[sg.sys].beta;
    for (int i = sg.row0 + threadIdx.x; i < sg.row1; i += TPB) d[i] = beta * d[i] + h[i];
  }
}

// ---------------------------------------------------------------------------
// the persistent form: one CTA per system at a time
//
// The systems are independent, so a CTA can run a whole system's iteration
// alone -- SpMV, the two reductions, the updates -- separated by CTA
// barriers only: no grid-wide step, no launch per iteration, and a converged
// system costs nothing.  CTAs take systems from a queue (largest first, so
// the longest solves start early) through one atomic counter; the kernel
// ends when the queue is empty.  Nothing waits on another CTA.  Each system's
// sums are formed in a fixed order (thread, then warp, then block), so a
// solve is repeatable bit for bit.
// ---------------------------------------------------------------------------
constexpr int PTPB = 512;

__device__ __forceinline__ void cta_sum2(double &a, double &b, double (*sh)[PTPB / 32]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) {
    sh[0][w] = a;
    sh[1][w] = b;
  }
  __syncthreads();
  double ta = 0.0, tb = 0.0;
  for (int k = 0; k < PTPB / 32; k++) {  // every thread sums the warp totals in order
    ta += sh[0][k];
    tb += sh[1][k];
  }
  a = ta;
  b = tb;
}

template <int L>
__global__ void __launch_bounds__(PTPB, 2) k_bpersist(int nsys, const int *__restrict__ order,
                                                      const long long *__restrict__ sysptr, int *next,
                                                      const int *__restrict__ rowptr, const int *__restrict__ col,
                                                      const double *__restrict__ val, const double *__restrict__ diag,
                                                      const double *__restrict__ f, double *__restrict__ x,
                                                      double *__restrict__ r, double *__restrict__ h,
                                                      double *__restrict__ d, double *__restrict__ p, SysState *st,
                                                      long long ni, double res, double zero) {
  __shared__ double sh[2][PTPB / 32];
  __shared__ int q_s;
  constexpr int GPW = 32 / L;
  const int lane = threadIdx.x & 31, g = lane / L, sub = lane % L, w = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) q_s = atomicAdd(next, 1);
    __syncthreads();
    const int q = q_s;
    __syncthreads();
    if (q >= nsys) return;
    const int k = order[q];
    const int r0 = (int)sysptr[k], r1 = (int)sysptr[k + 1];
    // start from x = 0: r = f, h = r/diag, d = h; f.f and r.h
    double a = 0.0, b = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += PTPB) {
      const double fi = f[i], hi = fi / diag[i];
      x[i] = 0.0;
      r[i] = fi;
      h[i] = hi;
      d[i] = hi;
      a += fi * fi;
      b += fi * hi;
    }
    cta_sum2(a, b, sh);
    SysState s = {};
    s.nory = a;
    s.nom = b;
    s.ani = -1;
    if (a < zero) {  // scr.cpp:1117-1120: reported, the iteration goes on
      s.status = SGPU_ZERO_RHS;
      s.ares = a;
      s.ani = 0;
      s.ani_set = 1;
    }
    if (ni <= 0) s.done = 1;
    while (!s.done) {
      __syncthreads();  // d complete
      // p = A d and d.p
      double dp = 0.0, unused = 0.0;
      for (int base = r0 + w * GPW; base < r1; base += (PTPB / 32) * GPW) {
        const int i = base + g;
        const int ii = i < r1 ? i : r1 - 1;  // every lane shuffles
        const double y = row_dot<L>(ii, rowptr, col, val, d, sub);
        if (sub == 0 && i < r1) {
          p[i] = y;
          dp += d[i] * y;
        }
      }
      cta_sum2(dp, unused, sh);
      s.denom = dp;
      if (fabs(dp) < zero) {  // scr.cpp:1146-1151
        s.ani = s.it;
        s.ares = s.nom;
        s.ani_set = 1;
        if (s.status == 0) s.status = SGPU_BREAKDOWN;
        s.done = 1;
        break;
      }
      const double alpha = s.nom / dp;
      // x += alpha d; r -= alpha p; h = r/diag; r.r and r.h
      double rr = 0.0, rh = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += PTPB) {
        x[i] += alpha * d[i];
        const double ri = r[i] - alpha * p[i], hi = ri / diag[i];
        r[i] = ri;
        h[i] = hi;
        rr += ri * ri;
        rh += ri * hi;
      }
      cta_sum2(rr, rh, sh);
      s.alpha = alpha;
      s.rr = rr;
      s.beta = rh / s.nom;
      s.nom = rh;
      const long long it = s.it;
      s.it = it + 1;
      if (fabs(rr / s.nory) < res) {  // scr.cpp:1188
        s.ani = it;
        s.ares = rh / s.nory;
        s.ani_set = 1;
        s.done = 1;
        break;
      }
      if (it + 1 >= ni) {
        s.done = 1;
        if (s.status == 0) s.status = SGPU_NOT_CONVERGED;
        break;
      }
      const double beta = s.beta;
      for (int i = r0 + threadIdx.x; i < r1; i += PTPB) d[i] = beta * d[i] + h[i];
    }
    if (threadIdx.x == 0) st[k] = s;
    __syncthreads();
  }
}

// the persistent solve of every system; hs gets the per-system results
int run_persistent(sgpu_matrix m, const std::vector<int64_t> &rows, int L, double *x, const double *f, double *r,
                   double *h, double *d, double *p, int64_t ni, double res, double zero, std::vector<SysState> &hs,
                   int64_t *iters, float *ms) {
  cudaStream_t s = m->stream;
  const Csr &c = m->csr;
  const int nsys = (int)rows.size();
  std::vector<long long> ptr(nsys + 1, 0);
  for (int k = 0; k < nsys; k++) ptr[k + 1] = ptr[k] + rows[k];
  std::vector<int> order(nsys);
  for (int k = 0; k < nsys; k++) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rows[a] > rows[b]; });
  DevBuf<long long> ptr_d;
  DevBuf<int> order_d, next_d;
  DevBuf<SysState> st;
  SGPU_TRY(ptr_d.alloc(nsys + 1));
  SGPU_TRY(order_d.alloc(nsys));
  SGPU_TRY(next_d.alloc(1));
  SGPU_TRY(st.alloc(nsys));
  SGPU_CUDA(cudaMemcpyAsync(ptr_d.p, ptr.data(), (nsys + 1) * sizeof(long long), cudaMemcpyHostToDevice, s));
  SGPU_CUDA(cudaMemcpyAsync(order_d.p, order.data(), nsys * sizeof(int), cudaMemcpyHostToDevice, s));
  SGPU_CUDA(cudaMemsetAsync(next_d.p, 0, sizeof(int), s));
  const int grid = std::min(nsys, kNumSMs * 2);
  SGPU_CUDA(cudaEventRecord(m->ev0, s));
  switch (L) {
    case 4:
      k_bpersist<4><<<grid, PTPB, 0, s>>>(nsys, order_d.p, ptr_d.p, next_d.p, c.rowptr.p, c.col.p, c.val.p, c.diag.p,
                                          f, x, r, h, d, p, st.p, (long long)ni, res, zero);
      break;
    case 16:
      k_bpersist<16><<<grid, PTPB, 0, s>>>(nsys, order_d.p, ptr_d.p, next_d.p, c.rowptr.p, c.col.p, c.val.p,
                                           c.diag.p, f, x, r, h, d, p, st.p, (long long)ni, res, zero);
      break;
    default:
      k_bpersist<8><<<grid, PTPB, 0, s>>>(nsys, order_d.p, ptr_d.p, next_d.p, c.rowptr.p, c.col.p, c.val.p, c.diag.p,
                                          f, x, r, h, d, p, st.p, (long long)ni, res, zero);
      break;
  }
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  SGPU_CUDA(cudaEventRecord(m->ev1, s));
  hs.resize(nsys);
  SGPU_CUDA(cudaMemcpyAsync(hs.data(), st.p, nsys * sizeof(SysState), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  if (ms) SGPU_CUDA(cudaEventElapsedTime(ms, m->ev0, m->ev1));
  int64_t mx = 0;
  for (const SysState &q : hs) mx = std::max<int64_t>(mx, q.it);
  if (iters) *iters = mx;
  return SGPU_OK;
}

struct Plan {
  int S = 1024, L = 8;
};

struct Batch {
  int nsys = 0, nsegs = 0;
  DevBuf<Seg> segs;
  DevBuf<int> seg0, nseg;
  DevBuf<SysState> st;
  DevBuf<unsigned> tickets;
  DevBuf<double> partials;
  DevBuf<int> live;
};

int build_segments(const std::vector<int64_t> &sys_rows, int S, Batch &b, cudaStream_t s) {
  std::vector<Seg> segs;
  std::vector<int> seg0, nseg;
  int64_t row = 0;
  for (size_t k = 0; k < sys_rows.size(); k++) {
    const int64_t r0 = row, r1 = row + sys_rows[k];
    seg0.push_back((int)segs.size());
    int idx = 0;
    for (int64_t a = r0; a < r1; a += S) segs.push_back(Seg{(int)k, (int)a, (int)std::min<int64_t>(a + S, r1), idx++});
    nseg.push_back(idx);
    row = r1;
  }
  b.nsys = (int)sys_rows.size();
  b.nsegs = (int)segs.size();
  SGPU_TRY(b.segs.alloc(segs.size()));
  SGPU_TRY(b.seg0.alloc(seg0.size()));
  SGPU_TRY(b.nseg.alloc(nseg.size()));
  SGPU_TRY(b.st.alloc(b.nsys));
  SGPU_TRY(b.tickets.alloc(b.nsys));
  SGPU_TRY(b.partials.alloc((size_t)2 * b.nsegs));
  SGPU_TRY(b.live.alloc(1));
  SGPU_CUDA(cudaMemcpyAsync(b.segs.p, segs.data(), segs.size() * sizeof(Seg), cudaMemcpyHostToDevice, s));
  SGPU_CUDA(cudaMemcpyAsync(b.seg0.p, seg0.data(), seg0.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  SGPU_CUDA(cudaMemcpyAsync(b.nseg.p, nseg.data(), nseg.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  SGPU_CUDA(cudaMemsetAsync(b.tickets.p, 0, b.nsys * sizeof(unsigned), s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  return SGPU_OK;
}

template <bool DOT>
int launch_bspmv(int L, int grid, Batch &b, const Csr &c, const double *v, double *y, cudaStream_t s, double zero) {
  switch (L) {
    case 4: k_bspmv<4, DOT><<<grid, TPB, 0, s>>>(b.nsegs, b.segs.p, c.rowptr.p, c.col.p, c.val.p, v, y, b.st.p, b.seg0.p,
                                                 b.nseg.p, b.partials.p, b.tickets.p, zero); break;
    case 16: k_bspmv<16, DOT><<<grid, TPB, 0, s>>>(b.nsegs, b.segs.p, c.rowptr.p, c.col.p, c.val.p, v, y, b.st.p,
                                                   b.seg0.p, b.nseg.p, b.partials.p, b.tickets.p, zero); break;
    default: k_bspmv<8, DOT><<<grid, TPB, 0, s>>>(b.nsegs, b.segs.p, c.rowptr.p, c.col.p, c.val.p, v, y, b.st.p, b.seg0.p,
                                                  b.nseg.p, b.partials.p, b.tickets.p, zero); break;
  }
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

// one batched solve; x, f device vectors (n); returns per-system results in hs
int run_batch(sgpu_matrix m, Batch &b, const Plan &pl, double *x, const double *f, double *r, double *h, double *d,
              double *p, int64_t ni, double res, double zero, std::vector<SysState> &hs, int64_t *iters,
              float *ms) {
  cudaStream_t s = m->stream;
  const Csr &c = m->csr;
  const int grid = std::min(b.nsegs, kNumSMs * 8);
  SGPU_CUDA(cudaMemsetAsync(b.tickets.p, 0, b.nsys * sizeof(unsigned), s));
  SGPU_CUDA(cudaEventRecord(m->ev0, s));
  SGPU_TRY(launch_bspmv<false>(pl.L, grid, b, c, x, p, s, zero));
  k_binit<<<grid, TPB, 0, s>>>(b.nsegs, b.segs.p, f, p, c.diag.p, r, h, d, b.st.p, b.seg0.p, b.nseg.p, b.partials.p,
                               b.tickets.p, zero, (long long)ni);
  count_launches(1);
  const int nsys = b.nsys;
  SGPU_CUDA(cudaMemcpyAsync(b.live.p, &nsys, sizeof(int), cudaMemcpyHostToDevice, s));
  // a graph of G iterations, relaunched until every system has stopped
  constexpr int G = 16;
  cudaGraph_t gph;
  cudaGraphExec_t exec;
  SGPU_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  for (int k = 0; k < G; k++) {
    launch_bspmv<true>(pl.L, grid, b, c, d, p, s, zero);
    k_bupdate<<<grid, TPB, 0, s>>>(b.nsegs, b.segs.p, x, r, h, d, p, c.diag.p, b.st.p, b.seg0.p, b.nseg.p,
                                   b.partials.p, b.tickets.p, res, (long long)ni, b.live.p);
    k_bdir<<<grid, TPB, 0, s>>>(b.nsegs, b.segs.p, d, h, b.st.p);
  }
  SGPU_CUDA(cudaStreamEndCapture(s, &gph));
  cudaError_t e = cudaGraphInstantiate(&exec, gph, 0);
  cudaGraphDestroy(gph);
  if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  int64_t it = 0;
  int live = nsys;
  int rc = SGPU_OK;
  while (live > 0 && it < ni) {
    e = cudaGraphLaunch(exec, s);
    if (e != cudaSuccess) { rc = fail(SGPU_CUDA_ERROR, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e)); break; }
    count_launches(3 * G);
    it += G;
    e = cudaMemcpyAsync(&live, b.live.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { rc = fail(SGPU_CUDA_ERROR, std::string("batch loop: ") + cudaGetErrorString(e)); break; }
  }
  cudaGraphExecDestroy(exec);
  if (rc != SGPU_OK) return rc;
  SGPU_CUDA(cudaEventRecord(m->ev1, s));
  hs.resize(nsys);
  SGPU_CUDA(cudaMemcpyAsync(hs.data(), b.st.p, nsys * sizeof(SysState), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  if (ms) SGPU_CUDA(cudaEventElapsedTime(ms, m->ev0, m->ev1));
  if (iters) *iters = it;
  return SGPU_OK;
}

}  // namespace

extern "C" SGPU_API int sgpu_matrix_pcg_batch(sgpu_matrix m, int32_t nsys, const int64_t *sys_rows, double *x,
                                              const double *f, int64_t ni, double res, double zero, int32_t tune,
                                              int64_t *ani, double *ares, int32_t *status, int64_t *iterations,
                                              sgpu_solve_info *info) {
  if (!m || !sys_rows || !x || !f) return fail(SGPU_BAD_INPUT, "null argument");
  if (nsys <= 0) return fail(SGPU_BAD_INPUT, "no systems");
  if (!m->csr.diag_positive) return fail(SGPU_BAD_INPUT, "Jacobi preconditioner needs a positive diagonal");
  std::vector<int64_t> rows(sys_rows, sys_rows + nsys);
  int64_t total = 0;
  for (int64_t v : rows) {
    if (v <= 0) return fail(SGPU_BAD_INPUT, "every system needs at least one equation");
    total += v;
  }
  if (total != m->n) return fail(SGPU_BAD_INPUT, "system sizes do not add up to the matrix size");
  if (info) memset(info, 0, sizeof(*info));
  SGPU_TRY(pcg_prepare(m, false));
  cudaStream_t s = m->stream;
  const size_t n = (size_t)m->n;
  Work &w = m->w;
  SGPU_CUDA(cudaMemcpyAsync(w.f.p, f, n * sizeof(double), cudaMemcpyHostToDevice, s));
  // the plan: segment rows S and lanes per row L; tuned on ~32 iterations of
  // this batch when asked (the iterate is reset for the real solve)
  // SGPU_BATCH_FORM=graph: the segmented graph-of-launches form below;
  // otherwise the persistent form (one CTA per system at a time)
  const char *form = getenv("SGPU_BATCH_FORM");
  const bool persistent = !(form && !strcmp(form, "graph"));
  Plan best;
  if (tune && !persistent) {
    float best_ms = 1e30f;
    for (int S : {512, 1024, 2048, 4096})
      for (int L : {4, 8, 16}) {
        Batch b;
        SGPU_TRY(build_segments(rows, S, b, s));
        std::vector<SysState> hs;
        float ms = 0.f;
        int64_t its = 0;
        SGPU_CUDA(cudaMemsetAsync(w.x.p, 0, n * sizeof(double), s));
        SGPU_TRY(run_batch(m, b, Plan{S, L}, w.x.p, w.f.p, w.r.p, w.h.p, w.d.p, w.p.p, 32, res, zero, hs, &its, &ms));
        if (ms < best_ms) { best_ms = ms; best = Plan{S, L}; }
      }
  }
  std::vector<SysState> hs;
  float ms = 0.f;
  int64_t its = 0;
  if (persistent) {
    // lanes per row from the rows' mean length
    const double mean = (double)m->csr.nnz / (double)m->n;
    best.L = mean > 40 ? 16 : (mean > 12 ? 8 : 4);
    best.S = 0;
    SGPU_TRY(run_persistent(m, rows, best.L, w.x.p, w.f.p, w.r.p, w.h.p, w.d.p, w.p.p, ni, res, zero, hs, &its,
                            &ms));
  } else {
    Batch b;
    SGPU_TRY(build_segments(rows, best.S, b, s));
    SGPU_CUDA(cudaMemsetAsync(w.x.p, 0, n * sizeof(double), s));
    SGPU_TRY(run_batch(m, b, best, w.x.p, w.f.p, w.r.p, w.h.p, w.d.p, w.p.p, ni, res, zero, hs, &its, &ms));
  }
  SGPU_CUDA(cudaMemcpyAsync(x, w.x.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  int worst = SGPU_OK;
  for (int k = 0; k < nsys; k++) {
    int st = hs[k].status;
    if (!hs[k].done && st == SGPU_OK) st = SGPU_NOT_CONVERGED;
    if (status) status[k] = st;
    if (iterations) iterations[k] = hs[k].it;
    if (hs[k].ani_set) {
      if (ani) ani[k] = hs[k].ani;
      if (ares) ares[k] = hs[k].ares;
    }
    if (st != SGPU_OK && worst == SGPU_OK) worst = st;
  }
  if (info) {
    info->iterations = its;
    info->solve_ms = ms;
    info->spmv_format = 0;
    info->spmv_variant = best.L;
    info->spmv_bytes = (double)m->csr.nnz * 12.0 + (m->n + 1) * 4.0 + 2.0 * m->n * 8.0;
    info->tile_rows = best.S;
  }
  return worst;
}
