// Jacobi-PCG on a caller-owned device CSR that allocates no device memory.
//
// Some callers of this library cannot allocate GPU memory while they solve:
// a host application that hands the GPU its whole memory pool up front (or
// runs under a custom allocator that owns every device byte), and code that
// must not call cudaMalloc/cudaFree at all because those calls synchronise
// the device and would stall the caller's other streams.  For them this file
// keeps the iteration's work vectors in one file-scope static device array
// of fixed size, created when the library is loaded and held by every GPU
// that loads it until the process exits.  The caller passes the matrix, the
// right-hand side and the solution; nothing else is allocated, by this code
// or by any library it calls (no cudaMalloc, cudaFree, graph, stream or
// event creation).
//
// Limits and sharing:
//  - at most SGPU_NOALLOC_MAX_N equations (131072): the array holds five
//    FP64 vectors of that length plus reduction slots, about 5 MiB;
//  - every call uses the same array, which keeps the last call's contents;
//    the entry point clears what must start at zero (reduction tickets,
//    iteration state) on every call;
//  - calls whose work overlaps on the GPU (two host threads, or two streams
//    of one process, at the same time on the same device) race on the
//    array: serialise them.
//
// Set-up: the array's name in host code is only a host-side stand-in, not a
// device address.  The first call on each device, with that device current,
// asks the runtime for the array's device address (cudaGetSymbolAddress) and
// keeps it; later calls reuse it.
//
// Host waits: every call reads the iteration state back after each chunk of
// iterations (cudaMemcpyAsync + cudaStreamSynchronize), so a call returns
// only when its solve has finished and cannot be recorded into a CUDA graph;
// a call made while its stream is capturing is refused with SGPU_BAD_INPUT
// before anything is enqueued.
//
// Input checks (on the device, before any iteration): every row must satisfy
// 0 <= rowptr[i] <= rowptr[i+1] <= rowptr[n], hold columns in [0, n) and a
// positive diagonal entry; otherwise the call returns SGPU_BAD_INPUT and
// leaves x untouched.  The caller's col/val arrays must hold rowptr[n]
// entries: the checks keep every read inside [0, rowptr[n]).
//
// The iteration is the reference's symcomprow::cg_prec with the diagonal
// preconditioner (GEFEL/scr.cpp:1093-1205): stop on (r.r)/(f.f) < res, and
// *ani = i, *ares = (r.h)/(f.f) written only on convergence.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "sgpu_internal.cuh"

namespace {

constexpr int kTPB = 256;
constexpr int kMaxN = SGPU_NOALLOC_MAX_N;
constexpr int kBlocks = 148 * 4;      // grid of every kernel here
constexpr int kChunk = 16;            // iterations launched between state reads

struct NaState {
  double nory, nom, denom, alpha, beta, rr, ares, res, zero;
  long long it, ni, ani;
  int done, status, ani_set, pad;
};

// byte layout of the scratch array
constexpr size_t kVecBytes = sizeof(double) * (size_t)kMaxN;
constexpr size_t kOffDiag = 0;
constexpr size_t kOffR = kOffDiag + kVecBytes;
constexpr size_t kOffH = kOffR + kVecBytes;
constexpr size_t kOffD = kOffH + kVecBytes;
constexpr size_t kOffP = kOffD + kVecBytes;
constexpr size_t kOffPart = kOffP + kVecBytes;                    // 2 * kBlocks doubles
constexpr size_t kOffState = kOffPart + 2 * kBlocks * sizeof(double);
constexpr size_t kOffTicket = kOffState + 256;                    // 4 unsigned
constexpr size_t kScratchBytes = kOffTicket + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct Scratch {
  double *diag, *r, *h, *d, *p, *part;
  NaState *st;
  unsigned *ticket;
};

Scratch carve(unsigned char *base) {
  Scratch s;
  s.diag = reinterpret_cast<double *>(base + kOffDiag);
  s.r = reinterpret_cast<double *>(base + kOffR);
  s.h = reinterpret_cast<double *>(base + kOffH);
  s.d = reinterpret_cast<double *>(base + kOffD);
  s.p = reinterpret_cast<double *>(base + kOffP);
  s.part = reinterpret_cast<double *>(base + kOffPart);
  s.st = reinterpret_cast<NaState *>(base + kOffState);
  s.ticket = reinterpret_cast<unsigned *>(base + kOffTicket);
  return s;
}

// device address of the scratch array, per device, found once
std::mutex g_mu;
unsigned char *g_addr[64] = {};

int scratch_address(unsigned char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sgpu::fail(SGPU_CUDA_ERROR, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return sgpu::fail(SGPU_BAD_INPUT, "device ordinal beyond 63");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return sgpu::fail(SGPU_CUDA_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_addr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_addr[dev];
  return SGPU_OK;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block sums of NV values; the last block to arrive adds the partials in
// block order and returns true in its thread 0
template <int NV>
__device__ bool grid_sum(double (&v)[NV], double *part, unsigned *ticket, double (&tot)[NV]) {
  __shared__ double sh[NV][kTPB / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q]);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) sh[q][w] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) {
      double t = 0.0;
      for (int k = 0; k < kTPB / 32; k++) t += sh[q][k];
      part[q * gridDim.x + blockIdx.x] = t;
    }
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NV; q++) {
    double t = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) t += __ldcg(part + q * gridDim.x + b);
    tot[q] = t;
  }
  *ticket = 0u;
  return true;
}

// clears the state and the reduction tickets (one thread: nothing else of the
// call runs before it)
__global__ void k_na_clear(Scratch s, long long ni, double res, double zero) {
  NaState z = {};
  z.ni = ni;
  z.res = res;
  z.zero = zero;
  z.ani = -1;
  *s.st = z;
  for (int k = 0; k < 4; k++) s.ticket[k] = 0u;
}

// checks every row and extracts the diagonal; a malformed row stops the call
// with SGPU_BAD_INPUT before any product reads the matrix
__global__ void k_na_setup(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                           const double *__restrict__ val, Scratch s) {
  const int nnz = rowptr[n];
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int b = rowptr[i], e = rowptr[i + 1];
    double dv = 0.0;
    if (b < 0 || e < b || e > nnz) {
      bad = true;
    } else {
      bool seen = false;
      for (int k = b; k < e; k++) {
        const int c = col[k];
        if (c < 0 || c >= n) { bad = true; break; }
        if (c == i && !seen) { dv = val[k]; seen = true; }
      }
      if (!(dv > 0.0)) bad = true;  // missing, zero, negative or NaN diagonal
    }
    s.diag[i] = dv;
  }
  if (bad) {  // every writer stores the same values
    s.st->status = SGPU_BAD_INPUT;
    s.st->done = 1;
  }
}

// y = A v, 16 lanes per row; with DOT, d.p -> alpha (and the breakdown test)
template <bool DOT>
__global__ void k_na_spmv(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                          const double *__restrict__ val, const double *__restrict__ v, double *__restrict__ y,
                          Scratch s) {
  if (s.st->done) return;
  const int lane = threadIdx.x & 31, g = lane >> 4, sub = lane & 15;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double acc = 0.0;
  for (int base = warp * 2; base < n; base += nw * 2) {
    const int i = base + g;
    int b = 0, e = 0;
    if (i < n) { b = rowptr[i]; e = rowptr[i + 1]; }
    double t = 0.0;
    for (int k = b + sub; k < e; k += 16) t += val[k] * v[col[k]];
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o, 16);
    if (sub == 0 && i < n) {
      y[i] = t;
      acc += v[i] * t;
    }
  }
  if (DOT) {
    double a[1] = {acc}, tot[1];
    if (grid_sum<1>(a, s.part, s.ticket + 0, tot)) {
      NaState *st = s.st;
      st->denom = tot[0];
      if (fabs(tot[0]) < st->zero) {  // scr.cpp:1146-1151
        st->ani = st->it;
        st->ares = st->nom;
        st->ani_set = 1;
        if (st->status == 0) st->status = SGPU_BREAKDOWN;  // a zero right-hand side keeps its status
        st->done = 1;
      } else {
        st->alpha = st->nom / tot[0];
      }
    }
  }
}

// r = f - p (p = A x0 when iv, else x = 0 and r = f), h = r/diag, d = h;
// f.f and r.h
__global__ void k_na_start(int n, const double *__restrict__ f, double *__restrict__ x, int iv, Scratch s) {
  if (s.st->done) return;  // malformed input: x stays as the caller left it
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double ri;
    if (iv) {
      ri = f[i] - s.p[i];
    } else {
      ri = f[i];
      x[i] = 0.0;
    }
    const double hi = ri / s.diag[i];
    s.r[i] = ri;
    s.h[i] = hi;
    s.d[i] = hi;
    v[0] += f[i] * f[i];
    v[1] += ri * hi;
  }
  double t[2];
  if (grid_sum<2>(v, s.part, s.ticket + 1, t)) {
    NaState *st = s.st;
    st->nory = t[0];
    st->nom = t[1];
    if (t[0] < st->zero) {  // scr.cpp:1117-1120: reported, the iteration goes on
      st->status = SGPU_ZERO_RHS;
      st->ares = t[0];
      st->ani = 0;
      st->ani_set = 1;
    }
    if (st->ni <= 0) st->done = 1;
  }
}

// x += alpha d; r -= alpha p; h = r/diag; stop test on (r.r)/(f.f)
__global__ void k_na_update(int n, double *__restrict__ x, Scratch s) {
  if (s.st->done) return;
  const double alpha = s.st->alpha;
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += alpha * s.d[i];
    const double ri = s.r[i] - alpha * s.p[i];
    const double hi = ri / s.diag[i];
    s.r[i] = ri;
    s.h[i] = hi;
    v[0] += ri * ri;
    v[1] += ri * hi;
  }
  double t[2];
  if (grid_sum<2>(v, s.part, s.ticket + 2, t)) {
    NaState *st = s.st;
    st->rr = t[0];
    st->beta = t[1] / st->nom;
    st->nom = t[1];
    const long long it = st->it;
    st->it = it + 1;
    if (fabs(t[0] / st->nory) < st->res) {  // scr.cpp:1188
      st->ani = it;
      st->ares = t[1] / st->nory;
      st->ani_set = 1;
      st->done = 1;
    } else if (it + 1 >= st->ni) {
      st->done = 1;
      if (st->status == 0) st->status = SGPU_NOT_CONVERGED;
    }
  }
}

// d = beta d + h
__global__ void k_na_dir(int n, Scratch s) {
  if (s.st->done) return;
  const double beta = s.st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s.d[i] = beta * s.d[i] + s.h[i];
}

}  // namespace

extern "C" SGPU_API int sgpu_csr_pcg_noalloc_d(int32_t n, const int32_t *rowptr_d, const int32_t *col_d,
                                               const double *val_d, const double *f_d, double *x_d, int64_t ni,
                                               double res, double zero, int64_t iv, void *stream, int64_t *ani,
                                               double *ares, int64_t *iterations) {
  if (n <= 0) return sgpu::fail(SGPU_BAD_INPUT, "n must be positive");
  if (n > kMaxN)
    return sgpu::fail(SGPU_BAD_INPUT, "n = " + std::to_string(n) + " exceeds the no-allocation solver's maximum of " +
                                          std::to_string(kMaxN) + " equations");
  if (!rowptr_d || !col_d || !val_d || !f_d || !x_d) return sgpu::fail(SGPU_BAD_INPUT, "null device pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t ce = cudaStreamIsCapturing(st, &cap);
  if (ce != cudaSuccess)
    return sgpu::fail(SGPU_CUDA_ERROR, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(ce));
  if (cap != cudaStreamCaptureStatusNone)
    return sgpu::fail(SGPU_BAD_INPUT,
                      "the no-allocation solver waits on the host between iterations and cannot run under "
                      "stream capture");
  unsigned char *base = nullptr;
  int rc = scratch_address(&base);
  if (rc != SGPU_OK) return rc;
  const Scratch s = carve(base);
  k_na_clear<<<1, 1, 0, st>>>(s, (long long)ni, res, zero);
  k_na_setup<<<kBlocks, kTPB, 0, st>>>(n, rowptr_d, col_d, val_d, s);
  if (iv) k_na_spmv<false><<<kBlocks, kTPB, 0, st>>>(n, rowptr_d, col_d, val_d, x_d, s.p, s);
  k_na_start<<<kBlocks, kTPB, 0, st>>>(n, f_d, x_d, iv != 0, s);
  sgpu::count_launches(iv ? 4 : 3);
  NaState h = {};
  for (;;) {
    for (int k = 0; k < kChunk; k++) {
      k_na_spmv<true><<<kBlocks, kTPB, 0, st>>>(n, rowptr_d, col_d, val_d, s.d, s.p, s);
      k_na_update<<<kBlocks, kTPB, 0, st>>>(n, x_d, s);
      k_na_dir<<<kBlocks, kTPB, 0, st>>>(n, s);
    }
    sgpu::count_launches(3 * kChunk);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, s.st, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return sgpu::fail(SGPU_CUDA_ERROR, std::string("no-allocation PCG: ") + cudaGetErrorString(e));
    if (h.done) break;
  }
  if (iterations) *iterations = h.it;
  if (h.ani_set) {
    if (ani) *ani = h.ani;
    if (ares) *ares = h.ares;
  }
  return h.status;
}
