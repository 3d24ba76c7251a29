// Device matrix handles: GEFEL CR/SCR storage -> full CSR (int32 indices),
// the FP32 Jacobi-scaled copy and the 3x3 block-row form.
//
// The reference keeps its matrix in `comprow` (GEFEL/cr.h:96-109) or
// `symcomprow` (GEFEL/scr.h:83-96).  The GPU iterates on the full CSR (or on
// its BSR3 refinement) because the lower-triangle-only SpMV of mxv_scr
// (GEFEL/scr.cpp:655-672) scatters into other rows, which on a GPU needs
// atomics; storing both halves costs 2x the value bytes but keeps every row
// a pure gather.
#include <cub/cub.cuh>

#include "sgpu_internal.cuh"

namespace sgpu {

namespace {

constexpr int TPB = 256;

inline int blocks_for(int64_t n, int tpb = TPB) {
  int64_t b = (n + tpb - 1) / tpb;
  return (int)(b < 1 ? 1 : (b > 1048576 ? 1048576 : b));
}

// -- validation of the source storage --------------------------------------
// err bits: 1 adr not monotone / adr[0] != 0 / a row outside [0, negm),
// 2 column out of range, 4 columns not strictly increasing, 8 SCR row does
// not end on its diagonal, 16 CR row has no diagonal.  A row whose bounds
// fail (bit 1) is not read, so every read stays inside the negm entries.
__global__ void k_validate(int64_t n, int64_t negm, const int64_t *__restrict__ adr, const int64_t *__restrict__ ci,
                           int sym, unsigned *err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t b = adr[i], e = adr[i + 1];
    unsigned bad = 0;
    if (b < 0 || e < b || e > negm || (i == 0 && b != 0)) bad |= 1;
    if (!(bad & 1)) {
      bool has_diag = false;
      for (int64_t k = b; k < e; k++) {
        int64_t c = ci[k];
        if (c < 0 || c >= n || (sym && c > i)) bad |= 2;
        if (k > b && ci[k - 1] >= c) bad |= 4;
        if (c == i) has_diag = true;
      }
      if (sym && (e == b || ci[e - 1] != i)) bad |= 8;
      if (!sym && !has_diag) bad |= 16;
    }
    if (bad) atomicOr(err, bad);
  }
}

// upper-part counts: number of off-diagonal SCR entries in each column
__global__ void k_count_upper(int64_t negm, const int64_t *__restrict__ ci, const int *__restrict__ row_of,
                              int *__restrict__ upcnt) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < negm;
       k += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)ci[k];
    if (c != row_of[k]) atomicAdd(&upcnt[c], 1);
  }
}

__global__ void k_row_of(int64_t n, const int64_t *__restrict__ adr, int *__restrict__ row_of) {
  // one warp per row writes the row id of each of its entries
  int lane = threadIdx.x & 31;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    for (int64_t k = adr[i] + lane; k < adr[i + 1]; k += 32) row_of[k] = (int)i;
  }
}

__global__ void k_full_len(int64_t n, const int64_t *__restrict__ adr, const int *__restrict__ upcnt,
                           int *__restrict__ len, int sym) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    len[i] = (int)(adr[i + 1] - adr[i]) + (sym ? upcnt[i] : 0);
}

// lower part (and the diagonal) of every SCR row lands at the start of the
// full row; a CR row is copied as is
__global__ void k_fill_lower(int64_t n, const int64_t *__restrict__ adr, const int64_t *__restrict__ ci,
                             const int *__restrict__ rowptr, int *__restrict__ col, int *__restrict__ map_lo) {
  int lane = threadIdx.x & 31;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    int64_t b = adr[i], e = adr[i + 1];
    int base = rowptr[i];
    for (int64_t k = b + lane; k < e; k += 32) {
      int pos = base + (int)(k - b);
      col[pos] = (int)ci[k];
      map_lo[k] = pos;
    }
  }
}

// off-diagonal SCR entries sorted (stably) by column: the s-th entry of
// column c is the (s - colstart[c])-th transposed entry of full row c, placed
// after that row's lower part; rows ascend within a column because the sort
// is stable and the input is row-major.
__global__ void k_fill_upper(int64_t m, const int *__restrict__ sorted_col, const int *__restrict__ sorted_k,
                             const int *__restrict__ colstart, const int64_t *__restrict__ adr,
                             const int *__restrict__ rowptr, const int *__restrict__ row_of,
                             int *__restrict__ col, int *__restrict__ map_up) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < m;
       s += (int64_t)gridDim.x * blockDim.x) {
    int c = sorted_col[s];
    int k = sorted_k[s];
    int rank = (int)(s - colstart[c]);
    int pos = rowptr[c] + (int)(adr[c + 1] - adr[c]) + rank;
    col[pos] = row_of[k];
    map_up[k] = pos;
  }
}

// sort keys for the transpose: the column of an off-diagonal entry, or
// INT_MAX for a diagonal entry so that all diagonals sort behind
__global__ void k_offdiag_keys(int64_t negm, const int64_t *__restrict__ ci, const int *__restrict__ row_of,
                               int *__restrict__ key, int *__restrict__ idx) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < negm;
       k += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)ci[k];
    key[k] = (c == row_of[k]) ? 0x7fffffff : c;
    idx[k] = (int)k;
  }
}

__global__ void k_scatter_values(int64_t negm, const double *__restrict__ a, const int *__restrict__ map_lo,
                                 const int *__restrict__ map_up, double *__restrict__ val, int sym) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < negm;
       k += (int64_t)gridDim.x * blockDim.x) {
    double v = a[k];
    val[map_lo[k]] = v;
    if (sym) {
      int u = map_up[k];
      if (u >= 0) val[u] = v;
    }
  }
}

__global__ void k_extract_diag(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                               const double *__restrict__ val, double *__restrict__ diag,
                               unsigned *err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    // binary search for the diagonal in the sorted row
    int lo = rowptr[i], hi = rowptr[i + 1] - 1;
    double d = 0.0;
    while (lo <= hi) {
      int mid = (lo + hi) >> 1;
      int c = col[mid];
      if (c == i) { d = val[mid]; break; }
      if (c < i) lo = mid + 1; else hi = mid - 1;
    }
    diag[i] = d;
    if (!(d > 0.0)) atomicOr(err, 32u);
  }
}

__global__ void k_scale32(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                          const double *__restrict__ val, const double *__restrict__ diag,
                          float *__restrict__ val32, double *__restrict__ dscale) {
  int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
    double si = 1.0 / sqrt(diag[i]);
    if (lane == 0) dscale[i] = si;
    for (int k = rowptr[i] + lane; k < rowptr[i + 1]; k += 32) {
      double sj = 1.0 / sqrt(diag[col[k]]);
      val32[k] = (float)(val[k] * si * sj);
    }
  }
}

// -- BSR3 detection and fill -------------------------------------------------
// block row b is valid if rows 3b..3b+2 have the same length and columns, and
// the columns are complete aligned triples
__global__ void k_bsr3_check(int nb, const int *__restrict__ rowptr, const int *__restrict__ col,
                             int *__restrict__ blen, unsigned *err) {
  int lane = threadIdx.x & 31;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += (gridDim.x * blockDim.x) >> 5) {
    int r0 = rowptr[3 * b], r1 = rowptr[3 * b + 1], r2 = rowptr[3 * b + 2], r3 = rowptr[3 * b + 3];
    int len = r1 - r0;
    bool ok = (r2 - r1 == len) && (r3 - r2 == len) && (len % 3 == 0);
    if (ok) {
      for (int k = lane; k < len; k += 32) {
        int c0 = col[r0 + k];
        if (col[r1 + k] != c0 || col[r2 + k] != c0) ok = false;
        int t = k % 3;
        if (c0 % 3 != t) ok = false;
        if (t > 0 && col[r0 + k - 1] != c0 - 1) ok = false;
      }
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
      blen[b] = ok ? len / 3 : 0;
      if (!ok) atomicOr(err, 1u);
    }
  }
}

// bval layout per block row: component-major, i.e. for block row b with
// blocks [s, e): bval[9*s + comp*(e-s) + j] holds component comp (row-major
// inside the 3x3 block) of block s+j; lanes of a warp reading component comp
// of consecutive blocks touch consecutive addresses
__global__ void k_bsr3_fill(int nb, const int *__restrict__ rowptr, const int *__restrict__ col,
                            const int *__restrict__ browptr, int *__restrict__ bcol,
                            int64_t *__restrict__ csr2bsr) {
  int lane = threadIdx.x & 31;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += (gridDim.x * blockDim.x) >> 5) {
    int s = browptr[b], e = browptr[b + 1], nbr = e - s;
    for (int r = 0; r < 3; r++) {
      int rs = rowptr[3 * b + r];
      for (int k = lane; k < 3 * nbr; k += 32) {
        int j = k / 3, cc = k % 3;
        if (r == 0 && cc == 0) bcol[s + j] = col[rs + k] / 3;
        int comp = 3 * r + cc;
        csr2bsr[rs + k] = 9LL * s + (int64_t)comp * nbr + j;
      }
    }
  }
}

__global__ void k_bsr3_values(int64_t nnz, const double *__restrict__ val, const int64_t *__restrict__ csr2bsr,
                              double *__restrict__ bval) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz;
       k += (int64_t)gridDim.x * blockDim.x)
    bval[csr2bsr[k]] = val[k];
}

__global__ void k_bsr3_values32(int64_t nnz, const float *__restrict__ val32, const int64_t *__restrict__ csr2bsr,
                                float *__restrict__ bval32) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz;
       k += (int64_t)gridDim.x * blockDim.x)
    bval32[csr2bsr[k]] = val32[k];
}

int read_err(const unsigned *err_d, cudaStream_t s, unsigned *out) {
  SGPU_CUDA(cudaMemcpyAsync(out, err_d, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  return SGPU_OK;
}

}  // namespace

// Build the full CSR of a handle from its (device) source pattern; values are
// filled by matrix_set_values_device.
int matrix_build_from_device_src(sgpu_matrix m) {
  cudaStream_t s = m->stream;
  const int64_t n = m->n, negm = m->src_negm;
  const int sym = m->src_sym;
  if (n <= 0 || n >= (1LL << 31) - 1) return fail(SGPU_BAD_INPUT, "n out of range for int32 device indices");
  DevBuf<unsigned> err;
  SGPU_TRY(err.alloc(1));
  SGPU_CUDA(cudaMemsetAsync(err.p, 0, sizeof(unsigned), s));
  k_validate<<<blocks_for(n), TPB, 0, s>>>(n, negm, m->src_adr.p, m->src_ci.p, sym, err.p);
  count_launches(1);
  unsigned e = 0;
  SGPU_TRY(read_err(err.p, s, &e));
  if (e) return fail(SGPU_BAD_INPUT, "malformed storage arrays (validation bits " + std::to_string(e) + ")");
  int64_t negm_chk = 0;
  SGPU_CUDA(cudaMemcpy(&negm_chk, m->src_adr.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost));
  if (negm_chk != negm) return fail(SGPU_BAD_INPUT, "adr[n] != number of entries");

  DevBuf<int> row_of, upcnt, len;
  SGPU_TRY(row_of.alloc(negm));
  SGPU_TRY(upcnt.alloc(n));
  SGPU_TRY(len.alloc(n));
  SGPU_CUDA(cudaMemsetAsync(upcnt.p, 0, n * sizeof(int), s));
  k_row_of<<<blocks_for(n * 32), TPB, 0, s>>>(n, m->src_adr.p, row_of.p);
  if (sym) k_count_upper<<<blocks_for(negm), TPB, 0, s>>>(negm, m->src_ci.p, row_of.p, upcnt.p);
  k_full_len<<<blocks_for(n), TPB, 0, s>>>(n, m->src_adr.p, upcnt.p, len.p, sym);
  count_launches(sym ? 3 : 2);

  Csr &c = m->csr;
  c.n = (int)n;
  SGPU_TRY(c.rowptr.alloc(n + 1));
  // rowptr = exclusive scan of len (n+1 entries: scan over len with a trailing 0)
  {
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, len.p, c.rowptr.p, (int)n, s);
    DevBuf<unsigned char> t;
    SGPU_TRY(t.alloc(tmp));
    cub::DeviceScan::ExclusiveSum(t.p, tmp, len.p, c.rowptr.p, (int)n, s);
    count_launches(2);
  }
  int last_ptr = 0, last_len = 0;
  SGPU_CUDA(cudaMemcpyAsync(&last_ptr, c.rowptr.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaMemcpyAsync(&last_len, len.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  int64_t nnz = (int64_t)last_ptr + last_len;
  if (nnz >= (1LL << 31) - 1) return fail(SGPU_BAD_INPUT, "matrix too large for int32 device indices");
  const int nnz32 = (int)nnz;
  SGPU_CUDA(cudaMemcpy(c.rowptr.p + n, &nnz32, sizeof(int), cudaMemcpyHostToDevice));
  c.nnz = nnz;
  SGPU_TRY(c.col.alloc(nnz));
  SGPU_TRY(c.val.alloc(nnz));
  SGPU_TRY(c.diag.alloc(n));
  SGPU_TRY(m->map_lo.alloc(negm));
  SGPU_TRY(m->map_up.alloc(negm));
  SGPU_CUDA(cudaMemsetAsync(m->map_up.p, 0xff, negm * sizeof(int), s));

  k_fill_lower<<<blocks_for(n * 32), TPB, 0, s>>>(n, m->src_adr.p, m->src_ci.p, c.rowptr.p, c.col.p,
                                                  m->map_lo.p);
  count_launches(1);
  if (sym) {
    DevBuf<int> key, idx, skey, sidx, colstart;
    SGPU_TRY(key.alloc(negm));
    SGPU_TRY(idx.alloc(negm));
    SGPU_TRY(skey.alloc(negm));
    SGPU_TRY(sidx.alloc(negm));
    SGPU_TRY(colstart.alloc(n));
    k_offdiag_keys<<<blocks_for(negm), TPB, 0, s>>>(negm, m->src_ci.p, row_of.p, key.p, idx.p);
    size_t tmp = 0;
    const int end_bit = 31;  // keys are non-negative int32
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, skey.p, idx.p, sidx.p, (int)negm, 0, end_bit, s);
    DevBuf<unsigned char> t;
    SGPU_TRY(t.alloc(tmp));
    cub::DeviceRadixSort::SortPairs(t.p, tmp, key.p, skey.p, idx.p, sidx.p, (int)negm, 0, end_bit, s);
    size_t tmp2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp2, upcnt.p, colstart.p, (int)n, s);
    DevBuf<unsigned char> t2;
    SGPU_TRY(t2.alloc(tmp2));
    cub::DeviceScan::ExclusiveSum(t2.p, tmp2, upcnt.p, colstart.p, (int)n, s);
    int64_t m_off = negm - n;  // every SCR row holds exactly one diagonal
    k_fill_upper<<<blocks_for(m_off), TPB, 0, s>>>(m_off, skey.p, sidx.p, colstart.p, m->src_adr.p,
                                                   c.rowptr.p, row_of.p, c.col.p, m->map_up.p);
    count_launches(6);
    SGPU_CUDA(cudaStreamSynchronize(s));
  }
  m->bsr.valid = false;
  m->bsr.nb = -1;  // not yet examined
  m->sell.examined = false;
  m->sell.valid = false;
  m->plan64 = SpmvPlan{};
  m->plan32 = SpmvPlan{};
  return SGPU_OK;
}

int matrix_set_values_device(sgpu_matrix m, const double *a_d) {
  cudaStream_t s = m->stream;
  Csr &c = m->csr;
  k_scatter_values<<<blocks_for(m->src_negm), TPB, 0, s>>>(m->src_negm, a_d, m->map_lo.p, m->map_up.p,
                                                          c.val.p, m->src_sym);
  count_launches(1);
  return finish_values(m);
}

__global__ void k_sell_values(int64_t nnz, const double *__restrict__ val, const int *__restrict__ csr2sell,
                              double *__restrict__ sval);

// After c.val changed: the diagonal, and the derived formats marked stale.
int finish_values(sgpu_matrix m) {
  cudaStream_t s = m->stream;
  Csr &c = m->csr;
  DevBuf<unsigned> err;
  SGPU_TRY(err.alloc(1));
  SGPU_CUDA(cudaMemsetAsync(err.p, 0, sizeof(unsigned), s));
  k_extract_diag<<<blocks_for(c.n), TPB, 0, s>>>(c.n, c.rowptr.p, c.col.p, c.val.p, c.diag.p, err.p);
  count_launches(1);
  unsigned e = 0;
  SGPU_TRY(read_err(err.p, s, &e));
  c.have32 = false;
  m->bsr.have32 = false;
  if (m->bsr.valid) {
    k_bsr3_values<<<blocks_for(c.nnz), TPB, 0, s>>>(c.nnz, c.val.p, m->bsr.csr2bsr.p, m->bsr.bval.p);
    count_launches(1);
  }
  if (m->sell.valid) {
    k_sell_values<<<blocks_for(c.nnz), TPB, 0, s>>>(c.nnz, c.val.p, m->sell.csr2sell.p, m->sell.sval.p);
    count_launches(1);
  }
  // a non-positive diagonal is kept (the FP64 CG without preconditioner can
  // still run); Jacobi and the scaled FP32 form refuse it later
  c.diag_positive = (e == 0);
  m->values_dirty32 = true;
  amg_values_changed(m);
  return SGPU_OK;
}

int ensure_fp32(sgpu_matrix m) {
  Csr &c = m->csr;
  if (c.have32) return SGPU_OK;
  cudaStream_t s = m->stream;
  SGPU_TRY(c.val32s.alloc(c.nnz));
  SGPU_TRY(c.dscale.alloc(c.n));
  k_scale32<<<blocks_for((int64_t)c.n * 32), TPB, 0, s>>>(c.n, c.rowptr.p, c.col.p, c.val.p, c.diag.p,
                                                          c.val32s.p, c.dscale.p);
  count_launches(1);
  c.have32 = true;
  if (m->bsr.valid) {
    SGPU_TRY(m->bsr.bval32s.alloc(m->bsr.nblk * 9 + 4));
    k_bsr3_values32<<<blocks_for(c.nnz), TPB, 0, s>>>(c.nnz, c.val32s.p, m->bsr.csr2bsr.p, m->bsr.bval32s.p);
    count_launches(1);
    m->bsr.have32 = true;
  }
  return SGPU_OK;
}

// ---------------------------------------------------------------------------
// sliced ELL
// ---------------------------------------------------------------------------
__global__ void k_sell_width(int n, int nslices, const int *__restrict__ rowptr, int64_t *__restrict__ width) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nslices; q += gridDim.x * blockDim.x) {
    int w = 0;
    for (int l = 0; l < 32; l++) {
      const int i = 32 * q + l;
      if (i < n) w = max(w, rowptr[i + 1] - rowptr[i]);
    }
    width[q] = 32ll * w;
  }
}

__global__ void k_sell_fill(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                            const int64_t *__restrict__ sptr, int *__restrict__ scol, double *__restrict__ sval,
                            int *__restrict__ csr2sell) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int q = i >> 5, l = i & 31;
    const int64_t base = sptr[q];
    const int w = (int)((sptr[q + 1] - base) >> 5);
    const int b = rowptr[i], len = rowptr[i + 1] - b;
    for (int k = 0; k < w; k++) {
      const int64_t pos = base + 32ll * k + l;
      if (k < len) {
        scol[pos] = col[b + k];
        csr2sell[b + k] = (int)pos;
      } else {
        scol[pos] = i;
        sval[pos] = 0.0;
      }
    }
  }
}

// the lanes past n in the last slice: padding too
__global__ void k_sell_tail(int n, int nslices, const int64_t *__restrict__ sptr, int *__restrict__ scol,
                            double *__restrict__ sval) {
  const int q = nslices - 1;
  const int w = (int)((sptr[q + 1] - sptr[q]) >> 5);
  for (int t = threadIdx.x; t < 32 * w; t += blockDim.x) {
    const int k = t >> 5, l = t & 31;
    if (32 * q + l >= n) {
      scol[sptr[q] + 32ll * k + l] = 0;
      sval[sptr[q] + 32ll * k + l] = 0.0;
    }
  }
}

__global__ void k_sell_values(int64_t nnz, const double *__restrict__ val, const int *__restrict__ csr2sell,
                              double *__restrict__ sval) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
    sval[csr2sell[k]] = val[k];
}

// Drops the sliced ELL copy; a later ensure_sell builds it again.
void release_sell(sgpu_matrix m) {
  Sell &e = m->sell;
  e.sptr.release();
  e.scol.release();
  e.sval.release();
  e.csr2sell.release();
  e.valid = false;
  e.examined = false;
  e.nslices = 0;
  e.nent = 0;
}

int ensure_sell(sgpu_matrix m) {
  Sell &e = m->sell;
  if (e.examined) return SGPU_OK;
  e.examined = true;
  e.valid = false;
  const Csr &c = m->csr;
  cudaStream_t s = m->stream;
  const int n = c.n, nslices = (n + 31) / 32;
  if (n <= 0) return SGPU_OK;
  DevBuf<int64_t> width;
  SGPU_TRY(width.alloc((size_t)nslices + 1));
  SGPU_CUDA(cudaMemsetAsync(width.p + nslices, 0, sizeof(int64_t), s));
  k_sell_width<<<blocks_for(nslices), TPB, 0, s>>>(n, nslices, c.rowptr.p, width.p);
  count_launches(1);
  SGPU_TRY(e.sptr.alloc((size_t)nslices + 1));
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, width.p, e.sptr.p, nslices + 1, s);
  DevBuf<unsigned char> t;
  SGPU_TRY(t.alloc(tmp));
  cub::DeviceScan::ExclusiveSum(t.p, tmp, width.p, e.sptr.p, nslices + 1, s);
  count_launches(1);
  int64_t nent = 0;
  SGPU_CUDA(cudaMemcpyAsync(&nent, e.sptr.p + nslices, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  // worth it only for rows of similar length: at most a quarter of padding
  if (nent >= (int64_t)INT32_MAX || (double)nent > 1.25 * (double)c.nnz) {
    e.sptr.release();
    return SGPU_OK;
  }
  e.nslices = nslices;
  e.nent = nent;
  SGPU_TRY(e.scol.alloc(nent));
  SGPU_TRY(e.sval.alloc(nent));
  SGPU_TRY(e.csr2sell.alloc(c.nnz));
  k_sell_fill<<<blocks_for(n), TPB, 0, s>>>(n, c.rowptr.p, c.col.p, e.sptr.p, e.scol.p, e.sval.p, e.csr2sell.p);
  k_sell_tail<<<1, TPB, 0, s>>>(n, nslices, e.sptr.p, e.scol.p, e.sval.p);
  k_sell_values<<<blocks_for(c.nnz), TPB, 0, s>>>(c.nnz, c.val.p, e.csr2sell.p, e.sval.p);
  count_launches(3);
  SGPU_CUDA(cudaGetLastError());
  SGPU_CUDA(cudaStreamSynchronize(s));
  e.valid = true;
  return SGPU_OK;
}

int ensure_bsr3(sgpu_matrix m) {
  Bsr3 &b = m->bsr;
  if (b.nb >= 0) return SGPU_OK;  // already examined
  Csr &c = m->csr;
  cudaStream_t s = m->stream;
  b.valid = false;
  b.nb = 0;
  if (c.n % 3 != 0) return SGPU_OK;
  int nb = c.n / 3;
  DevBuf<int> blen;
  DevBuf<unsigned> err;
  SGPU_TRY(blen.alloc(nb + 1));
  SGPU_TRY(err.alloc(1));
  SGPU_CUDA(cudaMemsetAsync(err.p, 0, sizeof(unsigned), s));
  k_bsr3_check<<<blocks_for((int64_t)nb * 32), TPB, 0, s>>>(nb, c.rowptr.p, c.col.p, blen.p, err.p);
  count_launches(1);
  unsigned e = 0;
  SGPU_TRY(read_err(err.p, s, &e));
  if (e) return SGPU_OK;  // not node-blocked: CSR only
  SGPU_TRY(b.browptr.alloc(nb + 1));
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, blen.p, b.browptr.p, nb + 1, s);
  DevBuf<unsigned char> t;
  SGPU_TRY(t.alloc(tmp));
  SGPU_CUDA(cudaMemsetAsync(blen.p + nb, 0, sizeof(int), s));
  cub::DeviceScan::ExclusiveSum(t.p, tmp, blen.p, b.browptr.p, nb + 1, s);
  count_launches(1);
  int nblk = 0;
  SGPU_CUDA(cudaMemcpyAsync(&nblk, b.browptr.p + nb, sizeof(int), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  b.nb = nb;
  b.nblk = nblk;
  // 16 bytes of slack after the columns and the FP32 values: bulk copies of
  // whole tiles round their end up to a 16-byte boundary
  SGPU_TRY(b.bcol.alloc((size_t)nblk + 4));
  SGPU_TRY(b.bval.alloc((size_t)nblk * 9));
  SGPU_TRY(b.csr2bsr.alloc(c.nnz));
  k_bsr3_fill<<<blocks_for((int64_t)nb * 32), TPB, 0, s>>>(nb, c.rowptr.p, c.col.p, b.browptr.p, b.bcol.p,
                                                           b.csr2bsr.p);
  k_bsr3_values<<<blocks_for(c.nnz), TPB, 0, s>>>(c.nnz, c.val.p, b.csr2bsr.p, b.bval.p);
  count_launches(2);
  b.valid = true;
  b.have32 = false;
  b.tile_cap = 0;
  if (c.have32) {
    SGPU_TRY(b.bval32s.alloc((size_t)nblk * 9 + 4));
    k_bsr3_values32<<<blocks_for(c.nnz), TPB, 0, s>>>(c.nnz, c.val32s.p, b.csr2bsr.p, b.bval32s.p);
    count_launches(1);
    b.have32 = true;
  }
  SGPU_CUDA(cudaStreamSynchronize(s));
  return SGPU_OK;
}

}  // namespace sgpu
