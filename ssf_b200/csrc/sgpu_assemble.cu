// Batched element integration fused with an atomic-free, colour-ordered
// scatter into the device CSR.
//
// Reference path: stiffness_matrix (MEFEL/SRC/globmat.cpp:41-143) loops over
// elements, calls linhex::res_stiffness_matrix (MEFEL/SRC/linhex.cpp:741 ->
// gl_stiffness_matrix :583) or planeelemlq::res_stiffness_matrix
// (MEFEL/SRC/plelemlq.cpp:785 -> :611), and localises each element matrix
// with symcomprow::localize (GEFEL/scr.cpp:422) / comprow::localize
// (GEFEL/cr.cpp:327).  TRFEL does the same with linhext::conductivity_matrix
// and capacity_matrix (TRFEL/SRC/linhext.cpp:774/979) in
// conductivity_matrix / capacity_matrix (TRFEL/SRC/globmatt.cpp:19/92).
//
// Here:
//  1. pattern: every element emits its (row, col <= row) equation pairs as
//     64-bit keys; one radix sort + unique gives the SCR pattern
//     (symcomprow::initiate, GEFEL/scr.cpp:556), from which the full CSR is
//     built (sgpu_matrix.cu);
//  2. colouring: greedy first-fit on the host over node masks -- elements of
//     one colour share no node, so their element matrices can be added into
//     the CSR without atomics, and the sum order is fixed (deterministic);
//  3. one launch per colour: one warp per element; lanes 0..G-1 compute the
//     Jacobian and Cartesian shape-function gradients of one Gauss point each
//     (derivatives_3d, GEFEL/difcalc.cpp:487) into shared memory, then every
//     lane forms whole node-pair blocks B_a^T D B_b summed over the Gauss
//     points and adds them into the CSR rows (binary search per row).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sgpu_internal.cuh"

namespace sgpu {

namespace {

constexpr int TPB = 256;
constexpr int WPB = TPB / 32;

inline int blocks_for(int64_t n, int tpb = TPB) {
  int64_t b = (n + tpb - 1) / tpb;
  return (int)(b < 1 ? 1 : (b > 1048576 ? 1048576 : b));
}

// Gauss rule of order 2 with the reference's 15-digit constant (GEFEL/intp.cpp:26-27)
__constant__ double c_gp2[2] = {-0.577350269189626, 0.577350269189626};

// ---------------------------------------------------------------------------
// pattern
// ---------------------------------------------------------------------------
__global__ void k_elem_codes(int64_t ne, int nne, int ndofn, const int64_t *__restrict__ elems,
                             const int64_t *__restrict__ cn, int *__restrict__ cne, unsigned *err, int64_t nn) {
  const int ndofe = nne * ndofn;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ne * ndofe;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / ndofe;
    const int q = (int)(t % ndofe), a = q / ndofn, i = q % ndofn;
    const int64_t node = elems[e * nne + a];
    int code = -1;
    if (node < 0 || node >= nn) {
      atomicOr(err, 1u);
    } else {
      const int64_t c = cn[node * ndofn + i];
      code = c > 0 ? (int)(c - 1) : -1;
    }
    cne[t] = code;
  }
}

// lower-triangle (row >= col) equation pairs of every element
__global__ void k_elem_pairs(int64_t ne, int ndofe, const int *__restrict__ cne,
                             unsigned long long *__restrict__ keys) {
  const int npair = ndofe * ndofe;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ne * npair;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / npair;
    const int q = (int)(t % npair), i = q / ndofe, j = q % ndofe;
    const int r = cne[e * ndofe + i], c = cne[e * ndofe + j];
    unsigned long long k = ~0ull;  // sorts last, dropped
    if (r >= 0 && c >= 0 && c <= r) k = ((unsigned long long)(unsigned)r << 32) | (unsigned)c;
    keys[t] = k;
  }
}

__global__ void k_keys_to_scr(int64_t m, int64_t n, const unsigned long long *__restrict__ keys,
                              int64_t *__restrict__ adr, int64_t *__restrict__ ci) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < m; s += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[s];
    const int64_t r = (int64_t)(k >> 32);
    ci[s] = (int64_t)(k & 0xffffffffull);
    if (s == 0 || (keys[s - 1] >> 32) != (unsigned long long)r) adr[r] = s;
    if (s == m - 1) adr[n] = m;
  }
}

// ---------------------------------------------------------------------------
// pattern from the node adjacency (no global sort of element pairs)
// ---------------------------------------------------------------------------

constexpr int kAdjCap = 512;  // candidate lower neighbours of one node (valence x nodes per element)

// node -> element incidence: counts, then the element ids of every node
__global__ void k_inc_count(int64_t m, const int64_t *__restrict__ elems, int *__restrict__ cnt) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(cnt + elems[t], 1);
}
__global__ void k_inc_fill(int64_t m, int nne, const int64_t *__restrict__ elems, const int *__restrict__ iptr,
                           int *__restrict__ cursor, int *__restrict__ inc) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t node = elems[t];
    inc[iptr[node] + atomicAdd(cursor + node, 1)] = (int)(t / nne);
  }
}

// one warp per node i: the sorted distinct nodes j <= i that share an element
// with i (bitonic sort of the candidates in shared memory).  FILL = false
// counts them into ucnt[i]; FILL = true writes them at nptr[i].  A node with
// more than kAdjCap candidates sets err bit 16 (the caller falls back).
template <bool FILL>
__global__ void __launch_bounds__(TPB) k_node_adj(int64_t nn, int nne, const int64_t *__restrict__ elems,
                                                  const int *__restrict__ iptr, const int *__restrict__ inc,
                                                  int *__restrict__ ucnt, const int64_t *__restrict__ nptr,
                                                  int *__restrict__ nadj, unsigned *err) {
  __shared__ int buf[WPB][kAdjCap];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int *sb = buf[wib];
  for (int64_t i = blockIdx.x * (int64_t)WPB + wib; i < nn; i += (int64_t)gridDim.x * WPB) {
    const int b = iptr[i], e = iptr[i + 1];
    const int ncand = (e - b) * nne;
    if (ncand > kAdjCap) {
      if (lane == 0) atomicOr(err, 16u);
      continue;
    }
    int P = 32;
    while (P < ncand) P <<= 1;
    for (int q = lane; q < P; q += 32) {
      int v = INT_MAX;
      if (q < ncand) {
        const int64_t j = elems[(int64_t)inc[b + q / nne] * nne + q % nne];
        if (j <= i) v = (int)j;
      }
      sb[q] = v;
    }
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int q = lane; q < P; q += 32) {
          const int x = q ^ j;
          if (x > q) {
            const int a = sb[q], c = sb[x];
            if ((a > c) == ((q & k) == 0)) {
              sb[q] = c;
              sb[x] = a;
            }
          }
        }
        __syncwarp();
      }
    int total = 0;
    for (int q0 = 0; q0 < P; q0 += 32) {
      const int q = q0 + lane;
      const bool keep = q < P && sb[q] != INT_MAX && (q == 0 || sb[q] != sb[q - 1]);
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (FILL && keep) nadj[nptr[i] + total + __popc(bal & ((1u << lane) - 1u))] = sb[q];
      total += __popc(bal);
    }
    if (!FILL && lane == 0) ucnt[i] = total;
    __syncwarp();
  }
}

// SCR row lengths from the node adjacency, for code numbers that grow with
// (node, component): row (i, c) holds the free components of every lower
// neighbour j < i and the free components d <= c of i itself
__global__ void k_scr_rowlen(int64_t nn, int ndofn, const int64_t *__restrict__ cn, const int64_t *__restrict__ nptr,
                             const int *__restrict__ nadj, int64_t *__restrict__ rowlen, int64_t n, unsigned *err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t base = 0;
    bool self = false;
    for (int64_t q = nptr[i]; q < nptr[i + 1]; q++) {
      const int j = nadj[q];
      if (j == i) {
        self = true;
        continue;
      }
      for (int d = 0; d < ndofn; d++) base += cn[(int64_t)j * ndofn + d] > 0;
    }
    int own = 0;
    for (int c = 0; c < ndofn; c++) {
      const int64_t r = cn[i * ndofn + c];
      if (r <= 0) continue;
      own++;
      if (r > n) {
        atomicOr(err, 1u);
        continue;
      }
      if (!self) atomicOr(err, 2u);  // an equation no element touches
      rowlen[r - 1] = base + own;
    }
  }
}

__global__ void k_scr_fill(int64_t nn, int ndofn, const int64_t *__restrict__ cn, const int64_t *__restrict__ nptr,
                           const int *__restrict__ nadj, const int64_t *__restrict__ adr, int64_t *__restrict__ ci,
                           int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
    for (int c = 0; c < ndofn; c++) {
      const int64_t r = cn[i * ndofn + c];
      if (r <= 0 || r > n) continue;
      int64_t w = adr[r - 1];
      for (int64_t q = nptr[i]; q < nptr[i + 1]; q++) {
        const int j = nadj[q];
        if (j == i) continue;
        for (int d = 0; d < ndofn; d++) {
          const int64_t cc = cn[(int64_t)j * ndofn + d];
          if (cc > 0) ci[w++] = cc - 1;
        }
      }
      for (int d = 0; d <= c; d++) {
        const int64_t cc = cn[i * ndofn + d];
        if (cc > 0) ci[w++] = cc - 1;
      }
    }
  }
}

__global__ void k_check_adr(int64_t n, const int64_t *__restrict__ adr, unsigned *err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (adr[i] < 0) atomicOr(err, 2u);  // an equation no element touches
}

// ---------------------------------------------------------------------------
// element kernels
// ---------------------------------------------------------------------------

// position of column c in the sorted CSR row [b, e), or -1
__device__ __forceinline__ int find_col(const int *__restrict__ col, int b, int e, int c) {
  int lo = b, hi = e - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = __ldg(col + mid);
    if (v == c) return mid;
    if (v < c) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// dN/dxi, dN/deta, dN/dzeta of the trilinear hexahedron (GEFEL/basefun.cpp:2316-2370)
__device__ __forceinline__ void hex_dnat(double xi, double eta, double zeta, double *nx, double *ny, double *nz) {
  const double sx[8] = {1, -1, -1, 1, 1, -1, -1, 1};
  const double sy[8] = {1, 1, -1, -1, 1, 1, -1, -1};
  const double sz[8] = {1, 1, 1, 1, -1, -1, -1, -1};
#pragma unroll
  for (int a = 0; a < 8; a++) {
    nx[a] = sx[a] * (1.0 + sy[a] * eta) * (1.0 + sz[a] * zeta) / 8.0;
    ny[a] = sy[a] * (1.0 + sx[a] * xi) * (1.0 + sz[a] * zeta) / 8.0;
    nz[a] = sz[a] * (1.0 + sx[a] * xi) * (1.0 + sy[a] * eta) / 8.0;
  }
}

__device__ __forceinline__ void hex_n(double xi, double eta, double zeta, double *n) {
  const double sx[8] = {1, -1, -1, 1, 1, -1, -1, 1};
  const double sy[8] = {1, 1, -1, -1, 1, 1, -1, -1};
  const double sz[8] = {1, 1, 1, 1, -1, -1, -1, -1};
#pragma unroll
  for (int a = 0; a < 8; a++) n[a] = (1.0 + sx[a] * xi) * (1.0 + sy[a] * eta) * (1.0 + sz[a] * zeta) / 8.0;
}

// Per-warp shared storage: Cartesian gradients at the Gauss points and
// |detJ| * weight (times the point's extra factor).
struct HexShared {
  double g[8][8][3];  // [gp][node][x,y,z]
  double w[8];
  double nb[8][8];    // shape functions at the Gauss points (capacity)
  double D[36];       // general material stiffness of the element (row-major)
};

// D B_b for a general 6 x 6 D (row-major) and the gradient (bx, by, bz) of
// node b: B_b columns u = (bx,0,0,0,bz,by), v = (0,by,0,bz,0,bx),
// w = (0,0,bz,by,bx,0) in the strain order [xx, yy, zz, yz, xz, xy]
__device__ __forceinline__ void elastic_db(const double *D, double bx, double by, double bz, double db[6][3]) {
#pragma unroll
  for (int r = 0; r < 6; r++) {
    db[r][0] = D[6 * r + 0] * bx + D[6 * r + 4] * bz + D[6 * r + 5] * by;
    db[r][1] = D[6 * r + 1] * by + D[6 * r + 3] * bz + D[6 * r + 5] * bx;
    db[r][2] = D[6 * r + 2] * bz + D[6 * r + 3] * by + D[6 * r + 4] * bx;
  }
}

// lanes 0..7: Gauss point `lane` (reference loop order xi, eta, zeta)
__device__ __forceinline__ void hex_gauss_point(int lane, const double *x, const double *y, const double *z,
                                                HexShared &sh, bool want_n) {
  if (lane < 8) {
    const double xi = c_gp2[(lane >> 2) & 1], eta = c_gp2[(lane >> 1) & 1], zeta = c_gp2[lane & 1];
    double nx[8], ny[8], nz[8];
    hex_dnat(xi, eta, zeta, nx, ny, nz);
    double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0, d9 = 0;
#pragma unroll
    for (int a = 0; a < 8; a++) {
      d1 += nx[a] * x[a]; d2 += ny[a] * x[a]; d3 += nz[a] * x[a];
      d4 += nx[a] * y[a]; d5 += ny[a] * y[a]; d6 += nz[a] * y[a];
      d7 += nx[a] * z[a]; d8 += ny[a] * z[a]; d9 += nz[a] * z[a];
    }
    const double jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 - d9 * d4 * d2;
#pragma unroll
    for (int a = 0; a < 8; a++) {
      const double ddx = nx[a], ddy = ny[a], ddz = nz[a];
      sh.g[lane][a][0] = (ddx * (d5 * d9 - d8 * d6) + ddy * (d7 * d6 - d9 * d4) + ddz * (d4 * d8 - d7 * d5)) / jac;
      sh.g[lane][a][1] = (ddx * (d8 * d3 - d9 * d2) + ddy * (d1 * d9 - d7 * d3) + ddz * (d7 * d2 - d8 * d1)) / jac;
      sh.g[lane][a][2] = (ddx * (d2 * d6 - d5 * d3) + ddy * (d4 * d3 - d6 * d1) + ddz * (d1 * d5 - d4 * d2)) / jac;
    }
    sh.w[lane] = fabs(jac);  // weights are 1 for the order-2 rule
    if (want_n) {
      double n[8];
      hex_n(xi, eta, zeta, n);
#pragma unroll
      for (int a = 0; a < 8; a++) sh.nb[lane][a] = n[a];
    }
  }
}

// add v into CSR entry (r, c); both >= 0
__device__ __forceinline__ void csr_add(const int *__restrict__ rowptr, const int *__restrict__ col,
                                        double *__restrict__ val, int r, int c, double v, unsigned *err) {
  const int p = find_col(col, __ldg(rowptr + r), __ldg(rowptr + r + 1), c);
  if (p >= 0) val[p] += v;
  else atomicOr(err, 4u);
}

// adds the 3 x 3 block k at rows r[0..2], columns c[0..2] (< 0: no
// equation).  When both triples are one node's consecutive equations, the
// three rows of a node hold the same column list in the full CSR, so one
// search finds the block's first entry and the other eight sit at fixed
// offsets -- each checked before it is used; otherwise nine searches.
__device__ __forceinline__ void block3_add(const int *__restrict__ rowptr, const int *__restrict__ col,
                                           double *__restrict__ val, const int r[3], const int c[3],
                                           const double k[3][3], unsigned *err) {
  if (r[0] >= 0 && r[1] == r[0] + 1 && r[2] == r[0] + 2 && c[0] >= 0 && c[1] == c[0] + 1 && c[2] == c[0] + 2) {
    const int b0 = __ldg(rowptr + r[0]), e0 = __ldg(rowptr + r[0] + 1);
    const int p = find_col(col, b0, e0, c[0]);
    if (p >= 0 && p + 2 < e0) {
      const int off = p - b0;
      int q[3];
      bool ok = true;
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int bi = __ldg(rowptr + r[i]), ei = __ldg(rowptr + r[i] + 1);
        q[i] = bi + off;
        ok = ok && q[i] + 2 < ei && __ldg(col + q[i]) == c[0] && __ldg(col + q[i] + 1) == c[1] &&
             __ldg(col + q[i] + 2) == c[2];
      }
      if (ok) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) val[q[i] + j] += k[i][j];
        return;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 3; i++) {
    if (r[i] < 0) continue;
#pragma unroll
    for (int j = 0; j < 3; j++)
      if (c[j] >= 0) csr_add(rowptr, col, val, r[i], c[j], k[i][j], err);
  }
}

// hex8 elasticity (linhex::gl_stiffness_matrix): block (a,b) of
// sum_gp |J| B_a^T D B_b with B rows [xx, yy, zz, yz, xz, xy]
// (linhex::geom_matrix, MEFEL/SRC/linhex.cpp:153-186) and isotropic D
// (elastisomat::matstiff_spacestr, MEFEL/SRC/elastisomat.cpp:395-420)
template <bool GEN>
__global__ void __launch_bounds__(TPB) k_hex8_elastic(int ne_c, const int *__restrict__ elist,
                                                      const double *__restrict__ coords,
                                                      const int64_t *__restrict__ elems,
                                                      const int *__restrict__ cne, const double *__restrict__ emat,
                                                      const int *__restrict__ rowptr, const int *__restrict__ col,
                                                      double *__restrict__ val, unsigned *err) {
  __shared__ HexShared shm[WPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  HexShared &sh = shm[wib];
  for (int t = blockIdx.x * WPB + wib; t < ne_c; t += gridDim.x * WPB) {
    const int e = elist[t];
    double x[8], y[8], z[8];
    double cx = 0, cy = 0, cz = 0;
    if (lane < 8) {
      const int64_t nd = elems[(int64_t)e * 8 + lane];
      cx = coords[3 * nd]; cy = coords[3 * nd + 1]; cz = coords[3 * nd + 2];
    }
#pragma unroll
    for (int a = 0; a < 8; a++) {
      x[a] = __shfl_sync(0xffffffffu, cx, a);
      y[a] = __shfl_sync(0xffffffffu, cy, a);
      z[a] = __shfl_sync(0xffffffffu, cz, a);
    }
    hex_gauss_point(lane, x, y, z, sh, false);
    if (GEN) {
      for (int q = lane; q < 36; q += 32) sh.D[q] = emat[36 * (int64_t)e + q];
    }
    __syncwarp();
    double d0 = 0.0, d1 = 0.0, G = 0.0;
    if (!GEN) {
      const double E = emat[2 * (int64_t)e], nu = emat[2 * (int64_t)e + 1];
      G = E / 2.0 / (1.0 + nu);
      const double s = E / (1.0 + nu) / (1.0 - 2.0 * nu);
      d0 = s * (1 - nu);
      d1 = s * nu;
    }
    int code[24];
#pragma unroll
    for (int q = 0; q < 24; q++) code[q] = __ldg(cne + (int64_t)e * 24 + q);
    for (int blk = lane; blk < 64; blk += 32) {
      const int a = blk >> 3, b = blk & 7;
      double k[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
      for (int gp = 0; gp < 8; gp++) {
        const double ax = sh.g[gp][a][0], ay = sh.g[gp][a][1], az = sh.g[gp][a][2];
        const double bx = sh.g[gp][b][0], by = sh.g[gp][b][1], bz = sh.g[gp][b][2];
        const double w = sh.w[gp];
        // D B_b: columns (u, v, w) of node b
        // rows: xx, yy, zz, yz, xz, xy
        double db[6][3];
        if (GEN) {
          elastic_db(sh.D, bx, by, bz, db);
        } else {
          db[0][0] = d0 * bx; db[0][1] = d1 * by; db[0][2] = d1 * bz;
          db[1][0] = d1 * bx; db[1][1] = d0 * by; db[1][2] = d1 * bz;
          db[2][0] = d1 * bx; db[2][1] = d1 * by; db[2][2] = d0 * bz;
          db[3][0] = 0.0;     db[3][1] = G * bz;  db[3][2] = G * by;
          db[4][0] = G * bz;  db[4][1] = 0.0;     db[4][2] = G * bx;
          db[5][0] = G * by;  db[5][1] = G * bx;  db[5][2] = 0.0;
        }
#pragma unroll
        for (int j = 0; j < 3; j++) {
          // B_a^T rows: u -> (xx: ax, xz: az, xy: ay); v -> (yy: ay, yz: az, xy: ax); w -> (zz: az, yz: ay, xz: ax)
          k[0][j] += w * (ax * db[0][j] + az * db[4][j] + ay * db[5][j]);
          k[1][j] += w * (ay * db[1][j] + az * db[3][j] + ax * db[5][j]);
          k[2][j] += w * (az * db[2][j] + ay * db[3][j] + ax * db[4][j]);
        }
      }
      const int rr[3] = {code[3 * a], code[3 * a + 1], code[3 * a + 2]};
      const int cc[3] = {code[3 * b], code[3 * b + 1], code[3 * b + 2]};
      block3_add(rowptr, col, val, rr, cc, k, err);
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// hex8 isotropic elasticity, colour-ordered like k_hex8_elastic, with the
// arithmetic cut down so that the kernel is bound by its scatter:
//   * every lane works on the Gauss points: lane = gp + 8 q forms the
//     Jacobian of point gp and the Cartesian gradients of nodes 2q, 2q+1
//     (one reciprocal of detJ instead of a division per gradient entry);
//   * for the isotropic D of elastisomat (MEFEL/SRC/elastisomat.cpp:395-420),
//     with lambda = E nu / ((1+nu)(1-2nu)) and mu = E / (2 (1+nu)), the block
//     (a,b) of sum_gp |J| B_a^T D B_b (linhex::gl_stiffness_matrix,
//     MEFEL/SRC/linhex.cpp:583-630) is
//         K_ab = lambda P + mu P^T + mu tr(P) I,  P = sum_gp |J| g_a g_b^T,
//     9 FMA per point instead of the full B^T D B product;
//   * the element matrix is symmetric: the 36 pairs a <= b are formed once
//     (lanes 0..27 the 28 pairs a < b, lanes 28..31 two diagonal pairs each)
//     and K_ba = K_ab^T is scattered beside K_ab, so every lane scatters two
//     blocks.
// The same sums as the reference's up to rounding (the reciprocal and the
// regrouped products: relative differences of a few units of 1e-16).
// ---------------------------------------------------------------------------
// dN_a/dxi, dN_a/deta, dN_a/dzeta of one node (the expressions of hex_dnat)
__device__ __forceinline__ void hex_dnat1(int a, double xi, double eta, double zeta, double &nx, double &ny,
                                          double &nz) {
  const double sx = ((a + 1) & 2) ? -1.0 : 1.0;  // +, -, -, +, +, -, -, +
  const double sy = (a & 2) ? -1.0 : 1.0;        // +, +, -, -, +, +, -, -
  const double sz = (a & 4) ? -1.0 : 1.0;        // +, +, +, +, -, -, -, -
  nx = sx * (1.0 + sy * eta) * (1.0 + sz * zeta) / 8.0;
  ny = sy * (1.0 + sx * xi) * (1.0 + sz * zeta) / 8.0;
  nz = sz * (1.0 + sx * xi) * (1.0 + sy * eta) / 8.0;
}

constexpr int kIsoRowCap = 96;  // columns of one row held in shared memory

struct HexIsoShared {
  double g[8][8][3];  // [gp][node][x, y, z]
  double w[8];        // |detJ| (weights are 1)
  int rp[24];         // rowptr of the element's equations
  int rl[8];          // length of node a's rows when its three equations are
                      // consecutive with rows of one length (<= kIsoRowCap), else -1
  int cols[8][kIsoRowCap];  // the column list of node a's first row
};

// 4-byte global -> shared copy that completes asynchronously (cp.async)
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// position of column c in the sorted shared list cols[0, len), or -1
__device__ __forceinline__ int find_in_shared(const int *cols, int len, int c) {
  int lo = 0, hi = len - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = cols[mid];
    if (v == c) return mid;
    if (v < c) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// adds block k at the rows of node A (equations rr) and the columns of node B
// (equations cc).  The three rows of a node whose equations are consecutive
// hold one column list in the full CSR (every row lists the free equations
// of the node's neighbours), so with node A's list in shared memory one
// search there places all nine entries; other blocks take block3_add.
template <bool ROWCACHE>
__device__ __forceinline__ void iso_scatter(const HexIsoShared &sh, int A, const int rr[3], const int cc[3],
                                            const double k[3][3], const int *__restrict__ rowptr,
                                            const int *__restrict__ col, double *__restrict__ val, unsigned *err) {
  if (ROWCACHE) {
    const int len = sh.rl[A];
    if (len > 0 && cc[0] >= 0 && cc[1] == cc[0] + 1 && cc[2] == cc[0] + 2) {
      const int p = find_in_shared(sh.cols[A], len, cc[0]);
      if (p >= 0 && p + 2 < len && sh.cols[A][p + 1] == cc[1] && sh.cols[A][p + 2] == cc[2]) {
#pragma unroll
        for (int i = 0; i < 3; i++) {
          double *v = val + sh.rp[3 * A + i] + p;
          v[0] += k[i][0];
          v[1] += k[i][1];
          v[2] += k[i][2];
        }
        return;
      }
    }
  }
  block3_add(rowptr, col, val, rr, cc, k, err);
}

// the pair (a, b), a < b, of index t in 0..27 (row-major over the upper triangle)
__device__ __forceinline__ void upper_pair(int t, int &a, int &b) {
  a = 0;
  int left = t;
  while (left >= 7 - a) { left -= 7 - a; a++; }
  b = a + 1 + left;
}

__device__ __forceinline__ void hex_iso_block(const HexIsoShared &sh, int a, int b, double lam, double mu,
                                              double k[3][3]) {
  double P[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int gp = 0; gp < 8; gp++) {
    const double w = sh.w[gp];
    const double ax = w * sh.g[gp][a][0], ay = w * sh.g[gp][a][1], az = w * sh.g[gp][a][2];
    const double bx = sh.g[gp][b][0], by = sh.g[gp][b][1], bz = sh.g[gp][b][2];
    P[0][0] += ax * bx; P[0][1] += ax * by; P[0][2] += ax * bz;
    P[1][0] += ay * bx; P[1][1] += ay * by; P[1][2] += ay * bz;
    P[2][0] += az * bx; P[2][1] += az * by; P[2][2] += az * bz;
  }
  const double tr = mu * (P[0][0] + P[1][1] + P[2][2]);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) k[i][j] = lam * P[i][j] + mu * P[j][i] + (i == j ? tr : 0.0);
}

// STORE: no scatter; the 36 blocks a <= b of element e go to
// kbuf[324 e + 9 slot + 3 i + j] (slot: the index of (a, b) among the pairs
// a < b in row-major order, 28 + a for (a, a)), every element in one launch
// (elist unused), for k_hex8_gather.
template <bool ROWCACHE, bool STORE>
__global__ void __launch_bounds__(TPB, 3) k_hex8_iso(int ne_c, const int *__restrict__ elist,
                                                     const double *__restrict__ coords,
                                                     const int64_t *__restrict__ elems,
                                                     const int *__restrict__ cne, const double *__restrict__ emat,
                                                     const int *__restrict__ rowptr, const int *__restrict__ col,
                                                     double *__restrict__ val, unsigned *err,
                                                     double *__restrict__ kbuf) {
  __shared__ HexIsoShared shm[WPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  HexIsoShared &sh = shm[wib];
  const int gp = lane & 7, q = lane >> 3;
  const double xi = c_gp2[(gp >> 2) & 1], eta = c_gp2[(gp >> 1) & 1], zeta = c_gp2[gp & 1];
  for (int t = blockIdx.x * WPB + wib; t < ne_c; t += gridDim.x * WPB) {
    const int e = STORE ? t : elist[t];
    double cx = 0, cy = 0, cz = 0;
    if (lane < 8) {
      const int64_t nd = elems[(int64_t)e * 8 + lane];
      cx = coords[3 * nd]; cy = coords[3 * nd + 1]; cz = coords[3 * nd + 2];
    }
    const int code = (lane < 24 && !STORE) ? __ldg(cne + (int64_t)e * 24 + lane) : -1;
    if (ROWCACHE && !STORE) {
      // the rows of the element's equations; node a's column list copied
      // into shared memory while the Gauss points are formed
      int rpv = -1, rlen = 0;
      if (code >= 0) {
        rpv = __ldg(rowptr + code);
        rlen = __ldg(rowptr + code + 1) - rpv;
      }
      const int na = lane & 7;
      const int c0 = __shfl_sync(0xffffffffu, code, 3 * na), c1 = __shfl_sync(0xffffffffu, code, 3 * na + 1),
                c2 = __shfl_sync(0xffffffffu, code, 3 * na + 2);
      const int l0 = __shfl_sync(0xffffffffu, rlen, 3 * na), l1 = __shfl_sync(0xffffffffu, rlen, 3 * na + 1),
                l2 = __shfl_sync(0xffffffffu, rlen, 3 * na + 2);
      if (lane < 24) sh.rp[lane] = rpv;
      if (lane < 8)
        sh.rl[lane] = (c0 >= 0 && c1 == c0 + 1 && c2 == c0 + 2 && l0 == l1 && l1 == l2 && l0 > 0 &&
                       l0 <= kIsoRowCap) ? l0 : -1;
      __syncwarp();
#pragma unroll
      for (int a = 0; a < 8; a++) {
        const int len = sh.rl[a];
        if (len > 0) {
          const int *src = col + sh.rp[3 * a];
          for (int j = lane; j < len; j += 32) cp_async4(&sh.cols[a][j], src + j);
        }
      }
    }
    // Jacobian of point gp (every lane of the point's four computes it)
    double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0, d9 = 0;
#pragma unroll
    for (int a = 0; a < 8; a++) {
      const double x = __shfl_sync(0xffffffffu, cx, a), y = __shfl_sync(0xffffffffu, cy, a),
                   z = __shfl_sync(0xffffffffu, cz, a);
      double nxa, nya, nza;
      hex_dnat1(a, xi, eta, zeta, nxa, nya, nza);
      d1 += nxa * x; d2 += nya * x; d3 += nza * x;
      d4 += nxa * y; d5 += nya * y; d6 += nza * y;
      d7 += nxa * z; d8 += nya * z; d9 += nza * z;
    }
    const double jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 - d9 * d4 * d2;
    const double ij = 1.0 / jac;
    // cofactors of derivatives_3d (GEFEL/difcalc.cpp:487-565), scaled by 1/detJ
    const double c11 = (d5 * d9 - d8 * d6) * ij, c12 = (d7 * d6 - d9 * d4) * ij, c13 = (d4 * d8 - d7 * d5) * ij;
    const double c21 = (d8 * d3 - d9 * d2) * ij, c22 = (d1 * d9 - d7 * d3) * ij, c23 = (d7 * d2 - d8 * d1) * ij;
    const double c31 = (d2 * d6 - d5 * d3) * ij, c32 = (d4 * d3 - d6 * d1) * ij, c33 = (d1 * d5 - d4 * d2) * ij;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int a = 2 * q + h;
      double ddx, ddy, ddz;
      hex_dnat1(a, xi, eta, zeta, ddx, ddy, ddz);
      sh.g[gp][a][0] = ddx * c11 + ddy * c12 + ddz * c13;
      sh.g[gp][a][1] = ddx * c21 + ddy * c22 + ddz * c23;
      sh.g[gp][a][2] = ddx * c31 + ddy * c32 + ddz * c33;
    }
    if (q == 0) sh.w[gp] = fabs(jac);
    const double E = __ldg(emat + 2 * (int64_t)e), nu = __ldg(emat + 2 * (int64_t)e + 1);
    const double mu = E / 2.0 / (1.0 + nu);
    const double lam = E / (1.0 + nu) / (1.0 - 2.0 * nu) * nu;
    if (ROWCACHE && !STORE) cp_async_wait_all();
    __syncwarp();
    // first block: lanes < 28 the pair a < b of their index, lanes 28..31
    // the diagonal pair (2 (lane - 28), same)
    int a0, b0;
    if (lane < 28) {
      upper_pair(lane, a0, b0);
    } else {
      a0 = b0 = 2 * (lane - 28);
    }
    double k[3][3];
    hex_iso_block(sh, a0, b0, lam, mu, k);
    if (STORE) {
      double *dst = kbuf + (size_t)e * 324 + 9 * (lane < 28 ? lane : 28 + a0);
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) dst[3 * i + j] = k[i][j];
      if (lane >= 28) {
        const int a1 = 2 * (lane - 28) + 1;
        hex_iso_block(sh, a1, a1, lam, mu, k);
        double *d1 = kbuf + (size_t)e * 324 + 9 * (28 + a1);
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) d1[3 * i + j] = k[i][j];
      }
      __syncwarp();
      continue;
    }
    int rr[3], cc[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      rr[i] = __shfl_sync(0xffffffffu, code, 3 * a0 + i);
      cc[i] = __shfl_sync(0xffffffffu, code, 3 * b0 + i);
    }
    iso_scatter<ROWCACHE>(sh, a0, rr, cc, k, rowptr, col, val, err);
    // second block: the transpose at (b, a), or the next diagonal pair
    int a1, b1;
    if (lane < 28) {
      a1 = b0;
      b1 = a0;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = i + 1; j < 3; j++) {
          const double tmp = k[i][j];
          k[i][j] = k[j][i];
          k[j][i] = tmp;
        }
    } else {
      a1 = b1 = 2 * (lane - 28) + 1;
      hex_iso_block(sh, a1, b1, lam, mu, k);
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
      rr[i] = __shfl_sync(0xffffffffu, code, 3 * a1 + i);
      cc[i] = __shfl_sync(0xffffffffu, code, 3 * b1 + i);
    }
    iso_scatter<ROWCACHE>(sh, a1, rr, cc, k, rowptr, col, val, err);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// hex8 isotropic elasticity by rows: one warp per node forms the node's CSR
// rows from its incident elements in shared memory and writes them once.
//
// The colour-ordered scatter above reads and writes every 3 x 3 block once
// per element that touches it (2.4 times per block on a structured mesh,
// 24-byte pieces of 32-byte sectors) -- about 3 GB of read-modify-write for
// the 630 MB value array of a 1M-equation cantilever.  Here each CSR entry is
// summed in shared memory and stored once, with no colours, no atomics and
// no zero fill of the value array; the summation order of every entry is
// fixed (incident elements by ascending id, Gauss points in the reference's
// order).  The price is that an element's Gauss-point gradients are formed
// by each of its 8 nodes' warps.
//
// For the isotropic D of elastisomat (MEFEL/SRC/elastisomat.cpp:395-420),
// with lambda = E nu / ((1+nu)(1-2nu)) and mu = E / (2 (1+nu)), block (a,b)
// of sum_gp |J| B_a^T D B_b (linhex::gl_stiffness_matrix,
// MEFEL/SRC/linhex.cpp:583-630) is
//     K_ab = lambda P + mu P^T + mu tr(P) I,   P = sum_gp |J| g_a g_b^T
// with g the Cartesian gradients of derivatives_3d (GEFEL/difcalc.cpp:487):
// 24 FMA per block row instead of the full B^T D B product.
// ---------------------------------------------------------------------------
constexpr int kRowCap = 96;    // CSR entries of one row held in shared memory
constexpr int kIncCap = 32;    // elements at one node
constexpr int kElemBatch = 4;  // elements whose Gauss-point gradients a warp forms at once
constexpr int kRowWarps = 4;   // warps per block of the row kernel

constexpr int kGpStride = 25;  // 8 nodes x 3 gradient components, padded: the
                               // 16 lanes of a half-warp storing their points'
                               // gradients hit distinct banks

struct HexRowShared {
  double g[kElemBatch][8][kGpStride];  // [element][gp][3 node + x/y/z]
  double w[kElemBatch][8];        // |detJ| (weights are 1)
  double acc[3][kRowCap];         // the node's rows
  int col[3][kRowCap];            // their column indices
  int inc[kIncCap];               // incident elements, ascending
};

// gradients of the 8 shape functions (g[3 a + c]) and |detJ| at Gauss point
// gp (0..7, xi outermost), as hex_gauss_point, with one reciprocal of detJ
// scaling the cofactors of derivatives_3d (GEFEL/difcalc.cpp:487-565)
__device__ __forceinline__ void hex_gp_gradients(int gp, const double *x, const double *y, const double *z,
                                                 double *g, double *w) {
  const double xi = c_gp2[(gp >> 2) & 1], eta = c_gp2[(gp >> 1) & 1], zeta = c_gp2[gp & 1];
  double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0, d9 = 0;
#pragma unroll
  for (int a = 0; a < 8; a++) {
    double nxa, nya, nza;
    hex_dnat1(a, xi, eta, zeta, nxa, nya, nza);
    d1 += nxa * x[a]; d2 += nya * x[a]; d3 += nza * x[a];
    d4 += nxa * y[a]; d5 += nya * y[a]; d6 += nza * y[a];
    d7 += nxa * z[a]; d8 += nya * z[a]; d9 += nza * z[a];
  }
  const double jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 - d9 * d4 * d2;
  const double ij = 1.0 / jac;
  const double c11 = (d5 * d9 - d8 * d6) * ij, c12 = (d7 * d6 - d9 * d4) * ij, c13 = (d4 * d8 - d7 * d5) * ij;
  const double c21 = (d8 * d3 - d9 * d2) * ij, c22 = (d1 * d9 - d7 * d3) * ij, c23 = (d7 * d2 - d8 * d1) * ij;
  const double c31 = (d2 * d6 - d5 * d3) * ij, c32 = (d4 * d3 - d6 * d1) * ij, c33 = (d1 * d5 - d4 * d2) * ij;
#pragma unroll
  for (int a = 0; a < 8; a++) {
    double ddx, ddy, ddz;
    hex_dnat1(a, xi, eta, zeta, ddx, ddy, ddz);
    g[3 * a] = ddx * c11 + ddy * c12 + ddz * c13;
    g[3 * a + 1] = ddx * c21 + ddy * c22 + ddz * c23;
    g[3 * a + 2] = ddx * c31 + ddy * c32 + ddz * c33;
  }
  *w = fabs(jac);
}

// position of column c in the sorted shared row cols[0, len), or -1
__device__ __forceinline__ int find_col_sh(const int *cols, int len, int c) {
  int lo = 0, hi = len - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = cols[mid];
    if (v == c) return mid;
    if (v < c) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// err bits: 4 an element entry has no CSR position; 32 a node exceeds
// kIncCap elements or kRowCap entries per row (the caller falls back to the
// colour-ordered kernel)
__global__ void __launch_bounds__(kRowWarps * 32) k_hex8_rows(int64_t nn, const int *__restrict__ iptr,
                                                              const int *__restrict__ inc,
                                                              const double *__restrict__ coords,
                                                              const int64_t *__restrict__ elems,
                                                              const int *__restrict__ cne,
                                                              const double *__restrict__ emat,
                                                              const int *__restrict__ rowptr,
                                                              const int *__restrict__ col,
                                                              double *__restrict__ val, unsigned *err) {
  __shared__ HexRowShared shm[kRowWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  HexRowShared &sh = shm[wib];
  for (int64_t node = blockIdx.x * (int64_t)kRowWarps + wib; node < nn; node += (int64_t)gridDim.x * kRowWarps) {
    const int ib = iptr[node], deg = iptr[node + 1] - ib;
    if (deg == 0) continue;
    if (deg > kIncCap) {
      if (lane == 0) atomicOr(err, 32u);
      continue;
    }
    // incident elements in ascending order (distinct ids: rank sort)
    const int mine = lane < deg ? inc[ib + lane] : INT_MAX;
    int rank = 0;
    for (int k = 0; k < deg; k++) rank += __shfl_sync(0xffffffffu, mine, k) < mine;
    if (lane < deg) sh.inc[rank] = mine;
    __syncwarp();
    // the node's rows: its code numbers in its first element
    int la0;
    {
      const int e0 = sh.inc[0];
      const bool hit = lane < 8 && elems[(int64_t)e0 * 8 + lane] == node;
      la0 = __ffs(__ballot_sync(0xffffffffu, hit)) - 1;
      if (la0 < 0) la0 = 0;  // not reached for a consistent incidence
    }
    int r[3], len[3];
    bool fits = true;
#pragma unroll
    for (int i = 0; i < 3; i++) {
      r[i] = __ldg(cne + (int64_t)sh.inc[0] * 24 + 3 * la0 + i);
      len[i] = 0;
      if (r[i] >= 0) {
        const int rb = __ldg(rowptr + r[i]);
        len[i] = __ldg(rowptr + r[i] + 1) - rb;
        if (len[i] > kRowCap) {
          fits = false;
        } else {
          for (int k = lane; k < len[i]; k += 32) {
            sh.col[i][k] = __ldg(col + rb + k);
            sh.acc[i][k] = 0.0;
          }
        }
      }
    }
    if (!fits) {
      if (lane == 0) atomicOr(err, 32u);
      __syncwarp();
      continue;
    }
    if (r[0] < 0 && r[1] < 0 && r[2] < 0) {
      __syncwarp();
      continue;  // a fully constrained node has no rows
    }
    __syncwarp();
    for (int q0 = 0; q0 < deg; q0 += kElemBatch) {
      const int nb = min(kElemBatch, deg - q0);
      {  // Gauss-point gradients of up to kElemBatch elements: lane = (element, gp)
        const int el = lane >> 3, gp = lane & 7;
        if (el < nb) {
          const int e = sh.inc[q0 + el];
          double x[8], y[8], z[8];
#pragma unroll
          for (int a = 0; a < 8; a++) {
            const int64_t nd = __ldg(elems + (int64_t)e * 8 + a);
            x[a] = __ldg(coords + 3 * nd);
            y[a] = __ldg(coords + 3 * nd + 1);
            z[a] = __ldg(coords + 3 * nd + 2);
          }
          hex_gp_gradients(gp, x, y, z, sh.g[el][gp], &sh.w[el][gp]);
        }
      }
      __syncwarp();
      for (int q = 0; q < nb; q++) {
        const int e = sh.inc[q0 + q];
        const bool hit = lane < 8 && elems[(int64_t)e * 8 + lane] == node;
        int la = __ffs(__ballot_sync(0xffffffffu, hit)) - 1;
        if (la < 0) la = 0;
        const double E = __ldg(emat + 2 * (int64_t)e), nu = __ldg(emat + 2 * (int64_t)e + 1);
        const double mu = E / 2.0 / (1.0 + nu);
        const double lam = E / (1.0 + nu) / (1.0 - 2.0 * nu) * nu;
        // lane (b, i), b = node of the element, i = row component: row i of
        // P_b = sum_gp |J| g_la g_b^T
        const int b = lane < 24 ? lane / 3 : 0, i = lane < 24 ? lane - 3 * (lane / 3) : 0;
        double p0 = 0.0, p1 = 0.0, p2 = 0.0;
        if (lane < 24) {
#pragma unroll
          for (int gp = 0; gp < 8; gp++) {
            const double wa = sh.w[q][gp] * sh.g[q][gp][3 * la + i];
            p0 += wa * sh.g[q][gp][3 * b];
            p1 += wa * sh.g[q][gp][3 * b + 1];
            p2 += wa * sh.g[q][gp][3 * b + 2];
          }
        }
        // column i of P_b (rows k = 0..2 live in lanes 3b + k) and its trace
        double pc[3], tr = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const int src = 3 * b + k;
          const double t0 = __shfl_sync(0xffffffffu, p0, src);
          const double t1 = __shfl_sync(0xffffffffu, p1, src);
          const double t2 = __shfl_sync(0xffffffffu, p2, src);
          pc[k] = i == 0 ? t0 : (i == 1 ? t1 : t2);
          tr += k == 0 ? t0 : (k == 1 ? t1 : t2);
        }
        if (lane < 24 && r[i] >= 0) {
          const double kr[3] = {lam * p0 + mu * pc[0] + (i == 0 ? mu * tr : 0.0),
                                lam * p1 + mu * pc[1] + (i == 1 ? mu * tr : 0.0),
                                lam * p2 + mu * pc[2] + (i == 2 ? mu * tr : 0.0)};
          const int *cb = cne + (int64_t)e * 24 + 3 * b;
          const int c0 = __ldg(cb), c1 = __ldg(cb + 1), c2 = __ldg(cb + 2);
          const int *cols = sh.col[i];
          double *acc = sh.acc[i];
          bool done = false;
          if (c0 >= 0 && c1 == c0 + 1 && c2 == c0 + 2) {  // a fully free node: one search
            const int p = find_col_sh(cols, len[i], c0);
            if (p >= 0 && p + 2 < len[i] && cols[p + 1] == c1 && cols[p + 2] == c2) {
              acc[p] += kr[0];
              acc[p + 1] += kr[1];
              acc[p + 2] += kr[2];
              done = true;
            }
          }
          if (!done) {
            const int cc[3] = {c0, c1, c2};
#pragma unroll
            for (int j = 0; j < 3; j++) {
              if (cc[j] < 0) continue;
              const int p = find_col_sh(cols, len[i], cc[j]);
              if (p >= 0) acc[p] += kr[j];
              else atomicOr(err, 4u);
            }
          }
        }
        __syncwarp();
      }
    }
    // every entry of the node's rows, written once
#pragma unroll
    for (int i = 0; i < 3; i++) {
      if (r[i] < 0) continue;
      double *dst = val + __ldg(rowptr + r[i]);
      for (int k = lane; k < len[i]; k += 32) dst[k] = sh.acc[i][k];
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// hex8 isotropic elasticity, write-once: k_hex8_iso<.., STORE> forms the 36
// blocks a <= b of every element into a buffer (one launch, no colours, no
// scatter), then one warp per node gathers the blocks of its incident
// elements into the node's (up to) three CSR rows in shared memory -- the
// elements by ascending id, so every entry's summation order is fixed -- and
// writes each entry once.  The colour-ordered scatter reads and writes every
// 3x3 block once per element that touches it, in 24-byte pieces of 32-byte
// sectors (about 7 GB of DRAM traffic for the 630 MB value array of the
// 1.01M-DOF cantilever); here the traffic is the buffer written and read
// once (324 doubles per element) and the values written once.
// ---------------------------------------------------------------------------
constexpr int kGatherBatch = 4;  // incident elements whose blocks a warp loads at once

struct HexGatherShared {
  double acc[3][kRowCap];  // the node's rows
  int col[3][kRowCap];     // their column indices
  int inc[kIncCap];        // incident elements, ascending
  int la[kIncCap];         // the node's index in each of them
};

// the slot of pair (a, b), a < b, among the 28 pairs in row-major order
__device__ __forceinline__ int upper_slot(int a, int b) { return 7 * a - (a * (a - 1)) / 2 + (b - a - 1); }

__global__ void __launch_bounds__(kRowWarps * 32) k_hex8_gather(int64_t nn, const int *__restrict__ iptr,
                                                                const int *__restrict__ inc,
                                                                const int64_t *__restrict__ elems,
                                                                const int *__restrict__ cne,
                                                                const double *__restrict__ kbuf,
                                                                const int *__restrict__ rowptr,
                                                                const int *__restrict__ col,
                                                                double *__restrict__ val, unsigned *err) {
  __shared__ HexGatherShared shm[kRowWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  HexGatherShared &sh = shm[wib];
  // lane (b, i): node b of the element, row component i
  const int b = lane < 24 ? lane / 3 : 0, i = lane < 24 ? lane - 3 * (lane / 3) : 0;
  for (int64_t node = blockIdx.x * (int64_t)kRowWarps + wib; node < nn; node += (int64_t)gridDim.x * kRowWarps) {
    const int ib = iptr[node], deg = iptr[node + 1] - ib;
    if (deg == 0) continue;
    if (deg > kIncCap) {
      if (lane == 0) atomicOr(err, 32u);
      continue;
    }
    // incident elements in ascending order (distinct ids: rank sort), and
    // the node's index in each
    const int mine = lane < deg ? inc[ib + lane] : INT_MAX;
    int rank = 0;
    for (int k = 0; k < deg; k++) rank += __shfl_sync(0xffffffffu, mine, k) < mine;
    if (lane < deg) sh.inc[rank] = mine;
    __syncwarp();
    for (int t = lane; t < 8 * deg; t += 32) {
      const int q = t >> 3, a = t & 7;
      if (elems[(int64_t)sh.inc[q] * 8 + a] == node) sh.la[q] = a;
    }
    __syncwarp();
    // the node's rows: its code numbers in its first element
    int r[3], len[3];
    bool fits = true;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      r[c] = __ldg(cne + (int64_t)sh.inc[0] * 24 + 3 * sh.la[0] + c);
      len[c] = 0;
      if (r[c] >= 0) {
        const int rb = __ldg(rowptr + r[c]);
        len[c] = __ldg(rowptr + r[c] + 1) - rb;
        if (len[c] > kRowCap) {
          fits = false;
        } else {
          for (int k = lane; k < len[c]; k += 32) {
            sh.col[c][k] = __ldg(col + rb + k);
            sh.acc[c][k] = 0.0;
          }
        }
      }
    }
    if (!fits) {
      if (lane == 0) atomicOr(err, 32u);
      __syncwarp();
      continue;
    }
    if (r[0] < 0 && r[1] < 0 && r[2] < 0) {
      __syncwarp();
      continue;  // a fully constrained node has no rows
    }
    __syncwarp();
    for (int q0 = 0; q0 < deg; q0 += kGatherBatch) {
      // row i of block (la, b) of up to kGatherBatch elements and node b's
      // code numbers, all loads issued before the first is used
      double kr[kGatherBatch][3];
      int cc[kGatherBatch][3];
#pragma unroll
      for (int u = 0; u < kGatherBatch; u++) {
        const int q = q0 + u;
        kr[u][0] = kr[u][1] = kr[u][2] = 0.0;
        cc[u][0] = cc[u][1] = cc[u][2] = -1;
        if (q < deg && lane < 24 && r[i] >= 0) {
          const int e = sh.inc[q], la = sh.la[q];
          const double *eb = kbuf + (size_t)e * 324;
          if (la == b) {
            const double *blk = eb + 9 * (28 + la);
#pragma unroll
            for (int j = 0; j < 3; j++) kr[u][j] = __ldg(blk + 3 * i + j);
          } else if (la < b) {
            const double *blk = eb + 9 * upper_slot(la, b);
#pragma unroll
            for (int j = 0; j < 3; j++) kr[u][j] = __ldg(blk + 3 * i + j);
          } else {  // K_{la,b} = K_{b,la}^T
            const double *blk = eb + 9 * upper_slot(b, la);
#pragma unroll
            for (int j = 0; j < 3; j++) kr[u][j] = __ldg(blk + 3 * j + i);
          }
#pragma unroll
          for (int j = 0; j < 3; j++) cc[u][j] = __ldg(cne + (int64_t)e * 24 + 3 * b + j);
        }
      }
#pragma unroll
      for (int u = 0; u < kGatherBatch; u++) {
        // the elements in ascending order: one element's blocks at a time
        if (q0 + u < deg && lane < 24 && r[i] >= 0) {
          const int *cols = sh.col[i];
          double *acc = sh.acc[i];
          const int c0 = cc[u][0], c1 = cc[u][1], c2 = cc[u][2];
          bool done = false;
          if (c0 >= 0 && c1 == c0 + 1 && c2 == c0 + 2) {  // a fully free node: one search
            const int p = find_col_sh(cols, len[i], c0);
            if (p >= 0 && p + 2 < len[i] && cols[p + 1] == c1 && cols[p + 2] == c2) {
              acc[p] += kr[u][0];
              acc[p + 1] += kr[u][1];
              acc[p + 2] += kr[u][2];
              done = true;
            }
          }
          if (!done) {
#pragma unroll
            for (int j = 0; j < 3; j++) {
              if (cc[u][j] < 0) continue;
              const int p = find_col_sh(cols, len[i], cc[u][j]);
              if (p >= 0) acc[p] += kr[u][j];
              else atomicOr(err, 4u);
            }
          }
        }
        __syncwarp();
      }
    }
    // every entry of the node's rows, written once
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (r[c] < 0) continue;
      double *dst = val + __ldg(rowptr + r[c]);
      for (int k = lane; k < len[c]; k += 32) dst[k] = sh.acc[c][k];
    }
    __syncwarp();
  }
}

// tet4 elasticity (lintet::stiffness_matrix, MEFEL/SRC/lintet.cpp:290-315):
// the linear tetrahedron's gradients are constant, so one integration point
// with weight det3d/6 (GEFEL/matrix.cpp:3629) gives block (a,b) =
// det/6 B_a^T D B_b, B rows [xx, yy, zz, yz, xz, xy] as for the hexahedron
// (lintet::geom_matrix, :213-240).  The gradients follow derivatives_3d
// (GEFEL/difcalc.cpp:487-565) with the natural derivatives
// (1,0,0,-1), (0,1,0,-1), (0,0,1,-1) of dx/dy/dz_bf_lin_tet.  A negative
// det3d sets err bit 8 (the reference aborts on wrong node numbering).
// Half a warp per element, lane (a,b) of the 4 x 4 node blocks; lanes 0..11
// of a half load the 12 coordinates.
template <bool GEN>
__global__ void __launch_bounds__(TPB) k_tet4_elastic(int ne_c, const int *__restrict__ elist,
                                                      const double *__restrict__ coords,
                                                      const int64_t *__restrict__ elems,
                                                      const int *__restrict__ cne, const double *__restrict__ emat,
                                                      const int *__restrict__ rowptr, const int *__restrict__ col,
                                                      double *__restrict__ val, unsigned *err) {
  const int lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
  const int warp = (int)((blockIdx.x * (unsigned)TPB + threadIdx.x) >> 5);
  const int nwarps = gridDim.x * WPB;
  // every lane runs the same trips (the shuffles need the whole warp)
  for (int t0 = 2 * warp; t0 < ne_c; t0 += 2 * nwarps) {
    const int t = t0 + half;
    const bool live = t < ne_c;
    const int e = live ? elist[t] : 0;
    double cv = 0.0;
    if (live && hl < 12) cv = coords[3 * elems[(int64_t)e * 4 + hl / 3] + hl % 3];
    double x[4], y[4], z[4];
#pragma unroll
    for (int a = 0; a < 4; a++) {
      x[a] = __shfl_sync(0xffffffffu, cv, 16 * half + 3 * a);
      y[a] = __shfl_sync(0xffffffffu, cv, 16 * half + 3 * a + 1);
      z[a] = __shfl_sync(0xffffffffu, cv, 16 * half + 3 * a + 2);
    }
    if (!live) continue;
    // det3d: (p0-p3) . ((p1-p3) x (p2-p3)); the Jacobian columns are the
    // same differences (d1..d9 of derivatives_3d)
    const double d1 = x[0] - x[3], d2 = x[1] - x[3], d3 = x[2] - x[3];
    const double d4 = y[0] - y[3], d5 = y[1] - y[3], d6 = y[2] - y[3];
    const double d7 = z[0] - z[3], d8 = z[1] - z[3], d9 = z[2] - z[3];
    const double det = d1 * d5 * d9 + d2 * d6 * d7 + d3 * d4 * d8 - d3 * d5 * d7 - d6 * d8 * d1 - d9 * d2 * d4;
    if (det < 0.0) {
      if (hl == 0) atomicOr(err, 8u);
      continue;
    }
    const double jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 - d9 * d4 * d2;
    // rows of the inverse Jacobian: gradient of node a = natural (nx,ny,nz) . rows
    const double r00 = (d5 * d9 - d8 * d6) / jac, r01 = (d7 * d6 - d9 * d4) / jac, r02 = (d4 * d8 - d7 * d5) / jac;
    const double r10 = (d8 * d3 - d9 * d2) / jac, r11 = (d1 * d9 - d7 * d3) / jac, r12 = (d7 * d2 - d8 * d1) / jac;
    const double r20 = (d2 * d6 - d5 * d3) / jac, r21 = (d4 * d3 - d6 * d1) / jac, r22 = (d1 * d5 - d4 * d2) / jac;
    const int a = hl >> 2, b = hl & 3;
    // node 3 has natural derivatives (-1,-1,-1); nodes 0..2 pick one column
    double ax, ay, az, bx, by, bz;
    if (a < 3) {
      ax = a == 0 ? r00 : (a == 1 ? r01 : r02);
      ay = a == 0 ? r10 : (a == 1 ? r11 : r12);
      az = a == 0 ? r20 : (a == 1 ? r21 : r22);
    } else {
      ax = -(r00 + r01 + r02); ay = -(r10 + r11 + r12); az = -(r20 + r21 + r22);
    }
    if (b < 3) {
      bx = b == 0 ? r00 : (b == 1 ? r01 : r02);
      by = b == 0 ? r10 : (b == 1 ? r11 : r12);
      bz = b == 0 ? r20 : (b == 1 ? r21 : r22);
    } else {
      bx = -(r00 + r01 + r02); by = -(r10 + r11 + r12); bz = -(r20 + r21 + r22);
    }
    const double w = det / 6.0;
    double db[6][3];
    if (GEN) {
      double D[36];
#pragma unroll
      for (int q = 0; q < 36; q++) D[q] = __ldg(emat + 36 * (int64_t)e + q);
      elastic_db(D, bx, by, bz, db);
    } else {
      const double E = emat[2 * (int64_t)e], nu = emat[2 * (int64_t)e + 1];
      const double G = E / 2.0 / (1.0 + nu);
      const double s = E / (1.0 + nu) / (1.0 - 2.0 * nu);
      const double c0 = s * (1 - nu), c1 = s * nu;
      db[0][0] = c0 * bx; db[0][1] = c1 * by; db[0][2] = c1 * bz;
      db[1][0] = c1 * bx; db[1][1] = c0 * by; db[1][2] = c1 * bz;
      db[2][0] = c1 * bx; db[2][1] = c1 * by; db[2][2] = c0 * bz;
      db[3][0] = 0.0;     db[3][1] = G * bz;  db[3][2] = G * by;
      db[4][0] = G * bz;  db[4][1] = 0.0;     db[4][2] = G * bx;
      db[5][0] = G * by;  db[5][1] = G * bx;  db[5][2] = 0.0;
    }
    double k[3][3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      k[0][j] = w * (ax * db[0][j] + az * db[4][j] + ay * db[5][j]);
      k[1][j] = w * (ay * db[1][j] + az * db[3][j] + ax * db[5][j]);
      k[2][j] = w * (az * db[2][j] + ay * db[3][j] + ax * db[4][j]);
    }
    int rr[3], cc[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      rr[i] = __ldg(cne + (int64_t)e * 12 + 3 * a + i);
      cc[i] = __ldg(cne + (int64_t)e * 12 + 3 * b + i);
    }
    block3_add(rowptr, col, val, rr, cc, k, err);
  }
}

// quad4 plane stress (planeelemlq::gl_stiffness_matrix, MEFEL/SRC/plelemlq.cpp:611-690):
// B rows [xx, yy, xy] (geom_matrix, :294-320), D plane stress
// (elastisomat::matstiff_plstress, MEFEL/SRC/elastisomat.cpp:255), thickness
// interpolated at the Gauss point from nodal values (here all equal to the
// element's cross-section thickness, mechcrsec::give_thickness :397-411)
struct QuadShared {
  double g[4][4][2];
  double w[4];
};

__global__ void __launch_bounds__(TPB) k_quad4_elastic(int ne_c, const int *__restrict__ elist,
                                                       const double *__restrict__ coords,
                                                       const int64_t *__restrict__ elems,
                                                       const int *__restrict__ cne, const double *__restrict__ emat,
                                                       const double *__restrict__ thick,
                                                       const int *__restrict__ rowptr, const int *__restrict__ col,
                                                       double *__restrict__ val, unsigned *err) {
  __shared__ QuadShared shm[WPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  QuadShared &sh = shm[wib];
  for (int t = blockIdx.x * WPB + wib; t < ne_c; t += gridDim.x * WPB) {
    const int e = elist[t];
    double x[4], y[4], cx = 0, cy = 0;
    if (lane < 4) {
      const int64_t nd = elems[(int64_t)e * 4 + lane];
      cx = coords[3 * nd]; cy = coords[3 * nd + 1];
    }
#pragma unroll
    for (int a = 0; a < 4; a++) {
      x[a] = __shfl_sync(0xffffffffu, cx, a);
      y[a] = __shfl_sync(0xffffffffu, cy, a);
    }
    const double t_e = thick[e];
    if (lane < 4) {
      const double xi = c_gp2[(lane >> 1) & 1], eta = c_gp2[lane & 1];
      // bf_lin_4_2d derivatives (GEFEL/basefun.cpp:609-655)
      const double nx[4] = {0.25 * (1.0 + eta), 0.25 * (-1.0 - eta), 0.25 * (-1.0 + eta), 0.25 * (1.0 - eta)};
      const double ny[4] = {0.25 * (1.0 + xi), 0.25 * (1.0 - xi), 0.25 * (-1.0 + xi), 0.25 * (-1.0 - xi)};
      const double n[4] = {0.25 * (1.0 + xi) * (1.0 + eta), 0.25 * (1.0 - xi) * (1.0 + eta),
                           0.25 * (1.0 - xi) * (1.0 - eta), 0.25 * (1.0 + xi) * (1.0 - eta)};
      double d1 = 0, d2 = 0, d3 = 0, d4 = 0, th = 0;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        d1 += nx[a] * x[a]; d2 += ny[a] * x[a]; d3 += nx[a] * y[a]; d4 += ny[a] * y[a];
        th += n[a] * t_e;
      }
      const double jac = d1 * d4 - d2 * d3;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        sh.g[lane][a][0] = (nx[a] * d4 - ny[a] * d3) / jac;
        sh.g[lane][a][1] = (ny[a] * d1 - nx[a] * d2) / jac;
      }
      sh.w[lane] = fabs(jac * th);
    }
    __syncwarp();
    const double E = emat[2 * (int64_t)e], nu = emat[2 * (int64_t)e + 1];
    const double c = E / (1.0 - nu * nu), d01 = c * nu, g3 = E / 2.0 / (1.0 + nu);
    if (lane < 16) {
      const int a = lane >> 2, b = lane & 3;
      double k00 = 0, k01 = 0, k10 = 0, k11 = 0;
#pragma unroll
      for (int gp = 0; gp < 4; gp++) {
        const double ax = sh.g[gp][a][0], ay = sh.g[gp][a][1];
        const double bx = sh.g[gp][b][0], by = sh.g[gp][b][1];
        const double w = sh.w[gp];
        // D B_b (rows xx, yy, xy; columns u, v)
        const double db00 = c * bx, db01 = d01 * by, db10 = d01 * bx, db11 = c * by, db20 = g3 * by, db21 = g3 * bx;
        k00 += w * (ax * db00 + ay * db20);
        k01 += w * (ax * db01 + ay * db21);
        k10 += w * (ay * db10 + ax * db20);
        k11 += w * (ay * db11 + ax * db21);
      }
      const int r0 = __ldg(cne + (int64_t)e * 8 + 2 * a), r1 = __ldg(cne + (int64_t)e * 8 + 2 * a + 1);
      const int c0 = __ldg(cne + (int64_t)e * 8 + 2 * b), c1 = __ldg(cne + (int64_t)e * 8 + 2 * b + 1);
      if (r0 >= 0) {
        if (c0 >= 0) csr_add(rowptr, col, val, r0, c0, k00, err);
        if (c1 >= 0) csr_add(rowptr, col, val, r0, c1, k01, err);
      }
      if (r1 >= 0) {
        if (c0 >= 0) csr_add(rowptr, col, val, r1, c0, k10, err);
        if (c1 >= 0) csr_add(rowptr, col, val, r1, c1, k11, err);
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// quadratic serendipity elements
// ---------------------------------------------------------------------------

// order-3 Gauss rule with the reference's constants (GEFEL/intp.cpp:34-43)
__constant__ double c_gp3[3] = {-0.774596669241483, 0.0, 0.774596669241483};
__constant__ double c_gw3[3] = {0.5555555555555555, 0.8888888888888888, 0.5555555555555555};
// natural node coordinates in SIFEL's order (bf_quad_hex_3d,
// GEFEL/basefun.cpp:2377-2403; bf_quad_4_2d, :708-718)
__constant__ signed char c_h20[20][3] = {
    {1, 1, 1},  {-1, 1, 1},  {-1, -1, 1},  {1, -1, 1},  {1, 1, -1},  {-1, 1, -1},  {-1, -1, -1},
    {1, -1, -1}, {0, 1, 1},  {-1, 0, 1},   {0, -1, 1},  {1, 0, 1},   {1, 1, 0},    {-1, 1, 0},
    {-1, -1, 0}, {1, -1, 0}, {0, 1, -1},   {-1, 0, -1}, {0, -1, -1}, {1, 0, -1}};
__constant__ signed char c_q8[8][2] = {{1, 1}, {-1, 1}, {-1, -1}, {1, -1}, {0, 1}, {-1, 0}, {0, -1}, {1, 0}};

// dN_a/d(xi, eta, zeta) of the 20-node serendipity hexahedron
__device__ __forceinline__ void hex20_dnat(int a, double xi, double eta, double zeta, double &nx, double &ny,
                                           double &nz) {
  const double p = c_h20[a][0], q = c_h20[a][1], r = c_h20[a][2];
  const double fx = 1.0 + xi * p, fy = 1.0 + eta * q, fz = 1.0 + zeta * r;
  if (p != 0.0 && q != 0.0 && r != 0.0) {
    nx = p * fy * fz * (2.0 * xi * p + eta * q + zeta * r - 1.0) / 8.0;
    ny = q * fx * fz * (xi * p + 2.0 * eta * q + zeta * r - 1.0) / 8.0;
    nz = r * fx * fy * (xi * p + eta * q + 2.0 * zeta * r - 1.0) / 8.0;
  } else if (p == 0.0) {
    nx = -xi * fy * fz / 2.0;
    ny = q * (1.0 - xi * xi) * fz / 4.0;
    nz = r * (1.0 - xi * xi) * fy / 4.0;
  } else if (q == 0.0) {
    nx = p * (1.0 - eta * eta) * fz / 4.0;
    ny = -eta * fx * fz / 2.0;
    nz = r * (1.0 - eta * eta) * fx / 4.0;
  } else {
    nx = p * (1.0 - zeta * zeta) * fy / 4.0;
    ny = q * (1.0 - zeta * zeta) * fx / 4.0;
    nz = -zeta * fx * fy / 2.0;
  }
}

struct Hex20Shared {
  double g[27][20][3];  // Cartesian gradients [gp][node][x,y,z]
  double w[27];         // detJ w_i w_j w_k
  double D[36];
  double xyz[20][3];
};
constexpr int TPB20 = 128;
constexpr int WPB20 = TPB20 / 32;

// node pair (a, b), a <= b, number blk of the 210 upper-triangle pairs of a
// 20-node element in row order
__device__ __forceinline__ void pair20(int blk, int &a, int &b) {
  a = 0;
  while (blk >= 20 - a) {
    blk -= 20 - a;
    a++;
  }
  b = a + blk;
}

// hex20 elasticity (quadhex::stiffness_matrix, MEFEL/SRC/quadhex.cpp:232-270):
// 3 x 3 x 3 Gauss points (lane gp = 9 i + 3 j + k, the reference's loop order),
// B as for the linear hexahedron (quadhex::geom_matrix, :150-180), weight
// detJ w_i w_j w_k without an absolute value.  One warp per element, the
// gradients of all points in shared memory; each lane forms whole 3 x 3
// blocks (a, b), a <= b, and writes the block and its transpose.
template <bool GEN>
__global__ void __launch_bounds__(TPB20) k_hex20_elastic(int ne_c, const int *__restrict__ elist,
                                                         const double *__restrict__ coords,
                                                         const int64_t *__restrict__ elems,
                                                         const int *__restrict__ cne, const double *__restrict__ emat,
                                                         const int *__restrict__ rowptr, const int *__restrict__ col,
                                                         double *__restrict__ val, unsigned *err) {
  extern __shared__ double smem20[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  Hex20Shared &sh = reinterpret_cast<Hex20Shared *>(smem20)[wib];
  for (int t = blockIdx.x * WPB20 + wib; t < ne_c; t += gridDim.x * WPB20) {
    const int e = elist[t];
    if (lane < 20) {
      const int64_t nd = elems[(int64_t)e * 20 + lane];
      sh.xyz[lane][0] = coords[3 * nd];
      sh.xyz[lane][1] = coords[3 * nd + 1];
      sh.xyz[lane][2] = coords[3 * nd + 2];
    }
    if (GEN) {
      for (int q = lane; q < 36; q += 32) sh.D[q] = emat[36 * (int64_t)e + q];
    }
    __syncwarp();
    if (lane < 27) {
      const int i = lane / 9, j = (lane / 3) % 3, k = lane % 3;
      const double xi = c_gp3[i], eta = c_gp3[j], zeta = c_gp3[k];
      double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0, d9 = 0;
      for (int a = 0; a < 20; a++) {
        double nx, ny, nz;
        hex20_dnat(a, xi, eta, zeta, nx, ny, nz);
        const double x = sh.xyz[a][0], y = sh.xyz[a][1], z = sh.xyz[a][2];
        d1 += nx * x; d2 += ny * x; d3 += nz * x;
        d4 += nx * y; d5 += ny * y; d6 += nz * y;
        d7 += nx * z; d8 += ny * z; d9 += nz * z;
      }
      const double jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 - d9 * d4 * d2;
      for (int a = 0; a < 20; a++) {
        double ddx, ddy, ddz;
        hex20_dnat(a, xi, eta, zeta, ddx, ddy, ddz);
        sh.g[lane][a][0] = (ddx * (d5 * d9 - d8 * d6) + ddy * (d7 * d6 - d9 * d4) + ddz * (d4 * d8 - d7 * d5)) / jac;
        sh.g[lane][a][1] = (ddx * (d8 * d3 - d9 * d2) + ddy * (d1 * d9 - d7 * d3) + ddz * (d7 * d2 - d8 * d1)) / jac;
        sh.g[lane][a][2] = (ddx * (d2 * d6 - d5 * d3) + ddy * (d4 * d3 - d6 * d1) + ddz * (d1 * d5 - d4 * d2)) / jac;
      }
      sh.w[lane] = jac * (c_gw3[i] * c_gw3[j] * c_gw3[k]);
    }
    __syncwarp();
    double d0 = 0.0, d1 = 0.0, G = 0.0;
    if (!GEN) {
      const double E = emat[2 * (int64_t)e], nu = emat[2 * (int64_t)e + 1];
      G = E / 2.0 / (1.0 + nu);
      const double s = E / (1.0 + nu) / (1.0 - 2.0 * nu);
      d0 = s * (1 - nu);
      d1 = s * nu;
    }
    for (int blk = lane; blk < 210; blk += 32) {
      int a, b;
      pair20(blk, a, b);
      double k[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int gp = 0; gp < 27; gp++) {
        const double ax = sh.g[gp][a][0], ay = sh.g[gp][a][1], az = sh.g[gp][a][2];
        const double bx = sh.g[gp][b][0], by = sh.g[gp][b][1], bz = sh.g[gp][b][2];
        const double w = sh.w[gp];
        double db[6][3];
        if (GEN) {
          elastic_db(sh.D, bx, by, bz, db);
        } else {
          db[0][0] = d0 * bx; db[0][1] = d1 * by; db[0][2] = d1 * bz;
          db[1][0] = d1 * bx; db[1][1] = d0 * by; db[1][2] = d1 * bz;
          db[2][0] = d1 * bx; db[2][1] = d1 * by; db[2][2] = d0 * bz;
          db[3][0] = 0.0;     db[3][1] = G * bz;  db[3][2] = G * by;
          db[4][0] = G * bz;  db[4][1] = 0.0;     db[4][2] = G * bx;
          db[5][0] = G * by;  db[5][1] = G * bx;  db[5][2] = 0.0;
        }
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
          k[0][jj] += w * (ax * db[0][jj] + az * db[4][jj] + ay * db[5][jj]);
          k[1][jj] += w * (ay * db[1][jj] + az * db[3][jj] + ax * db[5][jj]);
          k[2][jj] += w * (az * db[2][jj] + ay * db[3][jj] + ax * db[4][jj]);
        }
      }
      int rr[3], cc[3];
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        rr[ii] = __ldg(cne + (int64_t)e * 60 + 3 * a + ii);
        cc[ii] = __ldg(cne + (int64_t)e * 60 + 3 * b + ii);
      }
      block3_add(rowptr, col, val, rr, cc, k, err);
      if (a != b) {
        double kt[3][3];
#pragma unroll
        for (int ii = 0; ii < 3; ii++)
#pragma unroll
          for (int jj = 0; jj < 3; jj++) kt[ii][jj] = k[jj][ii];
        block3_add(rowptr, col, val, cc, rr, kt, err);
      }
    }
    __syncwarp();
  }
}

struct Quad8Shared {
  double g[9][8][2];
  double w[9];
};

// quad8 plane stress (planeelemqq::stiffness_matrix, MEFEL/SRC/plelemqq.cpp:215-270):
// 3 x 3 Gauss (lane gp = 3 i + j), gradients by derivatives_2d, a negative
// detJ sets err bit 8 (the reference aborts), thickness interpolated from the
// nodal values (planeelemqq::approx, :102-112), weight detJ t w_i w_j; B rows
// [xx, yy, xy] (geom_matrix, :150-170), plane-stress D.  One warp per
// element, lanes cover the 64 node blocks of 2 x 2.
__global__ void __launch_bounds__(TPB) k_quad8_elastic(int ne_c, const int *__restrict__ elist,
                                                       const double *__restrict__ coords,
                                                       const int64_t *__restrict__ elems,
                                                       const int *__restrict__ cne, const double *__restrict__ emat,
                                                       const double *__restrict__ thick,
                                                       const int *__restrict__ rowptr, const int *__restrict__ col,
                                                       double *__restrict__ val, unsigned *err) {
  __shared__ Quad8Shared shm[WPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  Quad8Shared &sh = shm[wib];
  for (int t = blockIdx.x * WPB + wib; t < ne_c; t += gridDim.x * WPB) {
    const int e = elist[t];
    double cx = 0, cy = 0;
    if (lane < 8) {
      const int64_t nd = elems[(int64_t)e * 8 + lane];
      cx = coords[3 * nd];
      cy = coords[3 * nd + 1];
    }
    double x[8], y[8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
      x[a] = __shfl_sync(0xffffffffu, cx, a);
      y[a] = __shfl_sync(0xffffffffu, cy, a);
    }
    const double t_e = thick[e];
    bool bad = false;
    if (lane < 9) {
      const double xi = c_gp3[lane / 3], eta = c_gp3[lane % 3];
      double nx[8], ny[8], th = 0.0, d1 = 0, d2 = 0, d3 = 0, d4 = 0;
#pragma unroll
      for (int a = 0; a < 8; a++) {
        const double p = c_q8[a][0], q = c_q8[a][1], fx = 1.0 + xi * p, fy = 1.0 + eta * q;
        double n;
        if (p != 0.0 && q != 0.0) {
          n = 0.25 * fx * fy * (xi * p + eta * q - 1.0);
          nx[a] = 0.25 * p * fy * (2.0 * xi * p + eta * q);
          ny[a] = 0.25 * q * fx * (xi * p + 2.0 * eta * q);
        } else if (p == 0.0) {
          n = 0.5 * (1.0 - xi * xi) * fy;
          nx[a] = -xi * fy;
          ny[a] = 0.5 * q * (1.0 - xi * xi);
        } else {
          n = 0.5 * fx * (1.0 - eta * eta);
          nx[a] = 0.5 * p * (1.0 - eta * eta);
          ny[a] = -eta * fx;
        }
        th += n * t_e;
        d1 += nx[a] * x[a]; d2 += ny[a] * x[a]; d3 += nx[a] * y[a]; d4 += ny[a] * y[a];
      }
      const double jac = d1 * d4 - d2 * d3;
      bad = jac < 0.0;
#pragma unroll
      for (int a = 0; a < 8; a++) {
        sh.g[lane][a][0] = (nx[a] * d4 - ny[a] * d3) / jac;
        sh.g[lane][a][1] = (ny[a] * d1 - nx[a] * d2) / jac;
      }
      sh.w[lane] = jac * (th * c_gw3[lane / 3] * c_gw3[lane % 3]);
    }
    if (__any_sync(0xffffffffu, bad)) {
      if (lane == 0) atomicOr(err, 8u);
      continue;
    }
    __syncwarp();
    const double E = emat[2 * (int64_t)e], nu = emat[2 * (int64_t)e + 1];
    const double c = E / (1.0 - nu * nu), d01 = c * nu, g3 = E / 2.0 / (1.0 + nu);
    for (int blk = lane; blk < 64; blk += 32) {
      const int a = blk >> 3, b = blk & 7;
      double k00 = 0, k01 = 0, k10 = 0, k11 = 0;
#pragma unroll
      for (int gp = 0; gp < 9; gp++) {
        const double ax = sh.g[gp][a][0], ay = sh.g[gp][a][1];
        const double bx = sh.g[gp][b][0], by = sh.g[gp][b][1];
        const double w = sh.w[gp];
        const double db00 = c * bx, db01 = d01 * by, db10 = d01 * bx, db11 = c * by, db20 = g3 * by, db21 = g3 * bx;
        k00 += w * (ax * db00 + ay * db20);
        k01 += w * (ax * db01 + ay * db21);
        k10 += w * (ay * db10 + ax * db20);
        k11 += w * (ay * db11 + ax * db21);
      }
      const int r0 = __ldg(cne + (int64_t)e * 16 + 2 * a), r1 = __ldg(cne + (int64_t)e * 16 + 2 * a + 1);
      const int c0 = __ldg(cne + (int64_t)e * 16 + 2 * b), c1 = __ldg(cne + (int64_t)e * 16 + 2 * b + 1);
      if (r0 >= 0) {
        if (c0 >= 0) csr_add(rowptr, col, val, r0, c0, k00, err);
        if (c1 >= 0) csr_add(rowptr, col, val, r0, c1, k01, err);
      }
      if (r1 >= 0) {
        if (c0 >= 0) csr_add(rowptr, col, val, r1, c0, k10, err);
        if (c1 >= 0) csr_add(rowptr, col, val, r1, c1, k11, err);
      }
    }
    __syncwarp();
  }
}

// tri3 plane stress, the constant-strain triangle (planeelemlt::stiffness_matrix,
// MEFEL/SRC/plelemlt.cpp:234-272): det = twice the signed area, B from the
// area-coordinate coefficients b_i = (y_j - y_k)/det, c_i = (x_k - x_j)/det
// (plsb/plsc, GEFEL/basefun.cpp:394-416; geom_matrix, plelemlt.cpp:166-192),
// weight thick*det/2 with the thickness interpolated at (1/3, 1/3) through
// area coordinates (approx_nat, :119-131).  No sign check, as in the
// reference.  One thread per element: 3 x 3 node blocks of 2 x 2.
__global__ void __launch_bounds__(TPB) k_tri3_elastic(int ne_c, const int *__restrict__ elist,
                                                      const double *__restrict__ coords,
                                                      const int64_t *__restrict__ elems,
                                                      const int *__restrict__ cne, const double *__restrict__ emat,
                                                      const double *__restrict__ thick,
                                                      const int *__restrict__ rowptr, const int *__restrict__ col,
                                                      double *__restrict__ val, unsigned *err) {
  for (int t = blockIdx.x * TPB + threadIdx.x; t < ne_c; t += gridDim.x * TPB) {
    const int e = elist[t];
    double x[3], y[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int64_t nd = elems[(int64_t)e * 3 + a];
      x[a] = coords[3 * nd];
      y[a] = coords[3 * nd + 1];
    }
    const double det = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
    const double b[3] = {(y[1] - y[2]) / det, (y[2] - y[0]) / det, (y[0] - y[1]) / det};
    const double c[3] = {(x[2] - x[1]) / det, (x[0] - x[2]) / det, (x[1] - x[0]) / det};
    const double t_e = thick[e];
    const double third = 1.0 / 3.0;
    const double th = third * t_e + third * t_e + (1.0 - third - third) * t_e;
    const double w = th * det / 2.0;
    const double E = emat[2 * (int64_t)e], nu = emat[2 * (int64_t)e + 1];
    const double cc = E / (1.0 - nu * nu), d01 = cc * nu, g3 = E / 2.0 / (1.0 + nu);
    int code[6];
#pragma unroll
    for (int q = 0; q < 6; q++) code[q] = __ldg(cne + (int64_t)e * 6 + q);
#pragma unroll
    for (int a = 0; a < 3; a++) {
#pragma unroll
      for (int bb = 0; bb < 3; bb++) {
        // B_a^T D B_b with B_n = [[b_n, 0], [0, c_n], [c_n, b_n]]
        const double k00 = w * (b[a] * cc * b[bb] + c[a] * g3 * c[bb]);
        const double k01 = w * (b[a] * d01 * c[bb] + c[a] * g3 * b[bb]);
        const double k10 = w * (c[a] * d01 * b[bb] + b[a] * g3 * c[bb]);
        const double k11 = w * (c[a] * cc * c[bb] + b[a] * g3 * b[bb]);
        const int r0 = code[2 * a], r1 = code[2 * a + 1], c0 = code[2 * bb], c1 = code[2 * bb + 1];
        if (r0 >= 0) {
          if (c0 >= 0) csr_add(rowptr, col, val, r0, c0, k00, err);
          if (c1 >= 0) csr_add(rowptr, col, val, r0, c1, k01, err);
        }
        if (r1 >= 0) {
          if (c0 >= 0) csr_add(rowptr, col, val, r1, c0, k10, err);
          if (c1 >= 0) csr_add(rowptr, col, val, r1, c1, k11, err);
        }
      }
    }
  }
}

// hex8 conduction (linhext::conductivity_matrix, TRFEL/SRC/linhext.cpp:774-840,
// isotropic D = k I, isotrmat::matcond3d) or capacity
// (linhext::capacity_matrix, :979-1030: N^T N rho c |J| w)
template <bool CAPACITY>
__global__ void __launch_bounds__(TPB) k_hex8_scalar(int ne_c, const int *__restrict__ elist,
                                                     const double *__restrict__ coords,
                                                     const int64_t *__restrict__ elems,
                                                     const int *__restrict__ cne, const double *__restrict__ emat,
                                                     const double *__restrict__ rho,
                                                     const int *__restrict__ rowptr, const int *__restrict__ col,
                                                     double *__restrict__ val, unsigned *err) {
  __shared__ HexShared shm[WPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  HexShared &sh = shm[wib];
  for (int t = blockIdx.x * WPB + wib; t < ne_c; t += gridDim.x * WPB) {
    const int e = elist[t];
    double x[8], y[8], z[8], cx = 0, cy = 0, cz = 0;
    if (lane < 8) {
      const int64_t nd = elems[(int64_t)e * 8 + lane];
      cx = coords[3 * nd]; cy = coords[3 * nd + 1]; cz = coords[3 * nd + 2];
    }
#pragma unroll
    for (int a = 0; a < 8; a++) {
      x[a] = __shfl_sync(0xffffffffu, cx, a);
      y[a] = __shfl_sync(0xffffffffu, cy, a);
      z[a] = __shfl_sync(0xffffffffu, cz, a);
    }
    hex_gauss_point(lane, x, y, z, sh, CAPACITY);
    __syncwarp();
    const double kc = emat[2 * (int64_t)e], cc = emat[2 * (int64_t)e + 1];
    const double re = rho ? rho[e] : 1.0;
    for (int blk = lane; blk < 64; blk += 32) {
      const int a = blk >> 3, b = blk & 7;
      double v = 0.0;
#pragma unroll
      for (int gp = 0; gp < 8; gp++) {
        if (CAPACITY) {
          // rho interpolated from equal nodal densities: sum_a N_a rho
          double r = 0.0;
#pragma unroll
          for (int q = 0; q < 8; q++) r += sh.nb[gp][q] * re;
          v += (sh.nb[gp][a] * sh.nb[gp][b]) * (sh.w[gp] * r * cc);
        } else {
          const double gg = sh.g[gp][a][0] * sh.g[gp][b][0] + sh.g[gp][a][1] * sh.g[gp][b][1] +
                            sh.g[gp][a][2] * sh.g[gp][b][2];
          v += gg * kc * sh.w[gp];
        }
      }
      const int r = __ldg(cne + (int64_t)e * 8 + a), c = __ldg(cne + (int64_t)e * 8 + b);
      if (r >= 0 && c >= 0) csr_add(rowptr, col, val, r, c, v, err);
    }
    __syncwarp();
  }
}

// Dirichlet lifting of TRFEL's assemble_init (TRFEL/SRC/globmatt.cpp:1635-1760):
// for every element, r_e = the nodal values prescvalues() gives (prescribed
// values on prescribed DOFs, the initial values on free DOFs,
// globmatt.cpp:1057-1075), f_e = -K_e r_e, added to rhs at the free DOFs
// (locglob).  With time-constant prescribed values the capacity term of
// assemble_init, -C_e (r - r_prev)/dt, is zero and is not formed.
__global__ void __launch_bounds__(TPB) k_hex8t_lift(int ne_c, const int *__restrict__ elist,
                                                    const double *__restrict__ coords,
                                                    const int64_t *__restrict__ elems,
                                                    const int *__restrict__ cne, const double *__restrict__ emat,
                                                    const double *__restrict__ rnode, double *__restrict__ rhs) {
  __shared__ HexShared shm[WPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  HexShared &sh = shm[wib];
  for (int t = blockIdx.x * WPB + wib; t < ne_c; t += gridDim.x * WPB) {
    const int e = elist[t];
    double x[8], y[8], z[8], cx = 0, cy = 0, cz = 0, rv = 0;
    if (lane < 8) {
      const int64_t nd = elems[(int64_t)e * 8 + lane];
      cx = coords[3 * nd]; cy = coords[3 * nd + 1]; cz = coords[3 * nd + 2];
      rv = rnode[nd];
    }
    double r[8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
      x[a] = __shfl_sync(0xffffffffu, cx, a);
      y[a] = __shfl_sync(0xffffffffu, cy, a);
      z[a] = __shfl_sync(0xffffffffu, cz, a);
      r[a] = __shfl_sync(0xffffffffu, rv, a);
    }
    hex_gauss_point(lane, x, y, z, sh, false);
    __syncwarp();
    const double kc = emat[2 * (int64_t)e];
    if (lane < 8) {
      const int a = lane;
      double f = 0.0;
#pragma unroll
      for (int b = 0; b < 8; b++) {
        double kab = 0.0;
#pragma unroll
        for (int gp = 0; gp < 8; gp++) {
          const double gg = sh.g[gp][a][0] * sh.g[gp][b][0] + sh.g[gp][a][1] * sh.g[gp][b][1] +
                            sh.g[gp][a][2] * sh.g[gp][b][2];
          kab += gg * kc * sh.w[gp];
        }
        f += kab * r[b];
      }
      const int row = __ldg(cne + (int64_t)e * 8 + a);
      if (row >= 0) rhs[row] -= f;
    }
    __syncwarp();
  }
}

// MEFEL's prescribed displacements (loadcase::prdisplcontrib,
// MEFEL/SRC/loadcase.cpp:615-664): rhs -= K_e r_e at the element's equations,
// r_e the element's nodal values of rnode (nn x 3: the prescribed
// displacement at a prescribed DOF, 0 elsewhere).  One warp per element, as
// k_hex8_elastic: lane pair (a, b) forms block K_ab and K_ab r_b; the eight
// lanes of a row node sum their products.  Elements whose r_e is zero add
// nothing and return at once.  Colour-ordered: no two elements of a launch
// share a node.
template <bool GEN>
__global__ void __launch_bounds__(TPB) k_hex8_lift(int ne_c, const int *__restrict__ elist,
                                                   const double *__restrict__ coords,
                                                   const int64_t *__restrict__ elems, const int *__restrict__ cne,
                                                   const double *__restrict__ emat, const double *__restrict__ rnode,
                                                   double *__restrict__ rhs) {
  __shared__ HexShared shm[WPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  HexShared &sh = shm[wib];
  for (int t = blockIdx.x * WPB + wib; t < ne_c; t += gridDim.x * WPB) {
    const int e = elist[t];
    double cx = 0, cy = 0, cz = 0, r0 = 0, r1 = 0, r2 = 0;
    if (lane < 8) {
      const int64_t nd = elems[(int64_t)e * 8 + lane];
      cx = coords[3 * nd]; cy = coords[3 * nd + 1]; cz = coords[3 * nd + 2];
      r0 = rnode[3 * nd]; r1 = rnode[3 * nd + 1]; r2 = rnode[3 * nd + 2];
    }
    if (!__any_sync(0xffffffffu, r0 != 0.0 || r1 != 0.0 || r2 != 0.0)) continue;
    double x[8], y[8], z[8], r[8][3];
#pragma unroll
    for (int a = 0; a < 8; a++) {
      x[a] = __shfl_sync(0xffffffffu, cx, a);
      y[a] = __shfl_sync(0xffffffffu, cy, a);
      z[a] = __shfl_sync(0xffffffffu, cz, a);
      r[a][0] = __shfl_sync(0xffffffffu, r0, a);
      r[a][1] = __shfl_sync(0xffffffffu, r1, a);
      r[a][2] = __shfl_sync(0xffffffffu, r2, a);
    }
    hex_gauss_point(lane, x, y, z, sh, false);
    if (GEN) {
      for (int q = lane; q < 36; q += 32) sh.D[q] = emat[36 * (int64_t)e + q];
    }
    __syncwarp();
    double d0 = 0.0, d1 = 0.0, G = 0.0;
    if (!GEN) {
      const double E = emat[2 * (int64_t)e], nu = emat[2 * (int64_t)e + 1];
      G = E / 2.0 / (1.0 + nu);
      const double sc = E / (1.0 + nu) / (1.0 - 2.0 * nu);
      d0 = sc * (1 - nu);
      d1 = sc * nu;
    }
    // lanes 0..31: (a, b) = (lane >> 3, lane & 7) and (4 + (lane >> 3), lane & 7)
    double f[2][3] = {{0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int a = 4 * h + (lane >> 3), b = lane & 7;
      double k[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
      for (int gp = 0; gp < 8; gp++) {
        const double ax = sh.g[gp][a][0], ay = sh.g[gp][a][1], az = sh.g[gp][a][2];
        const double bx = sh.g[gp][b][0], by = sh.g[gp][b][1], bz = sh.g[gp][b][2];
        const double w = sh.w[gp];
        double db[6][3];
        if (GEN) {
          elastic_db(sh.D, bx, by, bz, db);
        } else {
          db[0][0] = d0 * bx; db[0][1] = d1 * by; db[0][2] = d1 * bz;
          db[1][0] = d1 * bx; db[1][1] = d0 * by; db[1][2] = d1 * bz;
          db[2][0] = d1 * bx; db[2][1] = d1 * by; db[2][2] = d0 * bz;
          db[3][0] = 0.0;     db[3][1] = G * bz;  db[3][2] = G * by;
          db[4][0] = G * bz;  db[4][1] = 0.0;     db[4][2] = G * bx;
          db[5][0] = G * by;  db[5][1] = G * bx;  db[5][2] = 0.0;
        }
#pragma unroll
        for (int j = 0; j < 3; j++) {
          k[0][j] += w * (ax * db[0][j] + az * db[4][j] + ay * db[5][j]);
          k[1][j] += w * (ay * db[1][j] + az * db[3][j] + ax * db[5][j]);
          k[2][j] += w * (az * db[2][j] + ay * db[3][j] + ax * db[4][j]);
        }
      }
#pragma unroll
      for (int i = 0; i < 3; i++) f[h][i] = k[i][0] * r[b][0] + k[i][1] * r[b][1] + k[i][2] * r[b][2];
    }
    // sum over b: the 8 lanes of one row node
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) f[h][i] += __shfl_xor_sync(0xffffffffu, f[h][i], o);
    if ((lane & 7) == 0) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int a = 4 * h + (lane >> 3);
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const int row = __ldg(cne + (int64_t)e * 24 + 3 * a + i);
          if (row >= 0) rhs[row] -= f[h][i];
        }
      }
    }
    __syncwarp();
  }
}

// The same for the plane-stress quad (planeelemlq): rnode nn x 2; 16 lanes
// (a, b) form K_ab r_b, the 4 lanes of a row node sum them.
__global__ void __launch_bounds__(TPB) k_quad4_lift(int ne_c, const int *__restrict__ elist,
                                                    const double *__restrict__ coords,
                                                    const int64_t *__restrict__ elems, const int *__restrict__ cne,
                                                    const double *__restrict__ emat, const double *__restrict__ thick,
                                                    const double *__restrict__ rnode, double *__restrict__ rhs) {
  __shared__ QuadShared shm[WPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  QuadShared &sh = shm[wib];
  for (int t = blockIdx.x * WPB + wib; t < ne_c; t += gridDim.x * WPB) {
    const int e = elist[t];
    double x[4], y[4], cx = 0, cy = 0, r0 = 0, r1 = 0;
    if (lane < 4) {
      const int64_t nd = elems[(int64_t)e * 4 + lane];
      cx = coords[3 * nd]; cy = coords[3 * nd + 1];
      r0 = rnode[2 * nd]; r1 = rnode[2 * nd + 1];
    }
    if (!__any_sync(0xffffffffu, r0 != 0.0 || r1 != 0.0)) continue;
    double r[4][2];
#pragma unroll
    for (int a = 0; a < 4; a++) {
      x[a] = __shfl_sync(0xffffffffu, cx, a);
      y[a] = __shfl_sync(0xffffffffu, cy, a);
      r[a][0] = __shfl_sync(0xffffffffu, r0, a);
      r[a][1] = __shfl_sync(0xffffffffu, r1, a);
    }
    const double t_e = thick[e];
    if (lane < 4) {
      const double xi = c_gp2[(lane >> 1) & 1], eta = c_gp2[lane & 1];
      const double nx[4] = {0.25 * (1.0 + eta), 0.25 * (-1.0 - eta), 0.25 * (-1.0 + eta), 0.25 * (1.0 - eta)};
      const double ny[4] = {0.25 * (1.0 + xi), 0.25 * (1.0 - xi), 0.25 * (-1.0 + xi), 0.25 * (-1.0 - xi)};
      const double n[4] = {0.25 * (1.0 + xi) * (1.0 + eta), 0.25 * (1.0 - xi) * (1.0 + eta),
                           0.25 * (1.0 - xi) * (1.0 - eta), 0.25 * (1.0 + xi) * (1.0 - eta)};
      double d1 = 0, d2 = 0, d3 = 0, d4 = 0, th = 0;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        d1 += nx[a] * x[a]; d2 += ny[a] * x[a]; d3 += nx[a] * y[a]; d4 += ny[a] * y[a];
        th += n[a] * t_e;
      }
      const double jac = d1 * d4 - d2 * d3;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        sh.g[lane][a][0] = (nx[a] * d4 - ny[a] * d3) / jac;
        sh.g[lane][a][1] = (ny[a] * d1 - nx[a] * d2) / jac;
      }
      sh.w[lane] = fabs(jac * th);
    }
    __syncwarp();
    const double E = emat[2 * (int64_t)e], nu = emat[2 * (int64_t)e + 1];
    const double c = E / (1.0 - nu * nu), d01 = c * nu, g3 = E / 2.0 / (1.0 + nu);
    double f0 = 0.0, f1 = 0.0;
    if (lane < 16) {
      const int a = lane >> 2, b = lane & 3;
      double k00 = 0, k01 = 0, k10 = 0, k11 = 0;
#pragma unroll
      for (int gp = 0; gp < 4; gp++) {
        const double ax = sh.g[gp][a][0], ay = sh.g[gp][a][1];
        const double bx = sh.g[gp][b][0], by = sh.g[gp][b][1];
        const double w = sh.w[gp];
        const double db00 = c * bx, db01 = d01 * by, db10 = d01 * bx, db11 = c * by, db20 = g3 * by, db21 = g3 * bx;
        k00 += w * (ax * db00 + ay * db20);
        k01 += w * (ax * db01 + ay * db21);
        k10 += w * (ay * db10 + ax * db20);
        k11 += w * (ay * db11 + ax * db21);
      }
      f0 = k00 * r[b][0] + k01 * r[b][1];
      f1 = k10 * r[b][0] + k11 * r[b][1];
    }
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
      f0 += __shfl_xor_sync(0xffffffffu, f0, o);
      f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    }
    if (lane < 16 && (lane & 3) == 0) {
      const int a = lane >> 2;
      const int row0 = __ldg(cne + (int64_t)e * 8 + 2 * a), row1 = __ldg(cne + (int64_t)e * 8 + 2 * a + 1);
      if (row0 >= 0) rhs[row0] -= f0;
      if (row1 >= 0) rhs[row1] -= f1;
    }
    __syncwarp();
  }
}

int read_err(const unsigned *err_d, cudaStream_t s, unsigned *out) {
  SGPU_CUDA(cudaMemcpyAsync(out, err_d, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  return SGPU_OK;
}

// greedy first-fit colouring over per-node colour masks: an element takes the
// lowest colour no element sharing one of its nodes already has
int colour_elements(int64_t nn, int64_t ne, int nne, const int64_t *elems, std::vector<int> &order,
                    std::vector<int> &offsets) {
  std::vector<uint64_t> mask((size_t)nn, 0);
  std::vector<int> colour((size_t)ne);
  int ncol = 0;
  for (int64_t e = 0; e < ne; e++) {
    uint64_t used = 0;
    for (int a = 0; a < nne; a++) used |= mask[(size_t)elems[e * nne + a]];
    if (used == ~0ull) return fail(SGPU_BAD_INPUT, "mesh needs more than 64 element colours");
    const int c = __builtin_ctzll(~used);
    colour[(size_t)e] = c;
    ncol = std::max(ncol, c + 1);
    for (int a = 0; a < nne; a++) mask[(size_t)elems[e * nne + a]] |= (1ull << c);
  }
  offsets.assign(ncol + 1, 0);
  for (int64_t e = 0; e < ne; e++) offsets[colour[(size_t)e] + 1]++;
  for (int c = 0; c < ncol; c++) offsets[c + 1] += offsets[c];
  order.resize((size_t)ne);
  std::vector<int> fill(offsets.begin(), offsets.end() - 1);
  for (int64_t e = 0; e < ne; e++) order[(size_t)fill[colour[(size_t)e]]++] = (int)e;
  return SGPU_OK;
}

// stream-ordered temporaries of the pattern build (the device pool keeps the
// memory between calls, so no cudaMalloc / cudaFree synchronisation)
template <class T>
struct AsyncBuf {
  T *p = nullptr;
  cudaStream_t s = nullptr;
  explicit AsyncBuf(cudaStream_t st) : s(st) {}
  AsyncBuf(const AsyncBuf &) = delete;
  AsyncBuf &operator=(const AsyncBuf &) = delete;
  ~AsyncBuf() {
    if (p) cudaFreeAsync(p, s);
  }
  int alloc(size_t count) {
    static bool pool_kept = false;
    if (!pool_kept) {
      int dev = 0;
      cudaMemPool_t pool;
      if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
      pool_kept = true;
    }
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocAsync((void **)&p, count * sizeof(T), s);
    if (e != cudaSuccess) return fail(SGPU_CUDA_ERROR, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    return SGPU_OK;
  }
};

// exclusive scan of `len` (n entries) into out (n+1 entries, out[n] = total)
template <class In, class Out>
int scan_into(const In *len, Out *out, int64_t n, cudaStream_t s) {
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, len, out, (int)n + 1, s);
  AsyncBuf<unsigned char> t(s);
  SGPU_TRY(t.alloc(tmp));
  cub::DeviceScan::ExclusiveSum(t.p, tmp, len, out, (int)n + 1, s);
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

// node -> element incidence: iptr[nn + 1] and the element ids of every node
// (in no particular order) in inc[ne * nne].  Returns 1 when the incidence
// does not fit int32 offsets.
int build_incidence(const int64_t *elems_d, int64_t nn, int64_t ne, int nne, DevBuf<int> &iptr, DevBuf<int> &inc,
                    cudaStream_t s) {
  const int64_t m_inc = ne * nne;
  if (m_inc > (1LL << 31) - 1) return 1;
  AsyncBuf<int> cnt(s), cursor(s);
  SGPU_TRY(cnt.alloc(nn + 1));
  SGPU_TRY(cursor.alloc(nn));
  SGPU_TRY(iptr.alloc(nn + 1));
  SGPU_TRY(inc.alloc(m_inc));
  SGPU_CUDA(cudaMemsetAsync(cnt.p, 0, (nn + 1) * sizeof(int), s));
  SGPU_CUDA(cudaMemsetAsync(cursor.p, 0, nn * sizeof(int), s));
  k_inc_count<<<blocks_for(m_inc), TPB, 0, s>>>(m_inc, elems_d, cnt.p);
  count_launches(1);
  SGPU_TRY(scan_into(cnt.p, iptr.p, nn, s));
  k_inc_fill<<<blocks_for(m_inc), TPB, 0, s>>>(m_inc, nne, elems_d, iptr.p, cursor.p, inc.p);
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

// The SCR pattern from the node adjacency when the code numbers grow with
// (node, component) (gencodnum's numbering): from the node -> element
// incidence (build_incidence), per-node sorted lower neighbours, row
// lengths, scan, fill.  Returns
// SGPU_OK, or 1 when a node has too many candidate neighbours (the caller
// uses the element-pair sort instead).  Writes m->src_adr / src_ci / src_negm.
int pattern_adjacency(sgpu_matrix m, const int64_t *elems_d, const int64_t *cn_d, int64_t nn, int nne, int ndofn,
                      int64_t n, const int *iptr_d, const int *inc_d, unsigned *err_d, cudaStream_t s) {
  AsyncBuf<int> ucnt(s), nadj(s);
  AsyncBuf<int64_t> nptr(s), rowlen(s);
  SGPU_TRY(ucnt.alloc(nn + 1));
  SGPU_CUDA(cudaMemsetAsync(ucnt.p, 0, (nn + 1) * sizeof(int), s));
  const int gadj = (int)std::min<int64_t>((nn + WPB - 1) / WPB, (int64_t)kNumSMs * 32);
  k_node_adj<false><<<gadj, TPB, 0, s>>>(nn, nne, elems_d, iptr_d, inc_d, ucnt.p, nullptr, nullptr, err_d);
  count_launches(1);
  unsigned e = 0;
  SGPU_TRY(read_err(err_d, s, &e));
  if (e & 16u) {
    SGPU_CUDA(cudaMemsetAsync(err_d, 0, sizeof(unsigned), s));
    return 1;
  }
  SGPU_TRY(nptr.alloc(nn + 1));
  SGPU_TRY(scan_into(ucnt.p, nptr.p, nn, s));
  int64_t nadj_total = 0;
  SGPU_CUDA(cudaMemcpyAsync(&nadj_total, nptr.p + nn, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  SGPU_TRY(nadj.alloc((size_t)nadj_total));
  k_node_adj<true><<<gadj, TPB, 0, s>>>(nn, nne, elems_d, iptr_d, inc_d, nullptr, nptr.p, nadj.p, err_d);
  SGPU_TRY(rowlen.alloc(n + 1));
  SGPU_CUDA(cudaMemsetAsync(rowlen.p, 0, (n + 1) * sizeof(int64_t), s));
  k_scr_rowlen<<<blocks_for(nn), TPB, 0, s>>>(nn, ndofn, cn_d, nptr.p, nadj.p, rowlen.p, n, err_d);
  count_launches(2);
  SGPU_TRY(m->src_adr.alloc(n + 1));
  SGPU_TRY(scan_into(rowlen.p, m->src_adr.p, n, s));
  int64_t negm = 0;
  SGPU_CUDA(cudaMemcpyAsync(&negm, m->src_adr.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SGPU_TRY(read_err(err_d, s, &e));
  if (e) return fail(SGPU_BAD_INPUT, "code numbers: element node out of range or unused equation");
  m->src_negm = negm;
  SGPU_TRY(m->src_ci.alloc(negm));
  k_scr_fill<<<blocks_for(nn), TPB, 0, s>>>(nn, ndofn, cn_d, nptr.p, nadj.p, m->src_adr.p, m->src_ci.p, n);
  count_launches(1);
  SGPU_CUDA(cudaGetLastError());
  return SGPU_OK;
}

}  // namespace

// Assembly state kept with the matrix handle so that values can be
// re-integrated (new materials, the capacity form) on the same pattern.
struct AssemblyData {
  int kind = 0, nne = 0, ndofn = 0;
  bool general = false;  // emat holds a 6 x 6 material stiffness per element
  int64_t nn = 0, ne = 0;
  DevBuf<double> coords, emat, thick, rho;
  DevBuf<int64_t> elems;
  DevBuf<int> cne, elist;
  std::vector<int> offsets;
  std::vector<int> order;  // the per-colour element lists on the host (ascending ids per colour)
  // node -> element incidence, and whether every equation belongs to one
  // (node, component) (gencodnum's consecutive numbering): the row kernel's
  // precondition
  DevBuf<int> iptr, inc;
  bool node_rows = false;
};

// SGPU_HEX8_FULL=1: isotropic hexahedra through the full B^T D B product of
// k_hex8_elastic instead of k_hex8_iso (read at every assembly)
bool hex8_full_product() {
  const char *e = std::getenv("SGPU_HEX8_FULL");
  return e && !strcmp(e, "1");
}

// SGPU_HEX8_GATHER=1: isotropic hexahedra through the element buffer and
// the row gather instead of the colour-ordered scatter (k_hex8_iso)
bool hex8_gather() {
  const char *e = std::getenv("SGPU_HEX8_GATHER");
  return e && !strcmp(e, "1");
}

// SGPU_HEX8_ROWCACHE=0: k_hex8_iso searches every block's row in global
// memory instead of in the shared-memory copy of the element's rows
bool hex8_row_cache() {
  const char *e = std::getenv("SGPU_HEX8_ROWCACHE");
  return !(e && !strcmp(e, "0"));
}

int assemble_values(sgpu_matrix m, AssemblyData &ad, int kind, float *ms_out) {
  cudaStream_t s = m->stream;
  Csr &c = m->csr;
  DevBuf<unsigned> err;
  SGPU_TRY(err.alloc(1));
  SGPU_CUDA(cudaMemsetAsync(err.p, 0, sizeof(unsigned), s));
  SGPU_CUDA(cudaEventRecord(m->ev0, s));
  // isotropic hex8 elasticity on gencodnum's numbering, SGPU_ASSEMBLY_ROWS=1:
  // rows formed per node and written once.  Not the default: on the 1.01M-DOF
  // cantilever it takes 3.71 ms against 3.24 ms for the colour-ordered
  // scatter (each element's gradients are formed by all 8 of its nodes' warps,
  // and 124 registers with 40 KB of shared memory per block leave 16 warps per SM)
  bool rows_done = false;
  const char *rows_env = std::getenv("SGPU_ASSEMBLY_ROWS");
  const bool rows_wanted = rows_env && !strcmp(rows_env, "1");
  if (kind == SGPU_ELEM_HEX8 && !ad.general && ad.node_rows && ad.iptr.p && rows_wanted) {
    const int grid = (int)std::min<int64_t>((ad.nn + kRowWarps - 1) / kRowWarps, (int64_t)kNumSMs * 64);
    k_hex8_rows<<<grid, kRowWarps * 32, 0, s>>>(ad.nn, ad.iptr.p, ad.inc.p, ad.coords.p, ad.elems.p, ad.cne.p,
                                                ad.emat.p, c.rowptr.p, c.col.p, c.val.p, err.p);
    count_launches(1);
    SGPU_CUDA(cudaGetLastError());
    unsigned e = 0;
    SGPU_TRY(read_err(err.p, s, &e));
    if (e & 32u) {  // a node beyond the kernel's shared-memory capacity: colour-ordered scatter instead
      SGPU_CUDA(cudaMemsetAsync(err.p, 0, sizeof(unsigned), s));
    } else {
      rows_done = true;
    }
  }
  // isotropic hex8 on gencodnum's numbering, SGPU_HEX8_GATHER=1: element
  // blocks into a buffer, then every node's rows gathered and written once
  // (k_hex8_gather).  The value array is cleared first: a node without
  // elements has rows that no warp writes.
  if (!rows_done && kind == SGPU_ELEM_HEX8 && !ad.general && ad.node_rows && ad.iptr.p && hex8_gather() &&
      !hex8_full_product()) {
    AsyncBuf<double> kbuf(s);
    SGPU_TRY(kbuf.alloc((size_t)ad.ne * 324));
    SGPU_CUDA(cudaMemsetAsync(c.val.p, 0, (size_t)c.nnz * sizeof(double), s));
    const int g1 = (int)std::min<int64_t>((ad.ne + WPB - 1) / WPB, (int64_t)kNumSMs * 16);
    k_hex8_iso<false, true><<<g1, TPB, 0, s>>>((int)ad.ne, nullptr, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                c.rowptr.p, c.col.p, c.val.p, err.p, kbuf.p);
    const int g2 = (int)std::min<int64_t>((ad.nn + kRowWarps - 1) / kRowWarps, (int64_t)kNumSMs * 64);
    k_hex8_gather<<<g2, kRowWarps * 32, 0, s>>>(ad.nn, ad.iptr.p, ad.inc.p, ad.elems.p, ad.cne.p, kbuf.p,
                                                c.rowptr.p, c.col.p, c.val.p, err.p);
    count_launches(2);
    SGPU_CUDA(cudaGetLastError());
    unsigned e = 0;
    SGPU_TRY(read_err(err.p, s, &e));
    if (e & 32u) {  // a node beyond the gather's shared-memory capacity: colour-ordered scatter instead
      SGPU_CUDA(cudaMemsetAsync(err.p, 0, sizeof(unsigned), s));
    } else {
      rows_done = true;
    }
  }
  if (!rows_done) SGPU_CUDA(cudaMemsetAsync(c.val.p, 0, (size_t)c.nnz * sizeof(double), s));
  // SGPU_ASSEMBLY_SLABS=k: k slabs of element ids, all colours of a slab
  // before the next slab, so that the colours of a slab meet its rows in L2
  // instead of reading and writing the value array from DRAM once per colour.
  // Within a launch no two elements share a node (one colour) and launches
  // run in stream order, so the scatter needs no atomics either way; the order
  // of each entry's sum is fixed by the slab count.  Not the default: on the
  // 1.01M-DOF cantilever the colour-major order (one slab) takes 2.03 ms, 4
  // slabs 2.27 ms, 20 slabs (48 MB of rows each) 2.79 ms, 64 slabs 6.05 ms --
  // the smaller launches lose more than L2 reuse gains.
  const int ncol = rows_done ? 0 : (int)ad.offsets.size() - 1;
  int nslab = 1;
  if (const char *se = std::getenv("SGPU_ASSEMBLY_SLABS"))
    nslab = (int)std::max<int64_t>(1, std::min<int64_t>(std::min(256, atoi(se)), ad.ne));
  for (int pass = 0; pass < ncol * nslab; pass++) {
    const int sl = pass / ncol, col = pass % ncol;
    const int *cb = ad.order.data() + ad.offsets[col], *ce = ad.order.data() + ad.offsets[col + 1];
    const int lo = (int)(sl * ad.ne / nslab), hi = (int)((sl + 1) * ad.ne / nslab);
    const int beg = (int)(std::lower_bound(cb, ce, lo) - ad.order.data());
    const int end = (int)(std::lower_bound(cb, ce, hi) - ad.order.data());
    const int cnt = end - beg;
    if (cnt == 0) continue;
    const int grid = std::min((cnt + WPB - 1) / WPB, kNumSMs * 16);
    const int *el = ad.elist.p + beg;
    switch (kind) {
      case 0:
        if (ad.general)
          k_hex8_elastic<true><<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                    c.rowptr.p, c.col.p, c.val.p, err.p);
        else if (hex8_full_product())
          k_hex8_elastic<false><<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                     c.rowptr.p, c.col.p, c.val.p, err.p);
        else if (hex8_row_cache())
          k_hex8_iso<true, false><<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                       c.rowptr.p, c.col.p, c.val.p, err.p, nullptr);
        else
          k_hex8_iso<false, false><<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                        c.rowptr.p, c.col.p, c.val.p, err.p, nullptr);
        break;
      case 1:
        k_quad4_elastic<<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p, ad.thick.p,
                                             c.rowptr.p, c.col.p, c.val.p, err.p);
        break;
      case 4: {
        const int g4 = std::min((cnt + 2 * WPB - 1) / (2 * WPB), kNumSMs * 16);
        if (ad.general)
          k_tet4_elastic<true><<<g4, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                  c.rowptr.p, c.col.p, c.val.p, err.p);
        else
          k_tet4_elastic<false><<<g4, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                   c.rowptr.p, c.col.p, c.val.p, err.p);
        break;
      }
      case 6: {
        const int g6 = std::min((cnt + WPB20 - 1) / WPB20, kNumSMs * 8);
        const size_t sm = WPB20 * sizeof(Hex20Shared);
        if (ad.general) {
          SGPU_CUDA(cudaFuncSetAttribute(k_hex20_elastic<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
          k_hex20_elastic<true><<<g6, TPB20, sm, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                      c.rowptr.p, c.col.p, c.val.p, err.p);
        } else {
          SGPU_CUDA(cudaFuncSetAttribute(k_hex20_elastic<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
          k_hex20_elastic<false><<<g6, TPB20, sm, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                       c.rowptr.p, c.col.p, c.val.p, err.p);
        }
        break;
      }
      case 7:
        k_quad8_elastic<<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p, ad.thick.p,
                                             c.rowptr.p, c.col.p, c.val.p, err.p);
        break;
      case 5: {
        const int g5 = std::min((cnt + TPB - 1) / TPB, kNumSMs * 16);
        k_tri3_elastic<<<g5, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p, ad.thick.p,
                                          c.rowptr.p, c.col.p, c.val.p, err.p);
        break;
      }
      case 2:
        k_hex8_scalar<false><<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p, nullptr,
                                                  c.rowptr.p, c.col.p, c.val.p, err.p);
        break;
      default:
        k_hex8_scalar<true><<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p,
                                                 ad.rho.p ? ad.rho.p : nullptr, c.rowptr.p, c.col.p, c.val.p,
                                                 err.p);
        break;
    }
    count_launches(1);
    SGPU_CUDA(cudaGetLastError());
  }
  SGPU_CUDA(cudaEventRecord(m->ev1, s));
  unsigned e = 0;
  SGPU_TRY(read_err(err.p, s, &e));
  if (e & 8u) return fail(SGPU_BAD_INPUT, "element of negative volume or Jacobian (wrong node numbering)");
  if (e) return fail(SGPU_BAD_INPUT, "element scatter found no CSR entry (bits " + std::to_string(e) + ")");
  float ms = 0.f;
  SGPU_CUDA(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
  if (ms_out) *ms_out = ms;
  return SGPU_OK;
}

}  // namespace sgpu

using namespace sgpu;

struct sgpu_assembly_s {
  sgpu::AssemblyData d;
};

extern "C" {

SGPU_API int sgpu_assemble(const sgpu_mesh *mesh, sgpu_matrix *out, sgpu_assembly_info *info) {
  if (!mesh || !out) return fail(SGPU_BAD_INPUT, "null argument");
  *out = nullptr;
  if (info) memset(info, 0, sizeof(*info));
  const int kind = mesh->kind;
  int nne, ndofn;
  switch (kind) {
    case SGPU_ELEM_HEX8: nne = 8; ndofn = 3; break;
    case SGPU_ELEM_QUAD4: nne = 4; ndofn = 2; break;
    case SGPU_ELEM_TET4: nne = 4; ndofn = 3; break;
    case SGPU_ELEM_TRI3: nne = 3; ndofn = 2; break;
    case SGPU_ELEM_HEX20: nne = 20; ndofn = 3; break;
    case SGPU_ELEM_QUAD8: nne = 8; ndofn = 2; break;
    case SGPU_ELEM_HEX8T_K:
    case SGPU_ELEM_HEX8T_C: nne = 8; ndofn = 1; break;
    default: return fail(SGPU_BAD_INPUT, "unknown element kind");
  }
  if (mesh->ndofn != ndofn) return fail(SGPU_BAD_INPUT, "ndofn does not match the element kind");
  if (mesh->nn <= 0 || mesh->ne <= 0 || !mesh->coords || !mesh->elems || !mesh->cn || (!mesh->emat && !mesh->dmat))
    return fail(SGPU_BAD_INPUT, "empty mesh");
  if (mesh->dmat && kind != SGPU_ELEM_HEX8 && kind != SGPU_ELEM_TET4 && kind != SGPU_ELEM_HEX20)
    return fail(SGPU_BAD_INPUT, "general material matrices are defined for the 3D elasticity kinds");
  if ((kind == SGPU_ELEM_QUAD4 || kind == SGPU_ELEM_TRI3 || kind == SGPU_ELEM_QUAD8) && !mesh->thick)
    return fail(SGPU_BAD_INPUT, "plane elements need thicknesses");
  if (mesh->ne > (1LL << 31) - 1) return fail(SGPU_BAD_INPUT, "too many elements");
  const int64_t nn = mesh->nn, ne = mesh->ne;
  const int ndofe = nne * ndofn;
  // number of equations = largest code number
  int64_t n = 0;
  for (int64_t q = 0; q < nn * ndofn; q++) n = std::max<int64_t>(n, mesh->cn[q]);
  if (n <= 0) return fail(SGPU_BAD_INPUT, "no free equations");
  for (int64_t q = 0; q < ne * nne; q++)
    if (mesh->elems[q] < 0 || mesh->elems[q] >= nn) return fail(SGPU_BAD_INPUT, "element node out of range");

  sgpu_matrix m = new sgpu_matrix_s();
  m->n = n;
  m->src_sym = 1;
  auto bail = [&](int st) {
    if (m->stream) cudaStreamSynchronize(m->stream);
    cudaStream_t s = m->own_stream;
    cudaEvent_t a = m->ev0, b = m->ev1;
    delete m;
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (s) cudaStreamDestroy(s);
    return st;
  };
  if (cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&m->ev0) != cudaSuccess || cudaEventCreate(&m->ev1) != cudaSuccess)
    return bail(fail(SGPU_CUDA_ERROR, "stream/event creation failed"));
  m->stream = m->own_stream;
  cudaStream_t s = m->stream;
  m->asm_data = new sgpu_assembly_s();
  AssemblyData &ad = m->asm_data->d;
  ad.kind = kind; ad.nne = nne; ad.ndofn = ndofn; ad.nn = nn; ad.ne = ne;
  int st;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, s);
#define BAIL_ON(x)                        \
  do {                                    \
    st = (x);                             \
    if (st != SGPU_OK) {                  \
      cudaEventDestroy(t0);               \
      cudaEventDestroy(t1);               \
      return bail(st);                    \
    }                                     \
  } while (0)
  BAIL_ON(ad.coords.alloc(nn * 3));
  BAIL_ON(ad.elems.alloc(ne * nne));
  ad.general = mesh->dmat != nullptr;
  const int64_t nmatp = ad.general ? 36 : 2;
  BAIL_ON(ad.emat.alloc(ne * nmatp));
  DevBuf<int64_t> cn_d;
  BAIL_ON(cn_d.alloc(nn * ndofn));
  BAIL_ON(ad.cne.alloc(ne * ndofe));
  cudaMemcpyAsync(ad.coords.p, mesh->coords, nn * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(ad.elems.p, mesh->elems, ne * nne * sizeof(int64_t), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(ad.emat.p, ad.general ? mesh->dmat : mesh->emat, ne * nmatp * sizeof(double),
                  cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(cn_d.p, mesh->cn, nn * ndofn * sizeof(int64_t), cudaMemcpyHostToDevice, s);
  if (mesh->thick) {
    BAIL_ON(ad.thick.alloc(ne));
    cudaMemcpyAsync(ad.thick.p, mesh->thick, ne * sizeof(double), cudaMemcpyHostToDevice, s);
  }
  if (mesh->rho) {
    BAIL_ON(ad.rho.alloc(ne));
    cudaMemcpyAsync(ad.rho.p, mesh->rho, ne * sizeof(double), cudaMemcpyHostToDevice, s);
  }
  DevBuf<unsigned> err;
  BAIL_ON(err.alloc(1));
  cudaMemsetAsync(err.p, 0, sizeof(unsigned), s);
  k_elem_codes<<<blocks_for(ne * ndofe), TPB, 0, s>>>(ne, nne, ndofn, ad.elems.p, cn_d.p, ad.cne.p, err.p, nn);
  count_launches(1);

  // pattern: from the node adjacency when the code numbers grow with (node,
  // component), else (or for a node of very high valence) lower-triangle
  // element pairs -> sort -> unique -> SCR
  bool monotone = true;
  {
    int64_t last = 0;
    for (int64_t q = 0; q < nn * ndofn && monotone; q++) {
      const int64_t c = mesh->cn[q];
      if (c > 0) {
        monotone = c == last + 1;  // gencodnum's consecutive numbering
        last = c;
      }
    }
  }
  int adj_st = 1;
  int inc_st = 1;
  if (monotone) {
    inc_st = build_incidence(ad.elems.p, nn, ne, nne, ad.iptr, ad.inc, s);
    if (inc_st != SGPU_OK && inc_st != 1) BAIL_ON(inc_st);
    ad.node_rows = inc_st == SGPU_OK;
  }
  if (inc_st == SGPU_OK && !std::getenv("SGPU_PATTERN_SORT")) {
    adj_st = pattern_adjacency(m, ad.elems.p, cn_d.p, nn, nne, ndofn, n, ad.iptr.p, ad.inc.p, err.p, s);
    if (adj_st != SGPU_OK && adj_st != 1) BAIL_ON(adj_st);
  }
  if (adj_st != SGPU_OK) {
    const int64_t npairs = ne * (int64_t)ndofe * ndofe;
    if (npairs > (1LL << 31) - 1) return bail(fail(SGPU_BAD_INPUT, "mesh too large for one pattern sort"));
    DevBuf<unsigned long long> keys, skeys;
    BAIL_ON(keys.alloc(npairs));
    BAIL_ON(skeys.alloc(npairs));
    k_elem_pairs<<<blocks_for(npairs), TPB, 0, s>>>(ne, ndofe, ad.cne.p, keys.p);
    count_launches(1);
    const int end_bit = 64;  // invalid keys (~0) must sort last
    size_t tmp = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tmp, keys.p, skeys.p, (int)npairs, 0, end_bit, s);
    DevBuf<unsigned char> t;
    BAIL_ON(t.alloc(tmp));
    cub::DeviceRadixSort::SortKeys(t.p, tmp, keys.p, skeys.p, (int)npairs, 0, end_bit, s);
    DevBuf<int> nsel;
    BAIL_ON(nsel.alloc(1));
    size_t tmp2 = 0;
    cub::DeviceSelect::Unique(nullptr, tmp2, skeys.p, keys.p, nsel.p, (int)npairs, s);
    DevBuf<unsigned char> t2;
    BAIL_ON(t2.alloc(tmp2));
    cub::DeviceSelect::Unique(t2.p, tmp2, skeys.p, keys.p, nsel.p, (int)npairs, s);
    count_launches(6);
    int nuniq = 0;
    cudaMemcpyAsync(&nuniq, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(SGPU_CUDA_ERROR, "pattern sort failed"));
    // drop the trailing invalid key, if any
    unsigned long long lastk = 0;
    cudaMemcpy(&lastk, keys.p + nuniq - 1, sizeof(lastk), cudaMemcpyDeviceToHost);
    const int64_t negm = (lastk == ~0ull) ? nuniq - 1 : nuniq;
    m->src_negm = negm;
    BAIL_ON(m->src_adr.alloc(n + 1));
    BAIL_ON(m->src_ci.alloc(negm));
    cudaMemsetAsync(m->src_adr.p, 0xff, (n + 1) * sizeof(int64_t), s);
    k_keys_to_scr<<<blocks_for(negm), TPB, 0, s>>>(negm, n, keys.p, m->src_adr.p, m->src_ci.p);
    k_check_adr<<<blocks_for(n), TPB, 0, s>>>(n, m->src_adr.p, err.p);
    count_launches(2);
    unsigned e = 0;
    BAIL_ON(read_err(err.p, s, &e));
    if (e) return bail(fail(SGPU_BAD_INPUT, "code numbers: element node out of range or unused equation"));
  }
  BAIL_ON(matrix_build_from_device_src(m));
  cudaEventRecord(t1, s);
  cudaEventSynchronize(t1);
  float pattern_ms = 0.f;
  cudaEventElapsedTime(&pattern_ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);

  // colouring (host) and the per-colour element lists
  st = colour_elements(nn, ne, nne, mesh->elems, ad.order, ad.offsets);
  if (st != SGPU_OK) return bail(st);
  if (ad.elist.alloc(ne) != SGPU_OK) return bail(SGPU_CUDA_ERROR);
  cudaMemcpyAsync(ad.elist.p, ad.order.data(), ne * sizeof(int), cudaMemcpyHostToDevice, s);
  float asm_ms = 0.f;
  st = assemble_values(m, ad, kind, &asm_ms);
  if (st != SGPU_OK) return bail(st);
  st = finish_values(m);
  if (st != SGPU_OK) return bail(st);
  if (info) {
    info->n = n;
    info->negm_scr = m->src_negm;
    info->nnz_full = m->csr.nnz;
    info->colours = (int32_t)ad.offsets.size() - 1;
    info->pattern_ms = pattern_ms;
    info->integrate_ms = asm_ms;
  }
  *out = m;
  return SGPU_OK;
#undef BAIL_ON
}

SGPU_API int sgpu_assembly_lift(sgpu_matrix m, const double *rnode, double *rhs) {
  if (!m || !m->asm_data) return fail(SGPU_BAD_INPUT, "handle was not created by sgpu_assemble");
  if (!rnode || !rhs) return fail(SGPU_BAD_INPUT, "null argument");
  AssemblyData &ad = m->asm_data->d;
  const bool scalar = ad.kind == SGPU_ELEM_HEX8T_K || ad.kind == SGPU_ELEM_HEX8T_C;
  if (!scalar && ad.kind != SGPU_ELEM_HEX8 && ad.kind != SGPU_ELEM_QUAD4)
    return fail(SGPU_BAD_INPUT, "lifting is defined for hex8 conduction, hex8 and quad4 elasticity handles");
  cudaStream_t s = m->stream;
  DevBuf<double> rn, f;
  const int64_t nr = ad.nn * ad.ndofn;
  SGPU_TRY(rn.alloc(nr));
  SGPU_TRY(f.alloc(m->n));
  SGPU_CUDA(cudaMemcpyAsync(rn.p, rnode, nr * sizeof(double), cudaMemcpyHostToDevice, s));
  SGPU_CUDA(cudaMemcpyAsync(f.p, rhs, m->n * sizeof(double), cudaMemcpyHostToDevice, s));
  const int ncol = (int)ad.offsets.size() - 1;
  for (int col = 0; col < ncol; col++) {
    const int beg = ad.offsets[col], cnt = ad.offsets[col + 1] - beg;
    if (cnt == 0) continue;
    const int grid = std::min((cnt + WPB - 1) / WPB, kNumSMs * 16);
    const int *el = ad.elist.p + beg;
    if (scalar)
      k_hex8t_lift<<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p, rn.p, f.p);
    else if (ad.kind == SGPU_ELEM_QUAD4)
      k_quad4_lift<<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p, ad.thick.p, rn.p, f.p);
    else if (ad.general)
      k_hex8_lift<true><<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p, rn.p, f.p);
    else
      k_hex8_lift<false><<<grid, TPB, 0, s>>>(cnt, el, ad.coords.p, ad.elems.p, ad.cne.p, ad.emat.p, rn.p, f.p);
    count_launches(1);
  }
  SGPU_CUDA(cudaGetLastError());
  SGPU_CUDA(cudaMemcpyAsync(rhs, f.p, m->n * sizeof(double), cudaMemcpyDeviceToHost, s));
  SGPU_CUDA(cudaStreamSynchronize(s));
  return SGPU_OK;
}

SGPU_API int sgpu_assemble_copy(sgpu_matrix src, int32_t kind, const double *emat, const double *rho,
                                sgpu_matrix *out, sgpu_assembly_info *info) {
  if (!src || !src->asm_data || !out) return fail(SGPU_BAD_INPUT, "handle was not created by sgpu_assemble");
  *out = nullptr;
  const AssemblyData &sa = src->asm_data->d;
  const bool scalar_ok = (sa.kind == SGPU_ELEM_HEX8T_K || sa.kind == SGPU_ELEM_HEX8T_C) &&
                         (kind == SGPU_ELEM_HEX8T_K || kind == SGPU_ELEM_HEX8T_C);
  if (kind != sa.kind && !scalar_ok) return fail(SGPU_BAD_INPUT, "element kind differs from the pattern's");
  SGPU_CUDA(cudaStreamSynchronize(src->stream));
  sgpu_matrix m = new sgpu_matrix_s();
  auto bail = [&](int st) {
    if (m->stream) cudaStreamSynchronize(m->stream);
    cudaStream_t s = m->own_stream;
    cudaEvent_t a = m->ev0, b = m->ev1;
    delete m;
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (s) cudaStreamDestroy(s);
    return st;
  };
  if (cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&m->ev0) != cudaSuccess || cudaEventCreate(&m->ev1) != cudaSuccess)
    return bail(fail(SGPU_CUDA_ERROR, "stream/event creation failed"));
  m->stream = m->own_stream;
  cudaStream_t s = m->stream;
  m->n = src->n;
  m->src_sym = src->src_sym;
  m->src_negm = src->src_negm;
  m->asm_data = new sgpu_assembly_s();
  AssemblyData &ad = m->asm_data->d;
  ad.kind = kind; ad.nne = sa.nne; ad.ndofn = sa.ndofn; ad.nn = sa.nn; ad.ne = sa.ne;
  ad.general = sa.general;
  ad.offsets = sa.offsets;
  ad.order = sa.order;
  Csr &c = m->csr;
  c.n = src->csr.n;
  c.nnz = src->csr.nnz;
  int st = SGPU_OK;
#define DUP(dst, from)                                                                        \
  if (st == SGPU_OK && (from).p) {                                                            \
    st = (dst).alloc((from).n);                                                               \
    if (st == SGPU_OK &&                                                                      \
        cudaMemcpyAsync((dst).p, (from).p, (from).n * sizeof(*(from).p), cudaMemcpyDeviceToDevice, s) != cudaSuccess) \
      st = fail(SGPU_CUDA_ERROR, "device copy of the pattern failed");                        \
  }
  DUP(m->src_adr, src->src_adr);
  DUP(m->src_ci, src->src_ci);
  DUP(m->map_lo, src->map_lo);
  DUP(m->map_up, src->map_up);
  DUP(c.rowptr, src->csr.rowptr);
  DUP(c.col, src->csr.col);
  DUP(ad.coords, sa.coords);
  DUP(ad.elems, sa.elems);
  DUP(ad.cne, sa.cne);
  DUP(ad.elist, sa.elist);
  DUP(ad.emat, sa.emat);
  DUP(ad.thick, sa.thick);
  DUP(ad.rho, sa.rho);
  DUP(ad.iptr, sa.iptr);
  DUP(ad.inc, sa.inc);
  ad.node_rows = sa.node_rows;
#undef DUP
  if (st != SGPU_OK) return bail(st);
  if (c.val.alloc(c.nnz) != SGPU_OK || c.diag.alloc(c.n) != SGPU_OK) return bail(SGPU_CUDA_ERROR);
  m->bsr.valid = false;
  m->bsr.nb = -1;  // examined on first use
  if (emat && cudaMemcpyAsync(ad.emat.p, emat, ad.ne * (ad.general ? 36 : 2) * sizeof(double),
                              cudaMemcpyHostToDevice, s) != cudaSuccess)
    return bail(fail(SGPU_CUDA_ERROR, "copy of emat failed"));
  if (rho) {
    if (ad.rho.alloc(ad.ne) != SGPU_OK) return bail(SGPU_CUDA_ERROR);
    if (cudaMemcpyAsync(ad.rho.p, rho, ad.ne * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
      return bail(fail(SGPU_CUDA_ERROR, "copy of rho failed"));
  }
  float ms = 0.f;
  st = assemble_values(m, ad, kind, &ms);
  if (st == SGPU_OK) st = finish_values(m);
  if (st != SGPU_OK) return bail(st);
  if (info) {
    memset(info, 0, sizeof(*info));
    info->n = m->n;
    info->negm_scr = m->src_negm;
    info->nnz_full = c.nnz;
    info->colours = (int32_t)ad.offsets.size() - 1;
    info->integrate_ms = ms;
  }
  *out = m;
  return SGPU_OK;
}

SGPU_API int sgpu_reassemble(sgpu_matrix m, int32_t kind, const double *emat, const double *rho,
                             sgpu_assembly_info *info) {
  if (!m || !m->asm_data) return fail(SGPU_BAD_INPUT, "handle was not created by sgpu_assemble");
  AssemblyData &ad = m->asm_data->d;
  const bool scalar_ok = (ad.kind == SGPU_ELEM_HEX8T_K || ad.kind == SGPU_ELEM_HEX8T_C) &&
                         (kind == SGPU_ELEM_HEX8T_K || kind == SGPU_ELEM_HEX8T_C);
  if (kind != ad.kind && !scalar_ok) return fail(SGPU_BAD_INPUT, "element kind differs from the pattern's");
  cudaStream_t s = m->stream;
  if (emat)
    SGPU_CUDA(cudaMemcpyAsync(ad.emat.p, emat, ad.ne * (ad.general ? 36 : 2) * sizeof(double),
                              cudaMemcpyHostToDevice, s));
  if (rho) {
    SGPU_TRY(ad.rho.alloc(ad.ne));
    SGPU_CUDA(cudaMemcpyAsync(ad.rho.p, rho, ad.ne * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  float ms = 0.f;
  SGPU_TRY(assemble_values(m, ad, kind, &ms));
  SGPU_TRY(finish_values(m));
  if (info) {
    memset(info, 0, sizeof(*info));
    info->n = m->n;
    info->negm_scr = m->src_negm;
    info->nnz_full = m->csr.nnz;
    info->colours = (int32_t)ad.offsets.size() - 1;
    info->integrate_ms = ms;
  }
  return SGPU_OK;
}

}  // extern "C"

void sgpu_free_assembly(sgpu_assembly_s *a) { delete a; }
