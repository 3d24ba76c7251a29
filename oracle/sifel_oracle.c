/*
 * sifel_oracle.c -- CPU restatement of SIFEL's linear FE hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the GPU path is checked
 * against: tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py may call it; the product library never does.  Every routine
 * restates one reference routine in plain C, in the same operation order so
 * that, compiled with the reference's own flags (g++/gcc -O3, no FMA
 * contraction on x86-64), results agree with the compiled reference to the
 * last bit or very nearly so.  The restatement is pinned against the
 * compiled reference (oracle/_ref) by tests/test_oracle_vs_reference.py and
 * against committed golden fixtures by tests/test_oracle_golden.py.
 *
 * Conventions: `long` is int64 as in the reference; code numbers are 1-based,
 * 0 (or negative) means "no equation" (gtopology.cpp:1619-1680); matrices are
 * dense row-major.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Gauss rule of order 2, 15-digit constants (GEFEL/intp.cpp:15-40)          */
/* ------------------------------------------------------------------------ */
static const double GP2[2] = {-0.577350269189626, 0.577350269189626};
static const double GW2[2] = {1.0, 1.0};

/* trilinear hexahedron, GEFEL/basefun.cpp:2299-2370 */
static void bf_lin_hex_3d(double *n, double x, double y, double z) {
  n[0] = (1.0 + x) * (1.0 + y) * (1.0 + z) / 8.0;
  n[1] = (1.0 - x) * (1.0 + y) * (1.0 + z) / 8.0;
  n[2] = (1.0 - x) * (1.0 - y) * (1.0 + z) / 8.0;
  n[3] = (1.0 + x) * (1.0 - y) * (1.0 + z) / 8.0;
  n[4] = (1.0 + x) * (1.0 + y) * (1.0 - z) / 8.0;
  n[5] = (1.0 - x) * (1.0 + y) * (1.0 - z) / 8.0;
  n[6] = (1.0 - x) * (1.0 - y) * (1.0 - z) / 8.0;
  n[7] = (1.0 + x) * (1.0 - y) * (1.0 - z) / 8.0;
}
static void dx_bf_lin_hex_3d(double *n, double y, double z) {
  n[0] = (1.0 + y) * (1.0 + z) / 8.0;
  n[1] = (1.0 + y) * (1.0 + z) / (-8.0);
  n[2] = (1.0 - y) * (1.0 + z) / (-8.0);
  n[3] = (1.0 - y) * (1.0 + z) / 8.0;
  n[4] = (1.0 + y) * (1.0 - z) / 8.0;
  n[5] = (1.0 + y) * (1.0 - z) / (-8.0);
  n[6] = (1.0 - y) * (1.0 - z) / (-8.0);
  n[7] = (1.0 - y) * (1.0 - z) / 8.0;
}
static void dy_bf_lin_hex_3d(double *n, double x, double z) {
  n[0] = (1.0 + x) * (1.0 + z) / 8.0;
  n[1] = (1.0 - x) * (1.0 + z) / 8.0;
  n[2] = (1.0 - x) * (1.0 + z) / (-8.0);
  n[3] = (1.0 + x) * (1.0 + z) / (-8.0);
  n[4] = (1.0 + x) * (1.0 - z) / 8.0;
  n[5] = (1.0 - x) * (1.0 - z) / 8.0;
  n[6] = (1.0 - x) * (1.0 - z) / (-8.0);
  n[7] = (1.0 + x) * (1.0 - z) / (-8.0);
}
static void dz_bf_lin_hex_3d(double *n, double x, double y) {
  n[0] = (1.0 + x) * (1.0 + y) / 8.0;
  n[1] = (1.0 - x) * (1.0 + y) / 8.0;
  n[2] = (1.0 - x) * (1.0 - y) / 8.0;
  n[3] = (1.0 + x) * (1.0 - y) / 8.0;
  n[4] = (1.0 + x) * (1.0 + y) / (-8.0);
  n[5] = (1.0 - x) * (1.0 + y) / (-8.0);
  n[6] = (1.0 - x) * (1.0 - y) / (-8.0);
  n[7] = (1.0 + x) * (1.0 - y) / (-8.0);
}

/* bilinear quadrilateral, GEFEL/basefun.cpp:609-655 */
static void bf_lin_4_2d(double *n, double x, double y) {
  n[0] = 0.25 * (1.0 + x) * (1.0 + y);
  n[1] = 0.25 * (1.0 - x) * (1.0 + y);
  n[2] = 0.25 * (1.0 - x) * (1.0 - y);
  n[3] = 0.25 * (1.0 + x) * (1.0 - y);
}
static void dx_bf_lin_4_2d(double *n, double y) {
  n[0] = 0.25 * (1.0 + y);
  n[1] = 0.25 * (-1.0 - y);
  n[2] = 0.25 * (-1.0 + y);
  n[3] = 0.25 * (1.0 - y);
}
static void dy_bf_lin_4_2d(double *n, double x) {
  n[0] = 0.25 * (1.0 + x);
  n[1] = 0.25 * (1.0 - x);
  n[2] = 0.25 * (-1.0 + x);
  n[3] = 0.25 * (-1.0 - x);
}

/* derivatives_3d, GEFEL/difcalc.cpp:487-565 (8-node case): natural
 * derivatives in dx,dy,dz are replaced by Cartesian ones; returns detJ. */
static double derivatives_3d(double *dx, double *dy, double *dz, const double *x, const double *y,
                             const double *z, double xi, double eta, double zeta) {
  double nx[8], ny[8], nz[8];
  double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0, d9 = 0, jac;
  dx_bf_lin_hex_3d(nx, eta, zeta);
  dy_bf_lin_hex_3d(ny, xi, zeta);
  dz_bf_lin_hex_3d(nz, xi, eta);
  for (int i = 0; i < 8; i++) {
    d1 += nx[i] * x[i]; d2 += ny[i] * x[i]; d3 += nz[i] * x[i];
    d4 += nx[i] * y[i]; d5 += ny[i] * y[i]; d6 += nz[i] * y[i];
    d7 += nx[i] * z[i]; d8 += ny[i] * z[i]; d9 += nz[i] * z[i];
  }
  jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 - d9 * d4 * d2;
  for (int i = 0; i < 8; i++) {
    double ddx = dx[i], ddy = dy[i], ddz = dz[i];
    dx[i] = (ddx * (d5 * d9 - d8 * d6) + ddy * (d7 * d6 - d9 * d4) + ddz * (d4 * d8 - d7 * d5)) / jac;
    dy[i] = (ddx * (d8 * d3 - d9 * d2) + ddy * (d1 * d9 - d7 * d3) + ddz * (d7 * d2 - d8 * d1)) / jac;
    dz[i] = (ddx * (d2 * d6 - d5 * d3) + ddy * (d4 * d3 - d6 * d1) + ddz * (d1 * d5 - d4 * d2)) / jac;
  }
  return jac;
}

/* derivatives_2d, GEFEL/difcalc.cpp:86-138 (4-node case) */
static double derivatives_2d(double *dx, double *dy, const double *x, const double *y, double xi,
                             double eta) {
  double nx[4], ny[4], d1 = 0, d2 = 0, d3 = 0, d4 = 0, jac;
  dx_bf_lin_4_2d(nx, eta);
  dy_bf_lin_4_2d(ny, xi);
  for (int i = 0; i < 4; i++) {
    d1 += nx[i] * x[i]; d2 += ny[i] * x[i];
    d3 += nx[i] * y[i]; d4 += ny[i] * y[i];
  }
  jac = d1 * d4 - d2 * d3;
  for (int i = 0; i < 4; i++) {
    double ddx = dx[i], ddy = dy[i];
    dx[i] = (ddx * d4 - ddy * d3) / jac;
    dy[i] = (ddy * d1 - ddx * d2) / jac;
  }
  return jac;
}

/* bdbjac, GEFEL/matrix.cpp:3126: d += (A^T B) C * jac with mtxm then mxm
 * (matrix.cpp:1362, 1184), then cmulm and addm (y + d). A, C: m x n; B: m x m */
static void bdbjac(double *d, const double *a, const double *b, const double *c, double jac,
                   int m, int n) {
  double x[60 * 6];
  double y;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < m; j++) {
      double s = 0.0;
      for (int k = 0; k < m; k++) s += a[k * n + i] * b[k * m + j];
      x[i * m + j] = s;
    }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double s = 0.0;
      for (int k = 0; k < m; k++) s += x[i * m + k] * c[k * n + j];
      y = s * jac;
      d[i * n + j] = y + d[i * n + j];
    }
}

/* elastisomat::matstiff_spacestr, MEFEL/SRC/elastisomat.cpp:395-420 */
static void matstiff_spacestr(double e, double nu, double *d) {
  double g = e / 2.0 / (1.0 + nu);
  double s = e / (1.0 + nu) / (1.0 - 2.0 * nu);
  memset(d, 0, 36 * sizeof(double));
  d[0] = s * (1 - nu); d[1] = s * nu; d[2] = s * nu;
  d[6] = d[1]; d[7] = d[0]; d[8] = d[1];
  d[12] = d[1]; d[13] = d[1]; d[14] = d[0];
  d[21] = g; d[28] = g; d[35] = g;
}

/* elastisomat::matstiff_plstress, MEFEL/SRC/elastisomat.cpp:255-266 */
static void matstiff_plstress(double e, double nu, double *d) {
  double c = e / (1.0 - nu * nu);
  d[0] = c; d[1] = c * nu; d[2] = 0.0;
  d[3] = c * nu; d[4] = c; d[5] = 0.0;
  d[6] = 0.0; d[7] = 0.0; d[8] = e / 2.0 / (1.0 + nu);
}

/* linhex::gl_stiffness_matrix, MEFEL/SRC/linhex.cpp:583-630, with
 * linhex::geom_matrix (linhex.cpp:153-186).  xyz: 8 x (x,y,z).  dm: the
 * material stiffness (6 x 6, row-major) of every integration point, or NULL
 * for the isotropic (e, nu) of elastisomat. */
static void hex8_ke(const double *xyz, double e, double nu, const double *dm, double *ke) {
  double x[8], y[8], z[8], dx[8], dy[8], dz[8], gm[6 * 24], d[36];
  for (int i = 0; i < 8; i++) { x[i] = xyz[3 * i]; y[i] = xyz[3 * i + 1]; z[i] = xyz[3 * i + 2]; }
  memset(ke, 0, 576 * sizeof(double));
  for (int i = 0; i < 2; i++) {
    double xi = GP2[i];
    for (int j = 0; j < 2; j++) {
      double eta = GP2[j];
      for (int k = 0; k < 2; k++) {
        double zeta = GP2[k];
        dx_bf_lin_hex_3d(dx, eta, zeta);
        dy_bf_lin_hex_3d(dy, xi, zeta);
        dz_bf_lin_hex_3d(dz, xi, eta);
        double jac = derivatives_3d(dx, dy, dz, x, y, z, xi, eta, zeta);
        memset(gm, 0, sizeof(gm));
        for (int a = 0; a < 8; a++) {
          int jj = 3 * a, kk = 3 * a + 1, ll = 3 * a + 2;
          gm[0 * 24 + jj] = dx[a];
          gm[1 * 24 + kk] = dy[a];
          gm[2 * 24 + ll] = dz[a];
          gm[3 * 24 + kk] = dz[a]; gm[3 * 24 + ll] = dy[a];
          gm[4 * 24 + jj] = dz[a]; gm[4 * 24 + ll] = dx[a];
          gm[5 * 24 + jj] = dy[a]; gm[5 * 24 + kk] = dx[a];
        }
        if (dm) memcpy(d, dm, sizeof(d));
        else matstiff_spacestr(e, nu, d);
        jac *= GW2[i] * GW2[j] * GW2[k];
        if (jac < 0.0) jac = fabs(jac);
        bdbjac(ke, gm, d, gm, jac, 6, 24);
      }
    }
  }
}

void or_hex8_ke(const double *xyz, double e, double nu, double *ke) { hex8_ke(xyz, e, nu, NULL, ke); }
void or_hex8_ke_d(const double *xyz, const double *dm, double *ke) { hex8_ke(xyz, 0.0, 0.0, dm, ke); }

/* det3d, GEFEL/matrix.cpp:3629-3660 (the active branch): six times the signed
 * volume of the tetrahedron, (p0-p3) . ((p1-p3) x (p2-p3)). */
static double det3d(const double *x, const double *y, const double *z) {
  double a0 = x[0] - x[3], a1 = y[0] - y[3], a2 = z[0] - z[3];
  double b0 = x[1] - x[3], b1 = y[1] - y[3], b2 = z[1] - z[3];
  double c0 = x[2] - x[3], c1 = y[2] - y[3], c2 = z[2] - z[3];
  return a0 * b1 * c2 + b0 * c1 * a2 + c0 * a1 * b2 - c0 * b1 * a2 - c1 * b2 * a0 - c2 * b0 * a1;
}

/* lintet::stiffness_matrix, MEFEL/SRC/lintet.cpp:290-315: one integration
 * point; geom_matrix (lintet.cpp:213-240) takes the Cartesian gradients of the
 * natural derivatives dx/dy/dz_bf_lin_tet (GEFEL/basefun.cpp:1974-2000)
 * through derivatives_3d (GEFEL/difcalc.cpp:487-565, 4-node case) at
 * (0.25, 0.25, 0.25); the weight is det3d/6, and a negative det3d (wrong node
 * numbering) is an error.  xyz: 4 x (x,y,z).  Returns 0, or -1 on a negative
 * volume (ke untouched then). */
static int tet4_ke(const double *xyz, double e, double nu, const double *dm, double *ke) {
  static const double NX[4] = {1.0, 0.0, 0.0, -1.0}, NY[4] = {0.0, 1.0, 0.0, -1.0},
                      NZ[4] = {0.0, 0.0, 1.0, -1.0};
  double x[4], y[4], z[4], dx[4], dy[4], dz[4], gm[6 * 12], d[36];
  for (int i = 0; i < 4; i++) { x[i] = xyz[3 * i]; y[i] = xyz[3 * i + 1]; z[i] = xyz[3 * i + 2]; }
  double det = det3d(x, y, z);
  if (det < 0.0) return -1;
  double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0, d9 = 0, jac;
  for (int i = 0; i < 4; i++) {
    d1 += NX[i] * x[i]; d2 += NY[i] * x[i]; d3 += NZ[i] * x[i];
    d4 += NX[i] * y[i]; d5 += NY[i] * y[i]; d6 += NZ[i] * y[i];
    d7 += NX[i] * z[i]; d8 += NY[i] * z[i]; d9 += NZ[i] * z[i];
  }
  jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 - d9 * d4 * d2;
  for (int i = 0; i < 4; i++) {
    double ddx = NX[i], ddy = NY[i], ddz = NZ[i];
    dx[i] = (ddx * (d5 * d9 - d8 * d6) + ddy * (d7 * d6 - d9 * d4) + ddz * (d4 * d8 - d7 * d5)) / jac;
    dy[i] = (ddx * (d8 * d3 - d9 * d2) + ddy * (d1 * d9 - d7 * d3) + ddz * (d7 * d2 - d8 * d1)) / jac;
    dz[i] = (ddx * (d2 * d6 - d5 * d3) + ddy * (d4 * d3 - d6 * d1) + ddz * (d1 * d5 - d4 * d2)) / jac;
  }
  memset(gm, 0, sizeof(gm));
  for (int a = 0; a < 4; a++) {
    int jj = 3 * a, kk = 3 * a + 1, ll = 3 * a + 2;
    gm[0 * 12 + jj] = dx[a];
    gm[1 * 12 + kk] = dy[a];
    gm[2 * 12 + ll] = dz[a];
    gm[3 * 12 + kk] = dz[a]; gm[3 * 12 + ll] = dy[a];
    gm[4 * 12 + jj] = dz[a]; gm[4 * 12 + ll] = dx[a];
    gm[5 * 12 + jj] = dy[a]; gm[5 * 12 + kk] = dx[a];
  }
  if (dm) memcpy(d, dm, sizeof(d));
  else matstiff_spacestr(e, nu, d);
  memset(ke, 0, 144 * sizeof(double));
  bdbjac(ke, gm, d, gm, det / 6.0, 6, 12);
  return 0;
}

int or_tet4_ke(const double *xyz, double e, double nu, double *ke) { return tet4_ke(xyz, e, nu, NULL, ke); }
int or_tet4_ke_d(const double *xyz, const double *dm, double *ke) { return tet4_ke(xyz, 0.0, 0.0, dm, ke); }

/* elastortomat::matstiff, MEFEL/SRC/elastortomat.cpp:100-115, for a
 * transformation of constant general functions: lg_tens4transf
 * (MEFEL/SRC/vecttens.cpp:1561-1622) builds the 6 x 6 strain transformation
 * t from the 3 x 3 tmat (x_g = T x_l), then g = t^T l t by mtxm and mxm
 * (GEFEL/matrix.cpp:1362, 1184).  l, g: 6 x 6 row-major; tm: 3 x 3. */
void or_ortho_dmat(const double *l, const double *tm, double *g) {
#define TM(i, j) tm[3 * (i) + (j)]
  double t[36], aux[36];
  for (int c = 0; c < 3; c++) {
    /* rows 0..2: the squares of column c */
    t[6 * c + 0] = TM(0, c) * TM(0, c);
    t[6 * c + 1] = TM(1, c) * TM(1, c);
    t[6 * c + 2] = TM(2, c) * TM(2, c);
    t[6 * c + 3] = TM(1, c) * TM(2, c);
    t[6 * c + 4] = TM(0, c) * TM(2, c);
    t[6 * c + 5] = TM(0, c) * TM(1, c);
  }
  /* rows 3, 4, 5 pair the columns (2,1), (2,0), (1,0) */
  static const int P[3][2] = {{2, 1}, {2, 0}, {1, 0}};
  for (int r = 0; r < 3; r++) {
    int a = P[r][0], b = P[r][1];
    double *row = t + 6 * (3 + r);
    row[0] = 2.0 * TM(0, a) * TM(0, b);
    row[1] = 2.0 * TM(1, a) * TM(1, b);
    row[2] = 2.0 * TM(2, a) * TM(2, b);
    row[3] = TM(1, a) * TM(2, b) + TM(2, a) * TM(1, b);
    row[4] = TM(0, a) * TM(2, b) + TM(2, a) * TM(0, b);
    row[5] = TM(0, a) * TM(1, b) + TM(1, a) * TM(0, b);
  }
#undef TM
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double s = 0.0;
      for (int k = 0; k < 6; k++) s += t[6 * k + i] * l[6 * k + j];
      aux[6 * i + j] = s;
    }
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double s = 0.0;
      for (int k = 0; k < 6; k++) s += aux[6 * i + k] * t[6 * k + j];
      g[6 * i + j] = s;
    }
}

/* planeelemlq::gl_stiffness_matrix, MEFEL/SRC/plelemlq.cpp:611-690 with
 * geom_matrix (294-320); thickness interpolated from nodal values t[4]
 * (planeelemlq::approx, plelemlq.cpp:127). xy: 4 x (x,y). */
void or_quad4_ke(const double *xy, double e, double nu, const double *t, double *ke) {
  double x[4], y[4], dx[4], dy[4], gm[3 * 8], d[9], bf[4];
  for (int i = 0; i < 4; i++) { x[i] = xy[2 * i]; y[i] = xy[2 * i + 1]; }
  memset(ke, 0, 64 * sizeof(double));
  for (int i = 0; i < 2; i++) {
    double xi = GP2[i];
    for (int j = 0; j < 2; j++) {
      double eta = GP2[j];
      dx_bf_lin_4_2d(dx, eta);
      dy_bf_lin_4_2d(dy, xi);
      double jac = derivatives_2d(dx, dy, x, y, xi, eta);
      memset(gm, 0, sizeof(gm));
      for (int a = 0; a < 4; a++) {
        gm[0 * 8 + 2 * a] = dx[a];
        gm[1 * 8 + 2 * a + 1] = dy[a];
        gm[2 * 8 + 2 * a] = dy[a];
        gm[2 * 8 + 2 * a + 1] = dx[a];
      }
      matstiff_plstress(e, nu, d);
      bf_lin_4_2d(bf, xi, eta);
      double thick = 0.0;
      for (int a = 0; a < 4; a++) thick += bf[a] * t[a];
      jac *= thick * GW2[i] * GW2[j];
      if (jac < 0.0) jac = fabs(jac);
      bdbjac(ke, gm, d, gm, jac, 3, 8);
    }
  }
}

/* bdbj, GEFEL/matrix.cpp:3066-3110: symmetric fill of B^T D B jac */
static void bdbj(double *k, const double *b, const double *d, double jac, int m, int n) {
  double am[3 * 16];
  int ll = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < m; j++) {
      double s = 0.0;
      int ii = i, jj = j;
      for (int l = 0; l < m; l++) { s += b[ii] * d[jj]; ii += n; jj += m; }
      am[ll++] = s;
    }
  for (int i = 0; i < n; i++) {
    int ii = i * n + i, mm = ii, l0 = i * m, ul = l0 + m, jj = i;
    double s = 0.0;
    for (int l = l0; l < ul; l++) { s += am[l] * b[jj]; jj += n; }
    k[ii] += s * jac;
    ii++; mm += n;
    for (int j = i + 1; j < n; j++) {
      s = 0.0; jj = j;
      for (int l = l0; l < ul; l++) { s += am[l] * b[jj]; jj += n; }
      k[ii] += s * jac; k[mm] += s * jac;
      ii++; mm += n;
    }
  }
}

/* planeelemlt::stiffness_matrix, MEFEL/SRC/plelemlt.cpp:234-272: the
 * constant-strain triangle.  det = twice the signed area; B from the
 * area-coordinate coefficients plsb/plsc (GEFEL/basefun.cpp:394-416)
 * (planeelemlt::geom_matrix, plelemlt.cpp:166-192); plane-stress D; the
 * thickness interpolated at (1/3, 1/3) from nodal values t[3] through area
 * coordinates (planeelemlt::approx_nat, :119-131, scprd order); weight
 * thick*det/2 and the symmetric product bdbj.  No sign check: a clockwise
 * triangle gives the negative matrix, as in the reference.  xy: 3 x (x,y). */
void or_tri3_ke(const double *xy, double e, double nu, const double *t, double *ke) {
  double x[3], y[3], b[3], c[3], gm[3 * 6], d[9], ac[3];
  for (int i = 0; i < 3; i++) { x[i] = xy[2 * i]; y[i] = xy[2 * i + 1]; }
  double det = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
  b[0] = (y[1] - y[2]) / det; b[1] = (y[2] - y[0]) / det; b[2] = (y[0] - y[1]) / det;
  c[0] = (x[2] - x[1]) / det; c[1] = (x[0] - x[2]) / det; c[2] = (x[1] - x[0]) / det;
  memset(gm, 0, sizeof(gm));
  gm[0 * 6 + 0] = b[0]; gm[0 * 6 + 2] = b[1]; gm[0 * 6 + 4] = b[2];
  gm[1 * 6 + 1] = c[0]; gm[1 * 6 + 3] = c[1]; gm[1 * 6 + 5] = c[2];
  gm[2 * 6 + 0] = c[0]; gm[2 * 6 + 1] = b[0]; gm[2 * 6 + 2] = c[1];
  gm[2 * 6 + 3] = b[1]; gm[2 * 6 + 4] = c[2]; gm[2 * 6 + 5] = b[2];
  matstiff_plstress(e, nu, d);
  double xi = 1.0 / 3.0, eta = 1.0 / 3.0;
  ac[0] = xi; ac[1] = eta; ac[2] = 1.0 - ac[0] - ac[1];
  double thick = 0.0;
  for (int i = 0; i < 3; i++) thick += ac[i] * t[i];
  double jac = thick * det / 2.0;
  memset(ke, 0, 36 * sizeof(double));
  bdbj(ke, gm, d, jac, 3, 6);
}

/* ------------------------------------------------------------------------ */
/* Quadratic serendipity elements: quadhex (20 nodes), planeelemqq (8)      */
/* ------------------------------------------------------------------------ */

/* Gauss rule of order 3 with the reference's constants (gauss_points,
 * GEFEL/intp.cpp:34-43) */
static const double GP3[3] = {-0.774596669241483, 0.0, 0.774596669241483};
static const double GW3[3] = {0.5555555555555555, 0.8888888888888888, 0.5555555555555555};

/* natural coordinates of the 20 nodes in SIFEL's order (bf_quad_hex_3d,
 * GEFEL/basefun.cpp:2377-2403): corners as the linear hexahedron, then the
 * mid-edge nodes of the zeta = +1 face, the four vertical edges, and the
 * zeta = -1 face */
static const double H20[20][3] = {
    {1, 1, 1},  {-1, 1, 1},  {-1, -1, 1},  {1, -1, 1},  {1, 1, -1},  {-1, 1, -1},  {-1, -1, -1},
    {1, -1, -1}, {0, 1, 1},  {-1, 0, 1},   {0, -1, 1},  {1, 0, 1},   {1, 1, 0},    {-1, 1, 0},
    {-1, -1, 0}, {1, -1, 0}, {0, 1, -1},   {-1, 0, -1}, {0, -1, -1}, {1, 0, -1}};

/* derivatives of the 20-node serendipity functions with respect to the
 * natural coordinates (the functions of dx/dy/dz_bf_quad_hex_3d,
 * basefun.cpp:2413-2520, written from the corner and mid-edge formulas) */
static void hex20_dnat(double xi, double eta, double zeta, double *nx, double *ny, double *nz) {
  for (int a = 0; a < 20; a++) {
    double p = H20[a][0], q = H20[a][1], r = H20[a][2];
    double fx = 1.0 + xi * p, fy = 1.0 + eta * q, fz = 1.0 + zeta * r;
    if (p != 0.0 && q != 0.0 && r != 0.0) {
      nx[a] = p * fy * fz * (2.0 * xi * p + eta * q + zeta * r - 1.0) / 8.0;
      ny[a] = q * fx * fz * (xi * p + 2.0 * eta * q + zeta * r - 1.0) / 8.0;
      nz[a] = r * fx * fy * (xi * p + eta * q + 2.0 * zeta * r - 1.0) / 8.0;
    } else if (p == 0.0) {
      nx[a] = -xi * fy * fz / 2.0;
      ny[a] = q * (1.0 - xi * xi) * fz / 4.0;
      nz[a] = r * (1.0 - xi * xi) * fy / 4.0;
    } else if (q == 0.0) {
      nx[a] = p * (1.0 - eta * eta) * fz / 4.0;
      ny[a] = -eta * fx * fz / 2.0;
      nz[a] = r * (1.0 - eta * eta) * fx / 4.0;
    } else {
      nx[a] = p * (1.0 - zeta * zeta) * fy / 4.0;
      ny[a] = q * (1.0 - zeta * zeta) * fx / 4.0;
      nz[a] = -zeta * fx * fy / 2.0;
    }
  }
}

/* derivatives_3d (GEFEL/difcalc.cpp:487-565) for nn nodes: natural
 * derivatives in, Cartesian out; returns detJ */
static double derivatives_3d_n(int nn, double *dx, double *dy, double *dz, const double *x, const double *y,
                               const double *z) {
  double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0, d9 = 0, jac;
  for (int i = 0; i < nn; i++) {
    d1 += dx[i] * x[i]; d2 += dy[i] * x[i]; d3 += dz[i] * x[i];
    d4 += dx[i] * y[i]; d5 += dy[i] * y[i]; d6 += dz[i] * y[i];
    d7 += dx[i] * z[i]; d8 += dy[i] * z[i]; d9 += dz[i] * z[i];
  }
  jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 - d9 * d4 * d2;
  for (int i = 0; i < nn; i++) {
    double ddx = dx[i], ddy = dy[i], ddz = dz[i];
    dx[i] = (ddx * (d5 * d9 - d8 * d6) + ddy * (d7 * d6 - d9 * d4) + ddz * (d4 * d8 - d7 * d5)) / jac;
    dy[i] = (ddx * (d8 * d3 - d9 * d2) + ddy * (d1 * d9 - d7 * d3) + ddz * (d7 * d2 - d8 * d1)) / jac;
    dz[i] = (ddx * (d2 * d6 - d5 * d3) + ddy * (d4 * d3 - d6 * d1) + ddz * (d1 * d5 - d4 * d2)) / jac;
  }
  return jac;
}

/* quadhex::stiffness_matrix, MEFEL/SRC/quadhex.cpp:232-270: 3 x 3 x 3 Gauss
 * (loop order xi, eta, zeta), geom_matrix (:150-180) as for the linear
 * hexahedron, weight detJ w_i w_j w_k (no absolute value), bdbjac.
 * xyz: 20 x (x,y,z); dm: general 6 x 6 D or NULL for (e, nu). */
static void hex20_ke(const double *xyz, double e, double nu, const double *dm, double *ke) {
  double x[20], y[20], z[20], dx[20], dy[20], dz[20], gm[6 * 60], d[36];
  for (int i = 0; i < 20; i++) { x[i] = xyz[3 * i]; y[i] = xyz[3 * i + 1]; z[i] = xyz[3 * i + 2]; }
  memset(ke, 0, 3600 * sizeof(double));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) {
        hex20_dnat(GP3[i], GP3[j], GP3[k], dx, dy, dz);
        double jac = derivatives_3d_n(20, dx, dy, dz, x, y, z);
        memset(gm, 0, sizeof(gm));
        for (int a = 0; a < 20; a++) {
          int jj = 3 * a, kk = 3 * a + 1, ll = 3 * a + 2;
          gm[0 * 60 + jj] = dx[a];
          gm[1 * 60 + kk] = dy[a];
          gm[2 * 60 + ll] = dz[a];
          gm[3 * 60 + kk] = dz[a]; gm[3 * 60 + ll] = dy[a];
          gm[4 * 60 + jj] = dz[a]; gm[4 * 60 + ll] = dx[a];
          gm[5 * 60 + jj] = dy[a]; gm[5 * 60 + kk] = dx[a];
        }
        if (dm) memcpy(d, dm, sizeof(d));
        else matstiff_spacestr(e, nu, d);
        jac *= GW3[i] * GW3[j] * GW3[k];
        bdbjac(ke, gm, d, gm, jac, 6, 60);
      }
}

void or_hex20_ke(const double *xyz, double e, double nu, double *ke) { hex20_ke(xyz, e, nu, NULL, ke); }

/* natural coordinates of the 8 nodes (bf_quad_4_2d, GEFEL/basefun.cpp:708-718):
 * corners as the bilinear quad, then the mid-sides eta = +1, xi = -1,
 * eta = -1, xi = +1 */
static const double Q8[8][2] = {{1, 1}, {-1, 1}, {-1, -1}, {1, -1}, {0, 1}, {-1, 0}, {0, -1}, {1, 0}};

static void quad8_n(double xi, double eta, double *n, double *nx, double *ny) {
  for (int a = 0; a < 8; a++) {
    double p = Q8[a][0], q = Q8[a][1], fx = 1.0 + xi * p, fy = 1.0 + eta * q;
    if (p != 0.0 && q != 0.0) {
      n[a] = 0.25 * fx * fy * (xi * p + eta * q - 1.0);
      nx[a] = 0.25 * p * fy * (2.0 * xi * p + eta * q);
      ny[a] = 0.25 * q * fx * (xi * p + 2.0 * eta * q);
    } else if (p == 0.0) {
      n[a] = 0.5 * (1.0 - xi * xi) * fy;
      nx[a] = -xi * fy;
      ny[a] = 0.5 * q * (1.0 - xi * xi);
    } else {
      n[a] = 0.5 * fx * (1.0 - eta * eta);
      nx[a] = 0.5 * p * (1.0 - eta * eta);
      ny[a] = -eta * fx;
    }
  }
}

/* planeelemqq::stiffness_matrix, MEFEL/SRC/plelemqq.cpp:215-270: 3 x 3 Gauss,
 * geom_matrix (:150-170) with derivatives_2d (GEFEL/difcalc.cpp:86-138),
 * a negative detJ is an error (the reference aborts), thickness
 * interpolated from nodal values t[8] (planeelemqq::approx, :102-112),
 * weight detJ t w_i w_j, bdbj.  xy: 8 x (x,y).  Returns 0 or -1. */
int or_quad8_ke(const double *xy, double e, double nu, const double *t, double *ke) {
  double x[8], y[8], n[8], dx[8], dy[8], gm[3 * 16], d[9];
  for (int i = 0; i < 8; i++) { x[i] = xy[2 * i]; y[i] = xy[2 * i + 1]; }
  memset(ke, 0, 256 * sizeof(double));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double xi = GP3[i], eta = GP3[j];
      quad8_n(xi, eta, n, dx, dy);
      double d1 = 0, d2 = 0, d3 = 0, d4 = 0;
      for (int a = 0; a < 8; a++) {
        d1 += dx[a] * x[a]; d2 += dy[a] * x[a];
        d3 += dx[a] * y[a]; d4 += dy[a] * y[a];
      }
      double jac = d1 * d4 - d2 * d3;
      for (int a = 0; a < 8; a++) {
        double ddx = dx[a], ddy = dy[a];
        dx[a] = (ddx * d4 - ddy * d3) / jac;
        dy[a] = (ddy * d1 - ddx * d2) / jac;
      }
      if (jac < 0.0) return -1;
      memset(gm, 0, sizeof(gm));
      for (int a = 0; a < 8; a++) {
        gm[0 * 16 + 2 * a] = dx[a];
        gm[1 * 16 + 2 * a + 1] = dy[a];
        gm[2 * 16 + 2 * a] = dy[a];
        gm[2 * 16 + 2 * a + 1] = dx[a];
      }
      matstiff_plstress(e, nu, d);
      double thick = 0.0;
      for (int a = 0; a < 8; a++) thick += n[a] * t[a];
      jac *= thick * GW3[i] * GW3[j];
      bdbj(ke, gm, d, jac, 3, 16);
    }
  return 0;
}

/* nnj, GEFEL/matrix.cpp:3149-3174 (single row N) */
static void nnj(double *m, const double *n, double jac, int nn) {
  for (int i = 0; i < nn; i++) {
    int kk = i * nn + i, ll = kk;
    double s = 0.0 + n[i] * n[i];
    m[kk] += s * jac;
    kk++; ll += nn;
    for (int j = i + 1; j < nn; j++) {
      s = 0.0 + n[i] * n[j];
      m[kk] += s * jac; m[ll] += s * jac;
      kk++; ll += nn;
    }
  }
}

/* linhext::conductivity_matrix (TRFEL/SRC/linhext.cpp:774-840) for an
 * isotropic material D = k I3 (isotrmat::matcond3d, isotrmat.cpp:124) and
 * linhext::capacity_matrix (linhext.cpp:979-1030) with capacity c and
 * density rho (nodal values, interpolated by linhext::approx). */
void or_hex8t_kc(const double *xyz, double kcond, double c, const double *rho, double *ke,
                 double *ce) {
  double x[8], y[8], z[8], dx[8], dy[8], dz[8], gm[3 * 8], d[9], nb[8];
  for (int i = 0; i < 8; i++) { x[i] = xyz[3 * i]; y[i] = xyz[3 * i + 1]; z[i] = xyz[3 * i + 2]; }
  if (ke) {
    memset(ke, 0, 64 * sizeof(double));
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++)
        for (int k = 0; k < 2; k++) {
          double xi = GP2[i], eta = GP2[j], zeta = GP2[k];
          dx_bf_lin_hex_3d(dx, eta, zeta);
          dy_bf_lin_hex_3d(dy, xi, zeta);
          dz_bf_lin_hex_3d(dz, xi, eta);
          double jac = derivatives_3d(dx, dy, dz, x, y, z, xi, eta, zeta);
          for (int a = 0; a < 8; a++) { gm[a] = dx[a]; gm[8 + a] = dy[a]; gm[16 + a] = dz[a]; }
          memset(d, 0, sizeof(d));
          d[0] = kcond; d[4] = kcond; d[8] = kcond;
          if (jac < 0.0) jac = fabs(jac);
          jac *= GW2[i] * GW2[j] * GW2[k];
          bdbj(ke, gm, d, jac, 3, 8);
        }
  }
  if (ce) {
    memset(ce, 0, 64 * sizeof(double));
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++)
        for (int k = 0; k < 2; k++) {
          double xi = GP2[i], eta = GP2[j], zeta = GP2[k];
          /* jac_3d (GEFEL/difcalc.cpp:650): same Jacobian as derivatives_3d */
          double nx[8], ny[8], nz[8];
          double d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0, d9 = 0;
          dx_bf_lin_hex_3d(nx, eta, zeta);
          dy_bf_lin_hex_3d(ny, xi, zeta);
          dz_bf_lin_hex_3d(nz, xi, eta);
          for (int a = 0; a < 8; a++) {
            d1 += nx[a] * x[a]; d2 += ny[a] * x[a]; d3 += nz[a] * x[a];
            d4 += nx[a] * y[a]; d5 += ny[a] * y[a]; d6 += nz[a] * y[a];
            d7 += nx[a] * z[a]; d8 += ny[a] * z[a]; d9 += nz[a] * z[a];
          }
          double jac = d1 * d5 * d9 + d4 * d8 * d3 + d7 * d2 * d6 - d7 * d5 * d3 - d8 * d6 * d1 -
                       d9 * d4 * d2;
          bf_lin_hex_3d(nb, xi, eta, zeta);
          double r = 0.0;
          for (int a = 0; a < 8; a++) r += nb[a] * rho[a];
          if (jac < 0.0) jac = fabs(jac);
          jac *= GW2[i] * GW2[j] * GW2[k] * r * c;
          nnj(ce, nb, jac, 8);
        }
  }
}

/* ------------------------------------------------------------------------ */
/* Storage patterns (CR and SCR) and localisation                           */
/* ------------------------------------------------------------------------ */

/* comparison for qsort of long */
static int cmp_long(const void *a, const void *b) {
  long x = *(const long *)a, y = *(const long *)b;
  return (x > y) - (x < y);
}

/* Row-wise column sets of the global matrix from element code numbers:
 * symcomprow::initiate (GEFEL/scr.cpp:556; numcontr, addresses, fillarray,
 * sort_and_colindex_tko at 112-420) when sym != 0 (columns <= row, sorted, so
 * the diagonal is last), comprow::initiate (cr.cpp:454; sort_and_colindex at
 * 247) otherwise.  cn: ne x ndofe, 1-based, <= 0 skipped.
 * Two-phase: call with ci == NULL to get negm (adr filled), then again with
 * ci of that size. */
long or_pattern(long n, long ne, long ndofe, const long *cn, int sym, long *adr, long *ci) {
  long *cnt = (long *)calloc((size_t)n + 1, sizeof(long));
  for (long e = 0; e < ne; e++) {
    const long *c = cn + e * ndofe;
    for (long i = 0; i < ndofe; i++) {
      long ii = c[i] - 1;
      if (ii < 0) continue;
      for (long j = 0; j < ndofe; j++) {
        long jj = c[j] - 1;
        if (jj < 0) continue;
        if (sym && jj > ii) continue;
        cnt[ii]++;
      }
    }
  }
  long *start = (long *)malloc(((size_t)n + 1) * sizeof(long));
  start[0] = 0;
  for (long i = 0; i < n; i++) start[i + 1] = start[i] + cnt[i];
  long *aux = (long *)malloc((size_t)start[n] * sizeof(long) + 8);
  memset(cnt, 0, ((size_t)n + 1) * sizeof(long));
  for (long e = 0; e < ne; e++) {
    const long *c = cn + e * ndofe;
    for (long i = 0; i < ndofe; i++) {
      long ii = c[i] - 1;
      if (ii < 0) continue;
      for (long j = 0; j < ndofe; j++) {
        long jj = c[j] - 1;
        if (jj < 0) continue;
        if (sym && jj > ii) continue;
        aux[start[ii] + cnt[ii]++] = jj;
      }
    }
  }
  long negm = 0;
  for (long i = 0; i < n; i++) {
    long *row = aux + start[i];
    long m = cnt[i];
    qsort(row, (size_t)m, sizeof(long), cmp_long);
    long u = 0;
    for (long k = 0; k < m; k++)
      if (u == 0 || row[k] != row[u - 1]) row[u++] = row[k];
    cnt[i] = u;
    negm += u;
  }
  adr[0] = 0;
  for (long i = 0; i < n; i++) adr[i + 1] = adr[i] + cnt[i];
  if (ci)
    for (long i = 0; i < n; i++) memcpy(ci + adr[i], aux + start[i], (size_t)cnt[i] * sizeof(long));
  free(aux);
  free(start);
  free(cnt);
  return negm;
}

/* symcomprow::localize, GEFEL/scr.cpp:422-470 (searches restated as a direct
 * search from the row start; the entry hit is the same unique position). */
void or_scr_localize(long *adr, long *ci, double *a, const double *b, const long *cn, long m) {
  for (long i = 0; i < m; i++) {
    long ii = cn[i] - 1;
    if (ii < 0) continue;
    for (long j = 0; j < m; j++) {
      long jj = cn[j] - 1;
      if (jj < 0 || ii < jj) continue;
      for (long k = adr[ii]; k < adr[ii + 1]; k++)
        if (ci[k] == jj) { a[k] += b[i * m + j]; break; }
    }
  }
}

/* comprow::localize, GEFEL/cr.cpp:327-372 */
void or_cr_localize(long *adr, long *ci, double *a, const double *b, const long *cn, long m) {
  for (long i = 0; i < m; i++) {
    long ii = cn[i] - 1;
    if (ii < 0) continue;
    for (long j = 0; j < m; j++) {
      long jj = cn[j] - 1;
      if (jj < 0) continue;
      for (long k = adr[ii]; k < adr[ii + 1]; k++)
        if (ci[k] == jj) { a[k] += b[i * m + j]; break; }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Whole-mesh assembly: stiffness_matrix (MEFEL/SRC/globmat.cpp:41-143) and  */
/* conductivity_matrix / capacity_matrix (TRFEL/SRC/globmatt.cpp:19/92)     */
/* ------------------------------------------------------------------------ */

/* kind 0 = hex8 elasticity, 1 = quad4 plane stress, 2 = hex8 conduction,
 * 3 = hex8 capacity, 4 = tet4 elasticity, 5 = tri3 plane stress,
 * 6 = hex20 elasticity, 7 = quad8 plane stress.  coords: nn x 3; elems: ne x nne;
 * cn: ne x ndofe; mats: per element material row (E,nu) or (k,c); thick: per
 * element (quad4) or NULL; rho: per element density (capacity) or NULL
 * (then 1).  Returns 0, or -(e+1) for the first element e of negative volume
 * (tet4; the reference aborts there). */
long or_assemble(int kind, int sym, long ne, const double *coords, const long *elems,
                 const long *cn, const double *emat, const double *thick, const double *rho,
                 long *adr, long *ci, double *a) {
  static const long NNE[8] = {8, 4, 8, 8, 4, 3, 20, 8}, NDOFN[8] = {3, 2, 1, 1, 3, 2, 3, 2};
  long nne = NNE[kind], ndofe = NNE[kind] * NDOFN[kind];
  double xyz[60], xy[16], t[8], r[8];
  double *ke = (double *)malloc(3600 * sizeof(double));
  for (long e = 0; e < ne; e++) {
    const long *nd = elems + e * nne;
    if (kind == 6) {
      for (int i = 0; i < 20; i++)
        for (int c = 0; c < 3; c++) xyz[3 * i + c] = coords[3 * nd[i] + c];
      or_hex20_ke(xyz, emat[2 * e], emat[2 * e + 1], ke);
    } else if (kind == 7) {
      for (int i = 0; i < 8; i++) { xy[2 * i] = coords[3 * nd[i]]; xy[2 * i + 1] = coords[3 * nd[i] + 1]; t[i] = thick[e]; }
      if (or_quad8_ke(xy, emat[2 * e], emat[2 * e + 1], t, ke) != 0) { free(ke); return -(e + 1); }
    } else if (kind == 5) {
      for (int i = 0; i < 3; i++) { xy[2 * i] = coords[3 * nd[i]]; xy[2 * i + 1] = coords[3 * nd[i] + 1]; t[i] = thick[e]; }
      or_tri3_ke(xy, emat[2 * e], emat[2 * e + 1], t, ke);
    } else if (kind == 4) {
      for (int i = 0; i < 4; i++)
        for (int c = 0; c < 3; c++) xyz[3 * i + c] = coords[3 * nd[i] + c];
      if (or_tet4_ke(xyz, emat[2 * e], emat[2 * e + 1], ke) != 0) { free(ke); return -(e + 1); }
    } else if (kind == 1) {
      for (int i = 0; i < 4; i++) { xy[2 * i] = coords[3 * nd[i]]; xy[2 * i + 1] = coords[3 * nd[i] + 1]; t[i] = thick[e]; }
      or_quad4_ke(xy, emat[2 * e], emat[2 * e + 1], t, ke);
    } else {
      for (int i = 0; i < 8; i++)
        for (int c = 0; c < 3; c++) xyz[3 * i + c] = coords[3 * nd[i] + c];
      if (kind == 0) {
        or_hex8_ke(xyz, emat[2 * e], emat[2 * e + 1], ke);
      } else {
        for (int i = 0; i < 8; i++) r[i] = rho ? rho[e] : 1.0;
        if (kind == 2) or_hex8t_kc(xyz, emat[2 * e], emat[2 * e + 1], r, ke, NULL);
        else or_hex8t_kc(xyz, emat[2 * e], emat[2 * e + 1], r, NULL, ke);
      }
    }
    if (sym) or_scr_localize(adr, ci, a, ke, cn + e * ndofe, ndofe);
    else or_cr_localize(adr, ci, a, ke, cn + e * ndofe, ndofe);
  }
  free(ke);
  return 0;
}

/* or_assemble for the 3D elasticity kinds (0 hex8, 4 tet4, 6 hex20) with a general
 * material stiffness per element: dmat ne x 36 (row-major 6 x 6, global
 * system), as elastgmat3d::matstiff (MEFEL/SRC/elastgmat3d.cpp:69) or
 * elastortomat::matstiff give it.  Returns as or_assemble. */
long or_assemble_d(int kind, int sym, long ne, const double *coords, const long *elems, const long *cn,
                   const double *dmat, long *adr, long *ci, double *a) {
  long nne = (kind == 4) ? 4 : (kind == 6 ? 20 : 8), ndofe = 3 * nne;
  double xyz[60];
  double *ke = (double *)malloc(3600 * sizeof(double));
  for (long e = 0; e < ne; e++) {
    const long *nd = elems + e * nne;
    for (int i = 0; i < nne; i++)
      for (int c = 0; c < 3; c++) xyz[3 * i + c] = coords[3 * nd[i] + c];
    if (kind == 4) {
      if (or_tet4_ke_d(xyz, dmat + 36 * e, ke) != 0) { free(ke); return -(e + 1); }
    } else if (kind == 6) {
      hex20_ke(xyz, 0.0, 0.0, dmat + 36 * e, ke);
    } else {
      or_hex8_ke_d(xyz, dmat + 36 * e, ke);
    }
    if (sym) or_scr_localize(adr, ci, a, ke, cn + e * ndofe, ndofe);
    else or_cr_localize(adr, ci, a, ke, cn + e * ndofe, ndofe);
  }
  free(ke);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Matrix-vector products                                                   */
/* ------------------------------------------------------------------------ */

/* symcomprow::mxv_scr, GEFEL/scr.cpp:655-672 */
void or_scr_mxv(long n, const long *adr, const long *ci, const double *a, const double *b,
                double *c) {
  for (long i = 0; i < n; i++) {
    long lj = adr[i], uj = adr[i + 1];
    double s = 0.0, d = b[i];
    for (long j = lj; j < uj; j++) {
      long ii = ci[j];
      s += a[j] * b[ii];
      c[ii] += a[j] * d;
    }
    c[i] = s;
  }
}

/* comprow::mxv_cr, GEFEL/cr.cpp:653-700 (serial branch) */
void or_cr_mxv(long n, const long *adr, const long *ci, const double *a, const double *b,
               double *c) {
  for (long i = 0; i < n; i++) {
    double s = 0.0;
    for (long j = adr[i]; j < adr[i + 1]; j++) s += a[j] * b[ci[j]];
    c[i] = s;
  }
}

/* ss, GEFEL/vector.cpp:2052: plain serial dot product */
static double ss(const double *a, const double *b, long n) {
  double s = 0.0;
  for (long i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* ------------------------------------------------------------------------ */
/* Conjugate gradients                                                      */
/* Status: 0 converged, 1 iteration limit, 2 breakdown |d.p| < zero,        */
/*         5 zero right-hand side                                           */
/* ------------------------------------------------------------------------ */

/* symcomprow::cg_prec with tprec = 1 (Jacobi), GEFEL/scr.cpp:1093-1205.
 * Stops when (r.r)/(f.f) < res; on convergence ani = i, ares = (r.h)/(f.f);
 * otherwise ani/ares are left untouched (as in the reference). */
int or_scr_cg_prec(long n, const long *adr, const long *ci, const double *a, double *x,
                   const double *y, long ni, double res, double zero, long iv, long *ani,
                   double *ares) {
  double *d = (double *)malloc(n * sizeof(double)), *r = (double *)malloc(n * sizeof(double));
  double *p = (double *)malloc(n * sizeof(double)), *h = (double *)malloc(n * sizeof(double));
  int status = 1;
  if (iv == 0)
    for (long i = 0; i < n; i++) x[i] = 0.0;
  or_scr_mxv(n, adr, ci, a, x, p);
  double nory = 0.0;
  for (long i = 0; i < n; i++) { nory += y[i] * y[i]; r[i] = y[i] - p[i]; }
  if (nory < zero) { *ares = nory; *ani = 0; status = 5; }
  for (long i = 0; i < n; i++) h[i] = r[i] / a[adr[i + 1] - 1];
  double nom = ss(r, h, n);
  for (long i = 0; i < n; i++) d[i] = h[i];
  for (long it = 0; it < ni; it++) {
    or_scr_mxv(n, adr, ci, a, d, p);
    double denom = ss(d, p, n);
    if (fabs(denom) < zero) { *ares = nom; *ani = it; status = 2; break; }
    double alpha = nom / denom, rr = 0.0;
    for (long j = 0; j < n; j++) {
      x[j] += alpha * d[j];
      r[j] -= alpha * p[j];
      rr += r[j] * r[j];
    }
    for (long j = 0; j < n; j++) h[j] = r[j] / a[adr[j + 1] - 1];
    denom = nom;
    nom = ss(r, h, n);
    double beta = nom / denom;
    if (fabs(rr / nory) < res) { *ani = it; *ares = nom / nory; status = 0; break; }
    for (long j = 0; j < n; j++) d[j] = beta * d[j] + h[j];
  }
  free(h); free(p); free(r); free(d);
  return status;
}

/* comprow::cg_prec with a noprecond preconditioner (h = r, precond.cpp:166),
 * GEFEL/cr.cpp:1124-1240.  Stops when sqrt((r.h)/(f.f)) < res; then
 * ani = i, ares = r.h (the final assignment at cr.cpp:1236 overrides the
 * in-loop one); on exhaustion ani = ni, ares = r.h. */
int or_cr_cg_prec(long n, const long *adr, const long *ci, const double *a, double *x,
                  const double *y, long ni, double res, double zero, long iv, long *ani,
                  double *ares) {
  double *d = (double *)malloc(n * sizeof(double)), *r = (double *)malloc(n * sizeof(double));
  double *p = (double *)malloc(n * sizeof(double)), *h = (double *)malloc(n * sizeof(double));
  int status = 1;
  long it;
  if (iv == 0)
    for (long i = 0; i < n; i++) x[i] = 0.0;
  or_cr_mxv(n, adr, ci, a, x, p);
  double nory = 0.0;
  for (long i = 0; i < n; i++) { nory += y[i] * y[i]; r[i] = y[i] - p[i]; }
  if (nory < zero) {
    *ares = nory; *ani = 0;
    free(h); free(p); free(r); free(d);
    return 5;
  }
  for (long i = 0; i < n; i++) h[i] = r[i];
  double nom = ss(r, h, n);
  for (long i = 0; i < n; i++) d[i] = h[i];
  for (it = 0; it < ni; it++) {
    or_cr_mxv(n, adr, ci, a, d, p);
    double denom = ss(d, p, n);
    if (fabs(denom) < zero) { status = 2; break; }
    double alpha = nom / denom;
    for (long j = 0; j < n; j++) { x[j] += alpha * d[j]; r[j] -= alpha * p[j]; }
    for (long j = 0; j < n; j++) h[j] = r[j];
    denom = nom;
    nom = ss(r, h, n);
    double beta = nom / denom;
    if (sqrt(nom / nory) < res) { status = 0; break; }
    for (long j = 0; j < n; j++) d[j] = beta * d[j] + h[j];
  }
  *ani = it;
  *ares = nom;
  free(h); free(p); free(r); free(d);
  return status;
}

/* ------------------------------------------------------------------------ */
/* Transient d-form trapezoid, one step (TRFEL/SRC/npsolvert.cpp:1146-1230)  */
/* ------------------------------------------------------------------------ */

/* Given K and C in the same SCR pattern, the step's nodal flux vector rhs,
 * and (d, v) at t_n: builds A = alpha dt K + C (scalgm/addgm, index-aligned,
 * scr.cpp:760/682), p = C (d + (1-alpha) dt v) (mxv_scr), f = alpha dt rhs + p,
 * solves A d' = f by symcomprow::cg_prec (x starts from d when iv = 1, as the
 * reference passes lhs), sets v' = (d' - dd)/dt/alpha.  A is written into
 * `work_a` (length negm). */
int or_trfel_step(long n, const long *adr, const long *ci, const double *ka, const double *ca,
                  double *work_a, const double *rhs, double *d, double *v, double dt,
                  double alpha, long ni, double res, double zero, long iv, long *ani,
                  double *ares) {
  long negm = adr[n];
  double *dd = (double *)malloc(n * sizeof(double)), *p = (double *)malloc(n * sizeof(double));
  double *f = (double *)malloc(n * sizeof(double));
  for (long j = 0; j < n; j++) dd[j] = d[j] + (1.0 - alpha) * dt * v[j];
  or_scr_mxv(n, adr, ci, ca, dd, p);
  for (long k = 0; k < negm; k++) work_a[k] = ka[k] * (dt * alpha);
  for (long k = 0; k < negm; k++) work_a[k] += 1.0 * ca[k];
  for (long j = 0; j < n; j++) f[j] = rhs[j] * alpha * dt + p[j];
  int st = or_scr_cg_prec(n, adr, ci, work_a, d, f, ni, res, zero, iv, ani, ares);
  for (long j = 0; j < n; j++) v[j] = (d[j] - dd[j]) / dt / alpha;
  free(f); free(p); free(dd);
  return st;
}

/* One linear step of the v-form generalized trapezoid, one_step_linear of
 * nonstat_solv_vform_comp (TRFEL/SRC/npsolvert.cpp:367-480): predictor
 * dd = d + (1-alpha) dt v; p = K dd (Kmat->gmxv before K is overwritten);
 * A = alpha dt K + C (scalgm, addgm); f = rhs - p; A v = f (x from the
 * previous v when iv = 1); d = dd + alpha dt v.  solution_correction is the
 * identity for isotropic conduction. */
int or_trfel_step_v(long n, const long *adr, const long *ci, const double *ka, const double *ca,
                    double *work_a, const double *rhs, double *d, double *v, double dt,
                    double alpha, long ni, double res, double zero, long iv, long *ani,
                    double *ares) {
  long negm = adr[n];
  double *dd = (double *)malloc(n * sizeof(double)), *p = (double *)malloc(n * sizeof(double));
  double *f = (double *)malloc(n * sizeof(double));
  for (long j = 0; j < n; j++) dd[j] = d[j] + (1.0 - alpha) * dt * v[j];
  or_scr_mxv(n, adr, ci, ka, dd, p);
  for (long k = 0; k < negm; k++) work_a[k] = ka[k] * (dt * alpha);
  for (long k = 0; k < negm; k++) work_a[k] += 1.0 * ca[k];
  for (long j = 0; j < n; j++) f[j] = rhs[j] - p[j];
  int st = or_scr_cg_prec(n, adr, ci, work_a, v, f, ni, res, zero, iv, ani, ares);
  for (long j = 0; j < n; j++) d[j] = dd[j] + alpha * dt * v[j];
  free(f); free(p); free(dd);
  return st;
}

/* Dirichlet lifting of assemble_init (TRFEL/SRC/globmatt.cpp:1635-1760) for
 * linear hexahedra with isotropic conduction: r_e = nodal values given by
 * prescvalues() (globmatt.cpp:1057: prescribed values on prescribed DOFs,
 * initial values on free ones); f = -K_e r_e (mxv then cmulv(-1)); locglob
 * adds f at DOFs with code number > 0.  emat: ne x (k, c); cne: ne x 8. */
void or_trfel_lift(long ne, const double *coords, const long *elems, const long *cne, const double *emat,
                   const double *rnode, double *rhs) {
  double xyz[24], ke[64], r[8], f[8];
  for (long e = 0; e < ne; e++) {
    const long *nd = elems + e * 8;
    for (int i = 0; i < 8; i++) {
      for (int c = 0; c < 3; c++) xyz[3 * i + c] = coords[3 * nd[i] + c];
      r[i] = rnode[nd[i]];
    }
    double rho1[8] = {1, 1, 1, 1, 1, 1, 1, 1};
    or_hex8t_kc(xyz, emat[2 * e], emat[2 * e + 1], rho1, ke, NULL);
    for (int i = 0; i < 8; i++) {
      double s = 0.0;
      for (int j = 0; j < 8; j++) s += ke[i * 8 + j] * r[j];
      f[i] = -1.0 * s;
    }
    for (int i = 0; i < 8; i++) {
      long ii = cne[e * 8 + i] - 1;
      if (ii >= 0) rhs[ii] += f[i];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Element loads and prescribed displacements of a MEFEL load case          */
/* ------------------------------------------------------------------------ */

/* nnj with an mm x nn matrix N (GEFEL/matrix.cpp:3149-3174): m += N^T N jac,
 * symmetric fill, each product summed over the rows of N from 0. */
static void nnj_rows(double *m, const double *n, double jac, int mm, int nn) {
  for (int i = 0; i < nn; i++) {
    int kk = i * nn + i, ll = kk;
    double s = 0.0;
    for (int k = 0; k < mm; k++) s += n[k * nn + i] * n[k * nn + i];
    m[kk] += s * jac;
    kk++; ll += nn;
    for (int j = i + 1; j < nn; j++) {
      s = 0.0;
      for (int k = 0; k < mm; k++) s += n[k * nn + i] * n[k * nn + j];
      m[kk] += s * jac; m[ll] += s * jac;
      kk++; ll += nn;
    }
  }
}

/* Nodal forces of a surface load given in the global system (ls = 1) on the
 * faces of a linear hexahedron: linhex::node_forces_surf
 * (MEFEL/SRC/linhex.cpp:2543).  Face s (0..5) lies at xi = 1, eta = 1,
 * xi = -1, eta = -1, zeta = 1, zeta = -1; its nodes, in the order of the 4 x 3
 * load values nv[12 s ..] and of jac2d_3d's surface map
 * (GEFEL/difcalc.cpp:1065-1100), are HEX_FACE[s].  For every loaded face:
 * am = sum_{i,j} N^T N |J_s| w_i w_j (bf_matrix, linhex.cpp:126; nnj), with
 * the surface Jacobian of jac2d3d (GEFEL/difcalc.cpp:819-866), then
 * nf += am av where av holds the face's nodal loads (kept between faces, as
 * the reference's vector is).  Only ls = 1 is restated. */
static const int HEX_FACE[6][4] = {{0, 3, 7, 4}, {1, 0, 4, 5}, {2, 1, 5, 6},
                                   {3, 2, 6, 7}, {0, 1, 2, 3}, {4, 7, 6, 5}};

void or_hex8_surface_nf(const double *xyz, const long *ls, const double *nv, double *nf) {
  double x[8], y[8], z[8], am[24 * 24], av[24], v[24], n[3 * 24], bf[8];
  for (int i = 0; i < 8; i++) { x[i] = xyz[3 * i]; y[i] = xyz[3 * i + 1]; z[i] = xyz[3 * i + 2]; }
  memset(av, 0, sizeof(av));
  for (int s = 0; s < 6; s++) {
    if (ls[s] <= 0) continue;
    memset(am, 0, sizeof(am));
    double lx[4], ly[4], lz[4];
    for (int q = 0; q < 4; q++) {
      lx[q] = x[HEX_FACE[s][q]]; ly[q] = y[HEX_FACE[s][q]]; lz[q] = z[HEX_FACE[s][q]];
    }
    for (int i = 0; i < 2; i++) {
      for (int j = 0; j < 2; j++) {
        const double u = GP2[i], w = GP2[j];
        double xi, eta, zeta;
        switch (s) {
          case 0: xi = 1.0; eta = u; zeta = w; break;
          case 1: eta = 1.0; xi = u; zeta = w; break;
          case 2: xi = -1.0; eta = u; zeta = w; break;
          case 3: eta = -1.0; xi = u; zeta = w; break;
          case 4: zeta = 1.0; xi = u; eta = w; break;
          default: zeta = -1.0; xi = u; eta = w; break;
        }
        /* jac2d3d with (xi, eta) = (u, w) on the face's bilinear map */
        double nu4[4], nv4[4];
        dx_bf_lin_4_2d(nu4, w);
        dy_bf_lin_4_2d(nv4, u);
        double dxu = 0.0, dyu = 0.0, dzu = 0.0, dxv = 0.0, dyv = 0.0, dzv = 0.0;
        for (int q = 0; q < 4; q++) {
          dxu += nu4[q] * lx[q]; dyu += nu4[q] * ly[q]; dzu += nu4[q] * lz[q];
          dxv += nv4[q] * lx[q]; dyv += nv4[q] * ly[q]; dzv += nv4[q] * lz[q];
        }
        const double g11 = dxu * dxu + dyu * dyu + dzu * dzu;
        const double g22 = dxv * dxv + dyv * dyv + dzv * dzv;
        const double g12 = dxu * dxv + dyu * dyv + dzu * dzv;
        double jac = sqrt(g11 * g22 - g12 * g12);
        bf_lin_hex_3d(bf, xi, eta, zeta);
        memset(n, 0, sizeof(n));
        for (int a = 0; a < 8; a++) {
          n[0 * 24 + 3 * a] = bf[a];
          n[1 * 24 + 3 * a + 1] = bf[a];
          n[2 * 24 + 3 * a + 2] = bf[a];
        }
        jac = jac * GW2[i] * GW2[j];
        nnj_rows(am, n, jac, 3, 24);
      }
    }
    for (int q = 0; q < 4; q++)
      for (int c = 0; c < 3; c++) av[3 * HEX_FACE[s][q] + c] = nv[12 * s + 3 * q + c];
    for (int i = 0; i < 24; i++) {
      double t = 0.0;
      for (int j = 0; j < 24; j++) t += am[24 * i + j] * av[j];
      v[i] = t;
    }
    for (int i = 0; i < 24; i++) nf[i] = v[i] + nf[i];
  }
}

/* Nodal forces of edge loads (le = 1) on a plane-stress bilinear quad:
 * planeelemlq::nodeforces (MEFEL/SRC/plelemlq.cpp:2433-2514).  Edge e runs
 * from node e to node e+1 (mod 4) at eta = 1, xi = -1, eta = -1, xi = 1; its
 * 2 x 2 load values are nv[4 e ..]; am = sum_i N^T N |J_e| w_i with the edge
 * Jacobian of jac1d2d (GEFEL/difcalc.cpp:730-760), av zeroed per edge. */
void or_quad4_edge_nf(const double *xy, const long *le, const double *nv, double *nf) {
  double x[4], y[4], am[64], av[8], v[8], n[2 * 8], bf[4];
  for (int i = 0; i < 4; i++) { x[i] = xy[2 * i]; y[i] = xy[2 * i + 1]; }
  for (int e = 0; e < 4; e++) {
    if (le[e] != 1) continue;
    memset(am, 0, sizeof(am));
    const int a0 = e, a1 = (e + 1) & 3;
    for (int i = 0; i < 2; i++) {
      const double g = GP2[i];
      double xi, eta;
      switch (e) {
        case 0: eta = 1.0; xi = g; break;
        case 1: xi = -1.0; eta = g; break;
        case 2: eta = -1.0; xi = g; break;
        default: xi = 1.0; eta = g; break;
      }
      bf_lin_4_2d(bf, xi, eta);
      memset(n, 0, sizeof(n));
      for (int a = 0; a < 4; a++) {
        n[0 * 8 + 2 * a] = bf[a];
        n[1 * 8 + 2 * a + 1] = bf[a];
      }
      /* jac1d2d: dx_bf_lin_1d = (-0.5, 0.5) on the edge's two nodes */
      double dx = 0.0, dy = 0.0;
      dx += -0.5 * x[a0]; dy += -0.5 * y[a0];
      dx += 0.5 * x[a1]; dy += 0.5 * y[a1];
      double jac = sqrt(dx * dx + dy * dy);
      jac *= GW2[i];
      nnj_rows(am, n, jac, 2, 8);
    }
    memset(av, 0, sizeof(av));
    av[2 * a0] = nv[4 * e]; av[2 * a0 + 1] = nv[4 * e + 1];
    av[2 * a1] = nv[4 * e + 2]; av[2 * a1 + 1] = nv[4 * e + 3];
    for (int i = 0; i < 8; i++) {
      double t = 0.0;
      for (int j = 0; j < 8; j++) t += am[8 * i + j] * av[j];
      v[i] = t;
    }
    for (int i = 0; i < 8; i++) nf[i] = nf[i] + v[i];
  }
}

/* loadcase::prdisplcontrib (MEFEL/SRC/loadcase.cpp:615-664) for one element:
 * r_e from the prescribed displacements (elprdispl, globmat.cpp:1372: code
 * number c < 0 takes pd[-c-1], others 0), f = -(K_e r_e), added at the
 * element's DOFs with code number > 0.  ke: the element's stiffness
 * (ndofe x ndofe, as assembled). */
void or_prescribed_contrib(int ndofe, const double *ke, const long *cn, const double *pd, double *rhs) {
  double r[60], f[60];
  for (int i = 0; i < ndofe; i++) r[i] = cn[i] < 0 ? pd[-cn[i] - 1] : 0.0;
  for (int i = 0; i < ndofe; i++) {
    double s = 0.0;
    for (int j = 0; j < ndofe; j++) s += ke[i * ndofe + j] * r[j];
    f[i] = -1.0 * s;
  }
  for (int i = 0; i < ndofe; i++)
    if (cn[i] > 0) rhs[cn[i] - 1] += f[i];
}
