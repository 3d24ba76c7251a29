// Element loads of a MEFEL load case: consistent nodal forces of surface
// tractions on linear hexahedra and of edge loads on bilinear plane quads
// (host code; a load case touches a surface layer of the mesh, so the
// integrals are a few flops per loaded element and stay on the host, next to
// the deck reader that reads them).
//
// Reference path: loadcase::forcecontrib (MEFEL/SRC/loadcase.cpp:546-601)
// adds, after the nodal loads, every loaded element's nodal-force vector
// (loadel::surfaceload / edgeload, MEFEL/SRC/loadel.cpp:464/550) at the
// element's code numbers.  The vectors are
//   hexahedron, surface s:  nf += (sum_gp N^T N |J_s| w) av
//     (linhex::node_forces_surf, MEFEL/SRC/linhex.cpp:2543; surface Jacobian
//     jac2d3d, GEFEL/difcalc.cpp:819),
//   quad, edge e:           nf += (sum_gp N^T N |J_e| w) av
//     (planeelemlq::nodeforces, MEFEL/SRC/plelemlq.cpp:2433; jac1d2d,
//     GEFEL/difcalc.cpp:730),
// with av the load values at the face's (edge's) nodes.  N^T N is non-zero
// only between equal components of two nodes, so the products below run over
// node pairs of the face and the sums keep the reference's order (Gauss
// points outer, nodes inner), which reproduces its nodal forces exactly.
#include <cmath>
#include <cstring>
#include <string>

#include "sgpu_internal.cuh"

namespace sgpu {

namespace {

constexpr double kGp2[2] = {-0.577350269189626, 0.577350269189626};  // GEFEL/intp.cpp:26-27

// nodes of the hexahedron's faces in the order of their load values and of
// the surface map: xi = 1, eta = 1, xi = -1, eta = -1, zeta = 1, zeta = -1
constexpr int kHexFace[6][4] = {{0, 3, 7, 4}, {1, 0, 4, 5}, {2, 1, 5, 6}, {3, 2, 6, 7}, {0, 1, 2, 3}, {4, 7, 6, 5}};

void hex_n(double xi, double eta, double zeta, double *n) {
  static const double sx[8] = {1, -1, -1, 1, 1, -1, -1, 1};
  static const double sy[8] = {1, 1, -1, -1, 1, 1, -1, -1};
  static const double sz[8] = {1, 1, 1, 1, -1, -1, -1, -1};
  for (int a = 0; a < 8; a++) n[a] = (1.0 + sx[a] * xi) * (1.0 + sy[a] * eta) * (1.0 + sz[a] * zeta) / 8.0;
}

void quad_n(double xi, double eta, double *n) {
  n[0] = 0.25 * (1.0 + xi) * (1.0 + eta);
  n[1] = 0.25 * (1.0 - xi) * (1.0 + eta);
  n[2] = 0.25 * (1.0 - xi) * (1.0 - eta);
  n[3] = 0.25 * (1.0 + xi) * (1.0 - eta);
}

}  // namespace

// 24 nodal forces of the surface loads of one hexahedron: flags[6] (1 =
// loaded, values in the global system; 0 = not loaded), values[72] (face s:
// 4 nodes x 3 components at 12 s); xyz: the 8 nodes' coordinates.  Returns
// false for a flag this path does not take (2: values in a local system).
bool hex8_surface_forces(const double *xyz, const int32_t *flags, const double *values, double *nf) {
  double am[24][24], av[24], n8[8];
  std::memset(av, 0, sizeof(av));
  std::memset(nf, 0, 24 * sizeof(double));
  for (int s = 0; s < 6; s++) {
    if (flags[s] == 0) continue;
    if (flags[s] != 1) return false;
    std::memset(am, 0, sizeof(am));
    const int *fn = kHexFace[s];
    for (int i = 0; i < 2; i++) {
      for (int j = 0; j < 2; j++) {
        const double u = kGp2[i], w = kGp2[j];
        double xi, eta, zeta;
        switch (s) {
          case 0: xi = 1.0; eta = u; zeta = w; break;
          case 1: eta = 1.0; xi = u; zeta = w; break;
          case 2: xi = -1.0; eta = u; zeta = w; break;
          case 3: eta = -1.0; xi = u; zeta = w; break;
          case 4: zeta = 1.0; xi = u; eta = w; break;
          default: zeta = -1.0; xi = u; eta = w; break;
        }
        // tangents of the face's bilinear map at (u, w)
        const double du[4] = {0.25 * (1.0 + w), 0.25 * (-1.0 - w), 0.25 * (-1.0 + w), 0.25 * (1.0 - w)};
        const double dw[4] = {0.25 * (1.0 + u), 0.25 * (1.0 - u), 0.25 * (-1.0 + u), 0.25 * (-1.0 - u)};
        double tu[3] = {0.0, 0.0, 0.0}, tw[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < 4; q++)
          for (int c = 0; c < 3; c++) {
            tu[c] += du[q] * xyz[3 * fn[q] + c];
            tw[c] += dw[q] * xyz[3 * fn[q] + c];
          }
        const double g11 = tu[0] * tu[0] + tu[1] * tu[1] + tu[2] * tu[2];
        const double g22 = tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2];
        const double g12 = tu[0] * tw[0] + tu[1] * tw[1] + tu[2] * tw[2];
        const double jac = std::sqrt(g11 * g22 - g12 * g12);  // weights are 1
        hex_n(xi, eta, zeta, n8);
        for (int a = 0; a < 8; a++)
          for (int b = 0; b < 8; b++) {
            const double p = (0.0 + n8[a] * n8[b]) * jac;
            for (int c = 0; c < 3; c++) am[3 * a + c][3 * b + c] += p;
          }
      }
    }
    for (int q = 0; q < 4; q++)
      for (int c = 0; c < 3; c++) av[3 * fn[q] + c] = values[12 * s + 3 * q + c];
    for (int r = 0; r < 24; r++) {
      double t = 0.0;
      for (int k = 0; k < 24; k++) t += am[r][k] * av[k];
      nf[r] = t + nf[r];
    }
  }
  return true;
}

// 8 nodal forces of the edge loads of one plane quad: flags[4] (1 = loaded;
// other positive flags carry values that the reference reads and does not
// apply), values[16] (edge e from node e to node e+1: 2 nodes x 2 components
// at 4 e); xy: the 4 nodes' coordinates.
bool quad4_edge_forces(const double *xy, const int32_t *flags, const double *values, double *nf) {
  double am[8][8], av[8], n4[4];
  std::memset(nf, 0, 8 * sizeof(double));
  for (int e = 0; e < 4; e++) {
    if (flags[e] < 0) return false;
    if (flags[e] != 1) continue;
    std::memset(am, 0, sizeof(am));
    const int a0 = e, a1 = (e + 1) & 3;
    for (int i = 0; i < 2; i++) {
      const double g = kGp2[i];
      double xi, eta;
      switch (e) {
        case 0: eta = 1.0; xi = g; break;
        case 1: xi = -1.0; eta = g; break;
        case 2: eta = -1.0; xi = g; break;
        default: xi = 1.0; eta = g; break;
      }
      quad_n(xi, eta, n4);
      double dx = 0.0, dy = 0.0;
      dx += -0.5 * xy[2 * a0]; dy += -0.5 * xy[2 * a0 + 1];
      dx += 0.5 * xy[2 * a1]; dy += 0.5 * xy[2 * a1 + 1];
      const double jac = std::sqrt(dx * dx + dy * dy);  // weights are 1
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
          const double p = (0.0 + n4[a] * n4[b]) * jac;
          am[2 * a][2 * b] += p;
          am[2 * a + 1][2 * b + 1] += p;
        }
    }
    std::memset(av, 0, sizeof(av));
    av[2 * a0] = values[4 * e];
    av[2 * a0 + 1] = values[4 * e + 1];
    av[2 * a1] = values[4 * e + 2];
    av[2 * a1 + 1] = values[4 * e + 3];
    for (int r = 0; r < 8; r++) {
      double t = 0.0;
      for (int k = 0; k < 8; k++) t += am[r][k] * av[k];
      nf[r] = nf[r] + t;
    }
  }
  return true;
}

// adds the nodal forces of nle element-load records into f (equation order)
int add_element_loads(int kind, const double *coords, const int64_t *elems, const int64_t *cn, int64_t nn,
                      int64_t ne, int64_t nle, const int64_t *eid, const int32_t *flags, const double *values,
                      double *f) {
  if (nle <= 0) return SGPU_OK;
  const bool hex = kind == SGPU_ELEM_HEX8, quad = kind == SGPU_ELEM_QUAD4;
  if (!hex && !quad) return fail(SGPU_BAD_INPUT, "element loads are defined for hex8 surfaces and quad4 edges");
  const int nne = hex ? 8 : 4, ndofn = hex ? 3 : 2, nfl = hex ? 6 : 4, nval = hex ? 72 : 16;
  double xyz[24], nf[24];
  for (int64_t r = 0; r < nle; r++) {
    const int64_t e = eid[r];
    if (e < 0 || e >= ne) return fail(SGPU_BAD_INPUT, "element load " + std::to_string(r + 1) + ": element out of range");
    const int64_t *nd = elems + e * nne;
    for (int a = 0; a < nne; a++) {
      if (nd[a] < 0 || nd[a] >= nn) return fail(SGPU_BAD_INPUT, "element node out of range");
      for (int c = 0; c < (hex ? 3 : 2); c++) xyz[(hex ? 3 : 2) * a + c] = coords[3 * nd[a] + c];
    }
    const bool ok = hex ? hex8_surface_forces(xyz, flags + r * nfl, values + r * nval, nf)
                        : quad4_edge_forces(xyz, flags + r * nfl, values + r * nval, nf);
    if (!ok)
      return fail(SGPU_BAD_INPUT, "element load " + std::to_string(r + 1) +
                                      ": only loads given in the global system (flag 1) are supported");
    for (int a = 0; a < nne; a++)
      for (int c = 0; c < ndofn; c++) {
        const int64_t q = cn[nd[a] * ndofn + c];
        if (q > 0) f[q - 1] += nf[ndofn * a + c];
      }
  }
  return SGPU_OK;
}

}  // namespace sgpu

extern "C" SGPU_API int sgpu_mesh_element_loads(const sgpu_mesh *mesh, int64_t nle, const int64_t *eid,
                                                const int32_t *flags, const double *values, double *f) {
  if (!mesh || !f) return sgpu::fail(SGPU_BAD_INPUT, "null argument");
  if (nle < 0) return sgpu::fail(SGPU_BAD_INPUT, "negative element-load count");
  if (nle > 0 && (!eid || !flags || !values)) return sgpu::fail(SGPU_BAD_INPUT, "null element-load arrays");
  if (!mesh->coords || !mesh->elems || !mesh->cn) return sgpu::fail(SGPU_BAD_INPUT, "empty mesh");
  return sgpu::add_element_loads(mesh->kind, mesh->coords, mesh->elems, mesh->cn, mesh->nn, mesh->ne, nle, eid,
                                 flags, values, f);
}
