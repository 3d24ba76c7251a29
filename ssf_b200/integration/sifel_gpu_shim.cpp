// The binding a SIFEL maintainer adds to send GEFEL's Jacobi-PCG to the GPU.
//
// It replaces symcomprow::cg_prec (GEFEL/scr.cpp:1093) at link time:
// linking SIFEL's unchanged objects with
//   -Wl,--wrap=_ZN10symcomprow7cg_precEPdS0_ldRlRddlldP7ISolver
// makes every call to cg_prec from gmatrix::solve_system (GEFEL/gmatrix.cpp:
// 1225-1227) land here; the diagonal (Jacobi) case, tprec == 1, goes to
// sgpu_scr_cg_prec with the storage object's own arrays, every other case to
// the original routine.  SIFEL_GPU=off keeps the CPU routine, SIFEL_GPU=mixed
// selects the mixed-precision form, SIFEL_GPU=agg (agg64) the flexible CG with
// the aggregation multilevel preconditioner in FP32 (FP64) -- GEFEL's own
// precondtype boss = 101 -- on the same criterion.  Its near-null space is
// built from MEFEL's topology when the program has one (the rigid-body modes
// of the nodes' coordinates at their code numbers, as BOSS's gener_rbm_1/2,
// GEFEL/aggregator.cpp:638-700, build them per aggregate); otherwise (TRFEL,
// or nodes of mixed DOF counts) the library's default, one constant per node
// component.  Decks in SIFEL's input format run unchanged.
#include <cerrno>
#include <cstdlib>
#include <cstring>

#include <vector>

#include "gtopology.h"
#include "iotools.h"
#include "scr.h"
#include "sifelgpu.h"

// MEFEL's global topology (MEFEL/SRC/global.h:132); absent from TRFEL programs
extern gtopology *Gtm __attribute__((weak));

// Rigid-body modes of Gtm's nodes in equation order (n x k, column after
// column); k = 0 when there is no usable topology.
static int rigid_body_modes(long n, std::vector<double> &B) {
  if (&Gtm == nullptr || Gtm == nullptr || Gtm->nn <= 0 || Gtm->gnodes == nullptr) return 0;
  const long nn = Gtm->nn;
  const long ndofn = Gtm->gnodes[0].ndofn;
  if (ndofn != 2 && ndofn != 3) return 0;
  double cx = 0, cy = 0, cz = 0;
  for (long i = 0; i < nn; i++) {
    if (Gtm->gnodes[i].ndofn != ndofn) return 0;
    cx += Gtm->gnodes[i].x;
    cy += Gtm->gnodes[i].y;
    cz += Gtm->gnodes[i].z;
  }
  cx /= nn;
  cy /= nn;
  cz /= nn;
  const int k = ndofn == 3 ? 6 : 3;
  B.assign((size_t)n * k, 0.0);
  for (long i = 0; i < nn; i++) {
    const gnode &g = Gtm->gnodes[i];
    const double x = g.x - cx, y = g.y - cy, z = g.z - cz;
    for (long c = 0; c < ndofn; c++) {
      const long e = g.cn[c];
      if (e <= 0 || e > n) continue;
      double *row = &B[e - 1];
      if (ndofn == 3) {  // translations, then rotations about z, x, y
        const double r[3][6] = {{1, 0, 0, -y, 0, z}, {0, 1, 0, x, -z, 0}, {0, 0, 1, 0, y, -x}};
        for (int q = 0; q < 6; q++) row[(size_t)q * n] = r[c][q];
      } else {
        const double r[2][3] = {{1, 0, -y}, {0, 1, x}};
        for (int q = 0; q < 3; q++) row[(size_t)q * n] = r[c][q];
      }
    }
  }
  return k;
}

extern "C" {

void __real__ZN10symcomprow7cg_precEPdS0_ldRlRddlldP7ISolver(symcomprow *self, double *x, double *y, long ni,
                                                             double res, long &ani, double &ares, double zero,
                                                             long iv, long tprec, double par, ISolver *sdirect);

void __wrap__ZN10symcomprow7cg_precEPdS0_ldRlRddlldP7ISolver(symcomprow *self, double *x, double *y, long ni,
                                                             double res, long &ani, double &ares, double zero,
                                                             long iv, long tprec, double par, ISolver *sdirect) {
  const char *mode_env = getenv("SIFEL_GPU");
  if (tprec != 1 || (mode_env && !strcmp(mode_env, "off"))) {
    __real__ZN10symcomprow7cg_precEPdS0_ldRlRddlldP7ISolver(self, x, y, ni, res, ani, ares, zero, iv, tprec, par,
                                                            sdirect);
    return;
  }
  const bool agg = mode_env && (!strcmp(mode_env, "agg") || !strcmp(mode_env, "agg64"));
  const int mode = (mode_env && (!strcmp(mode_env, "mixed") || !strcmp(mode_env, "agg"))) ? SGPU_MIXED : SGPU_FP64;
  int64_t a_ni = ani;
  double a_res = ares;
  // SIFEL checks errno after the solve (check_math_err, GEFEL/mathem.cpp:1725)
  // and aborts on any value; the CUDA runtime may leave one behind (e.g. from
  // probing files while loading the driver), so errno is kept as it was
  const int saved_errno = errno;
  int st;
  if (agg) {
    sgpu_matrix m = NULL;
    st = sgpu_matrix_create(self->n, self->adr, self->ci, self->a, 1, &m);
    std::vector<double> B;
    const int k = st == SGPU_OK ? rigid_body_modes(self->n, B) : 0;
    if (k > 0) st = sgpu_matrix_set_nullspace(m, k, B.data());
    if (st == SGPU_OK)
      st = sgpu_matrix_pcg(m, x, y, ni, res, zero, iv, SGPU_CRIT_SCR_PREC, SGPU_PREC_AGG, mode, &a_ni, &a_res, NULL);
    if (m) sgpu_matrix_destroy(m);
  } else {
    st = sgpu_scr_cg_prec(self->n, self->adr, self->ci, self->a, x, y, ni, res, &a_ni, &a_res, zero, iv, mode, NULL);
  }
  errno = saved_errno;
  ani = (long)a_ni;
  ares = a_res;
  // the reference's own messages for the same outcomes (scr.cpp:1117-1151)
  if (st == SGPU_ZERO_RHS)
    print_err("right hand side vector has zero norm", __FILE__, __LINE__, __func__);
  else if (st == SGPU_BREAKDOWN)
    print_err("denominator in alpha expression is equal to zero", __FILE__, __LINE__, __func__);
  else if (st != SGPU_OK && st != SGPU_NOT_CONVERGED)
    print_err("GPU PCG failed: %s", __FILE__, __LINE__, __func__, sgpu_last_error());
}

}  // extern "C"
