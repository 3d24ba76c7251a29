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

// Node coordinates (nn x 3) and code numbers (nn x ndofn) of Gtm's nodes,
// from which sgpu_matrix_set_rigid_body_modes forms the rigid-body modes on
// the device; returns ndofn, 0 when there is no usable topology.
static int node_arrays(std::vector<double> &xyz, std::vector<int64_t> &cn) {
  if (&Gtm == nullptr || Gtm == nullptr || Gtm->nn <= 0 || Gtm->gnodes == nullptr) return 0;
  const long nn = Gtm->nn;
  const long ndofn = Gtm->gnodes[0].ndofn;
  if (ndofn < 1 || ndofn > 3) return 0;
  xyz.resize((size_t)nn * 3);
  cn.resize((size_t)nn * ndofn);
  for (long i = 0; i < nn; i++) {
    const gnode &g = Gtm->gnodes[i];
    if (g.ndofn != ndofn || g.cn == nullptr) return 0;
    xyz[3 * i] = g.x;
    xyz[3 * i + 1] = g.y;
    xyz[3 * i + 2] = g.z;
    for (long c = 0; c < ndofn; c++) cn[(size_t)i * ndofn + c] = g.cn[c];
  }
  return (int)ndofn;
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
    std::vector<double> xyz;
    std::vector<int64_t> cn;
    const int ndofn = st == SGPU_OK ? node_arrays(xyz, cn) : 0;
    if (ndofn > 0) st = sgpu_matrix_set_rigid_body_modes(m, (int64_t)(xyz.size() / 3), ndofn, xyz.data(), cn.data());
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
