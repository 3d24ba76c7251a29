// The binding that sends MEFEL's stiffness-matrix assembly to the GPU.
//
// It replaces stiffness_matrix (MEFEL/SRC/globmat.cpp:41-216) at link time:
// linking SIFEL's unchanged MEFEL objects with
//   -Wl,--wrap=_Z16stiffness_matrixl
// makes every call land here.  When the problem is one the GPU path covers
// -- linear statics, symmetric compressed-row storage, every element a
// linear hexahedron (linearhex, 102) of one isotropic elastic material
// (elisomat), no hanging nodes, no local node systems, all elements active,
// and no matrix assembled before -- the matrix is integrated and assembled
// by sgpu_assemble from MEFEL's topology (node coordinates, element nodes,
// gencodnum's code numbers, each element's E and nu) and copied back into
// the gmatrix's symcomprow arrays (n, negm, adr, adra, ci, a: the state
// symcomprow::initiate and localize leave, GEFEL/scr.cpp:556 and :422);
// then gmatrix::prepmat runs as in the reference.  Any other problem, or
// SIFEL_GPU=off / SIFEL_GPU_ASSEMBLY=off, calls the original routine.  The
// pattern is the reference's bit for bit; the values agree with its element
// loop to rounding (the GPU sums each entry in its own order).
//
// Link this file into MEFEL programs only (it uses MEFEL's globals); the
// solver binding sifel_gpu_shim.cpp serves both MEFEL and TRFEL.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "alias.h"
#include "elastisomat.h"
#include "element.h"
#include "galias.h"
#include "gmatrix.h"
#include "gtopology.h"
#include "mechmat.h"
#include "mechtop.h"
#include "node.h"
#include "probdesc.h"
#include "scr.h"
#include "sifelgpu.h"

// MEFEL's globals (MEFEL/SRC/global.h)
extern probdesc *Mp;
extern gtopology *Gtm;
extern mechtop *Mt;
extern mechmat *Mm;
extern gmatrix *Smat;
extern long Ndofm;
extern long Mespr;

namespace {

bool gpu_assembly_wanted() {
  const char *g = getenv("SIFEL_GPU"), *a = getenv("SIFEL_GPU_ASSEMBLY");
  return !(g && !strcmp(g, "off")) && !(a && !strcmp(a, "off"));
}

// the mesh of the problem in sgpu_assemble's terms, or false when the
// problem is outside what the GPU path assembles
bool mesh_arrays(std::vector<double> &xyz, std::vector<int64_t> &elems, std::vector<int64_t> &cn,
                 std::vector<double> &emat) {
  if (!Mp || !Gtm || !Mt || !Mm || Smat != nullptr) return false;
  if (Mp->tprob != linear_statics || Mp->tstorsm != symm_comp_rows) return false;
  const long nn = Gtm->nn, ne = Mt->ne;
  if (nn <= 0 || ne <= 0 || Gtm->ne != ne || !Gtm->gnodes || !Gtm->gelements || !Mt->elements) return false;
  xyz.resize((size_t)nn * 3);
  cn.resize((size_t)nn * 3);
  for (long i = 0; i < nn; i++) {
    const gnode &g = Gtm->gnodes[i];
    if (g.ndofn != 3 || !g.cn) return false;
    if (Mt->nodes && Mt->nodes[i].transf != 0) return false;
    xyz[3 * i] = g.x;
    xyz[3 * i + 1] = g.y;
    xyz[3 * i + 2] = g.z;
    for (int c = 0; c < 3; c++) cn[(size_t)3 * i + c] = g.cn[c];
  }
  elems.resize((size_t)ne * 8);
  emat.resize((size_t)ne * 2);
  for (long e = 0; e < ne; e++) {
    const element &el = Mt->elements[e];
    if (el.te != linearhex || (Gtm->leso && Gtm->leso[e] != 1)) return false;
    if (Mt->give_ndofe(e) != Gtm->give_ndofe(e)) return false;  // hanging nodes
    if (el.nm != 1 || el.tm[0] != elisomat || !Mm->eliso) return false;
    const gelement &ge = Gtm->gelements[e];
    if (ge.nne != 8 || !ge.nodes) return false;
    for (int a = 0; a < 8; a++) elems[(size_t)8 * e + a] = ge.nodes[a];
    const elastisomat &mat = Mm->eliso[el.idm[0]];
    emat[(size_t)2 * e] = mat.e;
    emat[(size_t)2 * e + 1] = mat.nu;
  }
  return true;
}

}  // namespace

extern "C" {

void __real__Z16stiffness_matrixl(long lcid);

void __wrap__Z16stiffness_matrixl(long lcid) {
  std::vector<double> xyz, emat;
  std::vector<int64_t> elems, cn;
  if (!gpu_assembly_wanted() || !mesh_arrays(xyz, elems, cn, emat)) {
    __real__Z16stiffness_matrixl(lcid);
    return;
  }
  // SIFEL checks errno after its computations (check_math_err,
  // GEFEL/mathem.cpp:1725) and aborts on any value; the CUDA runtime may
  // leave one behind while it starts (probing files), so errno is kept
  const int saved_errno = errno;
  sgpu_mesh mesh;
  memset(&mesh, 0, sizeof(mesh));
  mesh.kind = SGPU_ELEM_HEX8;
  mesh.ndofn = 3;
  mesh.nn = Gtm->nn;
  mesh.coords = xyz.data();
  mesh.ne = Mt->ne;
  mesh.elems = elems.data();
  mesh.cn = cn.data();
  mesh.emat = emat.data();
  sgpu_matrix h = nullptr;
  int64_t n = 0, negm = 0;
  int st = sgpu_assemble(&mesh, &h, nullptr);
  if (st == SGPU_OK) st = sgpu_matrix_info(h, &n, nullptr);
  if (st == SGPU_OK && n != Ndofm) st = SGPU_BAD_INPUT;
  if (st == SGPU_OK) st = sgpu_matrix_download(h, 1, nullptr, nullptr, nullptr, &negm);
  if (st != SGPU_OK) {
    fprintf(stderr, "\n GPU assembly not used (%s); assembling on the CPU\n", sgpu_last_error());
    if (h) sgpu_matrix_destroy(h);
    errno = saved_errno;
    __real__Z16stiffness_matrixl(lcid);
    return;
  }
  // the gmatrix and its symcomprow as gmatrix::initiate leaves them
  Smat = new gmatrix;
  Smat->setval(Mp->ssle);
  Smat->n = Ndofm;
  Smat->ts = symm_comp_rows;
  Smat->alloc();
  symcomprow *scr = Smat->scr;
  scr->allocadr(Ndofm);
  scr->negm = negm;
  scr->ci = new long[negm];
  scr->a = new double[negm];
  static_assert(sizeof(long) == sizeof(int64_t), "GEFEL's long is the ABI's int64_t");
  st = sgpu_matrix_download(h, 1, reinterpret_cast<int64_t *>(scr->adr), reinterpret_cast<int64_t *>(scr->ci),
                            scr->a, &negm);
  sgpu_matrix_destroy(h);
  if (st != SGPU_OK) {
    fprintf(stderr, "\n GPU assembly failed (%s)\n", sgpu_last_error());
    abort();
  }
  memcpy(scr->adra, scr->adr, (size_t)(Ndofm + 1) * sizeof(long));
  errno = saved_errno;
  Smat->prepmat(0.0, Mespr);
}

}  // extern "C"
