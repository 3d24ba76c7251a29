/*
 * sifelgpu.h -- C ABI of libsifelgpu.so, the B200 (sm_100a) implementation of
 * SIFEL's linear finite-element hot path: element integration, assembly into
 * GEFEL compressed-row storage and the Jacobi-preconditioned CG solve.
 *
 * Conventions shared by every entry point:
 *  - plain C types only; `int64_t` stands for the reference's `long`;
 *  - matrix storages are GEFEL's: CR (`comprow`, GEFEL/cr.h:96-109) holds all
 *    entries of each row with sorted columns; SCR (`symcomprow`,
 *    GEFEL/scr.h:83-96) holds the lower triangle of each row with sorted
 *    columns, so the diagonal is the last entry of its row; `adr` has n+1
 *    entries and adr[n] = negm;
 *  - code numbers are 1-based; 0 (or negative) means "no equation", as
 *    produced by gtopology::gencodnum (GEFEL/gtopology.cpp:1619);
 *  - pointers without a `_d` suffix on the function name are HOST pointers;
 *    the library copies in, computes on the current CUDA device and copies
 *    results back before returning;
 *  - every call returns an sgpu_status; nothing throws across the ABI;
 *    sgpu_last_error() gives a one-line description of the last failure.
 */
#ifndef SIFELGPU_H
#define SIFELGPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define SGPU_API __attribute__((visibility("default")))
#else
#define SGPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference reports through print_err (GEFEL/iotools.cpp:25)
 * and returns early; here every condition is a return value. */
typedef enum {
  SGPU_OK = 0,
  SGPU_NOT_CONVERGED = 1, /* iteration limit reached (reference: ani/ares untouched) */
  SGPU_BREAKDOWN = 2,     /* |d.p| < zero (scr.cpp:1146-1151, cr.cpp:1177-1181) */
  SGPU_BAD_INPUT = 3,     /* malformed storage, sizes, non-positive diagonal, ... */
  SGPU_CUDA_ERROR = 4,    /* a CUDA runtime call failed */
  SGPU_ZERO_RHS = 5       /* (f.f) < zero (scr.cpp:1117-1120, cr.cpp:1160-1164) */
} sgpu_status;

/* Stopping criteria of the reference routines (each keeps its own). */
typedef enum {
  SGPU_CRIT_SCR_PREC = 0, /* (r.r)/(f.f) < res   symcomprow::cg_prec, GEFEL/scr.cpp:1188 */
  SGPU_CRIT_CR_PREC = 1,  /* sqrt((r.h)/(f.f)) < res  comprow::cg_prec, GEFEL/cr.cpp:1217 */
  SGPU_CRIT_TRUE = 2      /* ||f - K x|| / ||f|| < res with the residual recomputed in FP64 */
} sgpu_criterion;

/* Arithmetic of the iteration. */
typedef enum {
  SGPU_FP64 = 0,  /* plain FP64 PCG: the drop-in for the reference call */
  SGPU_MIXED = 1  /* FP32 inner PCG on the Jacobi-scaled matrix, with the true
                     residual and the solution update recomputed in FP64
                     (reliable-update iterative refinement) */
} sgpu_mode;

/* Solve report; every field is written by every solve entry point. */
typedef struct {
  int64_t iterations;       /* PCG iterations performed (all inner ones for MIXED) */
  int64_t refinements;      /* FP64 residual recomputations (MIXED), else 0 */
  double crit_value;        /* value of the routine's own criterion at exit */
  double rh_over_ff;        /* (r.h)/(f.f) at exit, the reference's `ares` on convergence */
  double true_relres;       /* ||f - K x||_2 / ||f||_2, recomputed in FP64 on the GPU */
  double setup_ms;          /* upload + format conversion, device timed */
  double solve_ms;          /* iteration, device timed */
  double spmv_bytes;        /* algorithmic bytes of one SpMV of the iteration's format */
  int32_t spmv_format;      /* 0 = CSR, 3 = 3x3 block rows (BSR3) */
  int32_t spmv_variant;     /* autotuned kernel variant id */
  int32_t fallback;         /* MIXED: 1 if the FP32 iteration stagnated and the
                               solve was finished in FP64 from its iterate */
  int32_t tile_rows;        /* batched solves: rows per work segment picked by the tuner */
  double precond_setup_ms;  /* SGPU_PREC_AGG: hierarchy set-up of this call (0 when reused) */
  int32_t precond_levels;   /* SGPU_PREC_AGG: levels of the hierarchy, the dense one included */
  int32_t precond_coarse_n; /* SGPU_PREC_AGG: equations of the dense coarsest level */
} sgpu_solve_info;

/* Preconditioners (the `prec` argument of the sgpu_matrix_pcg* calls).  The
 * values follow GEFEL's precondtype (GEFEL/galias.h:103). */
typedef enum {
  SGPU_PREC_NONE = 0,   /* noprecond */
  SGPU_PREC_JACOBI = 1, /* diagprec: h = r / diag (scr.cpp:897-904) */
  SGPU_PREC_AGG = 101   /* boss: aggregation multilevel preconditioner (see
                           sgpu_matrix_set_nullspace); the iteration becomes a
                           flexible CG in FP64 whose preconditioner is one
                           V-cycle, in FP32 for SGPU_MIXED, FP64 for SGPU_FP64 */
} sgpu_precond;

/* ------------------------------------------------------------------------ */
/* Drop-in solver entry points (host arrays)                                */
/* ------------------------------------------------------------------------ */

/* Replaces symcomprow::cg_prec (GEFEL/scr.cpp:1093-1205) with tprec = 1, as
 * dispatched by gmatrix::solve_system (GEFEL/gmatrix.cpp:1225-1227).
 * Same arguments and meaning: x (in/out; used as start vector when iv = 1),
 * y = right-hand side (not modified), ni iteration limit, res threshold on
 * (r.r)/(f.f), zero = the gmatrix's computer zero (1e-30).  As in the
 * reference, *ani = i and *ares = (r.h)/(f.f) are written only on
 * convergence.  mode: SGPU_FP64 reproduces the reference's iteration;
 * SGPU_MIXED runs the FP32-inner / FP64-refined form to the same threshold
 * measured on the true FP64 residual.  info may be NULL. */
SGPU_API int sgpu_scr_cg_prec(int64_t n, const int64_t *adr, const int64_t *ci, const double *a, double *x,
                     const double *y, int64_t ni, double res, int64_t *ani, double *ares,
                     double zero, int64_t iv, int32_t mode, sgpu_solve_info *info);

/* Replaces comprow::cg_prec (GEFEL/cr.cpp:1124-1240) with a `noprecond`
 * preconditioner (h = r, GEFEL/precond.cpp:166-171), the only CR case the
 * reference can run (gmatrix.cpp:1213-1214).  Stops on sqrt((r.h)/(f.f)) < res;
 * afterwards *ani = i and *ares = r.h as the reference leaves them (cr.cpp:1236).
 * prec = 1 selects Jacobi instead (the reference's CR path has no working
 * Jacobi; the criterion is unchanged). */
SGPU_API int sgpu_cr_cg_prec(int64_t n, const int64_t *adr, const int64_t *ci, const double *a, double *x,
                    const double *y, int64_t ni, double res, int64_t *ani, double *ares,
                    double zero, int64_t iv, int32_t prec, int32_t mode, sgpu_solve_info *info);

/* ------------------------------------------------------------------------ */
/* Device-resident matrices                                                 */
/* ------------------------------------------------------------------------ */

typedef struct sgpu_matrix_s *sgpu_matrix;

/* Upload a GEFEL storage (symmetric != 0: SCR, else CR) and build the device
 * formats (full CSR with int32 indices; the FP32 Jacobi-scaled copy and the
 * 3x3 block form are built on first use).  Replaces the matrix half of
 * gmatrix::initiate + localize (GEFEL/gmatrix.cpp:268/499) for callers that
 * assemble on the host. */
SGPU_API int sgpu_matrix_create(int64_t n, const int64_t *adr, const int64_t *ci, const double *a,
                       int32_t symmetric, sgpu_matrix *out);
/* New values in the same pattern (the storage the handle was created from). */
SGPU_API int sgpu_matrix_update_values(sgpu_matrix m, const double *a);
SGPU_API int sgpu_matrix_destroy(sgpu_matrix m);
/* n and the number of stored entries of the full CSR form. */
SGPU_API int sgpu_matrix_info(sgpu_matrix m, int64_t *n, int64_t *nnz_full);
/* Copy the matrix back in GEFEL storage (symmetric != 0: SCR arrays of size
 * n+1 / negm; else CR).  Pass ci = a = NULL to get the sizes first. */
SGPU_API int sgpu_matrix_download(sgpu_matrix m, int32_t symmetric, int64_t *adr, int64_t *ci, double *a,
                         int64_t *negm);

/* y = A x (mxv_scr / mxv_cr semantics, GEFEL/scr.cpp:655, cr.cpp:653).
 * Host vectors. */
SGPU_API int sgpu_matrix_mxv(sgpu_matrix m, const double *x, double *y);
/* Same on device pointers (FP64), on the handle's stream. */
SGPU_API int sgpu_matrix_mxv_d(sgpu_matrix m, const double *x_d, double *y_d);

/* Run the handle's work on a caller's CUDA stream (cudaStream_t passed as a
 * pointer; NULL restores the handle's own stream). */
SGPU_API int sgpu_matrix_set_stream(sgpu_matrix m, void *stream);
/* y = (S A S) x in FP32 with S = diag(A)^-1/2: the operator of the mixed
 * iteration, device pointers, autotuned format/kernel. */
SGPU_API int sgpu_matrix_mxv32_d(sgpu_matrix m, const float *x_d, float *y_d);
/* Algorithmic bytes of one SpMV (precision 64 or 32) in the tuned format,
 * the format id (0 CSR, 2 sliced ELL, 3 BSR3) and the kernel variant; tunes
 * if needed. */
SGPU_API int sgpu_matrix_spmv_plan(sgpu_matrix m, int32_t precision, double *bytes, int32_t *format,
                                   int32_t *variant);

/* Override the autotuner: use SpMV `format` (0 CSR, 2 sliced ELL, 3 BSR3) and
 * `variant` (lanes per row: 4/8/16/32 for CSR, 8/16/32 for BSR3; 32 for the
 * sliced ELL, FP64 only) for `precision` (64 or 32).  For tests and
 * tuning studies; BAD_INPUT if the format is not available for the matrix. */
SGPU_API int sgpu_matrix_set_spmv(sgpu_matrix m, int32_t precision, int32_t format, int32_t variant);

/* PCG on a device-resident matrix, host vectors.  crit selects the reference
 * routine whose criterion is kept; prec is an sgpu_precond value. */
SGPU_API int sgpu_matrix_pcg(sgpu_matrix m, double *x, const double *f, int64_t ni, double res,
                    double zero, int64_t iv, int32_t crit, int32_t prec, int32_t mode,
                    int64_t *ani, double *ares, sgpu_solve_info *info);
/* Same on device vectors (x_d in/out, f_d read-only), no host copies. */
SGPU_API int sgpu_matrix_pcg_d(sgpu_matrix m, double *x_d, const double *f_d, int64_t ni, double res,
                      double zero, int64_t iv, int32_t crit, int32_t prec, int32_t mode,
                      int64_t *ani, double *ares, sgpu_solve_info *info);

/* Near-null space of the matrix for the aggregation preconditioner
 * (SGPU_PREC_AGG), the role the rigid-body modes play in GEFEL's BOSS
 * aggregator (aggregator::gener_rbm_1/2, GEFEL/aggregator.cpp:638-700): B is
 * k (<= 6) host vectors of n entries, column after column -- the 6 rigid-body
 * motions for 3D elasticity, 3 for plane problems, 1 (constants) for
 * conduction.  Without this call the preconditioner uses one constant vector
 * per equation of a node (translations only).  Setting it discards a built
 * hierarchy; new values (sgpu_matrix_update_values) do too. */
SGPU_API int sgpu_matrix_set_nullspace(sgpu_matrix m, int32_t k, const double *B);
/* The same near-null space built on the device from the mesh: the rigid-body
 * motions of the centred node coordinates (coords nn x 3) in the equations
 * the code numbers give (cn nn x ndofn, 1-based, <= 0 none): 6 vectors for
 * ndofn 3, 3 for ndofn 2, the constant for ndofn 1.  No n x k host array. */
SGPU_API int sgpu_matrix_set_rigid_body_modes(sgpu_matrix m, int64_t nn, int32_t ndofn, const double *coords,
                                              const int64_t *cn);
/* Discards the hierarchy of SGPU_PREC_AGG (the next such solve builds it
 * again); the near-null space is kept.  For timing set-up with the solve. */
SGPU_API int sgpu_matrix_precond_clear(sgpu_matrix m);

/* All load cases at once (solve_linear_statics, MEFEL/SRC/lssolver.cpp:78-80,
 * solves them one after the other): nrhs (<= 128) independent Jacobi-PCG
 * iterations with the criterion of symcomprow::cg_prec, advanced together so
 * that one sparse-matrix-times-block product per iteration reads the matrix
 * once for all of them.  X, F: nrhs column blocks of n (the lhsrhs layout,
 * lhsrhs.cpp:72-74), host; per column ani/ares as the reference (written only
 * on convergence) and status[c] (may be NULL).  Returns the first non-OK
 * column status, else OK. */
SGPU_API int sgpu_matrix_pcg_multi(sgpu_matrix m, int32_t nrhs, double *X, const double *F, int64_t ni,
                                   double res, double zero, int64_t iv, int64_t *ani, double *ares,
                                   int32_t *status, sgpu_solve_info *info);

/* All load cases with the aggregation preconditioner: nrhs (<= 128) flexible
 * CGs (FP64, each with the criterion of symcomprow::cg_prec on its own
 * column) sharing one hierarchy (built on first use, as for SGPU_PREC_AGG)
 * and advanced together, so every kernel of the cycle treats all columns --
 * each level's matrix is read once per sweep for all of them.  mode:
 * SGPU_MIXED (FP32 cycle) or SGPU_FP64.  Arguments as sgpu_matrix_pcg_multi;
 * info->iterations is the largest column count. */
SGPU_API int sgpu_matrix_pcg_multi_agg(sgpu_matrix m, int32_t nrhs, double *X, const double *F, int64_t ni,
                                       double res, double zero, int64_t iv, int32_t mode, int64_t *ani,
                                       double *ares, int32_t *status, sgpu_solve_info *info);

/* Many independent systems of uneven size (the diagonal blocks of m, in
 * order; sys_rows[k] equations each, summing to n) solved together: every
 * system its own Jacobi-PCG with the criterion of symcomprow::cg_prec, all
 * advanced by the same kernels (one block-diagonal SpMV and two vector
 * kernels per iteration, captured in a CUDA graph and relaunched until every
 * system has stopped); converged systems drop out of the work.  tune != 0
 * first times a few iterations with each segment size / lanes-per-row pair
 * and keeps the fastest.  x: n (host, out; the iteration starts from 0);
 * f: n; per system ani/ares (reference conventions), status and iterations
 * (arrays of nsys, may be NULL). */
SGPU_API int sgpu_matrix_pcg_batch(sgpu_matrix m, int32_t nsys, const int64_t *sys_rows, double *x,
                                   const double *f, int64_t ni, double res, double zero, int32_t tune,
                                   int64_t *ani, double *ares, int32_t *status, int64_t *iterations,
                                   sgpu_solve_info *info);

/* The same uneven batch with the aggregation preconditioner: every system its
 * own FP64 flexible CG (scalars, the criterion of symcomprow::cg_prec and
 * ani/ares per system) while the hierarchy of the whole block-diagonal
 * matrix -- whose aggregates never cross systems -- is shared, so every
 * cycle kernel runs once for all systems; per-system sums are formed from
 * per-row products in row order.  mode: SGPU_MIXED (FP32 cycle) or
 * SGPU_FP64.  The near-null space comes from sgpu_matrix_set_nullspace on m
 * (e.g. every plate's rigid-body modes).  x starts from 0. */
SGPU_API int sgpu_matrix_pcg_batch_agg(sgpu_matrix m, int32_t nsys, const int64_t *sys_rows, double *x,
                                       const double *f, int64_t ni, double res, double zero, int32_t mode,
                                       int64_t *ani, double *ares, int32_t *status, int64_t *iterations,
                                       sgpu_solve_info *info);

/* ------------------------------------------------------------------------ */
/* Assembly on the GPU                                                      */
/* ------------------------------------------------------------------------ */

/* Element kinds of the hot path. */
typedef enum {
  SGPU_ELEM_HEX8 = 0,    /* linhex, 3D elasticity, 2x2x2 Gauss (MEFEL/SRC/linhex.cpp:583) */
  SGPU_ELEM_QUAD4 = 1,   /* planeelemlq, plane stress, 2x2 Gauss (MEFEL/SRC/plelemlq.cpp:611) */
  SGPU_ELEM_HEX8T_K = 2, /* linhext conductivity (TRFEL/SRC/linhext.cpp:774) */
  SGPU_ELEM_HEX8T_C = 3, /* linhext capacity (TRFEL/SRC/linhext.cpp:979) */
  SGPU_ELEM_TET4 = 4,    /* lintet, 3D elasticity, 1 point (MEFEL/SRC/lintet.cpp:290) */
  SGPU_ELEM_TRI3 = 5,    /* planeelemlt, plane stress, 1 point (MEFEL/SRC/plelemlt.cpp:234) */
  SGPU_ELEM_HEX20 = 6,   /* quadhex, 3D elasticity, 3x3x3 Gauss (MEFEL/SRC/quadhex.cpp:232) */
  SGPU_ELEM_QUAD8 = 7    /* planeelemqq, plane stress, 3x3 Gauss (MEFEL/SRC/plelemqq.cpp:215) */
} sgpu_elem_kind;

/* A mesh in SIFEL's terms.  Node order inside an element follows SIFEL
 * (GEFEL/basefun.cpp:2299 for hexahedra, :609 for quadrilaterals, :2377 and
 * :708 for their serendipity forms); a quad8 with a negative Jacobian fails
 * like a tetrahedron of negative volume; a
 * tetrahedron must have det3d > 0 (GEFEL/matrix.cpp:3629), else
 * sgpu_assemble fails with SGPU_BAD_INPUT as the reference aborts. */
typedef struct {
  int32_t kind;          /* sgpu_elem_kind */
  int32_t ndofn;         /* DOFs per node: 3 (hex8, tet4, hex20), 2 (quad4, tri3, quad8), 1 (hex8t) */
  int64_t nn;            /* nodes */
  const double *coords;  /* nn x 3 (z ignored for the plane kinds) */
  int64_t ne;            /* elements */
  const int64_t *elems;  /* ne x nne, 0-based node ids */
  const int64_t *cn;     /* nn x ndofn code numbers (1-based, <= 0: no equation) */
  const double *emat;    /* ne x 2: (E, nu) for elasticity, (k, c) for hex8t */
  const double *thick;   /* ne thicknesses (plane kinds), else NULL */
  const double *rho;     /* ne densities (capacity), NULL = 1 */
  const double *dmat;    /* NULL, or ne x 36: a general material stiffness per
                            element (6 x 6 row-major, global axes, strain order
                            xx yy zz yz xz xy) for hex8 / tet4 / hex20, replacing emat:
                            elastgmat3d::matstiff (MEFEL/SRC/elastgmat3d.cpp:69)
                            or elastortomat::matstiff (elastortomat.cpp:100) */
} sgpu_mesh;

typedef struct {
  int64_t n;          /* equations */
  int64_t negm_scr;   /* entries of the SCR (lower-triangle) storage */
  int64_t nnz_full;   /* entries of the full CSR on the device */
  int32_t colours;    /* element colours of the atomic-free scatter */
  double pattern_ms;  /* pattern build (device timed) */
  double integrate_ms;/* element integration + scatter (device timed) */
} sgpu_assembly_info;

/* Assemble the global matrix of a mesh on the GPU into a new device-resident
 * handle.  Replaces stiffness_matrix (MEFEL/SRC/globmat.cpp:41) and
 * conductivity_matrix / capacity_matrix (TRFEL/SRC/globmatt.cpp:19/92)
 * including the storage initiation (symcomprow::initiate, GEFEL/scr.cpp:556).
 * sgpu_matrix_download gives the SCR or CR arrays the reference would hold. */
SGPU_API int sgpu_assemble(const sgpu_mesh *mesh, sgpu_matrix *out, sgpu_assembly_info *info);
/* Re-integrate the values of a handle made by sgpu_assemble, on the same
 * pattern: new per-element parameters (emat, rho; NULL keeps the old ones) or,
 * for hex8t handles, the other matrix (kind K <-> C).  For a handle built
 * with dmat, emat is the new ne x 36 array. */
SGPU_API int sgpu_reassemble(sgpu_matrix m, int32_t kind, const double *emat, const double *rho,
                             sgpu_assembly_info *info);

/* A second matrix of the same mesh on the pattern of a handle made by
 * sgpu_assemble, in a new handle: the pattern, the element colouring and the
 * element data are copied on the device, only the values are integrated
 * (kind: the handle's own, or for hex8t handles the other of K and C; emat /
 * rho replace the element parameters when not NULL).  TRFEL's conductivity
 * and capacity matrices (TRFEL/SRC/globmatt.cpp:19/92) share one pattern this
 * way instead of building it twice. */
SGPU_API int sgpu_assemble_copy(sgpu_matrix src, int32_t kind, const double *emat, const double *rho,
                                sgpu_matrix *out, sgpu_assembly_info *info);

/* Dirichlet lifting: add -K_e r_e of every element into rhs[n] (host,
 * accumulated) at its free DOFs, for a handle made by sgpu_assemble.
 *  - hex8 conduction handles: TRFEL's assemble_init
 *    (TRFEL/SRC/globmatt.cpp:1635); rnode[nn] holds the nodal values
 *    prescvalues() gives (globmatt.cpp:1057): prescribed values on prescribed
 *    nodes, initial values on free ones.  Time-constant prescribed values
 *    only (the capacity part of the lifting is then zero).
 *  - hex8 and quad4 elasticity handles: MEFEL's prescribed displacements,
 *    loadcase::prdisplcontrib (MEFEL/SRC/loadcase.cpp:615-664) with
 *    elprdispl (globmat.cpp:1372); rnode[nn * ndofn] holds the prescribed
 *    displacement of every DOF whose code number is negative (the load
 *    case's pd[-code-1]) and 0 elsewhere; elements whose values are all zero
 *    add nothing. */
SGPU_API int sgpu_assembly_lift(sgpu_matrix m, const double *rnode, double *rhs);

/* Element loads of a load case (loadcase::forcecontrib,
 * MEFEL/SRC/loadcase.cpp:546-601, after the nodal loads): the consistent
 * nodal forces of nle element-load records added into f[n] (host) at the
 * elements' code numbers.  eid[nle] 0-based elements; for a hex8 mesh,
 * surface loads (loadel type 3): flags nle x 6 (per face, in the order
 * xi = 1, eta = 1, xi = -1, eta = -1, zeta = 1, zeta = -1: 1 loaded, 0 not)
 * and values nle x 72 (face s: its 4 nodes x 3 components of the load in
 * the global system at 12 s; node order as linhex::node_forces_surf,
 * MEFEL/SRC/linhex.cpp:2543); for a quad4 mesh, edge loads (type 2): flags
 * nle x 4 (edge e from node e to node e+1; 1 loaded) and values nle x 16
 * (2 nodes x 2 components at 4 e; planeelemlq::nodeforces,
 * MEFEL/SRC/plelemlq.cpp:2433).  Loads given in a local system (flag 2) are
 * SGPU_BAD_INPUT.  Host computation; only mesh->kind, nn, coords, ne, elems
 * and cn are read. */
SGPU_API int sgpu_mesh_element_loads(const sgpu_mesh *mesh, int64_t nle, const int64_t *eid, const int32_t *flags,
                                     const double *values, double *f);

/* ------------------------------------------------------------------------ */
/* Linear transient conduction                                              */
/* ------------------------------------------------------------------------ */

/* out = a K + b C on the common pattern of two handles (gmatrix::scalgm and
 * addgm, GEFEL/gmatrix.cpp:1848/1791, index-aligned); a new handle. */
SGPU_API int sgpu_matrix_combine(sgpu_matrix K, sgpu_matrix C, double a, double b, sgpu_matrix *out);
/* nsteps steps of the d-form generalized trapezoid of
 * linear_nonstat_solv_dform (TRFEL/SRC/npsolvert.cpp:1071-1272) with a fixed
 * dt and alpha: dd = d + (1-alpha) dt v; A = alpha dt K + C; f = alpha dt rhs
 * + C dd; A d = f by PCG with the reference's criterion (ni, res, zero, iv as
 * for sgpu_scr_cg_prec; x starts from the previous d when iv = 1); v = (d -
 * dd)/dt/alpha.  prec: SGPU_PREC_JACOBI (the reference's) or SGPU_PREC_AGG
 * (the hierarchy is built on the first step and kept for all of them).  rhs[n] is the step's right-hand side
 * (constant: the lifting of time-constant prescribed values), d and v (host,
 * n) are read and overwritten; step_iterations (may be NULL) gets the
 * iterations of every step.  Everything between the first and the last copy
 * stays on the device. */
SGPU_API int sgpu_transient_dform(sgpu_matrix K, sgpu_matrix C, const double *rhs, double *d, double *v,
                                  double dt, double alpha, int64_t nsteps, int64_t ni, double res, double zero,
                                  int64_t iv, int32_t prec, int32_t mode, int64_t *step_iterations,
                                  sgpu_solve_info *info);
/* The v-form of the same trapezoid, nonstat_solv_vform_comp / one_step_linear
 * (TRFEL/SRC/npsolvert.cpp:62, 367-480; nonstatsolver trapezoidv): dd = d +
 * (1-alpha) dt v; f = rhs - K dd; A v = f (x starts from the previous v when
 * iv = 1); d = dd + alpha dt v.  Arguments as sgpu_transient_dform. */
SGPU_API int sgpu_transient_vform(sgpu_matrix K, sgpu_matrix C, const double *rhs, double *d, double *v,
                                  double dt, double alpha, int64_t nsteps, int64_t ni, double res, double zero,
                                  int64_t iv, int32_t prec, int32_t mode, int64_t *step_iterations,
                                  sgpu_solve_info *info);

/* ------------------------------------------------------------------------ */
/* Solving without allocating device memory                                 */
/* ------------------------------------------------------------------------ */

/* Largest system sgpu_csr_pcg_noalloc_d takes (equations). */
#define SGPU_NOALLOC_MAX_N 131072

/* No counterpart in the reference: an addition for callers that cannot
 * allocate GPU memory while they solve (an application that owns the whole
 * device memory pool through its own allocator, or one that must not call
 * cudaMalloc/cudaFree because they synchronise the device).
 *
 * Jacobi-preconditioned CG on a caller-owned device CSR: full rows, int32
 * indices, a positive diagonal entry in every row.  rowptr_d[n+1],
 * col_d/val_d[rowptr_d[n]], f_d[n] are read, x_d[n] is the start vector when
 * iv != 0 (else set to 0 first) and gets the solution; all device pointers,
 * work enqueued on `stream` (NULL = legacy default stream).  The iteration
 * stops when (r.r)/(f.f) < res for the recurrence residual r, or after ni
 * iterations (SGPU_NOT_CONVERGED), or when |d.p| < zero for a search
 * direction d and p = K d (SGPU_BREAKDOWN); on convergence *ani = the index
 * of the last iteration (counted from 0) and *ares = (r.h)/(f.f) with the
 * preconditioned residual h = r/diag, otherwise both are left as they were
 * (a zero right-hand side, (f.f) < zero, returns SGPU_ZERO_RHS after the
 * first direction fails the |d.p| test, with *ani = 0 and *ares = 0).
 * *iterations (may be NULL) gets the iterations done.
 *
 * The work vectors live in one static device array of the library (about
 * 5 MiB, held by every GPU that loads it until exit), so n <=
 * SGPU_NOALLOC_MAX_N (SGPU_BAD_INPUT beyond).  Nothing is allocated.  Every
 * call uses the same array: calls that overlap on the GPU race and must be
 * serialised.  The first call on each device looks up the array's device
 * address.  Each call waits on the host for its own solve (it reads the
 * iteration state back between chunks of iterations), so it cannot be
 * recorded into a CUDA graph: a call on a capturing stream returns
 * SGPU_BAD_INPUT without enqueuing anything.  Malformed rows (rowptr not
 * within 0..rowptr[n] and non-decreasing, a column outside [0, n), a missing
 * or non-positive diagonal) give SGPU_BAD_INPUT with x_d untouched. */
SGPU_API int sgpu_csr_pcg_noalloc_d(int32_t n, const int32_t *rowptr_d, const int32_t *col_d,
                                    const double *val_d, const double *f_d, double *x_d, int64_t ni,
                                    double res, double zero, int64_t iv, void *stream, int64_t *ani,
                                    double *ares, int64_t *iterations);

/* ------------------------------------------------------------------------ */
/* Deck input (host)                                                        */
/* ------------------------------------------------------------------------ */

/* A MEFEL linear-statics deck in SIFEL's positional format, read by all host
 * threads.  Replaces the reading part of mefel_init (MEFEL/SRC/mefelinit.cpp:47:
 * probdesc::read, mechtop::read, mechmat::read, mechcrsec::read,
 * mechbclc::read) and gtopology::gencodnum (GEFEL/gtopology.cpp:1619) for the
 * decks of the hot path: linear statics, one element type of the
 * sgpu_elem_kind list, one material type (elisomat, elgmat3d, elortomat with
 * constant axes), constraint codes 0 / 1 / -k (prescribed displacement k),
 * nodal loads, element loads in the global system (linearhex surfaces,
 * planeelementlq edges) and prescribed displacements.  Other decks fail
 * with SGPU_BAD_INPUT naming the record or token. */
typedef struct sgpu_deck_s *sgpu_deck;

typedef struct {
  int32_t kind;            /* sgpu_elem_kind */
  int32_t ndofn, nne;      /* DOFs per node, nodes per element */
  int32_t mtype;           /* material type: 1 elisomat, 2 elgmat3d, 3 elortomat */
  int64_t nn, ne, n;       /* nodes, elements, equations */
  int32_t nmat, nmatp;     /* material instances, parameters per instance (2, 21, 45) */
  int32_t nlc;             /* load cases */
  int32_t storage;         /* 10 compressed_rows, 11 symm_comp_rows */
  int32_t precond;         /* 0 none, 1 diagonal */
  int32_t iv;              /* initial-vector flag of the solver line */
  int64_t ni;              /* iteration limit */
  double res;              /* required residual */
  double parse_ms;         /* wall time of sgpu_deck_read_mefel */
  const double *coords;    /* nn x 3 */
  const int64_t *elems;    /* ne x nne, 0-based */
  const int64_t *dofflag;  /* nn x ndofn: 1 free, 0 fixed */
  const int64_t *cn;       /* nn x ndofn code numbers (1-based, 0 fixed) */
  const int64_t *emat_id;  /* ne material instances (0-based) */
  const double *mats;      /* nmat x nmatp as read */
  const double *thick;     /* ne (plane kinds) or NULL */
  const double *loads;     /* nlc x nn x ndofn nodal forces (MEFEL) */
  /* TRFEL decks (sgpu_deck_read_trfel) */
  int32_t problem;         /* 1 linear statics (MEFEL), 50 stationary, 60 nonstationary (TRFEL) */
  int32_t tform;           /* nonstationary solver: 1 trapezoidd (d-form), 2 trapezoidv (v-form) */
  double alpha, t0, t1, dt;/* trapezoid parameter, start and end time, constant time step */
  const double *rnode;     /* nn nodal values of the lifting: prescribed values on prescribed
                              nodes, initial values on free ones (prescvalues) */
  const double *rho;       /* ne densities of the elements' cross sections */
} sgpu_deck_view;

/* threads <= 0: all hardware threads (at most 64). */
SGPU_API int sgpu_deck_read_mefel(const char *path, int32_t threads, sgpu_deck *out);
/* A TRFEL linear heat-conduction deck (the reading part of trfel_init,
 * TRFEL/SRC/trfelinit.cpp:24): stationary (50) or nonstationary (60, d- or
 * v-form trapezoid with a fixed time step), linear hexahedra (linhext, 225),
 * isotropic materials (isotransmat "c k", one instance per element allowed),
 * crsec3dt densities, constant prescribed values, initial values.
 * sgpu_deck_mesh gives the conduction kind (set kind SGPU_ELEM_HEX8T_C for the
 * capacity matrix); the right-hand side is sgpu_assembly_lift of view.rnode. */
SGPU_API int sgpu_deck_read_trfel(const char *path, int32_t threads, sgpu_deck *out);
/* Arrays of the deck (owned by it, valid until sgpu_deck_free). */
SGPU_API int sgpu_deck_get(sgpu_deck d, sgpu_deck_view *view);
/* The deck as an sgpu_assemble input (pointers into the deck). */
SGPU_API int sgpu_deck_mesh(sgpu_deck d, sgpu_mesh *mesh);
/* Nodal and element loads of load case lc in equation order, f[n]
 * (mefel_right_hand_side, MEFEL/SRC/globmat.cpp:2369: loadcase::forcecontrib;
 * the element loads as sgpu_mesh_element_loads); MEFEL decks only.  The
 * prescribed displacements' part is sgpu_assembly_lift of
 * sgpu_deck_prescribed's values. */
SGPU_API int sgpu_deck_rhs(sgpu_deck d, int32_t lc, double *f);
/* Prescribed displacements of load case lc as nodal values r[nn * ndofn]
 * (the load case's pd[-code-1] at every DOF with a negative constraint code,
 * 0 elsewhere); *count (may be NULL) gets the number of such DOFs. */
SGPU_API int sgpu_deck_prescribed(sgpu_deck d, int32_t lc, double *r, int64_t *count);
SGPU_API void sgpu_deck_free(sgpu_deck d);

/* ------------------------------------------------------------------------ */
/* Library state                                                            */
/* ------------------------------------------------------------------------ */

SGPU_API const char *sgpu_last_error(void);
SGPU_API const char *sgpu_version(void);
/* Number of kernels this library launched in the calling process so far. */
SGPU_API int64_t sgpu_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* SIFELGPU_H */
