// C entry points into the compiled SIFEL/GEFEL reference solvers.
//
// Test infrastructure only: built by oracle/build_ref.py into
// oracle/_ref/libsifelref.so together with GEFEL's own objects, so the
// tests and the CPU-baseline leg of bench.py can run the reference's
// unchanged routines on exactly the arrays that the GPU path receives:
//
//   symcomprow::cg_prec  (GEFEL/scr.cpp:1093)  Jacobi-PCG on SCR storage
//   symcomprow::cg       (GEFEL/scr.cpp:786)   plain CG on SCR storage
//   comprow::cg_prec     (GEFEL/cr.cpp:1124)   CG on CR storage, precond object
//   comprow::cg          (GEFEL/cr.cpp:1022)   plain CG on CR storage
//   symcomprow::mxv_scr  (GEFEL/scr.cpp:655),  comprow::mxv_cr (GEFEL/cr.cpp:653)
//
// The storage objects borrow the caller's arrays and give them back before
// their destructors run.  `quiet` redirects the reference's per-iteration
// stdout prints (scr.cpp:1184, cr.cpp:1212) to /dev/null for timing.
#include <fcntl.h>
#include <unistd.h>
#include <cstdio>

#define EXTERN
#include "globalg.h"
#include "galias.h"
#include "scr.h"
#include "cr.h"
#include "precond.h"

namespace {
struct Quiet {
  int saved = -1;
  explicit Quiet(int on) {
    if (!on) return;
    fflush(stdout);
    saved = dup(1);
    int dn = open("/dev/null", O_WRONLY);
    dup2(dn, 1);
    close(dn);
  }
  ~Quiet() {
    if (saved < 0) return;
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};

template <class S>
struct Borrow {
  S s;
  Borrow(long n, long *adr, long *ci, double *a) {
    s.n = n; s.negm = adr[n]; s.adr = adr; s.ci = ci; s.a = a;
  }
  ~Borrow() { s.adr = nullptr; s.ci = nullptr; s.a = nullptr; }
};
}  // namespace

extern "C" {

void ref_scr_mxv(long n, long *adr, long *ci, double *a, double *b, double *c) {
  Borrow<symcomprow> m(n, adr, ci, a);
  m.s.mxv_scr(b, c);
}

void ref_cr_mxv(long n, long *adr, long *ci, double *a, double *b, double *c) {
  Borrow<comprow> m(n, adr, ci, a);
  m.s.mxv_cr(b, c);
}

// tprec: 1 = diagonal (Jacobi), as dispatched at GEFEL/gmatrix.cpp:1225-1227
void ref_scr_cg_prec(long n, long *adr, long *ci, double *a, double *x, double *y, long ni,
                     double res, double zero, long iv, long tprec, long *ani, double *ares,
                     int quiet) {
  Quiet q(quiet);
  Borrow<symcomprow> m(n, adr, ci, a);
  long an = *ani;
  double ar = *ares;
  m.s.cg_prec(x, y, ni, res, an, ar, zero, iv, tprec, 0.0, nullptr);
  *ani = an;
  *ares = ar;
}

void ref_scr_cg(long n, long *adr, long *ci, double *a, double *x, double *y, long ni, double res,
                double zero, long iv, long *ani, double *ares, int quiet) {
  Quiet q(quiet);
  Borrow<symcomprow> m(n, adr, ci, a);
  long an = *ani;
  double ar = *ares;
  m.s.cg(x, y, ni, res, an, ar, zero, iv);
  *ani = an;
  *ares = ar;
}

// precondtype: 0 = noprecond (the only working CR case, gmatrix.cpp:1213-1214)
void ref_cr_cg_prec(long n, long *adr, long *ci, double *a, double *x, double *y, long ni,
                    double res, double zero, long iv, int ptype, long *ani, double *ares,
                    int quiet) {
  Quiet q(quiet);
  Borrow<comprow> m(n, adr, ci, a);
  precond pr;
  pr.pt = (precondtype)ptype;
  pr.n = n;
  long an = *ani;
  double ar = *ares;
  m.s.cg_prec(pr, x, y, ni, res, an, ar, zero, iv);
  *ani = an;
  *ares = ar;
}

void ref_cr_cg(long n, long *adr, long *ci, double *a, double *x, double *y, long ni, double res,
               double zero, long iv, long *ani, double *ares, int quiet) {
  Quiet q(quiet);
  Borrow<comprow> m(n, adr, ci, a);
  long an = *ani;
  double ar = *ares;
  m.s.cg(x, y, ni, res, an, ar, zero, iv);
  *ani = an;
  *ares = ar;
}

}  // extern "C"
