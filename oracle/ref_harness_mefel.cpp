// In-process harness around the compiled SIFEL/MEFEL reference.
//
// Test infrastructure only (built by oracle/build_ref.py into oracle/_ref/):
// it runs the reference's own linear-statics pipeline on a deck in SIFEL's
// positional input format and dumps what the GPU path must reproduce.
//
//   mefel_dump <deck.in> <outdir> [nosolve]
//
// Mirrors solve_linear_statics (MEFEL/SRC/lssolver.cpp:31-80):
//   mefel_init (mefelinit.cpp:47)            -> parse deck, code numbers
//   stiffness_matrix(0) (globmat.cpp:41)     -> element loop + localize
//   mefel_right_hand_side(i,rhs) (globmat.cpp:2369) for every load case
//   Mp->ssle->solve_system(...) (slesolv.cpp:472) for every load case
// and writes into <outdir>:
//   meta.txt  key value lines (n, negm, storage, nlc, ani/ares per case, times)
//   K_adr.i64 K_ci.i64 K_a.f64   the assembled storage arrays (CR or SCR)
//   f.f64 u.f64                  nlc blocks of n (lhsrhs layout)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#define EXTERN
#define EXTENDED_GLOBINC
#include "global.h"
#include "globalg.h"
#include "mefelinit.h"
#include "globmat.h"
#include "lhsrhs.h"
#include "probdesc.h"
#include "gmatrix.h"
#include "slesolv.h"
#include "scr.h"
#include "cr.h"

static double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static void dump(const std::string &path, const void *p, size_t bytes) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
  if (bytes) fwrite(p, 1, bytes, f);
  fclose(f);
}

int main(int argc, const char *argv[]) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s deck.in outdir [nosolve]\n", argv[0]);
    return 2;
  }
  std::string out = argv[2];
  bool solve = !(argc > 3 && strcmp(argv[3], "nosolve") == 0);
  const char *iargv[2] = {argv[0], argv[1]};

  double t0 = now_s();
  mefel_init(2, iargv);
  double t1 = now_s();
  stiffness_matrix(0);
  double t2 = now_s();

  long n = Ndofm;
  long nlc = Lsrs->nlc;
  double *rhs = Lsrs->give_rhs(0);
  for (long i = 0; i < nlc; i++) mefel_right_hand_side(i, rhs);
  double t3 = now_s();

  // dump the matrix before the solve (the solver does not modify it)
  long negm = 0;
  int ts = (int)Smat->ts;
  if (Smat->ts == symm_comp_rows) {
    negm = Smat->scr->negm;
    dump(out + "/K_adr.i64", Smat->scr->adr, sizeof(long) * (n + 1));
    dump(out + "/K_ci.i64", Smat->scr->ci, sizeof(long) * negm);
    dump(out + "/K_a.f64", Smat->scr->a, sizeof(double) * negm);
  } else if (Smat->ts == compressed_rows) {
    negm = Smat->cr->negm;
    dump(out + "/K_adr.i64", Smat->cr->adr, sizeof(long) * (n + 1));
    dump(out + "/K_ci.i64", Smat->cr->ci, sizeof(long) * negm);
    dump(out + "/K_a.f64", Smat->cr->a, sizeof(double) * negm);
  }
  dump(out + "/f.f64", rhs, sizeof(double) * n * nlc);

  FILE *m = fopen((out + "/meta.txt").c_str(), "w");
  fprintf(m, "n %ld\nnegm %ld\nstorage %d\nnlc %ld\n", n, negm, ts, nlc);
  fprintf(m, "t_init %.9f\nt_stiffness %.9f\nt_rhs %.9f\n", t1 - t0, t2 - t1, t3 - t2);
  if (solve) {
    // the solver overwrites nothing in rhs; keep a copy anyway for safety
    for (long i = 0; i < nlc; i++) {
      double ts0 = now_s();
      Mp->ssle->solve_system(Gtm, Smat, Lsrs->give_lhs(i), Lsrs->give_rhs(i), Out);
      double ts1 = now_s();
      fprintf(m, "t_solve_%ld %.9f\nani_%ld %ld\nares_%ld %.17e\n", i, ts1 - ts0, i,
              Smat->ani, i, Smat->ares);
    }
    dump(out + "/u.f64", Lsrs->give_lhs(0), sizeof(double) * n * nlc);
  }
  fclose(m);
  return 0;
}
