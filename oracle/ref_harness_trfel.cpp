// In-process harness around the compiled SIFEL/TRFEL reference.
//
// Test infrastructure only (built by oracle/build_ref.py into oracle/_ref/).
//
//   trfel_dump <deck.in> <outdir> [nosolve]
//
// Runs trfel_init (TRFEL/SRC/trfelinit.cpp:24) and, unless "nosolve",
// solve_trfel_problem (solvert.cpp:17), which for a nonstationary linear
// deck with the d-form trapezoid runs linear_nonstat_solv_dform
// (npsolvert.cpp:1071-1272) up to the deck's end time.  Afterwards it
// re-assembles the conductivity and capacity matrices with the reference's
// own conductivity_matrix / capacity_matrix (globmatt.cpp:19/92) and writes
// into <outdir>:
//   meta.txt                    n, negm, storages, timings, last ani/ares
//   K_adr.i64 K_ci.i64 K_a.f64  conductivity matrix storage arrays
//   C_adr.i64 C_ci.i64 C_a.f64  capacity matrix storage arrays
//   T.f64 V.f64                 nodal values and their time derivatives at the end
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#define EXTERN
#include "globalt.h"
#include "globalg.h"
#include "trfelinit.h"
#include "solvert.h"
#include "globmatt.h"
#include "lhsrhst.h"
#include "probdesct.h"
#include "gmatrix.h"
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

static long dump_matrix(const std::string &out, const char *tag, gmatrix *g, long n) {
  const long *adr = nullptr, *ci = nullptr;
  const double *a = nullptr;
  long negm = 0;
  if (g->ts == symm_comp_rows) {
    adr = g->scr->adr; ci = g->scr->ci; a = g->scr->a; negm = g->scr->negm;
  } else if (g->ts == compressed_rows) {
    adr = g->cr->adr; ci = g->cr->ci; a = g->cr->a; negm = g->cr->negm;
  } else {
    return -1;
  }
  dump(out + "/" + tag + "_adr.i64", adr, sizeof(long) * (n + 1));
  dump(out + "/" + tag + "_ci.i64", ci, sizeof(long) * negm);
  dump(out + "/" + tag + "_a.f64", a, sizeof(double) * negm);
  return negm;
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
  trfel_init(2, iargv);
  double t1 = now_s();
  long n = Ndoft;
  FILE *m = fopen((out + "/meta.txt").c_str(), "w");
  fprintf(m, "n %ld\nt_init %.9f\n", n, t1 - t0);
  if (solve) {
    solve_trfel_problem();
    double t2 = now_s();
    fprintf(m, "t_solve_total %.9f\n", t2 - t1);
    if (Kmat) fprintf(m, "ani %ld\nares %.17e\n", Kmat->ani, Kmat->ares);
    fflush(m);
    dump(out + "/T.f64", Lsrst->give_lhs(0), sizeof(double) * n);
    // a stationary problem keeps no time derivatives
    if (Tp->tprob != stationary_problem && Lsrst->give_tdlhs(0))
      dump(out + "/V.f64", Lsrst->give_tdlhs(0), sizeof(double) * n);
  }
  double t3 = now_s();
  conductivity_matrix(0);
  double t4 = now_s();
  const bool transient = Tp->tprob != stationary_problem;
  if (transient) capacity_matrix(0);
  double t5 = now_s();
  long nk = dump_matrix(out, "K", Kmat, n);
  long nc = transient ? dump_matrix(out, "C", Cmat, n) : 0;
  fprintf(m, "negm_K %ld\nnegm_C %ld\nstorage_K %d\nstorage_C %d\n", nk, nc, (int)Kmat->ts,
          transient ? (int)Cmat->ts : -1);
  fprintf(m, "t_conductivity %.9f\nt_capacity %.9f\n", t4 - t3, t5 - t4);
  fclose(m);
  return 0;
}
