// Parallel reader of MEFEL linear-statics decks in SIFEL's positional input
// format (no keywords).  Host code only.
//
// The reference reads a deck token by token through xfscanf in mefel_init
// (MEFEL/SRC/mefelinit.cpp:47): probdesc::read (MEFEL/SRC/probdesc.cpp:204-452),
// mechtop::read (mechtop.cpp:124-262) with gnode::read / node::read
// (GEFEL/gnode.cpp:55, MEFEL/SRC/node.cpp:94), element::read
// (element.cpp:90-350), mechmat::read (mechmat.cpp:1042-1110),
// mechcrsec::read (mechcrsec.cpp:74), mechbclc::read / loadcase::read
// (mechbclc.cpp:99, loadcase.cpp:114).  On the 1.01M-DOF cantilever that is
// 8.5 s of one core before the stiffness matrix is formed.
//
// Here the file is read into memory once, every token start is found by all
// threads at once (a token starts where a non-blank follows a blank, a test
// that needs no neighbouring chunk), and the sections whose records have a
// fixed token count -- nodes, constraints, elements, nodal loads -- are
// converted by all threads at once with std::from_chars; the short sections
// are walked in order.  The result is a mesh in SIFEL's terms (coordinates,
// 0-based element nodes, constraint flags, code numbers by gencodnum, material
// per element, thickness, nodal loads) that sgpu_deck_mesh hands straight to
// sgpu_assemble.
//
// Supported subset (anything else is SGPU_BAD_INPUT with the token index):
// problem type linear statics with every optional computation off; storage
// 10/11, solver cg, precond 0/1; nodes without cross-section or local
// system; constraint codes 0 (fixed) and 1 (free); one element type per deck
// (lineartet 100, linearhex 102, quadrhex 103 with crst 0; planeelementlt 20,
// planeelementlq 23, planeelementqq 24 with plane stress and a csplanestr
// thickness set); one material type per deck (elisomat 1, elgmat3d 2,
// elortomat 3 with constant transformation functions); nodal loads only;
// no eigenstrains or output requests.

#include <algorithm>
#include <atomic>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sgpu_internal.cuh"

namespace sgpu {
namespace {

inline bool blank(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\f' || c == '\v'; }

template <class F>
void parallel_for(int64_t n, int threads, F &&f) {
  if (threads <= 1 || n < 4096) {
    f(0, n);
    return;
  }
  std::vector<std::thread> pool;
  const int64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    const int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
    if (b >= e) break;
    pool.emplace_back([&f, b, e] { f(b, e); });
  }
  for (auto &th : pool) th.join();
}

}  // namespace

struct DeckData {
  std::vector<char> buf;
  std::vector<int64_t> tok;  // start offset of every token after the title line
  int threads = 1;
  // header
  int32_t storage = 0, solver = 0, iv = 0, precond = 0;
  int64_t ni = 0;
  double res = 0.0;
  // mesh
  int32_t kind = -1, ndofn = 0, nne = 0, mtype = 0, nmatp = 0;
  int64_t nn = 0, ne = 0, n = 0;
  int32_t nmat = 0, nlc = 0;
  std::vector<double> coords, mats, thick, loads, emat2, dmat;
  std::vector<int64_t> elems, dofflag, cn, emat_id;
  double parse_ms = 0.0;

  // token access ------------------------------------------------------------
  const char *at(int64_t t) const { return buf.data() + tok[(size_t)t]; }
  const char *end() const { return buf.data() + buf.size(); }
  bool geti(int64_t t, int64_t &v) const {
    if (t < 0 || t >= (int64_t)tok.size()) return false;
    const char *p = at(t);
    auto r = std::from_chars(p, end(), v);
    return r.ec == std::errc() && (r.ptr == end() || blank(*r.ptr));
  }
  bool getd(int64_t t, double &v) const {
    if (t < 0 || t >= (int64_t)tok.size()) return false;
    const char *p = at(t);
    if (*p == '+') p++;  // from_chars takes no leading plus
    auto r = std::from_chars(p, end(), v);
    return r.ec == std::errc() && (r.ptr == end() || blank(*r.ptr));
  }
};

namespace {

struct Cursor {
  const DeckData &d;
  int64_t t = 0;
  std::string err;
  int64_t i() {
    int64_t v = 0;
    if (!d.geti(t, v) && err.empty()) err = "integer expected at token " + std::to_string(t);
    t++;
    return v;
  }
  double f() {
    double v = 0;
    if (!d.getd(t, v) && err.empty()) err = "number expected at token " + std::to_string(t);
    t++;
    return v;
  }
  void expect(int64_t want, const char *what) {
    const int64_t at = t;
    const int64_t v = i();
    if (v != want && err.empty())
      err = std::string(what) + " = " + std::to_string(v) + " at token " + std::to_string(at) + " is not supported";
  }
};

// element type (MEFEL/SRC/alias.h elemtype) -> kind, nodes, DOFs per node, plane
struct ElemType {
  int type, kind, nne, ndofn;
  bool plane;
};
const ElemType kElemTypes[] = {
    {100, SGPU_ELEM_TET4, 4, 3, false},  {102, SGPU_ELEM_HEX8, 8, 3, false},  {103, SGPU_ELEM_HEX20, 20, 3, false},
    {20, SGPU_ELEM_TRI3, 3, 2, true},    {23, SGPU_ELEM_QUAD4, 4, 2, true},   {24, SGPU_ELEM_QUAD8, 8, 2, true}};

// 6 x 6 strain transformation of lg_tens4transf (MEFEL/SRC/vecttens.cpp:1561)
// from the axes tm (x_global = T x_local), and g = t^T l t
void ortho_global(const double *l, const double *tm, double *g) {
  auto T = [&](int i, int j) { return tm[3 * i + j]; };
  double t[36], aux[36];
  for (int c = 0; c < 3; c++) {
    double *row = t + 6 * c;
    row[0] = T(0, c) * T(0, c); row[1] = T(1, c) * T(1, c); row[2] = T(2, c) * T(2, c);
    row[3] = T(1, c) * T(2, c); row[4] = T(0, c) * T(2, c); row[5] = T(0, c) * T(1, c);
  }
  const int P[3][2] = {{2, 1}, {2, 0}, {1, 0}};
  for (int r = 0; r < 3; r++) {
    const int a = P[r][0], b = P[r][1];
    double *row = t + 6 * (3 + r);
    row[0] = 2.0 * T(0, a) * T(0, b); row[1] = 2.0 * T(1, a) * T(1, b); row[2] = 2.0 * T(2, a) * T(2, b);
    row[3] = T(1, a) * T(2, b) + T(2, a) * T(1, b);
    row[4] = T(0, a) * T(2, b) + T(2, a) * T(0, b);
    row[5] = T(0, a) * T(1, b) + T(1, a) * T(0, b);
  }
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

int tokenize(DeckData &d, size_t start) {
  const int T = d.threads;
  const size_t N = d.buf.size();
  const size_t span = N > start ? N - start : 0;
  const int parts = (int)std::max<size_t>(1, std::min<size_t>((size_t)T, span / 65536 + 1));
  std::vector<int64_t> counts(parts + 1, 0);
  auto bounds = [&](int p, size_t &b, size_t &e) {
    b = start + span * (size_t)p / (size_t)parts;
    e = start + span * (size_t)(p + 1) / (size_t)parts;
  };
  auto is_start = [&](size_t q) { return !blank(d.buf[q]) && (q == start || blank(d.buf[q - 1])); };
  {
    std::vector<std::thread> pool;
    for (int p = 0; p < parts; p++)
      pool.emplace_back([&, p] {
        size_t b, e;
        bounds(p, b, e);
        int64_t c = 0;
        for (size_t q = b; q < e; q++) c += is_start(q);
        counts[p + 1] = c;
      });
    for (auto &th : pool) th.join();
  }
  for (int p = 0; p < parts; p++) counts[p + 1] += counts[p];
  d.tok.resize((size_t)counts[parts]);
  {
    std::vector<std::thread> pool;
    for (int p = 0; p < parts; p++)
      pool.emplace_back([&, p] {
        size_t b, e;
        bounds(p, b, e);
        int64_t w = counts[p];
        for (size_t q = b; q < e; q++)
          if (is_start(q)) d.tok[(size_t)w++] = (int64_t)q;
      });
    for (auto &th : pool) th.join();
  }
  return SGPU_OK;
}

// Reads `count` records of `stride` tokens starting at token `base` with all
// threads; rec(k, t, ok) parses record k at token t and clears ok on a bad
// record.  Returns the first bad record or -1.
template <class F>
int64_t parallel_records(const DeckData &d, int64_t base, int64_t count, int64_t stride, F &&rec) {
  if (base + count * stride > (int64_t)d.tok.size()) return 0;
  std::atomic<int64_t> bad{INT64_MAX};
  parallel_for(count, d.threads, [&](int64_t b, int64_t e) {
    for (int64_t k = b; k < e; k++) {
      bool ok = true;
      rec(k, base + k * stride, ok);
      if (!ok) {
        int64_t cur = bad.load();
        while (k < cur && !bad.compare_exchange_weak(cur, k)) {
        }
        return;
      }
    }
  });
  const int64_t v = bad.load();
  return v == INT64_MAX ? -1 : v;
}

int parse(DeckData &d) {
  // the title is the first line (probdesc::read reads it whole)
  size_t start = 0;
  while (start < d.buf.size() && d.buf[start] != '\n') start++;
  SGPU_TRY(tokenize(d, start));
  Cursor c{d};
  // --- problem description (probdesc::read, positional) ---
  c.i();                                // mespr
  c.expect(1, "problemtype");           // linear_statics
  for (int k = 0; k < 4; k++) c.expect(0, "strain/stress/other/reaction computation flag");
  for (int k = 0; k < 3; k++) c.expect(0, "adaptivity/stochastic/homogenization flag");
  c.expect(0, "noderenumber");
  d.storage = (int32_t)c.i();
  if (d.storage != 10 && d.storage != 11 && c.err.empty()) c.err = "storage " + std::to_string(d.storage) + " is not supported";
  d.solver = (int32_t)c.i();
  if (d.solver != 20 && c.err.empty()) c.err = "linear solver " + std::to_string(d.solver) + " is not supported";
  d.ni = c.i();
  d.res = c.f();
  d.iv = (int32_t)c.i();
  d.precond = (int32_t)c.i();
  if (d.precond != 0 && d.precond != 1 && c.err.empty()) c.err = "preconditioner " + std::to_string(d.precond) + " is not supported";
  if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);

  // --- nodes: "id x y z ndofn crst transf", crst = transf = 0 ---
  d.nn = c.i();
  if (!c.err.empty() || d.nn <= 0) return fail(SGPU_BAD_INPUT, "deck: bad node count");
  int64_t nd0 = 0;
  if (!d.geti(c.t + 4, nd0) || nd0 < 1 || nd0 > 3) return fail(SGPU_BAD_INPUT, "deck: bad DOF count of the first node");
  d.ndofn = (int32_t)nd0;
  d.coords.assign((size_t)d.nn * 3, 0.0);
  std::vector<std::atomic<uint8_t>> seen((size_t)d.nn);
  for (auto &s : seen) s.store(0, std::memory_order_relaxed);
  int64_t bad = parallel_records(d, c.t, d.nn, 7, [&](int64_t, int64_t t, bool &ok) {
    int64_t id = 0, ndofn = 0, crst = 0, transf = 0;
    ok = d.geti(t, id) && id >= 1 && id <= d.nn && d.geti(t + 4, ndofn) && ndofn == d.ndofn && d.geti(t + 5, crst) &&
         crst == 0 && d.geti(t + 6, transf) && transf == 0;
    if (!ok) return;
    double *x = &d.coords[(size_t)(id - 1) * 3];
    ok = d.getd(t + 1, x[0]) && d.getd(t + 2, x[1]) && d.getd(t + 3, x[2]) &&
         seen[(size_t)(id - 1)].exchange(1) == 0;
  });
  if (bad >= 0)
    return fail(SGPU_BAD_INPUT, "deck: node record " + std::to_string(bad + 1) +
                                    " is not 'id x y z ndofn 0 0' with one DOF count per deck and unique ids");
  c.t += d.nn * 7;

  // --- constraints: "id c1..c_ndofn" with 0 fixed, 1 free ---
  d.dofflag.assign((size_t)d.nn * d.ndofn, 1);
  const int64_t ncn = c.i();
  if (!c.err.empty() || ncn < 0 || ncn > d.nn) return fail(SGPU_BAD_INPUT, "deck: bad constraint count");
  bad = parallel_records(d, c.t, ncn, 1 + d.ndofn, [&](int64_t, int64_t t, bool &ok) {
    int64_t id = 0;
    ok = d.geti(t, id) && id >= 1 && id <= d.nn;
    for (int q = 0; ok && q < d.ndofn; q++) {
      int64_t v = 0;
      ok = d.geti(t + 1 + q, v) && (v == 0 || v == 1);
      if (ok) d.dofflag[(size_t)(id - 1) * d.ndofn + q] = v;
    }
  });
  if (bad >= 0)
    return fail(SGPU_BAD_INPUT, "deck: constraint record " + std::to_string(bad + 1) +
                                    " is not 'id c1..cn' with codes 0 (fixed) or 1 (free)");
  c.t += ncn * (1 + d.ndofn);

  // --- elements: "id type [ssst] n1..nk cne crst [idcs] ntm tm idm" ---
  d.ne = c.i();
  if (!c.err.empty() || d.ne <= 0 || d.ne > (1LL << 31) - 1) return fail(SGPU_BAD_INPUT, "deck: bad element count");
  int64_t type0 = 0;
  d.geti(c.t + 1, type0);
  const ElemType *et = nullptr;
  for (const ElemType &x : kElemTypes)
    if (x.type == type0) et = &x;
  if (!et) return fail(SGPU_BAD_INPUT, "deck: element type " + std::to_string(type0) + " is not supported");
  if (et->ndofn != d.ndofn) return fail(SGPU_BAD_INPUT, "deck: element type and node DOF count disagree");
  d.kind = et->kind;
  d.nne = et->nne;
  const int off_nodes = et->plane ? 3 : 2;
  const int64_t stride = off_nodes + d.nne + (et->plane ? 3 : 2) + 3;
  // the material type of the first element fixes the deck's one type
  int64_t mt0 = 0;
  d.geti(c.t + stride - 2, mt0);
  d.elems.assign((size_t)d.ne * d.nne, 0);
  d.emat_id.assign((size_t)d.ne, 0);
  std::vector<int64_t> tset;
  if (et->plane) tset.assign((size_t)d.ne, 0);
  std::vector<std::atomic<uint8_t>> eseen((size_t)d.ne);
  for (auto &s : eseen) s.store(0, std::memory_order_relaxed);
  bad = parallel_records(d, c.t, d.ne, stride, [&](int64_t, int64_t t, bool &ok) {
    int64_t id = 0, type = 0, v = 0;
    ok = d.geti(t, id) && id >= 1 && id <= d.ne && d.geti(t + 1, type) && type == et->type;
    if (ok && et->plane) ok = d.geti(t + 2, v) && v == 10;  // strastrestate planestress
    if (!ok) return;
    const size_t e = (size_t)(id - 1);
    for (int a = 0; ok && a < d.nne; a++) {
      ok = d.geti(t + off_nodes + a, v) && v >= 1 && v <= d.nn;
      if (ok) d.elems[e * d.nne + a] = v - 1;
    }
    int64_t q = t + off_nodes + d.nne;
    ok = ok && d.geti(q++, v) && v == 0;  // cne
    if (ok && et->plane) {
      ok = d.geti(q++, v) && v == 10 && d.geti(q++, v) && v >= 1;  // crst csplanestr, set id
      if (ok) tset[e] = v - 1;
    } else if (ok) {
      ok = d.geti(q++, v) && v == 0;  // crst
    }
    ok = ok && d.geti(q++, v) && v == 1 && d.geti(q++, v) && v == mt0 && d.geti(q++, v) && v >= 1;
    if (ok) d.emat_id[e] = v - 1;
    ok = ok && eseen[e].exchange(1) == 0;
  });
  if (bad >= 0)
    return fail(SGPU_BAD_INPUT, "deck: element record " + std::to_string(bad + 1) +
                                    " differs from the first in type, layout or material type, or repeats an id");
  c.t += d.ne * stride;

  // --- materials: one type, "mattype ninst", instances ---
  c.expect(1, "number of material types");
  d.mtype = (int32_t)c.i();
  if (d.mtype != mt0 && c.err.empty()) c.err = "material type differs from the elements'";
  d.nmat = (int32_t)c.i();
  if (c.err.empty() && (d.mtype < 1 || d.mtype > 3)) c.err = "material type " + std::to_string(d.mtype) + " is not supported";
  if (c.err.empty() && d.mtype != 1 && et->plane) c.err = "general materials are supported for the 3D elements";
  if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);
  d.nmatp = d.mtype == 1 ? 2 : (d.mtype == 2 ? 21 : 45);
  d.mats.assign((size_t)d.nmat * d.nmatp, 0.0);
  for (int32_t k = 0; k < d.nmat && c.err.empty(); k++) {
    const int64_t id = c.i();
    if (id < 1 || id > d.nmat) {
      c.err = "material instance " + std::to_string(id) + " out of range";
      break;
    }
    double *row = &d.mats[(size_t)(id - 1) * d.nmatp];
    if (d.mtype == 3) {
      for (int q = 0; q < 36; q++) row[q] = c.f();
      for (int q = 0; q < 9; q++) {
        c.expect(0, "transformation function type");  // constant
        row[36 + q] = c.f();
      }
    } else {
      for (int q = 0; q < d.nmatp; q++) row[q] = c.f();
    }
  }
  if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);
  for (int64_t e = 0; e < d.ne; e++)
    if (d.emat_id[(size_t)e] >= d.nmat) return fail(SGPU_BAD_INPUT, "deck: element material instance out of range");

  // --- cross sections ---
  const int64_t ncst = c.i();
  if (et->plane) {
    if (ncst != 1) return fail(SGPU_BAD_INPUT, "deck: plane elements need one cross-section type (csplanestr)");
    c.expect(10, "cross-section type");
    const int64_t nset = c.i();
    std::vector<double> tv((size_t)std::max<int64_t>(nset, 0), 0.0);
    for (int64_t k = 0; k < nset && c.err.empty(); k++) {
      const int64_t id = c.i();
      if (id < 1 || id > nset) c.err = "thickness set out of range";
      else tv[(size_t)(id - 1)] = c.f();
    }
    if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);
    d.thick.assign((size_t)d.ne, 0.0);
    for (int64_t e = 0; e < d.ne; e++) {
      if (tset[(size_t)e] >= nset) return fail(SGPU_BAD_INPUT, "deck: element thickness set out of range");
      d.thick[(size_t)e] = tv[(size_t)tset[(size_t)e]];
    }
  } else if (ncst != 0) {
    return fail(SGPU_BAD_INPUT, "deck: cross sections of 3D elements are not supported");
  }

  // --- load cases: nodal loads only ---
  d.nlc = (int32_t)c.i();
  if (!c.err.empty() || d.nlc < 1) return fail(SGPU_BAD_INPUT, "deck: bad load case count");
  d.loads.assign((size_t)d.nlc * d.nn * d.ndofn, 0.0);
  for (int32_t lc = 0; lc < d.nlc; lc++) {
    const int64_t nl = c.i();
    if (!c.err.empty() || nl < 0 || nl > d.nn) return fail(SGPU_BAD_INPUT, "deck: bad loaded-node count");
    double *L = &d.loads[(size_t)lc * d.nn * d.ndofn];
    // a node may be listed twice: its forces add up (loadn data are summed by
    // loadcase::assemble), so the loads of one case are read in order
    bool ok = true;
    for (int64_t k = 0; k < nl && ok; k++) {
      const int64_t t = c.t + k * (1 + d.ndofn);
      int64_t id = 0;
      ok = d.geti(t, id) && id >= 1 && id <= d.nn;
      for (int q = 0; ok && q < d.ndofn; q++) {
        double v = 0.0;
        ok = d.getd(t + 1 + q, v);
        L[(size_t)(id - 1) * d.ndofn + q] += v;
      }
    }
    if (!ok) return fail(SGPU_BAD_INPUT, "deck: bad nodal load record in load case " + std::to_string(lc + 1));
    c.t += nl * (1 + d.ndofn);
    c.expect(0, "loaded elements");
    c.expect(0, "prescribed displacements");
    c.expect(0, "temperature changes");
    if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);
  }

  // --- eigenstrains, text output, graphic output: all off ---
  c.expect(0, "eigenstrains");
  c.expect(0, "text output");
  c.expect(0, "graphic output");
  if (c.err.empty() && c.t != (int64_t)d.tok.size())
    c.err = "unexpected token " + std::to_string(c.t) + " after the deck";
  if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);

  // --- code numbers (gtopology::gencodnum, GEFEL/gtopology.cpp:1619) ---
  d.cn.assign(d.dofflag.size(), 0);
  int64_t next = 0;
  for (size_t q = 0; q < d.dofflag.size(); q++)
    if (d.dofflag[q] == 1) d.cn[q] = ++next;
  d.n = next;
  if (d.n == 0) return fail(SGPU_BAD_INPUT, "deck: no free DOFs");

  // --- per-element material rows for sgpu_assemble ---
  if (d.mtype == 1) {
    d.emat2.resize((size_t)d.ne * 2);
    parallel_for(d.ne, d.threads, [&](int64_t b, int64_t e) {
      for (int64_t k = b; k < e; k++) {
        const double *row = &d.mats[(size_t)d.emat_id[(size_t)k] * 2];
        d.emat2[(size_t)k * 2] = row[0];
        d.emat2[(size_t)k * 2 + 1] = row[1];
      }
    });
  } else {
    std::vector<double> g((size_t)d.nmat * 36);
    for (int32_t k = 0; k < d.nmat; k++) {
      const double *row = &d.mats[(size_t)k * d.nmatp];
      double *gk = &g[(size_t)k * 36];
      if (d.mtype == 2) {  // elastgmat3d::matstiff: symmetric fill of d11..d66
        int q = 0;
        for (int i = 0; i < 6; i++)
          for (int j = i; j < 6; j++, q++) gk[6 * i + j] = gk[6 * j + i] = row[q];
      } else {
        ortho_global(row, row + 36, gk);
      }
    }
    d.dmat.resize((size_t)d.ne * 36);
    parallel_for(d.ne, d.threads, [&](int64_t b, int64_t e) {
      for (int64_t k = b; k < e; k++)
        std::memcpy(&d.dmat[(size_t)k * 36], &g[(size_t)d.emat_id[(size_t)k] * 36], 36 * sizeof(double));
    });
  }
  return SGPU_OK;
}

}  // namespace
}  // namespace sgpu

using namespace sgpu;

struct sgpu_deck_s {
  DeckData d;
};

extern "C" {

SGPU_API int sgpu_deck_read_mefel(const char *path, int32_t threads, sgpu_deck *out) {
  if (!path || !out) return fail(SGPU_BAD_INPUT, "null argument");
  *out = nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  auto *h = new sgpu_deck_s();
  DeckData &d = h->d;
  d.threads = threads > 0 ? threads : (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    delete h;
    return fail(SGPU_BAD_INPUT, std::string("cannot open deck ") + path);
  }
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  d.buf.resize(size > 0 ? (size_t)size : 0);
  const size_t got = size > 0 ? std::fread(d.buf.data(), 1, (size_t)size, f) : 0;
  std::fclose(f);
  if (size <= 0 || got != (size_t)size) {
    delete h;
    return fail(SGPU_BAD_INPUT, std::string("cannot read deck ") + path);
  }
  const int st = parse(d);
  if (st != SGPU_OK) {
    delete h;
    return st;
  }
  d.tok.clear();
  d.tok.shrink_to_fit();
  d.buf.clear();
  d.buf.shrink_to_fit();
  d.parse_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = h;
  return SGPU_OK;
}

SGPU_API int sgpu_deck_get(sgpu_deck h, sgpu_deck_view *v) {
  if (!h || !v) return fail(SGPU_BAD_INPUT, "null argument");
  const DeckData &d = h->d;
  std::memset(v, 0, sizeof(*v));
  v->kind = d.kind;
  v->ndofn = d.ndofn;
  v->nne = d.nne;
  v->mtype = d.mtype;
  v->nn = d.nn;
  v->ne = d.ne;
  v->n = d.n;
  v->nmat = d.nmat;
  v->nmatp = d.nmatp;
  v->nlc = d.nlc;
  v->storage = d.storage;
  v->precond = d.precond;
  v->iv = d.iv;
  v->ni = d.ni;
  v->res = d.res;
  v->parse_ms = d.parse_ms;
  v->coords = d.coords.data();
  v->elems = d.elems.data();
  v->dofflag = d.dofflag.data();
  v->cn = d.cn.data();
  v->emat_id = d.emat_id.data();
  v->mats = d.mats.data();
  v->thick = d.thick.empty() ? nullptr : d.thick.data();
  v->loads = d.loads.data();
  return SGPU_OK;
}

SGPU_API int sgpu_deck_mesh(sgpu_deck h, sgpu_mesh *mesh) {
  if (!h || !mesh) return fail(SGPU_BAD_INPUT, "null argument");
  const DeckData &d = h->d;
  std::memset(mesh, 0, sizeof(*mesh));
  mesh->kind = d.kind;
  mesh->ndofn = d.ndofn;
  mesh->nn = d.nn;
  mesh->coords = d.coords.data();
  mesh->ne = d.ne;
  mesh->elems = d.elems.data();
  mesh->cn = d.cn.data();
  mesh->emat = d.emat2.empty() ? nullptr : d.emat2.data();
  mesh->thick = d.thick.empty() ? nullptr : d.thick.data();
  mesh->rho = nullptr;
  mesh->dmat = d.dmat.empty() ? nullptr : d.dmat.data();
  return SGPU_OK;
}

SGPU_API int sgpu_deck_rhs(sgpu_deck h, int32_t lc, double *f) {
  if (!h || !f) return fail(SGPU_BAD_INPUT, "null argument");
  const DeckData &d = h->d;
  if (lc < 0 || lc >= d.nlc) return fail(SGPU_BAD_INPUT, "load case out of range");
  std::memset(f, 0, (size_t)d.n * sizeof(double));
  const double *L = &d.loads[(size_t)lc * d.nn * d.ndofn];
  for (size_t q = 0; q < d.cn.size(); q++)
    if (d.cn[q] > 0) f[d.cn[q] - 1] += L[q];
  return SGPU_OK;
}

SGPU_API void sgpu_deck_free(sgpu_deck h) { delete h; }

}  // extern "C"
