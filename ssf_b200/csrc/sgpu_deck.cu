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
// system; constraint codes 0 (fixed), 1 (free) and -k (the k-th prescribed
// displacement of each load case); one element type per deck
// (lineartet 100, linearhex 102, quadrhex 103 with crst 0; planeelementlt 20,
// planeelementlq 23, planeelementqq 24 with plane stress and a csplanestr
// thickness set); one material type per deck (elisomat 1, elgmat3d 2,
// elortomat 3 with constant transformation functions); nodal loads, element
// loads in the global system (surface loads of linearhex, edge loads of
// planeelementlq) and prescribed displacements; no temperature changes,
// eigenstrains or output requests.

#include <algorithm>
#include <atomic>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <unistd.h>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

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

// an array whose resize leaves the memory uninitialised (the file buffer and
// the token table are hundreds of MB on large decks: a zero fill on one
// thread would cost more than reading and tokenising them on all)
template <class T>
struct RawArray {
  std::unique_ptr<T[]> p;
  size_t n = 0;
  void resize(size_t count) {
    p.reset(count ? new T[count] : nullptr);
    n = count;
  }
  void clear() {
    p.reset();
    n = 0;
  }
  T *data() { return p.get(); }
  const T *data() const { return p.get(); }
  size_t size() const { return n; }
  T &operator[](size_t i) { return p[i]; }
  const T &operator[](size_t i) const { return p[i]; }
};

// phase times on stderr when SGPU_DECK_TIMING is set
struct PhaseClock {
  bool on = std::getenv("SGPU_DECK_TIMING") != nullptr;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  void mark(const char *what) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "deck: %-12s %8.1f ms\n", what, std::chrono::duration<double, std::milli>(now - t).count());
    t = now;
  }
};

// allocator whose value-less construct leaves trivial elements uninitialised:
// vectors that the parallel record loops fill entry by entry (one record per
// id, every id present) need no zero fill first
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U> &) {}
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    if constexpr (sizeof...(A) == 0) ::new ((void *)p) U;
    else ::new ((void *)p) U(std::forward<A>(a)...);
  }
};
template <class T>
using FillVec = std::vector<T, NoInitAlloc<T>>;

struct DeckData {
  PhaseClock clk;
  RawArray<char> buf;
  RawArray<int64_t> tok;  // start offset of every token after the title line
  int threads = 1;
  // header
  int32_t storage = 0, solver = 0, iv = 0, precond = 0;
  int64_t ni = 0;
  double res = 0.0;
  // mesh
  int32_t kind = -1, ndofn = 0, nne = 0, mtype = 0, nmatp = 0;
  int64_t nn = 0, ne = 0, n = 0;
  int32_t nmat = 0, nlc = 0;
  FillVec<double> coords;
  FillVec<int64_t> elems, emat_id;
  std::vector<double> mats, thick, loads, emat2, dmat;
  // per load case: element-load records (element, flags, values) and the
  // prescribed displacements
  std::vector<std::vector<int64_t>> le_eid;
  std::vector<std::vector<int32_t>> le_flags;
  std::vector<std::vector<double>> le_vals, pd;
  int64_t max_pd = 0;  // largest prescribed-displacement index the constraints use
  std::vector<int64_t> dofflag, cn;
  double parse_ms = 0.0;
  // TRFEL
  int32_t problem = 1;  // 1 linear statics (MEFEL); 50 stationary, 60 nonstationary (TRFEL)
  int32_t tform = 0;    // nonstationary solver: 1 trapezoidd, 2 trapezoidv
  double alpha = 0.0, t0 = 0.0, t1 = 0.0, dt = 0.0;
  std::vector<double> rnode, rho;  // nodal values of the lifting; per-element density

  // token access ------------------------------------------------------------
  const char *at(int64_t t) const { return buf.data() + tok[(size_t)t]; }
  const char *end() const { return buf.data() + buf.size(); }
  bool geti(int64_t t, int64_t &v) const {
    if (t < 0 || t >= (int64_t)tok.size()) return false;
    const char *p = at(t);
    // fscanf's %ld takes a leading plus, from_chars does not; a sign after
    // the plus stays an error
    if (*p == '+' && p + 1 < end() && p[1] >= '0' && p[1] <= '9') p++;
    auto r = std::from_chars(p, end(), v);
    return r.ec == std::errc() && (r.ptr == end() || blank(*r.ptr));
  }
  bool getd(int64_t t, double &v) const {
    if (t < 0 || t >= (int64_t)tok.size()) return false;
    const char *p = at(t);
    if (*p == '+' && p + 1 < end() && p[1] != '-' && p[1] != '+') p++;  // as for integers
    auto r = std::from_chars(p, end(), v);
    return r.ec == std::errc() && (r.ptr == end() || blank(*r.ptr));
  }
};

// sgpu_loads.cu
int add_element_loads(int kind, const double *coords, const int64_t *elems, const int64_t *cn, int64_t nn,
                      int64_t ne, int64_t nle, const int64_t *eid, const int32_t *flags, const double *values,
                      double *f);

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

// Bit i of the result is set where byte p[i] is blank (space, \t \n \v \f \r),
// for the 64 bytes at p.
inline uint64_t blank_mask64(const char *p) {
#if defined(__SSE2__)
  const __m128i sp = _mm_set1_epi8(' '), nine = _mm_set1_epi8(9), four = _mm_set1_epi8(4);
  uint64_t m = 0;
  for (int k = 0; k < 4; k++) {
    const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i *>(p + 16 * k));
    const __m128i x = _mm_sub_epi8(c, nine);  // 9..13 -> 0..4 (unsigned)
    const __m128i ctl = _mm_cmpeq_epi8(_mm_min_epu8(x, four), x);
    const __m128i b = _mm_or_si128(_mm_cmpeq_epi8(c, sp), ctl);
    m |= (uint64_t)(uint32_t)_mm_movemask_epi8(b) << (16 * k);
  }
  return m;
#else
  uint64_t m = 0;
  for (int k = 0; k < 64; k++) m |= (uint64_t)blank(p[k]) << k;
  return m;
#endif
}

// Token starts of buf[b, e): where a non-blank follows a blank (or `start`,
// which counts as preceded by a blank).  F(q) is called for every start q in
// increasing order.  64 bytes per step: the blank mask of the block, shifted
// by one with the carry of the previous block, against the non-blank mask.
template <class F>
void for_token_starts(const DeckData &d, size_t start, size_t b, size_t e, F &&f) {
  const char *buf = d.buf.data();
  uint64_t carry = (b == start) ? 1u : (uint64_t)blank(buf[b - 1]);
  size_t q = b;
  for (; q + 64 <= e; q += 64) {
    const uint64_t B = blank_mask64(buf + q);
    uint64_t st = ~B & ((B << 1) | carry);
    carry = B >> 63;
    while (st) {
      f(q + (size_t)__builtin_ctzll(st));
      st &= st - 1;
    }
  }
  for (; q < e; q++) {
    const bool bl = blank(buf[q]);
    if (!bl && carry) f(q);
    carry = bl;
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
  {
    std::vector<std::thread> pool;
    for (int p = 0; p < parts; p++)
      pool.emplace_back([&, p] {
        size_t b, e;
        bounds(p, b, e);
        int64_t c = 0;
        for_token_starts(d, start, b, e, [&c](size_t) { c++; });
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
        int64_t *w = d.tok.data() + counts[p];
        for_token_starts(d, start, b, e, [&w](size_t q) { *w++ = (int64_t)q; });
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

int parse_mefel(DeckData &d) {
  // the title is the first line (probdesc::read reads it whole)
  size_t start = 0;
  while (start < d.buf.size() && d.buf[start] != '\n') start++;
  SGPU_TRY(tokenize(d, start));
  d.clk.mark("tokenize");
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
  d.coords.resize((size_t)d.nn * 3);  // every node record writes its row
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

  // --- constraints: "id c1..c_ndofn" with 0 fixed, 1 free, -k prescribed ---
  d.dofflag.assign((size_t)d.nn * d.ndofn, 1);
  const int64_t ncn = c.i();
  if (!c.err.empty() || ncn < 0 || ncn > d.nn) return fail(SGPU_BAD_INPUT, "deck: bad constraint count");
  std::atomic<int64_t> max_pd{0};
  bad = parallel_records(d, c.t, ncn, 1 + d.ndofn, [&](int64_t, int64_t t, bool &ok) {
    int64_t id = 0;
    ok = d.geti(t, id) && id >= 1 && id <= d.nn;
    for (int q = 0; ok && q < d.ndofn; q++) {
      int64_t v = 0;
      ok = d.geti(t + 1 + q, v) && v <= 1 && v > -(1LL << 40);
      if (ok) d.dofflag[(size_t)(id - 1) * d.ndofn + q] = v;
      if (ok && v < 0) {
        int64_t cur = max_pd.load();
        while (-v > cur && !max_pd.compare_exchange_weak(cur, -v)) {
        }
      }
    }
  });
  if (bad >= 0)
    return fail(SGPU_BAD_INPUT, "deck: constraint record " + std::to_string(bad + 1) +
                                    " is not 'id c1..cn' with codes 0 (fixed), 1 (free) or -k (prescribed)");
  d.max_pd = max_pd.load();
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
  d.elems.resize((size_t)d.ne * d.nne);  // every element record writes its row
  d.emat_id.resize((size_t)d.ne);
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
    // loaded elements (loadel::read, MEFEL/SRC/loadel.cpp:96): "eid type"
    // then, for a surface load (3) of a linear hexahedron, per face a flag
    // and 4 nodes x 3 values when the flag is 1 or 2; for an edge load (2) of
    // a plane quad, per edge a flag and 2 nodes x 2 values when positive
    const int64_t nle = c.i();
    if (!c.err.empty() || nle < 0 || nle > d.ne)
      return fail(SGPU_BAD_INPUT, "deck: bad loaded-element count in load case " + std::to_string(lc + 1));
    d.le_eid.emplace_back();
    d.le_flags.emplace_back();
    d.le_vals.emplace_back();
    const bool hexs = d.kind == SGPU_ELEM_HEX8, quade = d.kind == SGPU_ELEM_QUAD4;
    const int nfl = hexs ? 6 : 4, per = hexs ? 12 : 4;
    for (int64_t r = 0; r < nle; r++) {
      const std::string rec = "deck: loaded element " + std::to_string(r + 1) + " of load case " + std::to_string(lc + 1);
      const int64_t eid = c.i(), tel = c.i();
      if (!c.err.empty()) return fail(SGPU_BAD_INPUT, rec + ": " + c.err);
      if (eid < 1 || eid > d.ne) return fail(SGPU_BAD_INPUT, rec + ": element out of range");
      if (!((hexs && tel == 3) || (quade && tel == 2)))
        return fail(SGPU_BAD_INPUT, rec + ": load type " + std::to_string(tel) +
                                        " is not supported (surface loads of linearhex, edge loads of planeelementlq)");
      d.le_eid.back().push_back(eid - 1);
      for (int k = 0; k < nfl; k++) {
        const int64_t fl = c.i();
        if (!c.err.empty()) return fail(SGPU_BAD_INPUT, rec + ": " + c.err);
        if (hexs && fl != 0 && fl != 1)
          return fail(SGPU_BAD_INPUT, rec + ": surface flag " + std::to_string(fl) +
                                          " (only 0 and 1, loads in the global system, are supported)");
        if (fl < 0) return fail(SGPU_BAD_INPUT, rec + ": negative edge flag");
        d.le_flags.back().push_back((int32_t)fl);
        for (int q = 0; q < per; q++) d.le_vals.back().push_back(fl > 0 ? c.f() : 0.0);
        if (!c.err.empty()) return fail(SGPU_BAD_INPUT, rec + ": " + c.err);
      }
    }
    // prescribed displacements (loadcase::read, MEFEL/SRC/loadcase.cpp:135-140)
    const int64_t npd = c.i();
    if (!c.err.empty() || npd < 0 || npd > (int64_t)d.nn * d.ndofn)
      return fail(SGPU_BAD_INPUT, "deck: bad prescribed-displacement count in load case " + std::to_string(lc + 1));
    if (npd < d.max_pd)
      return fail(SGPU_BAD_INPUT, "deck: load case " + std::to_string(lc + 1) + " has " + std::to_string(npd) +
                                      " prescribed displacements, the constraints use " + std::to_string(d.max_pd));
    d.pd.emplace_back((size_t)npd, 0.0);
    for (int64_t k = 0; k < npd; k++) d.pd.back()[(size_t)k] = c.f();
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
  for (size_t q = 0; q < d.dofflag.size(); q++) {
    if (d.dofflag[q] == 1) d.cn[q] = ++next;
    else if (d.dofflag[q] < 0) d.cn[q] = d.dofflag[q];  // gencodnum keeps the prescribed index
  }
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

// TRFEL linear heat conduction with linear hexahedra (linhext, element type
// 225), as trfel_init (TRFEL/SRC/trfelinit.cpp:24) reads it: probdesct::read
// (TRFEL/SRC/probdesct.cpp:177-560, timecontr::read GEFEL/timecontr.cpp:70),
// transtop::read (transtop.cpp:93), elementt::read (elementt.cpp:72),
// transmat::read (isotrmat "c k", isotrmat.cpp:444), transcrsec::read
// (transcrsec.cpp:33, one crsec3dt density), transbclc::read / loadcaset::read
// (loadcaset.cpp:133, pvalt::read pvalt.cpp:24) and lhsrhst::initcond
// (lhsrhst.cpp:157).  Every element may carry its own material instance (the
// heterogeneous cube has one per element), so the material records are
// converted by all threads too.
int parse_trfel(DeckData &d) {
  size_t start = 0;
  while (start < d.buf.size() && d.buf[start] != '\n') start++;
  SGPU_TRY(tokenize(d, start));
  d.clk.mark("tokenize");
  Cursor c{d};
  c.i();  // mesprt
  d.problem = (int32_t)c.i();
  if (d.problem != 50 && d.problem != 60 && c.err.empty())
    c.err = "problem type " + std::to_string(d.problem) + " is not supported";
  c.expect(1, "transmatter (one medium)");
  c.expect(1, "medium (heat)");
  c.f();  // scale
  for (int k = 0; k < 11; k++) c.expect(0, "optional computation flag");
  if (d.problem == 50) {
    d.storage = (int32_t)c.i();
  } else {
    d.tform = (int32_t)c.i();
    if (d.tform != 1 && d.tform != 2 && c.err.empty()) c.err = "nonstationary solver " + std::to_string(d.tform) + " is not supported";
    d.alpha = c.f();
    c.expect(0, "time control type (fixed)");
    d.t0 = c.f();
    d.t1 = c.f();
    const int64_t nit = c.i();
    if (nit < 0 && c.err.empty()) c.err = "generated important times are not supported";
    for (int64_t k = 0; k < nit; k++) c.f();
    c.expect(0, "time step function (constant)");
    d.dt = c.f();
    c.i();  // timetypeprint
    c.expect(0, "hdbackup");
    d.storage = (int32_t)c.i();
    c.expect(d.storage, "capacity storage (as the conductivity's)");
  }
  if (d.storage != 11 && d.storage != 10 && c.err.empty()) c.err = "storage " + std::to_string(d.storage) + " is not supported";
  d.solver = (int32_t)c.i();
  if (d.solver != 20 && c.err.empty()) c.err = "linear solver " + std::to_string(d.solver) + " is not supported";
  d.ni = c.i();
  d.res = c.f();
  d.iv = (int32_t)c.i();
  d.precond = (int32_t)c.i();
  if (d.problem == 60) c.expect(0, "capacity diagonalization");
  if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);

  // nodes: "id x y z ndofn crst" with one DOF and no cross section
  d.ndofn = 1;
  d.nn = c.i();
  if (!c.err.empty() || d.nn <= 0) return fail(SGPU_BAD_INPUT, "deck: bad node count");
  d.coords.resize((size_t)d.nn * 3);  // every node record writes its row
  std::vector<std::atomic<uint8_t>> seen((size_t)d.nn);
  for (auto &q : seen) q.store(0, std::memory_order_relaxed);
  int64_t bad = parallel_records(d, c.t, d.nn, 6, [&](int64_t, int64_t t, bool &ok) {
    int64_t id = 0, nd = 0, crst = 0;
    ok = d.geti(t, id) && id >= 1 && id <= d.nn && d.geti(t + 4, nd) && nd == 1 && d.geti(t + 5, crst) && crst == 0;
    if (!ok) return;
    double *x = &d.coords[(size_t)(id - 1) * 3];
    ok = d.getd(t + 1, x[0]) && d.getd(t + 2, x[1]) && d.getd(t + 3, x[2]) && seen[(size_t)(id - 1)].exchange(1) == 0;
  });
  if (bad >= 0) return fail(SGPU_BAD_INPUT, "deck: node record " + std::to_string(bad + 1) + " is not 'id x y z 1 0'");
  c.t += d.nn * 6;
  d.clk.mark("nodes");

  // constraints: "id code", code < 0 the prescribed value -code, 1 free
  d.dofflag.assign((size_t)d.nn, 1);
  std::vector<int64_t> pv_of((size_t)d.nn, 0);
  const int64_t ncn = c.i();
  if (!c.err.empty() || ncn < 0 || ncn > d.nn) return fail(SGPU_BAD_INPUT, "deck: bad constraint count");
  bad = parallel_records(d, c.t, ncn, 2, [&](int64_t, int64_t t, bool &ok) {
    int64_t id = 0, code = 0;
    ok = d.geti(t, id) && id >= 1 && id <= d.nn && d.geti(t + 1, code) && (code < 0 || code == 1);
    if (ok && code < 0) {
      d.dofflag[(size_t)(id - 1)] = 0;
      pv_of[(size_t)(id - 1)] = -code;
    }
  });
  if (bad >= 0)
    return fail(SGPU_BAD_INPUT, "deck: constraint record " + std::to_string(bad + 1) +
                                    " is not 'id code' with a prescribed-value index (< 0) or 1");
  c.t += ncn * 2;

  // elements: "id 225 n1..n8 cne crst idcs tm idm"
  d.kind = SGPU_ELEM_HEX8T_K;
  d.nne = 8;
  d.ne = c.i();
  if (!c.err.empty() || d.ne <= 0 || d.ne > (1LL << 31) - 1) return fail(SGPU_BAD_INPUT, "deck: bad element count");
  d.elems.resize((size_t)d.ne * 8);  // every element record writes its row
  d.emat_id.resize((size_t)d.ne);
  FillVec<int64_t> cs_of((size_t)d.ne);
  std::vector<std::atomic<uint8_t>> eseen((size_t)d.ne);
  for (auto &q : eseen) q.store(0, std::memory_order_relaxed);
  bad = parallel_records(d, c.t, d.ne, 15, [&](int64_t, int64_t t, bool &ok) {
    int64_t id = 0, type = 0, v = 0;
    ok = d.geti(t, id) && id >= 1 && id <= d.ne && d.geti(t + 1, type) && type == 225;
    if (!ok) return;
    const size_t e = (size_t)(id - 1);
    for (int a = 0; ok && a < 8; a++) {
      ok = d.geti(t + 2 + a, v) && v >= 1 && v <= d.nn;
      if (ok) d.elems[e * 8 + a] = v - 1;
    }
    ok = ok && d.geti(t + 10, v) && v == 0 && d.geti(t + 11, v) && v == 3 && d.geti(t + 12, v) && v >= 1;
    if (ok) cs_of[e] = v - 1;
    ok = ok && d.geti(t + 13, v) && v == 100 && d.geti(t + 14, v) && v >= 1;
    if (ok) d.emat_id[e] = v - 1;
    ok = ok && eseen[e].exchange(1) == 0;
  });
  if (bad >= 0)
    return fail(SGPU_BAD_INPUT, "deck: element record " + std::to_string(bad + 1) +
                                    " is not 'id 225 n1..n8 0 3 cs 100 mat' or repeats an id");
  c.t += d.ne * 15;
  d.clk.mark("elements");

  // materials: one type isotransmat (100), instances "id c k"
  c.expect(1, "number of material types");
  c.expect(100, "material type (isotransmat)");
  d.nmat = (int32_t)c.i();
  if (!c.err.empty() || d.nmat <= 0) return fail(SGPU_BAD_INPUT, "deck: " + (c.err.empty() ? std::string("no materials") : c.err));
  d.mtype = 100;
  d.nmatp = 2;
  d.mats.assign((size_t)d.nmat * 2, 0.0);  // (k, c) per instance
  std::vector<std::atomic<uint8_t>> mseen((size_t)d.nmat);
  for (auto &q : mseen) q.store(0, std::memory_order_relaxed);
  bad = parallel_records(d, c.t, d.nmat, 3, [&](int64_t, int64_t t, bool &ok) {
    int64_t id = 0;
    double cc = 0.0, kk = 0.0;
    ok = d.geti(t, id) && id >= 1 && id <= d.nmat && d.getd(t + 1, cc) && d.getd(t + 2, kk) &&
         mseen[(size_t)(id - 1)].exchange(1) == 0;
    if (ok) {
      d.mats[(size_t)(id - 1) * 2] = kk;
      d.mats[(size_t)(id - 1) * 2 + 1] = cc;
    }
  });
  if (bad >= 0) return fail(SGPU_BAD_INPUT, "deck: material record " + std::to_string(bad + 1) + " is not 'id c k'");
  c.t += (int64_t)d.nmat * 3;
  d.clk.mark("materials");

  // cross sections: one type crsec3dt (3), instances "id rho"
  c.expect(1, "number of cross-section types");
  c.expect(3, "cross-section type (crsec3dt)");
  const int64_t ncs = c.i();
  std::vector<double> rho_cs((size_t)std::max<int64_t>(ncs, 0), 0.0);
  for (int64_t k = 0; k < ncs && c.err.empty(); k++) {
    const int64_t id = c.i();
    if (id < 1 || id > ncs) c.err = "cross section out of range";
    else rho_cs[(size_t)(id - 1)] = c.f();
  }
  if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);

  // one load case: prescribed values, nothing else
  c.expect(1, "number of load cases");
  const int64_t npv = c.i();
  std::vector<double> pv((size_t)std::max<int64_t>(npv, 0), 0.0);
  for (int64_t k = 0; k < npv && c.err.empty(); k++) {
    c.f();  // initial prescribed value
    if (d.problem == 60) c.expect(0, "prescribed-value function (constant)");
    pv[(size_t)k] = c.f();
  }
  for (int k = 0; k < 6; k++) c.expect(0, "sources / element loads / nodal values / climatic conditions / functions");
  c.expect(0, "boundary fluxes");
  if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);
  // initial values (nonstationary): "id value" for every node
  std::vector<double> init((size_t)d.nn, 0.0);
  if (d.problem == 60) {
    bad = parallel_records(d, c.t, d.nn, 2, [&](int64_t, int64_t t, bool &ok) {
      int64_t id = 0;
      double v = 0.0;
      ok = d.geti(t, id) && id >= 1 && id <= d.nn && d.getd(t + 1, v);
      if (ok) init[(size_t)(id - 1)] = v;
    });
    if (bad >= 0) return fail(SGPU_BAD_INPUT, "deck: initial-value record " + std::to_string(bad + 1));
    c.t += d.nn * 2;
  }
  d.clk.mark("initial");
  c.expect(0, "text output");
  c.expect(0, "graphic output");
  if (d.problem == 60) c.expect(0, "diagnostics");
  if (c.err.empty() && c.t != (int64_t)d.tok.size()) c.err = "unexpected token " + std::to_string(c.t) + " after the deck";
  if (!c.err.empty()) return fail(SGPU_BAD_INPUT, "deck: " + c.err);

  // validate indices, then: code numbers, per-element (k, c) rows and
  // density, the nodal values of the lifting (prescribed values on
  // prescribed nodes, initial values on free ones: prescvalues,
  // TRFEL/SRC/globmatt.cpp:1057)
  for (int64_t e = 0; e < d.ne; e++)
    if (d.emat_id[(size_t)e] >= d.nmat || cs_of[(size_t)e] >= ncs)
      return fail(SGPU_BAD_INPUT, "deck: element " + std::to_string(e + 1) + " names a missing material or cross section");
  d.rnode.assign((size_t)d.nn, 0.0);
  for (int64_t i = 0; i < d.nn; i++) {
    const int64_t k = pv_of[(size_t)i];
    if (k > npv) return fail(SGPU_BAD_INPUT, "deck: prescribed-value index out of range");
    d.rnode[(size_t)i] = k > 0 ? pv[(size_t)(k - 1)] : init[(size_t)i];
  }
  d.cn.assign((size_t)d.nn, 0);
  int64_t next = 0;
  for (int64_t i = 0; i < d.nn; i++)
    if (d.dofflag[(size_t)i] == 1) d.cn[(size_t)i] = ++next;
  d.n = next;
  if (d.n == 0) return fail(SGPU_BAD_INPUT, "deck: no free DOFs");
  d.emat2.resize((size_t)d.ne * 2);
  d.rho.resize((size_t)d.ne);
  parallel_for(d.ne, d.threads, [&](int64_t b, int64_t e) {
    for (int64_t k = b; k < e; k++) {
      const double *row = &d.mats[(size_t)d.emat_id[(size_t)k] * 2];
      d.emat2[(size_t)k * 2] = row[0];
      d.emat2[(size_t)k * 2 + 1] = row[1];
      d.rho[(size_t)k] = rho_cs[(size_t)cs_of[(size_t)k]];
    }
  });
  d.nlc = 1;
  return SGPU_OK;
}

// reads the file with all threads (pread of one chunk each)
int read_file(const char *path, DeckData &d) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(SGPU_BAD_INPUT, std::string("cannot open deck ") + path);
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fclose(f);
  if (size <= 0) return fail(SGPU_BAD_INPUT, std::string("empty deck ") + path);
  d.buf.resize((size_t)size);
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) return fail(SGPU_BAD_INPUT, std::string("cannot open deck ") + path);
  std::atomic<bool> ok{true};
  const int parts = std::max(1, std::min(d.threads, (int)(size / (1 << 22)) + 1));
  std::vector<std::thread> pool;
  for (int p = 0; p < parts; p++)
    pool.emplace_back([&, p] {
      size_t b = (size_t)size * p / parts, e = (size_t)size * (p + 1) / parts;
      while (b < e) {
        const ssize_t got = ::pread(fd, d.buf.data() + b, e - b, (off_t)b);
        if (got <= 0) {
          ok = false;
          return;
        }
        b += (size_t)got;
      }
    });
  for (auto &th : pool) th.join();
  ::close(fd);
  if (!ok) return fail(SGPU_BAD_INPUT, std::string("cannot read deck ") + path);
  return SGPU_OK;
}

int read_deck(const char *path, int32_t threads, bool trfel, sgpu_deck_s **out);

}  // namespace
}  // namespace sgpu

using namespace sgpu;

struct sgpu_deck_s {
  DeckData d;
};

namespace sgpu {
namespace {
int read_deck(const char *path, int32_t threads, bool trfel, sgpu_deck_s **out) {
  if (!path || !out) return fail(SGPU_BAD_INPUT, "null argument");
  *out = nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  auto *h = new sgpu_deck_s();
  DeckData &d = h->d;
  d.threads = threads > 0 ? threads : (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  int st = read_file(path, d);
  d.clk.mark("read");
  if (st == SGPU_OK) st = trfel ? parse_trfel(d) : parse_mefel(d);
  d.clk.mark("sections");
  if (st != SGPU_OK) {
    delete h;
    return st;
  }
  d.tok.clear();
  d.buf.clear();
  d.parse_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = h;
  return SGPU_OK;
}
}  // namespace
}  // namespace sgpu

extern "C" {

SGPU_API int sgpu_deck_read_mefel(const char *path, int32_t threads, sgpu_deck *out) {
  return sgpu::read_deck(path, threads, false, out);
}

SGPU_API int sgpu_deck_read_trfel(const char *path, int32_t threads, sgpu_deck *out) {
  return sgpu::read_deck(path, threads, true, out);
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
  v->problem = d.problem;
  v->tform = d.tform;
  v->alpha = d.alpha;
  v->t0 = d.t0;
  v->t1 = d.t1;
  v->dt = d.dt;
  v->rnode = d.rnode.empty() ? nullptr : d.rnode.data();
  v->rho = d.rho.empty() ? nullptr : d.rho.data();
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
  mesh->rho = d.rho.empty() ? nullptr : d.rho.data();
  mesh->dmat = d.dmat.empty() ? nullptr : d.dmat.data();
  return SGPU_OK;
}

SGPU_API int sgpu_deck_rhs(sgpu_deck h, int32_t lc, double *f) {
  if (!h || !f) return fail(SGPU_BAD_INPUT, "null argument");
  const DeckData &d = h->d;
  if (d.problem != 1)
    return fail(SGPU_BAD_INPUT, "a TRFEL deck's right-hand side is the lifting of rnode (sgpu_assembly_lift)");
  if (lc < 0 || lc >= d.nlc) return fail(SGPU_BAD_INPUT, "load case out of range");
  std::memset(f, 0, (size_t)d.n * sizeof(double));
  const double *L = &d.loads[(size_t)lc * d.nn * d.ndofn];
  for (size_t q = 0; q < d.cn.size(); q++)
    if (d.cn[q] > 0) f[d.cn[q] - 1] += L[q];
  // then the element loads, record by record (loadcase::forcecontrib)
  if ((size_t)lc < d.le_eid.size() && !d.le_eid[(size_t)lc].empty())
    return add_element_loads(d.kind, d.coords.data(), d.elems.data(), d.cn.data(), d.nn, d.ne,
                             (int64_t)d.le_eid[(size_t)lc].size(), d.le_eid[(size_t)lc].data(),
                             d.le_flags[(size_t)lc].data(), d.le_vals[(size_t)lc].data(), f);
  return SGPU_OK;
}

SGPU_API int sgpu_deck_prescribed(sgpu_deck h, int32_t lc, double *r, int64_t *count) {
  if (!h || !r) return fail(SGPU_BAD_INPUT, "null argument");
  const DeckData &d = h->d;
  if (d.problem != 1) return fail(SGPU_BAD_INPUT, "prescribed displacements belong to MEFEL decks");
  if (lc < 0 || lc >= d.nlc) return fail(SGPU_BAD_INPUT, "load case out of range");
  int64_t k = 0;
  const std::vector<double> &pd = d.pd[(size_t)lc];
  for (size_t q = 0; q < d.dofflag.size(); q++) {
    const int64_t c = d.dofflag[q];
    r[q] = 0.0;
    if (c < 0) {
      r[q] = pd[(size_t)(-c - 1)];
      k++;
    }
  }
  if (count) *count = k;
  return SGPU_OK;
}

SGPU_API void sgpu_deck_free(sgpu_deck h) { delete h; }

}  // extern "C"
