"""The drop-in solvers on the reference's exits and on malformed storage.

symcomprow::cg_prec (GEFEL/scr.cpp:1093-1205) and comprow::cg_prec
(GEFEL/cr.cpp:1124-1240) leave their loops in four ways: convergence, the
iteration limit (SCR leaves ani/ares untouched, scr.cpp:1196-1205; CR writes
ani = ni, ares = r.h, cr.cpp:1236), the zero denominator |d.p| < zero
(scr.cpp:1146-1151), and a zero right-hand side (reported at
scr.cpp:1117-1120 and followed by the zero-denominator exit; CR returns at
once, cr.cpp:1160-1164).  Each is run here on the GPU through the C ABI and
compared with the oracle (itself pinned to the compiled reference by the
golden fixtures).  Malformed storage must be refused with SGPU_BAD_INPUT
before any iteration, leaving x, ani and ares as the caller had them.  The
mixed form must report SGPU_OK only when the true FP64 residual meets the
threshold."""
import ctypes as C
import os

import numpy as np
import pytest

from ssf_b200 import _lib as L
from ssf_b200 import decks

pytestmark = pytest.mark.gpu

G = os.path.join(os.path.dirname(__file__), "golden")
SENT_ANI, SENT_ARES = -77, -7.5


def _golden(name):
    return dict(np.load(os.path.join(G, name)))


def _scr(lib, adr, ci, a, f, x, ni=20000, res=1e-20, zero=1e-30, iv=0, mode=L.FP64):
    ani, ares, info = C.c_int64(SENT_ANI), C.c_double(SENT_ARES), L.SolveInfo()
    st = lib.sgpu_scr_cg_prec(adr.size - 1, adr, ci, a, x, f, ni, res, C.byref(ani), C.byref(ares), zero, iv, mode,
                              C.byref(info))
    return st, ani.value, ares.value, info


def _cr(lib, adr, ci, a, f, x, ni=20000, res=1e-10, zero=1e-30, iv=0, prec=0, mode=L.FP64):
    ani, ares, info = C.c_int64(SENT_ANI), C.c_double(SENT_ARES), L.SolveInfo()
    st = lib.sgpu_cr_cg_prec(adr.size - 1, adr, ci, a, x, f, ni, res, C.byref(ani), C.byref(ares), zero, iv, prec,
                             mode, C.byref(info))
    return st, ani.value, ares.value, info


# -- the reference's exits --------------------------------------------------

def test_breakdown_exit_of_the_quad_plate(oracle, gpu_lib):
    # unit traction on a 0.02 m plate: |d.p| falls under the absolute zero
    # 1e-30 at iteration 49, before (r.r)/(f.f) < 1e-20; the reference leaves
    # with ani = i and ares = r.h (not divided by f.f)
    g = _golden("quad4_plate.npz")
    x = np.zeros_like(g["f"])
    st, ani, ares, info = _scr(gpu_lib, g["adr"], g["ci"], g["a"], g["f"], x)
    assert st == L.BREAKDOWN
    assert ani == int(g["ani"]) == 49
    assert ares == pytest.approx(float(g["ares"]), rel=1e-6)
    assert np.linalg.norm(x - g["u"]) / np.linalg.norm(g["u"]) <= 1e-8
    assert info.iterations == 49


def test_zero_rhs_scr(oracle, gpu_lib):
    # the reference reports the zero norm, goes on and leaves on the zero
    # denominator with ani = 0, ares = 0; the status says which happened first
    g = _golden("c1_cantilever.npz")
    f = np.zeros_like(g["f"])
    xo, st_o, ani_o, ares_o = oracle.scr_cg_prec(g["adr"], g["ci"], g["a"], f, ni=100, res=1e-20)
    assert (st_o, ani_o, ares_o) == (L.BREAKDOWN, 0, 0.0)
    x = np.full_like(f, 3.0)
    st, ani, ares, info = _scr(gpu_lib, g["adr"], g["ci"], g["a"], f, x, ni=100)
    assert st == L.ZERO_RHS
    assert (ani, ares) == (ani_o, ares_o)
    assert not x.any()


def test_zero_rhs_cr(oracle, gpu_lib):
    g = _golden("cr_cantilever.npz")
    f = np.zeros(g["adr"].size - 1)
    xo, st_o, ani_o, ares_o = oracle.cr_cg_prec(g["adr"], g["ci"], g["a"], f, ni=100, res=1e-10)
    assert st_o == L.ZERO_RHS
    x = np.full_like(f, 3.0)
    st, ani, ares, info = _cr(gpu_lib, g["adr"], g["ci"], g["a"], f, x, ni=100)
    assert st == L.ZERO_RHS and (ani, ares) == (ani_o, ares_o)
    assert not x.any() and info.iterations == 0


@pytest.mark.parametrize("ni", [1, 5, 37])
def test_iteration_limit_scr_leaves_ani_untouched(oracle, gpu_lib, ni):
    g = _golden("c1_cantilever.npz")
    xo, st_o, ani_o, _ = oracle.scr_cg_prec(g["adr"], g["ci"], g["a"], g["f"], ni=ni, res=1e-20)
    assert st_o == L.NOT_CONVERGED and ani_o == -1
    x = np.zeros_like(g["f"])
    st, ani, ares, info = _scr(gpu_lib, g["adr"], g["ci"], g["a"], g["f"], x, ni=ni)
    assert st == L.NOT_CONVERGED
    assert (ani, ares) == (SENT_ANI, SENT_ARES)
    assert info.iterations == ni
    # the same ni iterations: the iterate agrees with the oracle's
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-10


def test_iteration_limit_cr_writes_ni(oracle, gpu_lib):
    g = _golden("cr_cantilever.npz")
    f = oracle.load_vector(decks.cantilever_hex(10, 2, 2))
    xo, st_o, ani_o, ares_o = oracle.cr_cg_prec(g["adr"], g["ci"], g["a"], f, ni=9, res=1e-10)
    x = np.zeros_like(f)
    st, ani, ares, info = _cr(gpu_lib, g["adr"], g["ci"], g["a"], f, x, ni=9)
    assert st == st_o == L.NOT_CONVERGED
    assert ani == ani_o == 9
    assert ares == pytest.approx(ares_o, rel=1e-9)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-10


def test_start_vector_is_used(oracle, gpu_lib):
    # iv = 1: x on entry is the start vector (scr.cpp:1106-1112)
    g = _golden("c1_cantilever.npz")
    x0 = g["u"] * (1.0 + 1e-4)
    xo, st_o, ani_o, _ = oracle.scr_cg_prec(g["adr"], g["ci"], g["a"], g["f"], ni=20000, res=1e-20, x0=x0)
    x = x0.copy()
    st, ani, ares, info = _scr(gpu_lib, g["adr"], g["ci"], g["a"], g["f"], x, iv=1)
    assert st == st_o == L.OK and abs(ani - ani_o) <= 2 and ani < int(g["ani"])
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


# -- malformed storage ------------------------------------------------------

def _row_with_room(adr, ci, below):
    """A row i >= 2 whose last off-diagonal column leaves room for one more
    column just below (below=True) or above (below=False) the diagonal."""
    for i in range(2, adr.size - 1):
        cols = ci[adr[i]:adr[i + 1]]
        if cols.size < 3:
            continue
        if below and cols[-1] == i and cols[-2] < i - 1:
            return i
        if not below:
            k = int(np.nonzero(cols == i)[0][0])
            if k + 1 < cols.size and cols[k + 1] > i + 1:
                return i
    raise AssertionError("no suitable row")


def _scr_cases():
    def swap_adr(adr, ci, a):
        adr[5], adr[6] = adr[6], adr[5]
    def adr0(adr, ci, a):
        adr[0] = 1
    def adr_beyond(adr, ci, a):
        adr[3] = adr[-1] + 100
    def col_beyond(adr, ci, a):
        ci[adr[3]] = adr.size + 5
    def col_negative(adr, ci, a):
        ci[adr[10]] = -1
    def unsorted(adr, ci, a):
        k = adr[10]
        ci[k], ci[k + 1] = ci[k + 1], ci[k]
    def duplicate(adr, ci, a):
        k = adr[10]
        ci[k + 1] = ci[k]
    def upper_entry(adr, ci, a):
        ci[adr[12] - 1] = 12  # row 11 ends on column 12 instead of its diagonal
    def diag_not_last(adr, ci, a):
        i = _row_with_room(adr, ci, below=True)
        ci[adr[i + 1] - 1] = i - 1  # sorted, below the diagonal, no diagonal
    def zero_diag(adr, ci, a):
        a[adr[8] - 1] = 0.0
    def negative_diag(adr, ci, a):
        a[adr[8] - 1] *= -1.0
    return [("adr_not_monotone", swap_adr), ("adr0_not_zero", adr0), ("adr_beyond_negm", adr_beyond),
            ("column_beyond_n", col_beyond), ("negative_column", col_negative), ("unsorted_row", unsorted),
            ("duplicate_column", duplicate), ("entry_above_diagonal", upper_entry),
            ("diagonal_not_last", diag_not_last), ("zero_diagonal", zero_diag), ("negative_diagonal", negative_diag)]


@pytest.mark.parametrize("mode", [L.FP64, L.MIXED])
@pytest.mark.parametrize("name,edit", _scr_cases())
def test_malformed_scr_storage_is_refused(oracle, gpu_lib, name, edit, mode):
    g = _golden("c1_cantilever.npz")
    adr, ci, a = g["adr"].copy(), g["ci"].copy(), g["a"].copy()
    edit(adr, ci, a)
    x0 = np.linspace(-1.0, 2.0, g["f"].size)
    x = x0.copy()
    st, ani, ares, info = _scr(gpu_lib, adr, ci, a, g["f"], x, mode=mode)
    assert st == L.BAD_INPUT, (name, L.STATUS_NAMES.get(st))
    assert (ani, ares) == (SENT_ANI, SENT_ARES)
    assert np.array_equal(x, x0) and info.iterations == 0


def _cr_cases():
    def swap_adr(adr, ci, a):
        adr[7], adr[8] = adr[8], adr[7]
    def col_beyond(adr, ci, a):
        ci[adr[4] + 2] = adr.size + 1
    def unsorted(adr, ci, a):
        k = adr[20]
        ci[k], ci[k + 1] = ci[k + 1], ci[k]
    def no_diag(adr, ci, a):
        i = _row_with_room(adr, ci, below=False)
        k = adr[i] + int(np.nonzero(ci[adr[i]:adr[i + 1]] == i)[0][0])
        ci[k] = i + 1  # still sorted and distinct, the diagonal gone
    return [("adr_not_monotone", swap_adr), ("column_beyond_n", col_beyond), ("unsorted_row", unsorted),
            ("missing_diagonal", no_diag)]


@pytest.mark.parametrize("name,edit", _cr_cases())
def test_malformed_cr_storage_is_refused(oracle, gpu_lib, name, edit):
    g = _golden("cr_cantilever.npz")
    adr, ci, a = g["adr"].copy(), g["ci"].copy(), g["a"].copy()
    edit(adr, ci, a)
    f = np.ones(adr.size - 1)
    x0 = np.linspace(-1.0, 2.0, f.size)
    x = x0.copy()
    st, ani, ares, info = _cr(gpu_lib, adr, ci, a, f, x)
    assert st == L.BAD_INPUT, (name, L.STATUS_NAMES.get(st))
    assert (ani, ares) == (SENT_ANI, SENT_ARES)
    assert np.array_equal(x, x0) and info.iterations == 0


def test_cr_jacobi_refuses_a_non_positive_diagonal(oracle, gpu_lib):
    # the unpreconditioned CR iteration runs on any diagonal; Jacobi cannot
    g = _golden("cr_cantilever.npz")
    adr, ci, a = g["adr"], g["ci"], g["a"].copy()
    i = 6
    a[adr[i] + int(np.nonzero(ci[adr[i]:adr[i + 1]] == i)[0][0])] = 0.0
    f = np.ones(adr.size - 1)
    x = np.zeros_like(f)
    st, ani, ares, info = _cr(gpu_lib, adr, ci, a, f, x, prec=1)
    assert st == L.BAD_INPUT and (ani, ares) == (SENT_ANI, SENT_ARES) and info.iterations == 0


def test_sizes_and_null_arrays_are_refused(gpu_lib):
    g = _golden("c1_cantilever.npz")
    x = np.zeros_like(g["f"])
    ani, ares = C.c_int64(SENT_ANI), C.c_double(SENT_ARES)
    st = gpu_lib.sgpu_scr_cg_prec(0, g["adr"], g["ci"], g["a"], x, g["f"], 10, 1e-20, C.byref(ani), C.byref(ares),
                                  1e-30, 0, L.FP64, None)
    assert st == L.BAD_INPUT
    # a NULL array through a handle of the library without the binding's
    # array argument types
    raw = C.CDLL(L.LIB_PATH).sgpu_scr_cg_prec
    raw.restype = C.c_int
    vp = lambda arr: arr.ctypes.data_as(C.c_void_p)  # noqa: E731
    st = raw(C.c_int64(x.size), None, vp(g["ci"]), vp(g["a"]), vp(x), vp(g["f"]), C.c_int64(10), C.c_double(1e-20),
             C.byref(ani), C.byref(ares), C.c_double(1e-30), C.c_int64(0), C.c_int32(L.FP64), None)
    assert st == L.BAD_INPUT and (ani.value, ares.value) == (SENT_ANI, SENT_ARES)


# -- the mixed form's contract ----------------------------------------------

def _laplace_1d(n):
    """SCR storage of the 1D Laplacian (2 on the diagonal, -1 beside it)."""
    adr = np.zeros(n + 1, dtype=np.int64)
    adr[1:] = np.cumsum(np.where(np.arange(n) == 0, 1, 2))
    ci = np.empty(adr[-1], dtype=np.int64)
    a = np.empty(adr[-1])
    for i in range(n):
        if i == 0:
            ci[0], a[0] = 0, 2.0
        else:
            k = adr[i]
            ci[k], a[k] = i - 1, -1.0
            ci[k + 1], a[k + 1] = i, 2.0
    return adr, ci, a


def test_mixed_ok_only_on_the_true_residual(oracle, gpu_lib):
    g = _golden("c1_cantilever.npz")
    x = np.zeros_like(g["f"])
    st, ani, ares, info = _scr(gpu_lib, g["adr"], g["ci"], g["a"], g["f"], x, res=1e-20, mode=L.MIXED)
    assert st == L.OK and info.true_relres < 1e-10 and ani >= 0
    # a threshold below FP64's rounding floor of f - K x cannot be met: the
    # solve must say so instead of returning OK (it ends on the iteration's
    # stall or on the zero-denominator exit, whichever comes first)
    x = np.zeros_like(g["f"])
    st, ani, ares, info = _scr(gpu_lib, g["adr"], g["ci"], g["a"], g["f"], x, res=1e-36, mode=L.MIXED)
    assert st in (L.NOT_CONVERGED, L.BREAKDOWN), L.STATUS_NAMES.get(st)
    assert (ani, ares) == (SENT_ANI, SENT_ARES)
    assert info.true_relres >= 1e-18


def test_mixed_fallback_reports_the_true_residual(oracle, gpu_lib):
    # cond(S K S) ~ 4e6: the FP32 iteration stagnates and the solve goes on in
    # FP64 from its iterate, to the same threshold on the true residual
    n = 3000
    adr, ci, a = _laplace_1d(n)
    f = np.sin(np.linspace(0.0, 3.0, n)) + 0.1
    x = np.zeros(n)
    st, ani, ares, info = _scr(gpu_lib, adr, ci, a, f, x, ni=400000, res=1e-20, mode=L.MIXED)
    assert info.fallback == 1
    if st == L.OK:
        assert info.true_relres < 1e-10 and ani >= 0
    else:
        assert st == L.NOT_CONVERGED and info.true_relres >= 1e-10 and (ani, ares) == (SENT_ANI, SENT_ARES)
    # the reported residual is the returned x's (near FP64's rounding floor the
    # two evaluations differ in their own rounding, hence the factor 2)
    K = oracle.scr_to_dense(adr, ci, a)
    r_np = np.linalg.norm(f - K @ x) / np.linalg.norm(f)
    assert 0.5 * info.true_relres - 1e-15 <= r_np <= 2.0 * info.true_relres + 1e-15
