"""Host-side mirror of GEFEL's storage classes and solver dispatch, running on
the B200 through libsifelgpu.so.

Names, arguments and outcomes follow the reference:

* ``symcomprow`` -- GEFEL/scr.h:34 (lower triangle per row, diagonal last);
  ``mxv_scr`` (scr.cpp:655) and ``cg_prec`` (scr.cpp:1093, Jacobi, stop on
  (r.r)/(f.f) < res, ``ani``/``ares`` written only on convergence);
* ``comprow`` -- GEFEL/cr.h:34; ``mxv_cr`` (cr.cpp:653) and ``cg_prec``
  (cr.cpp:1124 with a ``noprecond`` preconditioner, stop on
  sqrt((r.h)/(f.f)) < res, ``ani``/``ares`` always written);
* ``gmatrix.solve_system`` -- the ``case cg`` dispatch of
  GEFEL/gmatrix.cpp:1184-1265 for the two storages above.

Every method runs on the GPU; there is no CPU path.  Solver methods return a
:class:`Result` with the reference's outputs (``ani``, ``ares``) and the
GPU's report (true FP64 relative residual, iterations, timings).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

storagetype = {"compressed_rows": 10, "symm_comp_rows": 11}
precondtype = {"noprecond": 0, "diagprec": 1}


@dataclass
class Result:
    status: int
    ani: int | None
    ares: float | None
    info: dict = field(default_factory=dict)

    @property
    def converged(self) -> bool:
        return self.status == L.OK


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _mode(mode):
    if isinstance(mode, str):
        return {"fp64": L.FP64, "mixed": L.MIXED}[mode]
    return int(mode)


class _Storage:
    symmetric = 0

    def __init__(self, adr, ci, a):
        self.adr = _i64(adr)
        self.ci = _i64(ci)
        self.a = _f64(a)
        self.n = self.adr.size - 1
        self.negm = int(self.adr[-1])

    def device(self) -> "DeviceMatrix":
        """A device-resident copy (for repeated products/solves)."""
        return DeviceMatrix(self.adr, self.ci, self.a, self.symmetric)


class symcomprow(_Storage):
    """GEFEL symmetric compressed rows (GEFEL/scr.h:34)."""

    symmetric = 1

    def mxv_scr(self, b):
        with self.device() as d:
            return d.mxv(b)

    def cg_prec(self, x, y, ni, res, zero=1.0e-30, iv=0, tprec=1, mode="fp64") -> Result:
        """symcomprow::cg_prec (GEFEL/scr.cpp:1093) with tprec = 1; x is
        updated in place."""
        if tprec != 1:
            raise ValueError("only the diagonal (Jacobi) preconditioner, tprec = 1, is on the GPU path")
        ani, ares = C.c_int64(-1), C.c_double(float("nan"))
        info = L.SolveInfo()
        x_ = _f64(x)
        st = L.lib().sgpu_scr_cg_prec(self.n, self.adr, self.ci, self.a, x_, _f64(y), int(ni), float(res),
                                      C.byref(ani), C.byref(ares), float(zero), int(iv), _mode(mode),
                                      C.byref(info))
        L.check(st, (L.OK, L.NOT_CONVERGED, L.BREAKDOWN, L.ZERO_RHS))
        if x_ is not x:
            x[...] = x_
        got = ani.value != -1
        return Result(st, ani.value if got else None, ares.value if got else None, info.as_dict())


class comprow(_Storage):
    """GEFEL compressed rows (GEFEL/cr.h:34)."""

    symmetric = 0

    def mxv_cr(self, b):
        with self.device() as d:
            return d.mxv(b)

    def cg_prec(self, x, y, ni, res, zero=1.0e-30, iv=0, prec="noprecond", mode="fp64") -> Result:
        """comprow::cg_prec (GEFEL/cr.cpp:1124); x is updated in place."""
        ani, ares = C.c_int64(-1), C.c_double(float("nan"))
        info = L.SolveInfo()
        x_ = _f64(x)
        p = precondtype[prec] if isinstance(prec, str) else int(prec)
        st = L.lib().sgpu_cr_cg_prec(self.n, self.adr, self.ci, self.a, x_, _f64(y), int(ni), float(res),
                                     C.byref(ani), C.byref(ares), float(zero), int(iv), p, _mode(mode),
                                     C.byref(info))
        L.check(st, (L.OK, L.NOT_CONVERGED, L.BREAKDOWN, L.ZERO_RHS))
        if x_ is not x:
            x[...] = x_
        got = ani.value != -1
        return Result(st, ani.value if got else None, ares.value if got else None, info.as_dict())


PREC = {"none": 0, "jacobi": 1, "agg": 101}


class DeviceMatrix:
    """A matrix held in HBM (handle of the C ABI), created from GEFEL storage."""

    def __init__(self, adr, ci, a, symmetric):
        adr, ci, a = _i64(adr), _i64(ci), _f64(a)
        self.n = adr.size - 1
        self.symmetric = int(symmetric)
        h = C.c_void_p()
        L.check(L.lib().sgpu_matrix_create(self.n, adr, ci, a, self.symmetric, C.byref(h)))
        self.h = h

    @classmethod
    def from_handle(cls, h, n, symmetric=1):
        obj = cls.__new__(cls)
        obj.h, obj.n, obj.symmetric = h, int(n), int(symmetric)
        return obj

    def close(self):
        if self.h:
            L.lib().sgpu_matrix_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def nnz(self) -> int:
        n, z = C.c_int64(), C.c_int64()
        L.check(L.lib().sgpu_matrix_info(self.h, C.byref(n), C.byref(z)))
        return z.value

    def update_values(self, a):
        L.check(L.lib().sgpu_matrix_update_values(self.h, _f64(a)))

    def set_spmv(self, precision, fmt, variant=0):
        """Pin the SpMV kernel (format 0 CSR / 2 sliced ELL (FP64) / 3 BSR3;
        lanes per row)."""
        L.check(L.lib().sgpu_matrix_set_spmv(self.h, int(precision), int(fmt), int(variant)))

    def spmv_plan(self, precision):
        b, f, v = C.c_double(), C.c_int32(), C.c_int32()
        L.check(L.lib().sgpu_matrix_spmv_plan(self.h, int(precision), C.byref(b), C.byref(f), C.byref(v)))
        return {"bytes": b.value, "format": f.value, "variant": v.value}

    def mxv(self, b):
        y = np.zeros(self.n)
        L.check(L.lib().sgpu_matrix_mxv(self.h, _f64(b), y))
        return y

    def download(self, symmetric=None):
        sym = self.symmetric if symmetric is None else int(symmetric)
        negm = C.c_int64()
        adr = np.zeros(self.n + 1, dtype=np.int64)
        L.check(L.lib().sgpu_matrix_download(self.h, sym, adr.ctypes.data, None, None, C.byref(negm)))
        ci = np.zeros(negm.value, dtype=np.int64)
        a = np.zeros(negm.value)
        L.check(L.lib().sgpu_matrix_download(self.h, sym, adr.ctypes.data, ci.ctypes.data, a.ctypes.data,
                                             C.byref(negm)))
        return adr, ci, a

    def set_nullspace(self, B):
        """Near-null space (n x k, k = 1, 3 or 6) for the aggregation
        preconditioner, e.g. :func:`ssf_b200.mefel.rigid_body_modes`."""
        B = np.asarray(B, dtype=np.float64)
        if B.ndim == 1:
            B = B[:, None]
        cols = np.ascontiguousarray(B.T)  # column after column
        L.check(L.lib().sgpu_matrix_set_nullspace(self.h, cols.shape[0], cols.ravel()))

    def set_rigid_body_modes(self, coords, cn):
        """The rigid-body near-null space built on the device from node
        coordinates (nn x 3) and code numbers (nn x ndofn)."""
        xyz = np.ascontiguousarray(coords, dtype=np.float64)
        c = np.ascontiguousarray(cn, dtype=np.int64)
        L.check(L.lib().sgpu_matrix_set_rigid_body_modes(self.h, xyz.shape[0], c.shape[1], xyz.ctypes.data,
                                                         c.ctypes.data))

    def precond_clear(self):
        """Discard the aggregation hierarchy (rebuilt by the next solve)."""
        L.check(L.lib().sgpu_matrix_precond_clear(self.h))

    def pcg(self, f, x=None, ni=100000, res=1e-20, zero=1e-30, crit="scr", prec=1, mode="fp64") -> tuple:
        """PCG with the criterion of the reference routine ``crit``; ``prec``
        0 / "none", 1 / "jacobi" or 101 / "agg" (aggregation multilevel
        preconditioner, flexible CG)."""
        crit_id = {"scr": L.CRIT_SCR_PREC, "cr": L.CRIT_CR_PREC, "true": L.CRIT_TRUE}[crit]
        prec = PREC.get(prec, prec)
        iv = 0 if x is None else 1
        xx = np.zeros(self.n) if x is None else _f64(x).copy()
        ani, ares = C.c_int64(-1), C.c_double(float("nan"))
        info = L.SolveInfo()
        st = L.lib().sgpu_matrix_pcg(self.h, xx, _f64(f), int(ni), float(res), float(zero), iv, crit_id, int(prec),
                                     _mode(mode), C.byref(ani), C.byref(ares), C.byref(info))
        L.check(st, (L.OK, L.NOT_CONVERGED, L.BREAKDOWN, L.ZERO_RHS))
        got = ani.value != -1
        return xx, Result(st, ani.value if got else None, ares.value if got else None, info.as_dict())


def pcg_multi(dm: "DeviceMatrix", F, ni=100000, res=1e-20, zero=1e-30, X0=None, prec="jacobi", mode="fp64"):
    """Every column of F (n x R) solved together: prec "jacobi" is the batched
    Jacobi-PCG (one SpMM per iteration, FP64), "agg" the batched flexible CG
    with the aggregation cycle (FP32 for mode "mixed").  Returns X (n x R)
    and a list of per-column Results."""
    F = np.asarray(F, dtype=np.float64)
    Fc = np.ascontiguousarray(F.T)  # R column blocks of n
    X0c = None if X0 is None else np.ascontiguousarray(np.asarray(X0, dtype=np.float64).T)
    Xc, out = pcg_multi_blocks(dm, Fc, ni, res, zero, X0c, prec, mode)
    return Xc.T.copy(), out


def pcg_multi_blocks(dm: "DeviceMatrix", Fc, ni=100000, res=1e-20, zero=1e-30, X0c=None, prec="jacobi",
                     mode="fp64", Xc=None):
    """pcg_multi on the reference's own layout (lhsrhs.cpp:72-74): Fc holds R
    column blocks of n (an R x n C array), as does the returned Xc (written
    into ``Xc`` when given, e.g. pinned host memory)."""
    R = Fc.shape[0]
    if Xc is None:
        Xc = np.zeros_like(Fc) if X0c is None else np.array(X0c, dtype=np.float64)
    elif X0c is not None:
        Xc[...] = X0c
    else:
        Xc[...] = 0.0
    X0 = X0c
    ani = np.full(R, -1, dtype=np.int64)
    ares = np.full(R, np.nan)
    st = np.zeros(R, dtype=np.int32)
    info = L.SolveInfo()
    if PREC.get(prec, prec) == L.PREC_AGG:
        rc = L.lib().sgpu_matrix_pcg_multi_agg(dm.h, R, Xc, Fc, int(ni), float(res), float(zero),
                                               0 if X0 is None else 1, _mode(mode), ani.ctypes.data,
                                               ares.ctypes.data, st.ctypes.data, C.byref(info))
    else:
        rc = L.lib().sgpu_matrix_pcg_multi(dm.h, R, Xc, Fc, int(ni), float(res), float(zero), 0 if X0 is None else 1,
                                           ani.ctypes.data, ares.ctypes.data, st.ctypes.data, C.byref(info))
    L.check(rc, (L.OK, L.NOT_CONVERGED, L.BREAKDOWN, L.ZERO_RHS))
    out = [Result(int(st[c]), int(ani[c]) if ani[c] >= 0 else None, float(ares[c]) if ani[c] >= 0 else None,
                  info.as_dict()) for c in range(R)]
    return Xc, out


class gmatrix:
    """The solver-dispatch facade of GEFEL/gmatrix.cpp for the CG cases.

    ``ts`` storage (10 / 11), ``tprec`` preconditioner (0 / 1), ``ni``,
    ``res``, ``iv`` as read by slesolv::read (GEFEL/slesolv.cpp:92-100);
    ``zero`` = 1e-30 as set by the gmatrix constructor (gmatrix.cpp:9)."""

    def __init__(self, ts=11, tprec=1, ni=100000, res=1e-20, iv=0, mode="fp64"):
        self.ts, self.tprec, self.ni, self.res, self.iv, self.mode = ts, tprec, ni, res, iv, mode
        self.zero = 1.0e-30
        self.ani = 0
        self.ares = 0.0
        self.storage = None

    def set_storage(self, adr, ci, a):
        self.storage = (symcomprow if self.ts == 11 else comprow)(adr, ci, a)

    def solve_system(self, lhs, rhs) -> Result:
        """gmatrix::solve_system, case cg (GEFEL/gmatrix.cpp:1184-1265)."""
        s = self.storage
        if self.ts == 11:
            if self.tprec != 1:
                raise ValueError("SCR on the GPU path supports diagprec only")
            r = s.cg_prec(lhs, rhs, self.ni, self.res, self.zero, self.iv, 1, self.mode)
        elif self.ts == 10:
            r = s.cg_prec(lhs, rhs, self.ni, self.res, self.zero, self.iv, self.tprec, self.mode)
        else:
            raise ValueError("storage type not on the GPU path")
        if r.ani is not None:
            self.ani, self.ares = r.ani, r.ares
        return r
