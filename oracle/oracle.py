"""ctypes front end of the CPU oracle (oracle/sifel_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the cpu_baseline leg of bench.py -- never by the product package.  ``build()``
compiles the restatement with gcc -O3 (no FMA contraction, like the
reference's own -O3 x86-64 build) into ``oracle/liboracle.so``.

Also wraps the compiled reference itself (``oracle/_ref/libsifelref.so``,
built by oracle/build_ref.py) where present: ``ref_*`` functions run SIFEL's
own GEFEL solvers on the same arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "sifel_oracle.c")
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libsifelref.so")

_lib = None
_ref = None

P = np.ctypeslib.ndpointer
_L = C.c_long
_D = C.c_double
_pL = P(np.int64, flags="C_CONTIGUOUS")
_pD = P(np.float64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.run(["gcc", "-O3", "-ffp-contract=off", "-fPIC", "-shared", SRC, "-o", LIB, "-lm"],
                       check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.or_hex8_ke.argtypes = [_pD, _D, _D, _pD]
        L.or_quad4_ke.argtypes = [_pD, _D, _D, _pD, _pD]
        L.or_hex8t_kc.argtypes = [_pD, _D, _D, _pD, C.c_void_p, C.c_void_p]
        L.or_pattern.argtypes = [_L, _L, _L, _pL, C.c_int, _pL, C.c_void_p]
        L.or_pattern.restype = _L
        L.or_assemble.argtypes = [C.c_int, C.c_int, _L, _pD, _pL, _pL, _pD, C.c_void_p, C.c_void_p,
                                  _pL, _pL, _pD]
        L.or_assemble.restype = _L
        L.or_tet4_ke.argtypes = [_pD, _D, _D, _pD]
        L.or_tri3_ke.argtypes = [_pD, _D, _D, _pD, _pD]
        L.or_assemble_d.argtypes = [C.c_int, C.c_int, _L, _pD, _pL, _pL, _pD, _pL, _pL, _pD]
        L.or_assemble_d.restype = _L
        L.or_ortho_dmat.argtypes = [_pD, _pD, _pD]
        L.or_hex20_ke.argtypes = [_pD, _D, _D, _pD]
        L.or_quad8_ke.argtypes = [_pD, _D, _D, _pD, _pD]
        L.or_quad8_ke.restype = C.c_int
        L.or_tet4_ke.restype = C.c_int
        L.or_scr_mxv.argtypes = [_L, _pL, _pL, _pD, _pD, _pD]
        L.or_cr_mxv.argtypes = [_L, _pL, _pL, _pD, _pD, _pD]
        for f in (L.or_scr_cg_prec, L.or_cr_cg_prec):
            f.argtypes = [_L, _pL, _pL, _pD, _pD, _pD, _L, _D, _D, _L, C.POINTER(_L), C.POINTER(_D)]
            f.restype = C.c_int
        for f in (L.or_trfel_step, L.or_trfel_step_v):
            f.argtypes = [_L, _pL, _pL, _pD, _pD, _pD, _pD, _pD, _pD, _D, _D, _L, _D, _D,
                          _L, C.POINTER(_L), C.POINTER(_D)]
            f.restype = C.c_int
        L.or_trfel_lift.argtypes = [_L, _pD, _pL, _pL, _pD, _pD, _pD]
        L.or_hex8_surface_nf.argtypes = [_pD, _pL, _pD, _pD]
        L.or_quad4_edge_nf.argtypes = [_pD, _pL, _pD, _pD]
        L.or_prescribed_contrib.argtypes = [C.c_int, _pD, _pL, _pD, _pD]
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


# ----------------------------------------------------------------------------
# element matrices
# ----------------------------------------------------------------------------

def hex8_ke(xyz, E, nu):
    ke = np.zeros(576)
    lib().or_hex8_ke(_f64(xyz).reshape(-1), float(E), float(nu), ke)
    return ke.reshape(24, 24)


def tet4_ke(xyz, E, nu):
    ke = np.zeros(144)
    if lib().or_tet4_ke(_f64(xyz).reshape(-1), float(E), float(nu), ke) != 0:
        raise ValueError("negative volume (wrong node numbering)")
    return ke.reshape(12, 12)


def hex20_ke(xyz, E, nu):
    ke = np.zeros(3600)
    lib().or_hex20_ke(_f64(xyz).reshape(-1), float(E), float(nu), ke)
    return ke.reshape(60, 60)


def quad8_ke(xy, E, nu, t):
    ke = np.zeros(256)
    tt = _f64(np.broadcast_to(np.asarray(t, dtype=np.float64), (8,)))
    if lib().or_quad8_ke(_f64(xy).reshape(-1), float(E), float(nu), tt, ke) != 0:
        raise ValueError("negative Jacobian (wrong node numbering)")
    return ke.reshape(16, 16)


def tri3_ke(xy, E, nu, t):
    ke = np.zeros(36)
    tt = _f64(np.broadcast_to(np.asarray(t, dtype=np.float64), (3,)))
    lib().or_tri3_ke(_f64(xy).reshape(-1), float(E), float(nu), tt, ke)
    return ke.reshape(6, 6)


def quad4_ke(xy, E, nu, t):
    ke = np.zeros(64)
    tt = _f64(np.broadcast_to(np.asarray(t, dtype=np.float64), (4,)))
    lib().or_quad4_ke(_f64(xy).reshape(-1), float(E), float(nu), tt, ke)
    return ke.reshape(8, 8)


def hex8t_kc(xyz, k, c, rho=1.0):
    ke = np.zeros(64)
    ce = np.zeros(64)
    r = _f64(np.broadcast_to(np.asarray(rho, dtype=np.float64), (8,)))
    lib().or_hex8t_kc(_f64(xyz).reshape(-1), float(k), float(c), r, ke.ctypes.data, ce.ctypes.data)
    return ke.reshape(8, 8), ce.reshape(8, 8)


# ----------------------------------------------------------------------------
# mesh-level assembly
# ----------------------------------------------------------------------------

KIND = {"hex8": 0, "quad4": 1, "hex8t_k": 2, "hex8t_c": 3, "tet4": 4, "tri3": 5, "hex20": 6, "quad8": 7}


def element_code_numbers(mesh):
    cn = mesh.code_numbers()  # (nn, ndofn)
    return _i64(cn[mesh.elems].reshape(mesh.ne, -1))


def pattern(n, cne, sym):
    cne = _i64(cne)
    adr = np.zeros(n + 1, dtype=np.int64)
    negm = lib().or_pattern(n, cne.shape[0], cne.shape[1], cne, int(sym), adr, None)
    ci = np.zeros(negm, dtype=np.int64)
    lib().or_pattern(n, cne.shape[0], cne.shape[1], cne, int(sym), adr, ci.ctypes.data)
    return adr, ci


def material_dmat(mesh):
    """Per-material 6 x 6 global stiffness (nmat, 36) of a "gen3d" mesh
    (elastgmat3d::matstiff, symmetric fill of the 21 read entries) or an
    "ortho" mesh (elastortomat::matstiff with constant transformation
    functions, through the C restatement of lg_tens4transf)."""
    out = np.zeros((mesh.mats.shape[0], 36))
    for k, row in enumerate(np.asarray(mesh.mats, dtype=np.float64)):
        if mesh.mtype == "gen3d":
            D = np.zeros((6, 6))
            D[np.triu_indices(6)] = row[:21]
            D = np.triu(D) + np.triu(D, 1).T
            out[k] = D.ravel()
        else:
            g = np.zeros(36)
            lib().or_ortho_dmat(_f64(row[:36]), _f64(row[36:45]), g)
            out[k] = g
    return out


def assemble(mesh, sym=True, kind=None, rho=None):
    """Global matrix of ``mesh`` in SCR (sym) or CR storage: (adr, ci, a)."""
    kind = kind or mesh.kind
    k = KIND[kind]
    n = mesh.ndof
    cne = element_code_numbers(mesh)
    adr, ci = pattern(n, cne, sym)
    a = np.zeros(ci.size)
    if getattr(mesh, "mtype", "iso") != "iso":
        if kind not in ("hex8", "tet4", "hex20"):
            raise ValueError("general materials are defined for the 3D elements")
        dm = _f64(material_dmat(mesh)[mesh.emat])
        st = lib().or_assemble_d(k, int(sym), mesh.ne, _f64(mesh.coords), _i64(mesh.elems), cne, dm, adr, ci, a)
        if st != 0:
            raise ValueError(f"element {-st} has a negative volume (wrong node numbering)")
        return adr, ci, a
    emat = _f64(mesh.mats[mesh.emat])
    thick = _f64(mesh.thick) if mesh.thick is not None else None
    rr = _f64(rho) if rho is not None else None
    st = lib().or_assemble(k, int(sym), mesh.ne, _f64(mesh.coords), _i64(mesh.elems), cne, emat,
                           thick.ctypes.data if thick is not None else None,
                           rr.ctypes.data if rr is not None else None, adr, ci, a)
    if st != 0:
        raise ValueError(f"element {-st} has a negative volume (wrong node numbering)")
    return adr, ci, a


def element_load_forces(mesh, eid, flags, values):
    """Nodal forces of one element load record (loadel::surfaceload /
    edgeload): linhex::node_forces_surf or planeelemlq::nodeforces."""
    nd = mesh.elems[eid]
    if mesh.kind == "hex8":
        nf = np.zeros(24)
        lib().or_hex8_surface_nf(_f64(mesh.coords[nd].reshape(-1)), _i64(flags), _f64(values), nf)
    elif mesh.kind == "quad4":
        nf = np.zeros(8)
        lib().or_quad4_edge_nf(_f64(mesh.coords[nd, :2].reshape(-1)), _i64(flags), _f64(values), nf)
    else:
        raise ValueError("element loads are restated for hex8 surfaces and quad4 edges")
    return nf


def element_stiffness(mesh, e):
    """The element matrix stiffness_matrix localises for element e."""
    nd = mesh.elems[e]
    E, nu = mesh.mats[mesh.emat[e]][:2]
    if mesh.kind == "hex8":
        ke = np.zeros(24 * 24)
        lib().or_hex8_ke(_f64(mesh.coords[nd].reshape(-1)), E, nu, ke)
    elif mesh.kind == "quad4":
        ke = np.zeros(64)
        lib().or_quad4_ke(_f64(mesh.coords[nd, :2].reshape(-1)), E, nu, _f64(np.full(4, mesh.thick[e])), ke)
    else:
        raise ValueError("prescribed displacements are restated for hex8 and quad4")
    return ke


def load_vector(mesh, lc=0):
    """Right-hand side of load case lc in equation order: loadcase::assemble
    (MEFEL/SRC/loadcase.cpp:400) -- forcecontrib (:546: nodal loads in record
    order, then the element loads' nodal forces, locglob) and, for elements
    with prescribed displacements, prdisplcontrib (:615: f -= K_e r_e)."""
    cn = mesh.code_numbers().reshape(-1)
    f = np.zeros(mesh.ndof)
    vals = mesh.loads[lc].reshape(-1)
    m = cn > 0
    np.add.at(f, cn[m] - 1, vals[m])
    cne = None
    if mesh.eloads and mesh.eloads[lc]:
        cne = element_code_numbers(mesh)
        for eid, flags, values in mesh.eloads[lc]:
            nf = element_load_forces(mesh, int(eid), flags, values)
            for j, c in enumerate(cne[int(eid)]):
                if c > 0:
                    f[c - 1] += nf[j]
    if mesh.pd is not None and mesh.pd.shape[1] > 0:
        cne = element_code_numbers(mesh) if cne is None else cne
        pd = _f64(mesh.pd[lc])
        for e in np.nonzero((cne < 0).any(axis=1))[0]:
            ke = element_stiffness(mesh, int(e))
            lib().or_prescribed_contrib(cne.shape[1], ke, _i64(cne[e]), pd, f)
    return f


# ----------------------------------------------------------------------------
# products and solvers
# ----------------------------------------------------------------------------

def scr_mxv(adr, ci, a, b):
    n = adr.size - 1
    c = np.zeros(n)
    lib().or_scr_mxv(n, _i64(adr), _i64(ci), _f64(a), _f64(b), c)
    return c


def cr_mxv(adr, ci, a, b):
    n = adr.size - 1
    c = np.zeros(n)
    lib().or_cr_mxv(n, _i64(adr), _i64(ci), _f64(a), _f64(b), c)
    return c


def scr_cg_prec(adr, ci, a, f, ni=100000, res=1e-20, zero=1e-30, x0=None):
    n = adr.size - 1
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    ani, ares = _L(-1), _D(float("nan"))
    st = lib().or_scr_cg_prec(n, _i64(adr), _i64(ci), _f64(a), x, _f64(f), ni, res, zero,
                              0 if x0 is None else 1, C.byref(ani), C.byref(ares))
    return x, st, ani.value, ares.value


def cr_cg_prec(adr, ci, a, f, ni=100000, res=1e-10, zero=1e-30, x0=None):
    n = adr.size - 1
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    ani, ares = _L(-1), _D(float("nan"))
    st = lib().or_cr_cg_prec(n, _i64(adr), _i64(ci), _f64(a), x, _f64(f), ni, res, zero,
                             0 if x0 is None else 1, C.byref(ani), C.byref(ares))
    return x, st, ani.value, ares.value


def trfel_lift(mesh, rnode):
    """-K r lifting of assemble_init over all elements, in equation order."""
    cne = element_code_numbers(mesh)
    rhs = np.zeros(mesh.ndof)
    lib().or_trfel_lift(mesh.ne, _f64(mesh.coords), _i64(mesh.elems), cne, _f64(mesh.mats[mesh.emat]),
                        _f64(rnode), rhs)
    return rhs


def trfel_steps(mesh, nsteps, dt, alpha=1.0, ni=100000, res=1e-20, zero=1e-30, iv=1, rnode=None, form="d",
                rho=None):
    """nsteps of linear_nonstat_solv_dform (TRFEL/SRC/npsolvert.cpp:1146-1230,
    form "d") or of the v-form's one_step_linear (npsolvert.cpp:367-480,
    form "v") with K and C assembled once (their values do not change for
    linear materials) and the lifting of time-constant prescribed values."""
    adr, ci, ka = assemble(mesh, sym=True, kind="hex8t_k")
    _, _, ca = assemble(mesh, sym=True, kind="hex8t_c", rho=rho)
    n = adr.size - 1
    if rnode is None:
        rnode = mesh.meta["prescribed"][:, 0]
    rhs = trfel_lift(mesh, rnode)
    d = np.zeros(n)
    v = np.zeros(n)
    work = np.zeros(ka.size)
    its = []
    for _ in range(nsteps):
        ani, ares = _L(-1), _D(0.0)
        step = lib().or_trfel_step if form == "d" else lib().or_trfel_step_v
        st = step(n, adr, ci, ka, ca, work, rhs, d, v, dt, alpha, ni, res, zero, iv,
                                 C.byref(ani), C.byref(ares))
        its.append((st, ani.value))
    return d, v, its


def trfel_stationary(mesh, ni=100000, res=1e-20, zero=1e-30, rnode=None):
    """solve_stationary_problem (TRFEL/SRC/spsolvert.cpp:13): K assembled,
    right-hand side = the lifting of assemble_init, Jacobi-PCG."""
    adr, ci, ka = assemble(mesh, sym=True, kind="hex8t_k")
    if rnode is None:
        rnode = mesh.meta["prescribed"][:, 0]
    rhs = trfel_lift(mesh, rnode)
    return scr_cg_prec(adr, ci, ka, rhs, ni=ni, res=res, zero=zero)


def scr_to_dense(adr, ci, a):
    n = adr.size - 1
    K = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(adr))
    K[rows, ci] = a
    K[ci, rows] = a
    return K


def cr_to_dense(adr, ci, a):
    n = adr.size - 1
    K = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(adr))
    K[rows, ci] = a
    return K


# ----------------------------------------------------------------------------
# the compiled reference (oracle/_ref), when built
# ----------------------------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(REF_LIB) and os.path.exists(os.path.join(REF_DIR, "mefel_dump"))


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(REF_LIB)
        R.ref_scr_mxv.argtypes = [_L, _pL, _pL, _pD, _pD, _pD]
        R.ref_cr_mxv.argtypes = [_L, _pL, _pL, _pD, _pD, _pD]
        R.ref_scr_cg_prec.argtypes = [_L, _pL, _pL, _pD, _pD, _pD, _L, _D, _D, _L, _L,
                                      C.POINTER(_L), C.POINTER(_D), C.c_int]
        R.ref_cr_cg_prec.argtypes = [_L, _pL, _pL, _pD, _pD, _pD, _L, _D, _D, _L, C.c_int,
                                     C.POINTER(_L), C.POINTER(_D), C.c_int]
        _ref = R
    return _ref


def ref_scr_cg_prec(adr, ci, a, f, ni=100000, res=1e-20, zero=1e-30, x0=None, quiet=True):
    n = adr.size - 1
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    ani, ares = _L(-1), _D(float("nan"))
    ref().ref_scr_cg_prec(n, _i64(adr), _i64(ci), _f64(a).copy(), x, _f64(f).copy(), ni, res, zero,
                          0 if x0 is None else 1, 1, C.byref(ani), C.byref(ares), int(quiet))
    return x, ani.value, ares.value


def ref_cr_cg_prec(adr, ci, a, f, ni=100000, res=1e-10, zero=1e-30, x0=None, quiet=True):
    n = adr.size - 1
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    ani, ares = _L(-1), _D(float("nan"))
    ref().ref_cr_cg_prec(n, _i64(adr), _i64(ci), _f64(a).copy(), x, _f64(f).copy(), ni, res, zero,
                         0 if x0 is None else 1, 0, C.byref(ani), C.byref(ares), int(quiet))
    return x, ani.value, ares.value


def run_mefel_dump(deck_path: str, outdir: str, solve: bool = True) -> dict:
    """Run the reference pipeline on a deck; return its dumped arrays."""
    os.makedirs(outdir, exist_ok=True)
    exe = os.path.join(REF_DIR, "mefel_dump")
    args = [exe, os.path.abspath(deck_path), "."] + ([] if solve else ["nosolve"])
    with open(os.path.join(outdir, "run.log"), "w") as log:
        subprocess.run(args, cwd=outdir, stdout=log, stderr=subprocess.STDOUT, check=True)
    return read_dump(outdir)


def run_trfel_dump(deck_path: str, outdir: str, solve: bool = True) -> dict:
    """Run the reference TRFEL pipeline on a deck; return its dumped arrays."""
    os.makedirs(outdir, exist_ok=True)
    exe = os.path.join(REF_DIR, "trfel_dump")
    args = [exe, os.path.abspath(deck_path), "."] + ([] if solve else ["nosolve"])
    with open(os.path.join(outdir, "run.log"), "w") as log:
        subprocess.run(args, cwd=outdir, stdout=log, stderr=subprocess.STDOUT, check=True)
    return read_dump(outdir)


def read_dump(outdir: str) -> dict:
    meta = {}
    with open(os.path.join(outdir, "meta.txt")) as fh:
        for line in fh:
            k, v = line.split()
            meta[k] = float(v) if ("." in v or "e" in v) else int(v)
    out = {"meta": meta}
    for name, dt in (("K_adr", np.int64), ("K_ci", np.int64), ("K_a", np.float64),
                     ("C_adr", np.int64), ("C_ci", np.int64), ("C_a", np.float64),
                     ("f", np.float64), ("u", np.float64), ("T", np.float64), ("V", np.float64)):
        ext = "i64" if dt == np.int64 else "f64"
        p = os.path.join(outdir, f"{name}.{ext}")
        if os.path.exists(p):
            out[name] = np.fromfile(p, dtype=dt)
    return out
