"""Host-side mirror of the MEFEL / TRFEL assembly entry points on the GPU.

* ``stiffness_matrix(mesh)`` -- MEFEL/SRC/globmat.cpp:41: element loop +
  localisation, here one call of ``sgpu_assemble`` (pattern, colouring,
  batched integration and scatter on the device);
* ``conductivity_matrix`` / ``capacity_matrix`` -- TRFEL/SRC/globmatt.cpp:19/92;
* ``mefel_right_hand_side(mesh, lc)`` -- globmat.cpp:2369 for nodal loads
  (loadcase::assemble, MEFEL/SRC/loadcase.cpp:400);
* ``solve_linear_statics(mesh, ...)`` -- MEFEL/SRC/lssolver.cpp:31-80:
  assemble once, solve every load case.

Meshes are :class:`ssf_b200.decks.Mesh` objects (nodes, elements, constraint
flags, materials and loads as a SIFEL deck describes them).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .gefel import DeviceMatrix, Result

KIND = {"hex8": L.ELEM_HEX8, "quad4": L.ELEM_QUAD4, "hex8t_k": L.ELEM_HEX8T_K, "hex8t_c": L.ELEM_HEX8T_C,
        "tet4": L.ELEM_TET4, "tri3": L.ELEM_TRI3, "hex20": L.ELEM_HEX20, "quad8": L.ELEM_QUAD8}


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def strain_transformation(T) -> np.ndarray:
    """6 x 6 transformation of strain vectors [xx, yy, zz, yz, xz, xy]
    (engineering shears) built from the 3 x 3 axes T (x_global = T x_local),
    as lg_tens4transf (MEFEL/SRC/vecttens.cpp:1561-1615) lays it out."""
    t = np.zeros((6, 6))
    for c in range(3):
        t[c] = [T[0, c] ** 2, T[1, c] ** 2, T[2, c] ** 2, T[1, c] * T[2, c], T[0, c] * T[2, c], T[0, c] * T[1, c]]
    for r, (a, b) in enumerate(((2, 1), (2, 0), (1, 0))):
        t[3 + r] = [2.0 * T[0, a] * T[0, b], 2.0 * T[1, a] * T[1, b], 2.0 * T[2, a] * T[2, b],
                    T[1, a] * T[2, b] + T[2, a] * T[1, b], T[0, a] * T[2, b] + T[2, a] * T[0, b],
                    T[0, a] * T[1, b] + T[1, a] * T[0, b]]
    return t


def material_matrices(mesh) -> np.ndarray:
    """Global 6 x 6 material stiffness per material instance, (nmat, 36), of a
    mesh with general materials: "gen3d" rows are the 21 upper-triangle
    entries (elastgmat3d::matstiff, MEFEL/SRC/elastgmat3d.cpp:69); "ortho"
    rows are the local stiffness (36) and the constant axes T (9), turned
    into the global system as t^T D t (elastortomat::matstiff,
    MEFEL/SRC/elastortomat.cpp:100-115)."""
    mats = np.asarray(mesh.mats, dtype=np.float64)
    out = np.zeros((mats.shape[0], 36))
    for k, row in enumerate(mats):
        if mesh.mtype == "gen3d":
            D = np.zeros((6, 6))
            D[np.triu_indices(6)] = row[:21]
            out[k] = (np.triu(D) + np.triu(D, 1).T).ravel()
        elif mesh.mtype == "ortho":
            t = strain_transformation(row[36:45].reshape(3, 3))
            out[k] = (t.T @ row[:36].reshape(6, 6) @ t).ravel()
        else:
            raise ValueError(f"material type {mesh.mtype!r} has no general matrix")
    return out


def _assemble(mesh, kind: str, rho=None):
    coords = _c(mesh.coords, np.float64)
    elems = _c(mesh.elems, np.int64)
    cn = _c(mesh.code_numbers(), np.int64)
    general = getattr(mesh, "mtype", "iso") != "iso"
    emat = None if general else _c(mesh.mats[mesh.emat], np.float64)
    dmat = _c(material_matrices(mesh)[mesh.emat], np.float64) if general else None
    thick = _c(mesh.thick, np.float64) if mesh.thick is not None else None
    rr = _c(rho, np.float64) if rho is not None else None
    keep = (coords, elems, cn, emat, dmat, thick, rr)
    m = L.Mesh(KIND[kind], cn.shape[1], coords.shape[0], coords.ctypes.data, elems.shape[0], elems.ctypes.data,
               cn.ctypes.data, emat.ctypes.data if emat is not None else None,
               thick.ctypes.data if thick is not None else None,
               rr.ctypes.data if rr is not None else None, dmat.ctypes.data if dmat is not None else None)
    h = C.c_void_p()
    info = L.AssemblyInfo()
    L.check(L.lib().sgpu_assemble(C.byref(m), C.byref(h), C.byref(info)))
    del keep
    dm = DeviceMatrix.from_handle(h, info.n, 1)
    dm.assembly = info.as_dict()
    return dm


def stiffness_matrix(mesh) -> DeviceMatrix:
    """Global stiffness matrix of a hex8 / tet4 / hex20 / quad4 / tri3 / quad8
    mesh, assembled on the GPU."""
    return _assemble(mesh, mesh.kind)


def conductivity_matrix(mesh) -> DeviceMatrix:
    return _assemble(mesh, "hex8t_k")


def capacity_matrix(mesh, rho=None) -> DeviceMatrix:
    return _assemble(mesh, "hex8t_c", rho)


def assemble_copy(K: DeviceMatrix, kind: str, emat=None, rho=None) -> DeviceMatrix:
    """Another matrix of K's mesh on K's pattern (``sgpu_assemble_copy``):
    e.g. the capacity matrix of a conduction handle, without a second
    pattern build and colouring."""
    em = None if emat is None else _c(emat, np.float64)
    rr = None if rho is None else _c(rho, np.float64)
    h = C.c_void_p()
    info = L.AssemblyInfo()
    L.check(L.lib().sgpu_assemble_copy(K.h, KIND[kind], em.ctypes.data if em is not None else None,
                                       rr.ctypes.data if rr is not None else None, C.byref(h), C.byref(info)))
    dm = DeviceMatrix.from_handle(h, info.n, 1)
    dm.assembly = info.as_dict()
    return dm


def rigid_body_modes(mesh) -> np.ndarray:
    """Near-null space of the mesh's operator in equation order (n x k): the
    6 rigid-body motions of a 3D elastic body, the 3 of a plane one, or the
    constant of a conduction problem -- the vectors GEFEL's BOSS aggregator
    builds per aggregate (aggregator::gener_rbm_1/2, GEFEL/aggregator.cpp:638-700),
    here for the whole mesh at once (each aggregate's QR restricts them).
    Coordinates are centred so the rotations are well scaled."""
    cn = mesh.code_numbers()
    n = int(cn.max())
    ndofn = cn.shape[1]
    xyz = np.asarray(mesh.coords, dtype=np.float64)
    xyz = xyz - xyz.mean(axis=0)
    if ndofn == 1:
        B = np.zeros((n, 1))
        c = cn[:, 0]
        B[c[c > 0] - 1, 0] = 1.0
        return B
    if ndofn == 2:
        B = np.zeros((n, 3))
        x, y = xyz[:, 0], xyz[:, 1]
        rows = [(1.0, 0.0, -y), (0.0, 1.0, x)]
    else:
        B = np.zeros((n, 6))
        x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
        o = np.zeros_like(x)
        # translations, then rotations about z, x, y
        rows = [(1.0, 0.0, 0.0, -y, o, z), (0.0, 1.0, 0.0, x, -z, o), (0.0, 0.0, 1.0, o, y, -x)]
    for comp in range(ndofn):
        c = cn[:, comp]
        keep = c > 0
        for q, v in enumerate(rows[comp]):
            B[c[keep] - 1, q] = v[keep] if np.ndim(v) else v
    return B


def _element_loads_into(mesh, lc: int, f: np.ndarray) -> None:
    """Adds load case lc's element loads (hex8 surfaces, quad4 edges) into f
    through the library (sgpu_mesh_element_loads)."""
    recs = mesh.eloads[lc] if mesh.eloads else []
    if not recs:
        return
    nfl = 6 if mesh.kind == "hex8" else 4
    eid = _c([r[0] for r in recs], np.int64)
    flags = _c(np.concatenate([np.asarray(r[1]).reshape(nfl) for r in recs]), np.int32)
    vals = _c(np.concatenate([np.asarray(r[2], dtype=np.float64).reshape(-1) for r in recs]), np.float64)
    coords = _c(mesh.coords, np.float64)
    elems = _c(mesh.elems, np.int64)
    cn = _c(mesh.code_numbers(), np.int64)
    m = L.Mesh(KIND[mesh.kind], cn.shape[1], coords.shape[0], coords.ctypes.data, elems.shape[0],
               elems.ctypes.data, cn.ctypes.data, None, None, None, None)
    L.check(L.lib().sgpu_mesh_element_loads(C.byref(m), eid.size, eid.ctypes.data, flags.ctypes.data,
                                            vals.ctypes.data, f))


def prescribed_displacements(mesh, lc: int = 0) -> np.ndarray | None:
    """Nodal prescribed displacements of load case lc (nn x ndofn: the value
    at a DOF flagged -k, 0 elsewhere), or None when the mesh has none."""
    neg = mesh.dofflag < 0
    if not neg.any():
        return None
    r = np.zeros(mesh.dofflag.shape)
    r[neg] = mesh.pd[lc][-mesh.dofflag[neg] - 1]
    return r


def mefel_right_hand_side(mesh, lc: int = 0, K: DeviceMatrix | None = None) -> np.ndarray:
    """Right-hand side of load case ``lc`` in equation order, as
    loadcase::assemble (MEFEL/SRC/loadcase.cpp:400) forms it: nodal forces,
    the element loads' nodal forces (loadcase::forcecontrib, :546), and for
    prescribed displacements -K_e r_e over the elements that have them
    (prdisplcontrib, :615) -- formed on the GPU from the assembled handle K,
    which a mesh with prescribed displacements must pass."""
    cn = mesh.code_numbers().reshape(-1)
    f = np.zeros(mesh.ndof)
    vals = mesh.loads[lc].reshape(-1)
    m = cn > 0
    np.add.at(f, cn[m] - 1, vals[m])
    _element_loads_into(mesh, lc, f)
    r = prescribed_displacements(mesh, lc)
    if r is not None:
        if K is None:
            raise ValueError("prescribed displacements need the assembled stiffness matrix (argument K)")
        L.check(L.lib().sgpu_assembly_lift(K.h, _c(r, np.float64), f))
    return f


def solve_linear_statics(mesh, ni=100000, res=1e-20, mode="fp64", batched=None):
    """Assemble K once, then solve every load case (lssolver.cpp:78-80).
    With several load cases (and FP64) they are solved together by the
    batched PCG unless batched=False."""
    from .gefel import pcg_multi
    K = stiffness_matrix(mesh)
    nlc = mesh.loads.shape[0]
    if batched is None:
        batched = nlc > 1 and mode == "fp64"
    out, results = [], []
    try:
        if batched:
            F = np.stack([mefel_right_hand_side(mesh, lc, K) for lc in range(nlc)], axis=1)
            X, results = pcg_multi(K, F, ni=ni, res=res)
            return X.T.copy(), results
        for lc in range(nlc):
            f = mefel_right_hand_side(mesh, lc, K)
            x, r = K.pcg(f, ni=ni, res=res, crit="scr", prec=1, mode=mode)
            out.append(x)
            results.append(r)
    finally:
        K.close()
    return np.stack(out), results


class Deck:
    """A MEFEL linear-statics deck read by the library's parallel reader
    (``sgpu_deck_read_mefel``: the reading part of mefel_init,
    MEFEL/SRC/mefelinit.cpp:47, and gtopology::gencodnum)."""

    def __init__(self, path: str, threads: int = 0, front: str = "mefel"):
        self.h = C.c_void_p()
        read = {"mefel": L.lib().sgpu_deck_read_mefel, "trfel": L.lib().sgpu_deck_read_trfel}[front]
        L.check(read(str(path).encode(), int(threads), C.byref(self.h)))
        v = L.DeckView()
        L.check(L.lib().sgpu_deck_get(self.h, C.byref(v)))
        self.view = v
        self.front = front
        self.info = {k: getattr(v, k) for k in ("kind", "ndofn", "nne", "mtype", "nn", "ne", "n", "nmat", "nlc",
                                                "storage", "precond", "iv", "ni", "res", "parse_ms", "problem",
                                                "tform", "alpha", "t0", "t1", "dt")}

    def _arr(self, ptr, shape, dt):
        n = int(np.prod(shape))
        ctype = C.c_double if dt == np.float64 else C.c_int64
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,)).reshape(shape).copy()

    def mesh(self):
        """The deck as a :class:`ssf_b200.decks.Mesh` (copies)."""
        from .decks import Mesh
        v = self.view
        if self.front == "trfel":
            rnode = self._arr(v.rnode, (v.nn,), np.float64)
            dofflag = self._arr(v.dofflag, (v.nn, 1), np.int64)
            presc = np.where(dofflag[:, 0] == 1, 0.0, rnode)[:, None]
            return Mesh(kind="hex8t", coords=self._arr(v.coords, (v.nn, 3), np.float64),
                        elems=self._arr(v.elems, (v.ne, 8), np.int64), dofflag=dofflag,
                        emat=self._arr(v.emat_id, (v.ne,), np.int64),
                        mats=self._arr(v.mats, (v.nmat, 2), np.float64), loads=np.zeros((1, v.nn, 1)),
                        meta=dict(prescribed=presc, rnode=rnode, rho=self._arr(v.rho, (v.ne,), np.float64)))
        kinds = {L.ELEM_HEX8: "hex8", L.ELEM_QUAD4: "quad4", L.ELEM_TET4: "tet4", L.ELEM_TRI3: "tri3",
                 L.ELEM_HEX20: "hex20", L.ELEM_QUAD8: "quad8"}
        return Mesh(kind=kinds[v.kind], coords=self._arr(v.coords, (v.nn, 3), np.float64),
                    elems=self._arr(v.elems, (v.ne, v.nne), np.int64),
                    dofflag=self._arr(v.dofflag, (v.nn, v.ndofn), np.int64),
                    emat=self._arr(v.emat_id, (v.ne,), np.int64),
                    mats=self._arr(v.mats, (v.nmat, v.nmatp), np.float64),
                    loads=self._arr(v.loads, (v.nlc, v.nn, v.ndofn), np.float64),
                    thick=self._arr(v.thick, (v.ne,), np.float64) if v.thick else None,
                    mtype={1: "iso", 2: "gen3d", 3: "ortho"}[v.mtype])

    def stiffness_matrix(self, kind=None) -> DeviceMatrix:
        """sgpu_assemble straight from the deck's arrays (TRFEL decks: the
        conductivity matrix, or the capacity matrix for kind "hex8t_c")."""
        m = L.Mesh()
        L.check(L.lib().sgpu_deck_mesh(self.h, C.byref(m)))
        if kind is not None:
            m.kind = KIND[kind]
        h = C.c_void_p()
        info = L.AssemblyInfo()
        L.check(L.lib().sgpu_assemble(C.byref(m), C.byref(h), C.byref(info)))
        dm = DeviceMatrix.from_handle(h, info.n, 1)
        dm.assembly = info.as_dict()
        return dm

    def rhs(self, lc: int = 0, K: DeviceMatrix | None = None) -> np.ndarray:
        """Load case lc's right-hand side: nodal and element loads
        (sgpu_deck_rhs), then the prescribed displacements' -K_e r_e on the
        GPU when the deck has any (K: the deck's assembled matrix)."""
        f = np.zeros(self.view.n)
        L.check(L.lib().sgpu_deck_rhs(self.h, int(lc), f))
        if self.front == "mefel":
            r = np.zeros(self.view.nn * self.view.ndofn)
            cnt = C.c_int64(0)
            L.check(L.lib().sgpu_deck_prescribed(self.h, int(lc), r, C.byref(cnt)))
            if cnt.value:
                if K is None:
                    raise ValueError("the deck prescribes displacements: pass its stiffness matrix K")
                L.check(L.lib().sgpu_assembly_lift(K.h, r, f))
        return f

    def close(self):
        if self.h:
            L.lib().sgpu_deck_free(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_deck(path: str, prec=None, mode="fp64", threads: int = 0, nullspace: bool = True):
    """What SIFEL's ``mefel deck.in`` does for linear statics, on the GPU:
    read the deck, assemble K, solve every load case with the deck's solver
    line (ni, res, diagonal or no preconditioner, the storage's criterion).
    ``prec`` "agg" swaps in the aggregation preconditioner (with the rigid-body
    modes when ``nullspace``).  Returns (X (nlc x n), results, info)."""
    import time
    t0 = time.perf_counter()
    with Deck(path, threads) as d:
        info = dict(d.info)
        K = d.stiffness_matrix()
        try:
            info["assembly"] = K.assembly
            crit = "scr" if d.info["storage"] == 11 else "cr"
            p = prec if prec is not None else d.info["precond"]
            if p == "agg" and nullspace:
                v = d.view
                L.check(L.lib().sgpu_matrix_set_rigid_body_modes(K.h, v.nn, v.ndofn, v.coords, v.cn))
            out, results = [], []
            for lc in range(d.info["nlc"]):
                x, r = K.pcg(d.rhs(lc, K), ni=d.info["ni"], res=d.info["res"], crit=crit, prec=p, mode=mode)
                out.append(x)
                results.append(r)
        finally:
            K.close()
    info["wall_s"] = time.perf_counter() - t0
    return np.stack(out), results, info


def solve_trfel_deck(path: str, prec="jacobi", mode="fp64", threads: int = 0, zero: float = 1e-30):
    """What SIFEL's ``trfel deck.in`` does for linear heat conduction, on the
    GPU: read the deck, assemble K (and C), lift the prescribed values, then
    the stationary solve (solve_stationary_problem, TRFEL/SRC/spsolvert.cpp:13)
    or every time step of the d- or v-form trapezoid the deck names
    (npsolvert.cpp:1071 / :62).  Returns (d, v, per-step iterations, info)."""
    import time
    t0 = time.perf_counter()
    with Deck(path, threads, front="trfel") as dk:
        info = dict(dk.info)
        v = dk.view
        K = dk.stiffness_matrix()
        Cm = None
        try:
            rnode = np.ctypeslib.as_array(C.cast(v.rnode, C.POINTER(C.c_double)), shape=(v.nn,))
            rhs = np.zeros(K.n)
            L.check(L.lib().sgpu_assembly_lift(K.h, np.ascontiguousarray(rnode), rhs))
            info["assembly"] = K.assembly
            if v.problem == 50:
                x, r = K.pcg(rhs, ni=v.ni, res=v.res, zero=zero, crit="scr" if v.storage == 11 else "cr",
                             prec=prec, mode=mode)
                info["wall_s"] = time.perf_counter() - t0
                return x, None, np.array([r.info["iterations"]]), dict(info, solve=r.info)
            Cm = assemble_copy(K, "hex8t_c")
            cn = np.ctypeslib.as_array(C.cast(v.cn, C.POINTER(C.c_int64)), shape=(v.nn,))
            free = cn > 0
            d = np.zeros(K.n)
            d[cn[free] - 1] = rnode[free]  # initial values (lhsrhst::initcond)
            vel = np.zeros(K.n)
            nsteps = int(round((v.t1 - v.t0) / v.dt))
            its = np.zeros(max(nsteps, 1), dtype=np.int64)
            sinfo = L.SolveInfo()
            fn = L.lib().sgpu_transient_dform if v.tform == 1 else L.lib().sgpu_transient_vform
            st = fn(K.h, Cm.h, rhs, d, vel, float(v.dt), float(v.alpha), nsteps, int(v.ni), float(v.res),
                    float(zero), int(v.iv), {"jacobi": L.PREC_JACOBI, "agg": L.PREC_AGG}[prec],
                    {"fp64": L.FP64, "mixed": L.MIXED}[mode], its.ctypes.data, C.byref(sinfo))
            L.check(st, (L.OK, L.NOT_CONVERGED, L.BREAKDOWN))
            info["nsteps"] = nsteps
            info["wall_s"] = time.perf_counter() - t0
            return d, vel, its[:nsteps], dict(info, solve=sinfo.as_dict())
        finally:
            K.close()
            if Cm is not None:
                Cm.close()


def trfel_lift(K: DeviceMatrix, rnode) -> np.ndarray:
    """Right-hand side of TRFEL's assemble_init for time-constant prescribed
    values: -sum_e K_e r_e at the free DOFs (TRFEL/SRC/globmatt.cpp:1635)."""
    rhs = np.zeros(K.n)
    L.check(L.lib().sgpu_assembly_lift(K.h, _c(rnode, np.float64), rhs))
    return rhs


def linear_nonstat_solv_dform(mesh, nsteps, dt, alpha=1.0, ni=100000, res=1e-20, zero=1e-30, iv=1,
                              mode="fp64", rnode=None, d0=None, v0=None, prec="jacobi", form="d"):
    """The d-form generalized trapezoid (TRFEL/SRC/npsolvert.cpp:1071) on the
    GPU: K and C assembled once, `nsteps` steps with everything on the device;
    ``prec`` "jacobi" (the reference's) or "agg" (aggregation multilevel, its
    hierarchy built once for all steps); ``form`` "v" runs the v-form of
    nonstat_solv_vform_comp (npsolvert.cpp:62, trapezoidv) instead.  Returns (d, v, per-step iterations,
    solve info)."""
    K = conductivity_matrix(mesh)
    Cm = assemble_copy(K, "hex8t_c")
    try:
        if rnode is None:
            rnode = mesh.meta["prescribed"][:, 0]
        rhs = trfel_lift(K, rnode)
        d = np.zeros(K.n) if d0 is None else _c(d0, np.float64).copy()
        v = np.zeros(K.n) if v0 is None else _c(v0, np.float64).copy()
        its = np.zeros(max(nsteps, 1), dtype=np.int64)
        info = L.SolveInfo()
        m = {"fp64": L.FP64, "mixed": L.MIXED}[mode]
        p = {"jacobi": L.PREC_JACOBI, "agg": L.PREC_AGG}[prec]
        fn = L.lib().sgpu_transient_dform if form == "d" else L.lib().sgpu_transient_vform
        st = fn(K.h, Cm.h, rhs, d, v, float(dt), float(alpha), int(nsteps), int(ni), float(res), float(zero),
                int(iv), p, m, its.ctypes.data, C.byref(info))
        L.check(st, (L.OK, L.NOT_CONVERGED, L.BREAKDOWN))
        return d, v, its[:nsteps], info.as_dict()
    finally:
        K.close()
        Cm.close()


def nonstat_solv_vform_comp(mesh, nsteps, dt, alpha=1.0, **kw):
    """The v-form generalized trapezoid (TRFEL/SRC/npsolvert.cpp:62,
    one_step_linear at 367-480) on the GPU."""
    return linear_nonstat_solv_dform(mesh, nsteps, dt, alpha=alpha, form="v", **kw)


def solve_batch(meshes, ni=200000, res=1e-20, zero=1e-30, tune=True, prec="jacobi", mode="fp64"):
    """Many independent meshes (e.g. the uneven plate batch) assembled in one
    call and solved together: prec "jacobi" is the batched Jacobi-PCG (FP64,
    segment work units), "agg" the batched flexible CGs with the aggregation
    cycle of the whole block-diagonal matrix (FP32 cycle for mode "mixed").
    Returns the list of solutions, per-system (status, ani, ares, iterations)
    and info."""
    from .decks import merge_meshes
    merged, rows = merge_meshes(meshes)
    K = stiffness_matrix(merged)
    try:
        f = mefel_right_hand_side(merged)
        x = np.zeros(K.n)
        nsys = rows.size
        ani = np.full(nsys, -1, dtype=np.int64)
        ares = np.full(nsys, np.nan)
        st = np.zeros(nsys, dtype=np.int32)
        its = np.zeros(nsys, dtype=np.int64)
        info = L.SolveInfo()
        if prec == "agg":
            K.set_rigid_body_modes(merged.coords, merged.code_numbers())
            rc = L.lib().sgpu_matrix_pcg_batch_agg(K.h, nsys, rows, x, f, int(ni), float(res), float(zero),
                                                   {"fp64": L.FP64, "mixed": L.MIXED}[mode], ani.ctypes.data,
                                                   ares.ctypes.data, st.ctypes.data, its.ctypes.data, C.byref(info))
        else:
            rc = L.lib().sgpu_matrix_pcg_batch(K.h, nsys, rows, x, f, int(ni), float(res), float(zero), int(tune),
                                               ani.ctypes.data, ares.ctypes.data, st.ctypes.data, its.ctypes.data,
                                               C.byref(info))
        L.check(rc, (L.OK, L.NOT_CONVERGED, L.BREAKDOWN, L.ZERO_RHS))
        offs = np.concatenate([[0], np.cumsum(rows)])
        xs = [x[offs[k]:offs[k + 1]] for k in range(nsys)]
        out = dict(status=st, ani=ani, ares=ares, iterations=its, info=info.as_dict(), assembly=K.assembly)
        return xs, out
    finally:
        K.close()


def solve_stationary_problem(mesh, ni=100000, res=1e-20, zero=1e-30, mode="fp64", rnode=None):
    """solve_stationary_problem (TRFEL/SRC/spsolvert.cpp:13) on the GPU:
    conductivity matrix assembled on the device, the lifting of the
    prescribed values as right-hand side, Jacobi-PCG."""
    K = conductivity_matrix(mesh)
    try:
        if rnode is None:
            rnode = mesh.meta["prescribed"][:, 0]
        rhs = trfel_lift(K, rnode)
        return K.pcg(rhs, ni=ni, res=res, zero=zero, crit="scr", prec=1, mode=mode)
    finally:
        K.close()
