"""Synthetic SIFEL problems: structured meshes, loads and positional decks.

The benchmark problems of this project are generated, never downloaded:

* ``cantilever_hex``   -- 3D linear-elastic cantilever of 8-node hexahedra,
  clamped at x = 0, uniform traction on the x = L face as consistent nodal
  forces (each face quad gives a quarter of its force to each corner);
* ``cantilever_top_loads`` -- independent N(0,1) x 1 kN z-forces on every
  free node of the top face, one column per load case;
* ``plate_quad``       -- 2D plane-stress plate of 4-node quads, left edge
  clamped, unit traction x thickness on the right edge;
* ``heat_cube``        -- unit cube of linear hexahedra for transient
  conduction with one conductivity per element;
* ``cantilever_tet``   -- the cantilever of ``cantilever_hex`` meshed with
  linear tetrahedra (six per grid cell);
* ``plate_tri``        -- the plate of ``plate_quad`` meshed with
  constant-strain triangles (two per quad);
* ``cantilever_hex20`` / ``plate_quad8`` -- the same problems with the
  quadratic serendipity elements.

``write_mefel_deck`` writes a deck in SIFEL's positional (``-kwd`` absent)
MEFEL input format, token order as read by ``probdesc::read``
(MEFEL/SRC/probdesc.cpp:204-452), ``mechtop::read`` (mechtop.cpp:124-262),
``element::read`` (element.cpp:90-350), ``mechmat::read`` (mechmat.cpp:1042),
``mechcrsec::read`` (mechcrsec.cpp:74), ``mechbclc::read`` / ``loadcase::read``
(mechbclc.cpp:99, loadcase.cpp:114) and ``outdriverm::read``
(outdriverm.cpp:96).  ``write_trfel_deck`` does the same for TRFEL.

Node order of a hexahedron follows SIFEL (GEFEL/basefun.cpp:2299):
n0 (+,+,+), n1 (-,+,+), n2 (-,-,+), n3 (+,-,+), n4..n7 likewise at zeta = -1.
Quadrilaterals: n0 (+,+), n1 (-,+), n2 (-,-), n3 (+,-) (basefun.cpp:609).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Mesh:
    """A mesh with nodal DOF flags, per-element materials and nodal loads.

    coords   (nn, 3) float64 node coordinates (z = 0 for 2D meshes)
    elems    (ne, nne) int64 0-based node ids in SIFEL element node order
    dofflag  (nn, ndofn) int64 constraint codes as in the deck: 1 free, 0 fixed
    emat     (ne,) int64 0-based material instance per element
    mats     (nmat, k) float64 material parameters: (E, nu) or (k, c) for
             mtype "iso"; the 21 upper-triangle entries d11..d16, d22..d66 of
             the 6 x 6 stiffness for "gen3d" (elastgmat3d); the 36 entries
             of the local stiffness then the 9 of the transformation T
             (x_global = T x_local), both row-major, for "ortho" (elastortomat)
    thick    (ne,) float64 element thickness (plane stress) or None
    loads    (nlc, nn, ndofn) float64 nodal forces per load case
    eloads   None, or per load case a list of element loads (eid, flags,
             values): a surface load of a hex8 (6 face flags, 1 = loaded in
             the global system, and 6 x 4 nodes x 3 values) or an edge load
             of a quad4 (4 edge flags, 4 x 2 nodes x 2 values), in the layout
             loadel::readsurfaceload / readedgeload read
             (MEFEL/SRC/loadel.cpp:204-279)
    pd       None, or (nlc, npd) float64 prescribed displacements: a DOF flag
             -k in dofflag takes pd[lc, k-1] (elprdispl, MEFEL/SRC/globmat.cpp:1372)
    """

    kind: str
    coords: np.ndarray
    elems: np.ndarray
    dofflag: np.ndarray
    emat: np.ndarray
    mats: np.ndarray
    loads: np.ndarray
    thick: np.ndarray | None = None
    meta: dict = field(default_factory=dict)
    mtype: str = "iso"
    eloads: list | None = None
    pd: np.ndarray | None = None

    @property
    def nn(self) -> int:
        return int(self.coords.shape[0])

    @property
    def ne(self) -> int:
        return int(self.elems.shape[0])

    @property
    def ndofn(self) -> int:
        return int(self.dofflag.shape[1])

    def code_numbers(self) -> np.ndarray:
        """DOF numbering of ``gtopology::gencodnum`` (GEFEL/gtopology.cpp:1619).

        Nodes in order, DOFs of a node in order; every free DOF (flag 1) gets
        the next 1-based number, fixed DOFs get 0 and DOFs with a prescribed
        displacement keep their negative flag (-k: the k-th prescribed value).
        """
        flat = self.dofflag.reshape(-1)
        cn = np.zeros_like(flat)
        free = flat == 1
        cn[free] = np.arange(1, int(free.sum()) + 1)
        neg = flat < 0
        cn[neg] = flat[neg]
        return cn.reshape(self.dofflag.shape)

    @property
    def ndof(self) -> int:
        return int((self.dofflag == 1).sum())


MATTYPE = {"iso": 1, "gen3d": 2, "ortho": 3}


def orthotropic_local(E1, E2, E3, nu12, nu13, nu23, G23, G13, G12) -> np.ndarray:
    """6 x 6 stiffness of an orthotropic material in its own axes, strain
    order [xx, yy, zz, yz, xz, xy] with engineering shears: the inverse of the
    compliance (nu_ij E_j = nu_ji E_i)."""
    S = np.zeros((6, 6))
    S[0, 0], S[1, 1], S[2, 2] = 1.0 / E1, 1.0 / E2, 1.0 / E3
    S[0, 1] = S[1, 0] = -nu12 / E1
    S[0, 2] = S[2, 0] = -nu13 / E1
    S[1, 2] = S[2, 1] = -nu23 / E2
    S[3, 3], S[4, 4], S[5, 5] = 1.0 / G23, 1.0 / G13, 1.0 / G12
    D = np.linalg.inv(S)
    return 0.5 * (D + D.T)


def rotation(angles) -> np.ndarray:
    """x_global = R x_local for rotations by angles (radians) about x, then y,
    then z."""
    ax, ay, az = angles
    cx, sx, cy, sy, cz, sz = np.cos(ax), np.sin(ax), np.cos(ay), np.sin(ay), np.cos(az), np.sin(az)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def _hex_grid(nx, ny, nz, lx, ly, lz):
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    # node id = i + (nx+1)*(j + (ny+1)*k): x fastest
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    elems = np.stack(
        [
            nid(i + 1, j + 1, k + 1),
            nid(i, j + 1, k + 1),
            nid(i, j, k + 1),
            nid(i + 1, j, k + 1),
            nid(i + 1, j + 1, k),
            nid(i, j + 1, k),
            nid(i, j, k),
            nid(i + 1, j, k),
        ],
        axis=1,
    ).astype(np.int64)
    return coords, elems, nid


def cantilever_hex(nx=20, ny=4, nz=4, L=1.0, B=0.2, H=0.2, E=210e9, nu=0.3,
                   traction=1.0e6) -> Mesh:
    """Clamped cantilever of linear hexahedra with an end traction in -z."""
    coords, elems, nid = _hex_grid(nx, ny, nz, L, B, H)
    nn = coords.shape[0]
    dofflag = np.ones((nn, 3), dtype=np.int64)
    dofflag[np.isclose(coords[:, 0], 0.0)] = 0
    loads = np.zeros((1, nn, 3))
    # consistent nodal forces of a uniform traction on bilinear face quads
    fq = traction * (B / ny) * (H / nz) / 4.0
    for k in range(nz):
        for j in range(ny):
            for (jj, kk) in ((j, k), (j + 1, k), (j + 1, k + 1), (j, k + 1)):
                loads[0, nid(nx, jj, kk), 2] -= fq
    return Mesh(
        kind="hex8",
        coords=coords,
        elems=elems,
        dofflag=dofflag,
        emat=np.zeros(elems.shape[0], dtype=np.int64),
        mats=np.array([[E, nu]]),
        loads=loads,
        meta=dict(nx=nx, ny=ny, nz=nz, L=L, B=B, H=H),
    )


def cantilever_surface_traction(mesh: Mesh, traction=(0.0, 0.0, -1.0e6)) -> Mesh:
    """The cantilever's end traction stated the way a SIFEL deck states a
    surface load: an element load (surface, global system) on face 1 (xi = 1,
    the x = L face) of every hexahedron of the last element layer, with the
    traction vector at the face's 4 nodes; the nodal loads are dropped."""
    nx = mesh.meta["nx"]
    ny, nz = mesh.meta["ny"], mesh.meta["nz"]
    # elements are numbered x fastest: the last layer is i = nx - 1
    k, j = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
    last = (nx - 1) + nx * (j.ravel() + ny * k.ravel())
    rec = []
    for e in last:
        vals = np.zeros(72)
        vals[0:12] = np.tile(np.asarray(traction, dtype=float), 4)
        rec.append((int(e), [1, 0, 0, 0, 0, 0], vals))
    out = Mesh(**{**mesh.__dict__})
    out.loads = np.zeros_like(mesh.loads[:1])
    out.eloads = [rec]
    return out


def plate_edge_traction(mesh: Mesh, traction=(1.0, 0.0)) -> Mesh:
    """The plate's right-edge load as element edge loads (edge 4: xi = 1,
    from node 4 to node 1 of planeelemlq) with the load vector at both edge
    nodes; the nodal loads are dropped."""
    nx, ny = mesh.meta["nx"], mesh.meta["ny"]
    last = (nx - 1) + nx * np.arange(ny)
    rec = []
    for e in last:
        vals = np.zeros(16)
        vals[12:16] = np.tile(np.asarray(traction, dtype=float), 2)
        rec.append((int(e), [0, 0, 0, 1], vals))
    out = Mesh(**{**mesh.__dict__})
    out.loads = np.zeros_like(mesh.loads[:1])
    out.eloads = [rec]
    return out


def prescribe(mesh: Mesh, nodes, comp: int, values) -> Mesh:
    """Prescribed displacements: DOF `comp` of each node in `nodes` takes the
    matching entry of `values` (one load case); the DOFs get the negative
    flags -1, -2, ... of a SIFEL deck's constraint records."""
    out = Mesh(**{**mesh.__dict__})
    out.dofflag = mesh.dofflag.copy()
    nodes = np.asarray(nodes, dtype=np.int64)
    values = np.broadcast_to(np.asarray(values, dtype=float), nodes.shape)
    base = 0 if mesh.pd is None else mesh.pd.shape[1]
    out.dofflag[nodes, comp] = -(base + 1 + np.arange(nodes.size))
    old = np.zeros((mesh.loads.shape[0], 0)) if mesh.pd is None else mesh.pd
    out.pd = np.concatenate([old, np.tile(values, (mesh.loads.shape[0], 1))], axis=1)
    return out


def cantilever_top_loads(mesh: Mesh, nlc: int, seed: int = 1234, scale: float = 1.0e3) -> Mesh:
    """Replace the loads by ``nlc`` cases of N(0,1)*scale z-forces on the
    free nodes of the top face (z = H)."""
    H = mesh.meta["H"]
    rng = np.random.default_rng(seed)
    top = np.where(np.isclose(mesh.coords[:, 2], H) & (mesh.dofflag[:, 2] == 1))[0]
    loads = np.zeros((nlc, mesh.nn, 3))
    loads[:, top, 2] = rng.standard_normal((nlc, top.size)) * scale
    out = Mesh(**{**mesh.__dict__})
    out.loads = loads
    return out


def plate_quad(nx, ny, Lx=None, Ly=None, E=1.0e10, nu=0.25, t=0.01, traction=1.0) -> Mesh:
    """Plane-stress plate of bilinear quads; left edge clamped, uniform
    traction (per unit area) x thickness on the right edge, in +x."""
    Lx = float(nx) if Lx is None else Lx
    Ly = float(ny) if Ly is None else Ly
    xs = np.linspace(0.0, Lx, nx + 1)
    ys = np.linspace(0.0, Ly, ny + 1)
    Y, X = np.meshgrid(ys, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)

    def nid(i, j):
        return i + (nx + 1) * j

    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    i, j = i.ravel(), j.ravel()
    elems = np.stack([nid(i + 1, j + 1), nid(i, j + 1), nid(i, j), nid(i + 1, j)], axis=1)
    nn = coords.shape[0]
    dofflag = np.ones((nn, 2), dtype=np.int64)
    dofflag[np.isclose(coords[:, 0], 0.0)] = 0
    loads = np.zeros((1, nn, 2))
    fe = traction * t * (Ly / ny) / 2.0
    for jj in range(ny):
        loads[0, nid(nx, jj), 0] += fe
        loads[0, nid(nx, jj + 1), 0] += fe
    return Mesh(
        kind="quad4",
        coords=coords,
        elems=elems.astype(np.int64),
        dofflag=dofflag,
        emat=np.zeros(elems.shape[0], dtype=np.int64),
        mats=np.array([[E, nu]]),
        loads=loads,
        thick=np.full(elems.shape[0], t),
        meta=dict(nx=nx, ny=ny, Lx=Lx, Ly=Ly),
    )


def plate_tri(nx, ny, Lx=None, Ly=None, E=1.0e10, nu=0.25, t=0.01, traction=1.0) -> Mesh:
    """The plate of ``plate_quad`` meshed with constant-strain triangles
    (planeelemlt, 3 nodes): every quad cut along its n0-n2 diagonal into
    (n0, n1, n2) and (n0, n2, n3), both counter-clockwise (positive area, the
    orientation the element's formulas assume); same supports and loads."""
    q = plate_quad(nx, ny, Lx, Ly, E, nu, t, traction)
    e = q.elems
    tris = np.stack([e[:, [0, 1, 2]], e[:, [0, 2, 3]]], axis=1).reshape(-1, 3)
    return Mesh(kind="tri3", coords=q.coords, elems=tris.astype(np.int64), dofflag=q.dofflag,
                emat=np.zeros(tris.shape[0], dtype=np.int64), mats=q.mats, loads=q.loads,
                thick=np.full(tris.shape[0], t), meta=q.meta)


def plate_batch(count=512, seed=0, lo=16, hi=128):
    """The uneven batch: ``count`` plates with side counts uniform in
    [lo, hi], E uniform in [1e9, 1e11], nu uniform in [0.2, 0.35]."""
    rng = np.random.default_rng(seed)
    nx = rng.integers(lo, hi + 1, size=count)
    ny = rng.integers(lo, hi + 1, size=count)
    E = rng.uniform(1.0e9, 1.0e11, size=count)
    nu = rng.uniform(0.2, 0.35, size=count)
    return [plate_quad(int(a), int(b), E=float(e), nu=float(v)) for a, b, e, v in zip(nx, ny, E, nu)]


def heat_cube(n=8, L=1.0, sigma=1.0, mu=0.0, seed=1234, rhoc=2.0e6, T_left=1.0) -> Mesh:
    """Unit cube of n^3 linear hexahedra; per-element conductivity
    exp(N(mu, sigma)) from ``seed`` in element order (x fastest); T fixed
    to ``T_left`` on the x = 0 face (prescribed-value DOFs)."""
    coords, elems, _ = _hex_grid(n, n, n, L, L, L)
    rng = np.random.default_rng(seed)
    k = np.exp(rng.normal(mu, sigma, size=elems.shape[0]))
    nn = coords.shape[0]
    dofflag = np.ones((nn, 1), dtype=np.int64)
    left = np.isclose(coords[:, 0], 0.0)
    dofflag[left] = 0
    presc = np.zeros((nn, 1))
    presc[left, 0] = T_left
    return Mesh(
        kind="hex8t",
        coords=coords,
        elems=elems,
        dofflag=dofflag,
        emat=np.arange(elems.shape[0], dtype=np.int64),
        mats=np.stack([k, np.full_like(k, rhoc)], axis=1),
        loads=np.zeros((1, nn, 1)),
        meta=dict(n=n, L=L, prescribed=presc),
    )


# ----------------------------------------------------------------------------
# deck writers
# ----------------------------------------------------------------------------

def det3d(coords: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """Six times the signed volume of every tetrahedron, with the reference's
    formula and sign (det3d, GEFEL/matrix.cpp:3629): (p0-p3).((p1-p3)x(p2-p3))."""
    p = coords[tets]
    a, b, c = p[:, 0] - p[:, 3], p[:, 1] - p[:, 3], p[:, 2] - p[:, 3]
    return np.einsum("ij,ij->i", a, np.cross(b, c))


def cantilever_tet(nx=20, ny=4, nz=4, L=1.0, B=0.2, H=0.2, E=210e9, nu=0.3,
                   traction=1.0e6) -> Mesh:
    """Clamped cantilever of linear tetrahedra (lintet, 4 nodes).

    Every cell of the nx x ny x nz grid is split into six tetrahedra along its
    diagonal from the lowest to the highest corner (one per ordering of the
    three axes, so neighbouring cells split their shared face the same way),
    nodes ordered so that det3d > 0, the orientation the reference requires
    (lintet::stiffness_matrix aborts on a negative volume).  The end traction
    in -z goes to the nodes of the x = L face triangles, a third of each
    triangle's force per corner.
    """
    coords, _, nid = _hex_grid(nx, ny, nz, L, B, H)
    nn = coords.shape[0]
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    unit = np.eye(3, dtype=np.int64)
    tets = []
    for perm in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        o1 = unit[perm[0]]
        o2 = o1 + unit[perm[1]]
        tets.append(np.stack([nid(i, j, k), nid(i + o1[0], j + o1[1], k + o1[2]),
                              nid(i + o2[0], j + o2[1], k + o2[2]), nid(i + 1, j + 1, k + 1)], axis=1))
    elems = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int64)
    neg = det3d(coords, elems) < 0.0
    elems[neg, 0], elems[neg, 1] = elems[neg, 1].copy(), elems[neg, 0].copy()
    dofflag = np.ones((nn, 3), dtype=np.int64)
    dofflag[np.isclose(coords[:, 0], 0.0)] = 0
    loads = np.zeros((1, nn, 3))
    onface = np.isclose(coords[:, 0], L)
    faces = np.concatenate([elems[:, [0, 1, 2]], elems[:, [0, 1, 3]], elems[:, [0, 2, 3]], elems[:, [1, 2, 3]]])
    faces = faces[onface[faces].all(axis=1)]
    p = coords[faces]
    area = 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1)
    np.add.at(loads[0, :, 2], faces.ravel(), np.repeat(-traction * area / 3.0, 3))
    return Mesh(
        kind="tet4",
        coords=coords,
        elems=elems,
        dofflag=dofflag,
        emat=np.zeros(elems.shape[0], dtype=np.int64),
        mats=np.array([[E, nu]]),
        loads=loads,
        meta=dict(nx=nx, ny=ny, nz=nz, L=L, B=B, H=H),
    )


# natural coordinates of the serendipity nodes in SIFEL's order
# (bf_quad_hex_3d, GEFEL/basefun.cpp:2377; bf_quad_4_2d, :708)
HEX20_NODES = np.array([[1, 1, 1], [-1, 1, 1], [-1, -1, 1], [1, -1, 1], [1, 1, -1], [-1, 1, -1], [-1, -1, -1],
                        [1, -1, -1], [0, 1, 1], [-1, 0, 1], [0, -1, 1], [1, 0, 1], [1, 1, 0], [-1, 1, 0],
                        [-1, -1, 0], [1, -1, 0], [0, 1, -1], [-1, 0, -1], [0, -1, -1], [1, 0, -1]])
QUAD8_NODES = np.array([[1, 1], [-1, 1], [-1, -1], [1, -1], [0, 1], [-1, 0], [0, -1], [1, 0]])


def cantilever_hex20(nx=10, ny=2, nz=2, L=1.0, B=0.2, H=0.2, E=210e9, nu=0.3, traction=1.0e6) -> Mesh:
    """The cantilever of ``cantilever_hex`` with 20-node serendipity
    hexahedra (quadhex, element type 103): grid corners plus one node in the
    middle of every cell edge.  The end traction in -z goes to the 8 nodes of
    every face quad as consistent forces: -1/12 of the quad's force at each
    corner, 1/3 at each mid-side."""
    mx, my, mz = 2 * nx + 1, 2 * ny + 1, 2 * nz + 1
    I, J, K = np.meshgrid(np.arange(mx), np.arange(my), np.arange(mz), indexing="ij")
    keep = ((I % 2) + (J % 2) + (K % 2)) <= 1  # no face or cell centres
    lid = -np.ones((mx, my, mz), dtype=np.int64)
    # node numbering x fastest, then y, then z (as the grid of cantilever_hex)
    order = np.argsort((K * my + J) * mx + I, axis=None, kind="stable")
    flat_keep = keep.ravel()[order]
    lid.ravel()[order[flat_keep]] = np.arange(int(flat_keep.sum()))
    pts = np.stack([I.ravel()[order[flat_keep]], J.ravel()[order[flat_keep]], K.ravel()[order[flat_keep]]], 1)
    coords = pts * np.array([L / (2 * nx), B / (2 * ny), H / (2 * nz)])
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    elems = np.stack([lid[2 * i + 1 + p, 2 * j + 1 + q, 2 * k + 1 + r] for p, q, r in HEX20_NODES], axis=1)
    nn = coords.shape[0]
    dofflag = np.ones((nn, 3), dtype=np.int64)
    dofflag[np.isclose(coords[:, 0], 0.0)] = 0
    loads = np.zeros((1, nn, 3))
    fq = traction * (B / ny) * (H / nz)
    for kk in range(nz):
        for jj in range(ny):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    if dj == 0 and dk == 0:
                        continue
                    share = -1.0 / 12.0 if (dj != 0 and dk != 0) else 1.0 / 3.0
                    loads[0, lid[2 * nx, 2 * jj + 1 + dj, 2 * kk + 1 + dk], 2] -= share * fq
    return Mesh(kind="hex20", coords=coords, elems=elems.astype(np.int64), dofflag=dofflag,
                emat=np.zeros(elems.shape[0], dtype=np.int64), mats=np.array([[E, nu]]), loads=loads,
                meta=dict(nx=nx, ny=ny, nz=nz, L=L, B=B, H=H))


def plate_quad8(nx, ny, Lx=None, Ly=None, E=1.0e10, nu=0.25, t=0.01, traction=1.0) -> Mesh:
    """The plate of ``plate_quad`` with 8-node serendipity quads
    (planeelemqq, element type 24); the right-edge traction goes to each
    3-node edge as 1/6, 2/3, 1/6 of its force."""
    Lx = float(nx) if Lx is None else Lx
    Ly = float(ny) if Ly is None else Ly
    mx, my = 2 * nx + 1, 2 * ny + 1
    J, I = np.meshgrid(np.arange(my), np.arange(mx), indexing="ij")
    keep = ((I % 2) + (J % 2)) <= 1
    lid = -np.ones((my, mx), dtype=np.int64)
    lid[keep] = np.arange(int(keep.sum()))
    coords = np.stack([I[keep] * (Lx / (2 * nx)), J[keep] * (Ly / (2 * ny)), np.zeros(int(keep.sum()))], axis=1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    i, j = i.ravel(), j.ravel()
    elems = np.stack([lid[2 * j + 1 + q, 2 * i + 1 + p] for p, q in QUAD8_NODES], axis=1)
    nn = coords.shape[0]
    dofflag = np.ones((nn, 2), dtype=np.int64)
    dofflag[np.isclose(coords[:, 0], 0.0)] = 0
    loads = np.zeros((1, nn, 2))
    fe = traction * t * (Ly / ny)
    for jj in range(ny):
        for dj, share in ((-1, 1.0 / 6.0), (0, 2.0 / 3.0), (1, 1.0 / 6.0)):
            loads[0, lid[2 * jj + 1 + dj, 2 * nx], 0] += share * fe
    return Mesh(kind="quad8", coords=coords, elems=elems.astype(np.int64), dofflag=dofflag,
                emat=np.zeros(elems.shape[0], dtype=np.int64), mats=np.array([[E, nu]]), loads=loads,
                thick=np.full(elems.shape[0], t), meta=dict(nx=nx, ny=ny, Lx=Lx, Ly=Ly))


def _fmt(v: float) -> str:
    return repr(float(v))


def write_mefel_deck(mesh: Mesh, path: str, storage: int = 11, ni: int = 20000,
                     res: float = 1.0e-20, iv: int = 0, precond: int = 1,
                     title: str = "sifel-b200 synthetic deck") -> None:
    """Write a linear-statics MEFEL deck (positional format).

    storage 11 = symm_comp_rows, 10 = compressed_rows; solver cg (20);
    precond 1 = diagprec, 0 = noprecond.  For SCR + diagprec the reference
    stops on (r.r)/(f.f) < res, so res = 1e-20 means relative residual 1e-10.
    """
    nd = mesh.ndofn
    lines: list[str] = [title]
    # mespr problemtype straincomp stresscomp othercomp reactcomp
    # adaptivity stochasticcalc homogenization noderenumber
    lines.append("0\n1\n0 0 0 0\n0 0 0\n0")
    lines.append(f"{storage}")
    lines.append(f"20 {ni} {_fmt(res)} {iv}")
    lines.append(f"{precond}")
    lines.append(f"{mesh.nn}")
    is2d = mesh.kind in ("quad4", "tri3", "quad8")
    for i, (x, y, z) in enumerate(mesh.coords):
        lines.append(f"{i + 1} {_fmt(x)} {_fmt(y)} {_fmt(z)} {nd} 0 0")
    con = np.where((mesh.dofflag != 1).any(axis=1))[0]
    lines.append(f"{con.size}")
    for i in con:
        lines.append(f"{i + 1} " + " ".join(str(int(c)) for c in mesh.dofflag[i]))
    lines.append(f"{mesh.ne}")
    for e, nodes in enumerate(mesh.elems):
        ns = " ".join(str(int(v) + 1) for v in nodes)
        m = int(mesh.emat[e]) + 1
        if is2d:
            # type planeelementlt (20), planeelementlq (23) or
            # planeelementqq (24), strastrestate
            # planestress (10), cne 0, crst csplanestr (10) with the
            # element's thickness set, one material
            et = {"tri3": 20, "quad4": 23, "quad8": 24}[mesh.kind]
            lines.append(f"{e + 1} {et} 10 {ns} 0 10 {int(mesh.meta.get('tset', [0] * mesh.ne)[e]) + 1 if 'tset' in mesh.meta else 1} 1 1 {m}")
        else:
            # type lineartet (100), linearhex (102) or quadrhex (103), cne 0,
            # crst 0, one material
            et = {"tet4": 100, "hex8": 102, "hex20": 103}[mesh.kind]
            lines.append(f"{e + 1} {et} {ns} 0 0 1 {MATTYPE[mesh.mtype]} {m}")
    # materials: one type, mats.shape[0] instances: "id e nu" (elisomat = 1),
    # "id d11 .. d16 d22 .. d66" (elgmat3d = 2, elastgmat3d::read), or
    # "id" + the 36 local stiffness entries + 9 transformation functions,
    # each "0 value" (funct_type stat, const_val) (elortomat = 3,
    # elastortomat::read and gfunct::read)
    lines.append("1")
    lines.append(f"{MATTYPE[mesh.mtype]} {mesh.mats.shape[0]}")
    for k, row in enumerate(mesh.mats):
        if mesh.mtype == "ortho":
            lines.append(f"{k + 1} " + " ".join(_fmt(v) for v in row[:36]) + " "
                         + " ".join(f"0 {_fmt(v)}" for v in row[36:45]))
        else:
            lines.append(f"{k + 1} " + " ".join(_fmt(v) for v in row))
    # cross sections
    if is2d:
        tvals = mesh.meta.get("tvals", [float(mesh.thick[0])])
        lines.append("1")
        lines.append(f"10 {len(tvals)}")
        for k, t in enumerate(tvals):
            lines.append(f"{k + 1} {_fmt(t)}")
    else:
        lines.append("0")
    # load cases
    nlc = mesh.loads.shape[0]
    lines.append(f"{nlc}")
    for lc in range(nlc):
        ld = np.where(np.abs(mesh.loads[lc]).sum(axis=1) != 0.0)[0]
        lines.append(f"{ld.size}")
        for i in ld:
            lines.append(f"{i + 1} " + " ".join(_fmt(v) for v in mesh.loads[lc, i]))
        el = mesh.eloads[lc] if mesh.eloads else []
        lines.append(f"{len(el)}")  # loaded elements: eid, load type, then per face / edge a flag and its values
        for eid, flags, values in el:
            tel = 3 if mesh.kind == "hex8" else 2  # surface (linhex) / edge (planeelemlq) load
            per = 12 if mesh.kind == "hex8" else 4
            toks = [str(int(eid) + 1), str(tel)]
            for k, fl in enumerate(flags):
                toks.append(str(int(fl)))
                if fl > 0:
                    toks += [_fmt(v) for v in values[per * k:per * (k + 1)]]
            lines.append(" ".join(toks))
        pdv = mesh.pd[lc] if mesh.pd is not None else np.zeros(0)
        lines.append(f"{pdv.size}")  # prescribed displacements
        if pdv.size:
            lines.append(" ".join(_fmt(v) for v in pdv))
        lines.append("0")  # temperature changes
    lines.append("0")  # eigenstrains
    lines.append("0")  # textout
    lines.append("0")  # outgr_format
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_trfel_deck(mesh: Mesh, path: str, dt: float = 1.0, nsteps: int = 1, alpha: float = 1.0, ni: int = 20000,
                     res: float = 1.0e-20, iv: int = 1, precond: int = 1, rho: float = 1.0,
                     title: str = "sifel-b200 synthetic transport deck", stationary: bool = False,
                     form: str = "d") -> None:
    """Write a linear nonstationary heat-conduction TRFEL deck (positional).

    Token order as read by probdesct::read (TRFEL/SRC/probdesct.cpp:177-560;
    timecontr::read, GEFEL/timecontr.cpp:70), transtop::read
    (transtop.cpp:93), elementt::read (elementt.cpp:72), transmat::read
    (transmat.cpp:794; isotrmat "c k", isotrmat.cpp:444), transcrsec::read
    (transcrsec.cpp:33), transbclc::read / loadcaset::read (transbclc.cpp:33,
    loadcaset.cpp:133; one constant prescribed value per distinct value),
    lhsrhst::initcond (lhsrhst.cpp:157) and outdrivert::read.  Every element
    has its own isotropic material instance (mesh.mats rows (k, c)); storage
    SCR (11) for K and C, cg (20) with the diagonal preconditioner.
    """
    presc = mesh.meta["prescribed"][:, 0]
    end = dt * nsteps
    L = [title]
    # mesprt problemtype(nonstationary 60) transmatter(onemedium 1) mednames(heat 1) scale
    L.append(f"0\n{50 if stationary else 60}\n1\n1\n1.0")
    # gradcomp fluxcomp othercomp eqothercomp gravity adaptivity stochastic homog noderenumber advection reaction
    L.append("0\n0\n0\n0\n0\n0\n0\n0\n0\n0\n0")
    if stationary:  # conductmatstor, solver (probdesct.cpp:189-196)
        L.append("11")
        L.append(f"20 {ni} {_fmt(res)} {iv}")
        L.append(f"{precond}")
    else:
        # nonstatsolver trapezoidd(1) / trapezoidv(2) alpha; timecontr fixed(0) start end, one
        # important time, constant dt
        L.append(f"{1 if form == 'd' else 2} {_fmt(alpha)}")
        L.append(f"0 0.0 {_fmt(end)} 1 {_fmt(end)} 0 {_fmt(dt)}")
        # timetypeprint, hdbackup, storages, solver, capdiagonalization
        L.append("1\n0\n11 11")
        L.append(f"20 {ni} {_fmt(res)} {iv}")
        L.append(f"{precond}\n0")
    L.append(f"{mesh.nn}")
    for i, (x, y, z) in enumerate(mesh.coords):
        L.append(f"{i + 1} {_fmt(x)} {_fmt(y)} {_fmt(z)} 1 0")
    # constraints: prescribed nodes get code -(index of their prescribed value)
    fixed = np.where(mesh.dofflag[:, 0] != 1)[0]
    values = sorted(set(float(presc[i]) for i in fixed))
    pv_index = {v: k + 1 for k, v in enumerate(values)}
    L.append(f"{fixed.size}")
    for i in fixed:
        L.append(f"{i + 1} {-pv_index[float(presc[i])]}")
    L.append(f"{mesh.ne}")
    for e, nodes in enumerate(mesh.elems):
        ns = " ".join(str(int(v) + 1) for v in nodes)
        # cne 0, cross section crsec3dt (3) instance 1 (the density), material isotransmat (100)
        L.append(f"{e + 1} 225 {ns} 0 3 1 100 {int(mesh.emat[e]) + 1}")
    # materials: isotransmat (100), one instance per row of mats: "id c k"
    L.append("1")
    L.append(f"100 {mesh.mats.shape[0]}")
    for k, (kc, c) in enumerate(mesh.mats):
        L.append(f"{k + 1} {_fmt(c)} {_fmt(kc)}")
    # cross sections: one 3D section carrying the density (capacity = rho c N^T N)
    L.append("1\n3 1")
    L.append(f"1 {_fmt(rho)}")
    # one load case: prescribed values, no sources / element loads / nodal values / climatic conditions
    L.append("1")
    L.append(f"{len(values)}")
    for v in values:  # pvalt::read: initial value, then (nonstationary) a constant time function
        L.append(f"{_fmt(v)} {_fmt(v)}" if stationary else f"{_fmt(v)} 0 {_fmt(v)}")
    L.append("0\n0\n0\n0\n0\n0")  # nqs neb nnv ncc ncc2 nmultfunc
    L.append("0")  # boundary fluxes: neb
    if not stationary:
        for i in range(mesh.nn):  # initial values (lhsrhst::initcond)
            L.append(f"{i + 1} 0.0")
    L.append("0\n0" if stationary else "0\n0\n0")  # textout outgr_format [numdiag]
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")


def merge_meshes(meshes) -> tuple[Mesh, np.ndarray]:
    """Concatenate independent meshes of one kind into one mesh with disjoint
    node ranges (node ids shifted, one material row per mesh kept).  The code
    numbers of the merged mesh run mesh by mesh, so every mesh is a
    contiguous diagonal block of the global matrix.  Returns the merged mesh
    and the equation count of each part."""
    kind = meshes[0].kind
    coords, elems, dofflag, emat, mats, thick, loads, rows = [], [], [], [], [], [], [], []
    node0 = 0
    mat0 = 0
    for m in meshes:
        if m.kind != kind:
            raise ValueError("meshes of different kinds")
        coords.append(m.coords)
        elems.append(m.elems + node0)
        dofflag.append(m.dofflag)
        emat.append(m.emat + mat0)
        mats.append(m.mats)
        if m.thick is not None:
            thick.append(m.thick)
        loads.append(m.loads[0])
        rows.append(m.ndof)
        node0 += m.nn
        mat0 += m.mats.shape[0]
    merged = Mesh(kind=kind, coords=np.concatenate(coords), elems=np.concatenate(elems),
                  dofflag=np.concatenate(dofflag), emat=np.concatenate(emat), mats=np.concatenate(mats),
                  loads=np.concatenate(loads)[None], thick=np.concatenate(thick) if thick else None,
                  meta=dict(parts=len(meshes)))
    return merged, np.asarray(rows, dtype=np.int64)
