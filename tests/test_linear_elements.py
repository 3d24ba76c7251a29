"""Linear tetrahedra (lintet, MEFEL element type 100), constant-strain
triangles (planeelemlt, type 20), the serendipity hexahedron and quad
(quadhex 103, planeelemqq 24) and general material matrices: the oracle
pinned to the compiled reference's fixtures, the elements' own invariants,
the generated meshes, and the GPU assembly and solves against the oracle."""
import os

import numpy as np
import pytest

from ssf_b200 import decks

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden_mesh(g, kind="tet4"):
    return decks.Mesh(kind=kind, coords=g["coords"], elems=g["elems"], dofflag=g["dofflag"], emat=g["emat"],
                      mats=g["mats"], loads=g["loads"], thick=g["thick"] if "thick" in g else None)


def test_tet4_cantilever_golden(oracle):
    g = np.load(os.path.join(GOLDEN, "tet4_cantilever.npz"))
    m = _golden_mesh(g)
    adr, ci, a = oracle.assemble(m, sym=True)
    assert np.array_equal(adr, g["adr"]) and np.array_equal(ci, g["ci"])
    assert np.array_equal(a, g["a"])
    f = oracle.load_vector(m)
    assert np.array_equal(f, g["f"])
    x, st, ani, ares = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert ani == int(g["ani"]) and ares == float(g["ares"])
    assert np.array_equal(x, g["u"])


def test_tet4_element_invariants(oracle):
    rng = np.random.default_rng(21)
    xyz = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    xyz = xyz + rng.uniform(-0.1, 0.1, xyz.shape)
    if decks.det3d(xyz, np.arange(4)[None])[0] < 0:
        xyz[[0, 1]] = xyz[[1, 0]]
    ke = oracle.tet4_ke(xyz, 70e9, 0.33)
    assert np.allclose(ke, ke.T, rtol=0, atol=1e-12 * np.abs(ke).max())
    # the six rigid-body motions produce no forces
    for i in range(3):
        v = np.zeros((4, 3)); v[:, i] = 1.0
        assert np.abs(ke @ v.ravel()).max() < 1e-9 * np.abs(ke).max()
    for i, j in ((0, 1), (1, 2), (0, 2)):
        v = np.zeros((4, 3)); v[:, i] = -xyz[:, j]; v[:, j] = xyz[:, i]
        assert np.abs(ke @ v.ravel()).max() < 1e-9 * np.abs(ke).max()
    # 6 independent deformation modes: rank 12 - 6
    assert np.linalg.matrix_rank(ke, tol=1e-9 * np.abs(ke).max()) == 6
    # K scales with the length (B ~ 1/h, volume ~ h^3)
    assert np.allclose(oracle.tet4_ke(2.0 * xyz, 70e9, 0.33), 2.0 * ke, rtol=1e-12, atol=0)
    # wrong node numbering (negative det3d) is an error, as in the reference
    with pytest.raises(ValueError):
        oracle.tet4_ke(xyz[[1, 0, 2, 3]], 70e9, 0.33)


def test_tet_mesh_is_conforming():
    m = decks.cantilever_tet(4, 3, 2, L=1.0, B=0.3, H=0.2)
    det = decks.det3d(m.coords, m.elems)
    assert (det > 0).all() and np.isclose(det.sum() / 6.0, 1.0 * 0.3 * 0.2)
    faces = np.sort(np.concatenate([m.elems[:, [0, 1, 2]], m.elems[:, [0, 1, 3]], m.elems[:, [0, 2, 3]],
                                    m.elems[:, [1, 2, 3]]]), axis=1)
    _, counts = np.unique(faces, axis=0, return_counts=True)
    # every face is shared by two tetrahedra or lies on the boundary: 2 x 2
    # triangles per boundary cell face
    nb = 2 * 2 * (4 * 3 + 4 * 2 + 3 * 2)
    assert counts.max() == 2 and (counts == 1).sum() == nb
    # consistent nodal forces add up to traction x end area
    assert np.isclose(m.loads.sum(), -1.0e6 * 0.3 * 0.2)


def test_negative_volume_rejected_by_oracle(oracle):
    m = decks.cantilever_tet(2, 1, 1)
    m.elems[3, [0, 1]] = m.elems[3, [1, 0]]
    with pytest.raises(ValueError, match="element 4"):
        oracle.assemble(m, sym=True)


@pytest.mark.gpu
def test_tet4_assembly_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import mefel
    m = decks.cantilever_tet(6, 3, 3)
    rng = np.random.default_rng(6)
    m.coords = m.coords + rng.uniform(-0.005, 0.005, m.coords.shape)
    m.emat = np.arange(m.ne) % 3
    m.mats = np.array([[210e9, 0.3], [70e9, 0.25], [30e9, 0.2]])
    adr, ci, a = oracle.assemble(m, sym=True)
    with mefel.stiffness_matrix(m) as K:
        assert K.assembly["colours"] <= 64
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, adr) and np.array_equal(g_ci, ci)
    assert np.allclose(g_a, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


@pytest.mark.gpu
def test_tet4_golden_on_device(gpu_lib):
    from ssf_b200 import mefel
    g = np.load(os.path.join(GOLDEN, "tet4_cantilever.npz"))
    m = _golden_mesh(g)
    with mefel.stiffness_matrix(m) as K:
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, g["adr"]) and np.array_equal(g_ci, g["ci"])
    assert np.allclose(g_a, g["a"], rtol=1e-12, atol=1e-12 * np.abs(g["a"]).max())


@pytest.mark.gpu
def test_tet4_negative_volume_rejected_on_device(gpu_lib):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.cantilever_tet(2, 1, 1)
    m.elems[3, [0, 1]] = m.elems[3, [1, 0]]
    with pytest.raises(L.SgpuError, match="negative volume"):
        mefel.stiffness_matrix(m)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,mode", [("jacobi", "fp64"), ("agg", "mixed"), ("agg", "fp64")])
def test_tet_cantilever_solve_matches_oracle(oracle, gpu_lib, prec, mode):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.cantilever_tet(30, 6, 6)
    adr, ci, a = oracle.assemble(m, sym=True)
    f = oracle.load_vector(m)
    xo, st, ani_o, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with mefel.stiffness_matrix(m) as K:
        if prec == "agg":
            K.set_nullspace(mefel.rigid_body_modes(m))
        x, r = K.pcg(f, res=1e-22, prec=prec, mode=mode)
    assert r.status == L.OK
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8
    if prec == "agg":
        assert r.info["iterations"] * 3 < ani_o


# ---------------------------------------------------------------------------
# tri3
# ---------------------------------------------------------------------------

def test_tri3_plate_golden(oracle):
    g = np.load(os.path.join(GOLDEN, "tri3_plate.npz"))
    m = _golden_mesh(g, "tri3")
    adr, ci, a = oracle.assemble(m, sym=True)
    assert np.array_equal(adr, g["adr"]) and np.array_equal(ci, g["ci"])
    assert np.array_equal(a, g["a"])
    f = oracle.load_vector(m)
    assert np.array_equal(f, g["f"])
    x, st, ani, ares = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert ani == int(g["ani"]) and ares == float(g["ares"])
    assert np.array_equal(x, g["u"])


def test_tri3_element_invariants(oracle):
    xy = np.array([[0.1, 0.0], [1.2, 0.2], [0.3, 0.9]])
    ke = oracle.tri3_ke(xy, 3e10, 0.22, 0.02)
    assert np.allclose(ke, ke.T, rtol=0, atol=1e-12 * np.abs(ke).max())
    for v in (np.tile([1.0, 0.0], 3), np.tile([0.0, 1.0], 3), np.stack([-xy[:, 1], xy[:, 0]], 1).ravel()):
        assert np.abs(ke @ v).max() < 1e-9 * np.abs(ke).max()
    assert np.linalg.matrix_rank(ke, tol=1e-9 * np.abs(ke).max()) == 3
    # K does not change with the size of a plane element (B ~ 1/h, area ~ h^2)
    assert np.allclose(oracle.tri3_ke(3.0 * xy, 3e10, 0.22, 0.02), ke, rtol=1e-12, atol=0)
    # a clockwise triangle gives the negative matrix (no orientation check)
    assert np.allclose(oracle.tri3_ke(xy[[1, 0, 2]], 3e10, 0.22, 0.02)[np.ix_([2, 3, 0, 1, 4, 5], [2, 3, 0, 1, 4, 5])],
                       -ke, rtol=1e-12, atol=1e-12 * np.abs(ke).max())


def test_tri_plate_mesh():
    m = decks.plate_tri(5, 3, Lx=2.0, Ly=1.0)
    p = m.coords[m.elems]
    area2 = (p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1])
    assert (area2 > 0).all() and np.isclose(area2.sum() / 2.0, 2.0)
    assert m.ne == 2 * 5 * 3 and np.isclose(m.loads.sum(), 1.0 * 0.01 * 1.0)


@pytest.mark.gpu
def test_tri3_assembly_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import mefel
    m = decks.plate_tri(9, 6, E=3e10, nu=0.22)
    rng = np.random.default_rng(8)
    m.coords[:, :2] += rng.uniform(-0.1, 0.1, (m.nn, 2))
    m.emat = np.arange(m.ne) % 2
    m.mats = np.array([[3e10, 0.22], [7e10, 0.31]])
    m.thick = rng.uniform(0.01, 0.03, m.ne)
    adr, ci, a = oracle.assemble(m, sym=True)
    with mefel.stiffness_matrix(m) as K:
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, adr) and np.array_equal(g_ci, ci)
    assert np.allclose(g_a, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


@pytest.mark.gpu
def test_tri3_golden_on_device(gpu_lib):
    from ssf_b200 import mefel
    g = np.load(os.path.join(GOLDEN, "tri3_plate.npz"))
    with mefel.stiffness_matrix(_golden_mesh(g, "tri3")) as K:
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, g["adr"]) and np.array_equal(g_ci, g["ci"])
    assert np.allclose(g_a, g["a"], rtol=1e-12, atol=1e-12 * np.abs(g["a"]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("prec,mode", [("jacobi", "fp64"), ("agg", "mixed")])
def test_tri_plate_solve_matches_oracle(oracle, gpu_lib, prec, mode):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.plate_tri(60, 30, E=3e10, nu=0.22)
    adr, ci, a = oracle.assemble(m, sym=True)
    f = oracle.load_vector(m)
    xo, st, ani_o, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26, zero=1e-300)
    with mefel.stiffness_matrix(m) as K:
        if prec == "agg":
            K.set_nullspace(mefel.rigid_body_modes(m))
        x, r = K.pcg(f, res=1e-22, zero=1e-300, prec=prec, mode=mode)
    assert r.status == L.OK
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


# ---------------------------------------------------------------------------
# general material matrices (elastgmat3d, elastortomat) on hex8 / tet4
# ---------------------------------------------------------------------------

def _ortho_mesh(kind, nx=6, ny=3, nz=3):
    m = decks.cantilever_hex(nx, ny, nz) if kind == "hex8" else decks.cantilever_tet(nx, ny, nz)
    Dl = decks.orthotropic_local(150e9, 10e9, 9e9, 0.3, 0.28, 0.45, 3.5e9, 5e9, 5.5e9)
    rows = [np.concatenate([Dl.ravel(), decks.rotation(a).ravel()]) for a in ((0.0, 0.0, 0.0), (0.3, -0.5, 0.9))]
    m.mtype, m.mats = "ortho", np.array(rows)
    m.emat = np.arange(m.ne) % 2
    return m


def test_material_matrices_host_mirror(oracle):
    # the product's host-side transformation against the oracle's restatement
    from ssf_b200 import mefel
    m = _ortho_mesh("hex8", 2, 1, 1)
    a, b = mefel.material_matrices(m), oracle.material_dmat(m)
    assert np.allclose(a, b, rtol=1e-14, atol=1e-14 * np.abs(b).max())
    # the identity transformation leaves the local matrix unchanged
    assert np.array_equal(b[0], m.mats[0, :36])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["hex8", "tet4"])
@pytest.mark.parametrize("mtype", ["ortho", "gen3d"])
def test_general_material_assembly_matches_oracle(oracle, gpu_lib, kind, mtype):
    from ssf_b200 import mefel
    m = _ortho_mesh(kind)
    if mtype == "gen3d":
        D = mefel.material_matrices(m)
        m.mtype = "gen3d"
        m.mats = np.array([d.reshape(6, 6)[np.triu_indices(6)] for d in D])
    rng = np.random.default_rng(9)
    m.coords = m.coords + rng.uniform(-0.004, 0.004, m.coords.shape)
    adr, ci, a = oracle.assemble(m, sym=True)
    with mefel.stiffness_matrix(m) as K:
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, adr) and np.array_equal(g_ci, ci)
    assert np.allclose(g_a, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


@pytest.mark.gpu
def test_orthotropic_cantilever_solve_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = _ortho_mesh("hex8", 30, 6, 6)
    adr, ci, a = oracle.assemble(m, sym=True)
    f = oracle.load_vector(m)
    xo, st, ani_o, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with mefel.stiffness_matrix(m) as K:
        K.set_nullspace(mefel.rigid_body_modes(m))
        x, r = K.pcg(f, res=1e-22, prec="agg", mode="mixed")
    assert r.status == L.OK
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


# ---------------------------------------------------------------------------
# serendipity elements: hex20 (quadhex), quad8 (planeelemqq)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("name,kind", [("hex20_cantilever", "hex20"), ("quad8_plate", "quad8")])
def test_serendipity_golden(oracle, name, kind):
    # the oracle's shape-function derivatives are written differently from
    # the reference's, so K agrees to rounding, not bit for bit
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    m = _golden_mesh(g, kind)
    adr, ci, a = oracle.assemble(m, sym=True)
    assert np.array_equal(adr, g["adr"]) and np.array_equal(ci, g["ci"])
    assert np.abs(a - g["a"]).max() <= 1e-14 * np.abs(g["a"]).max()
    f = oracle.load_vector(m)
    assert np.array_equal(f, g["f"])
    x, st, ani, ares = oracle.scr_cg_prec(g["adr"], g["ci"], g["a"], f, ni=20000, res=1e-20)
    assert ani == int(g["ani"]) and np.array_equal(x, g["u"])


def test_serendipity_element_invariants(oracle):
    m = decks.cantilever_hex20(1, 1, 1, L=1.0, B=0.8, H=0.6)
    xyz = m.coords[m.elems[0]] + np.random.default_rng(22).uniform(-0.03, 0.03, (20, 3))
    ke = oracle.hex20_ke(xyz, 70e9, 0.33)
    assert np.allclose(ke, ke.T, rtol=0, atol=1e-12 * np.abs(ke).max())
    for i in range(3):
        v = np.zeros((20, 3)); v[:, i] = 1.0
        assert np.abs(ke @ v.ravel()).max() < 1e-9 * np.abs(ke).max()
    for i, j in ((0, 1), (1, 2), (0, 2)):
        v = np.zeros((20, 3)); v[:, i] = -xyz[:, j]; v[:, j] = xyz[:, i]
        assert np.abs(ke @ v.ravel()).max() < 1e-9 * np.abs(ke).max()
    assert np.linalg.matrix_rank(ke, tol=1e-9 * np.abs(ke).max()) == 54
    q = decks.plate_quad8(1, 1, Lx=1.3, Ly=0.9)
    xy = q.coords[q.elems[0], :2] + np.random.default_rng(23).uniform(-0.05, 0.05, (8, 2))
    kq = oracle.quad8_ke(xy, 3e10, 0.22, 0.02)
    assert np.allclose(kq, kq.T, rtol=0, atol=1e-12 * np.abs(kq).max())
    assert np.linalg.matrix_rank(kq, tol=1e-9 * np.abs(kq).max()) == 13
    # a reflected quad (negative Jacobian) is an error, as in the reference
    with pytest.raises(ValueError):
        oracle.quad8_ke(xy * np.array([-1.0, 1.0]), 3e10, 0.22, 0.02)


def test_serendipity_meshes():
    m = decks.cantilever_hex20(3, 2, 2)
    assert m.nn == 4 * 3 * 3 + 3 * 3 * 3 + 4 * 2 * 3 + 4 * 3 * 2 and np.isclose(m.loads.sum(), -1.0e6 * 0.04)
    assert (m.elems >= 0).all() and len(np.unique(m.elems)) == m.nn
    q = decks.plate_quad8(4, 3)
    assert q.nn == 5 * 4 + 4 * 4 + 5 * 3 and np.isclose(q.loads.sum(), 1.0 * 0.01 * 3.0)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,mtype", [("hex20", "iso"), ("hex20", "ortho"), ("quad8", "iso")])
def test_serendipity_assembly_matches_oracle(oracle, gpu_lib, kind, mtype):
    from ssf_b200 import mefel
    rng = np.random.default_rng(10)
    if kind == "hex20":
        m = decks.cantilever_hex20(5, 3, 2)
        m.coords = m.coords + rng.uniform(-0.004, 0.004, m.coords.shape)
        if mtype == "ortho":
            o = _ortho_mesh("hex8")
            m.mtype, m.mats = "ortho", o.mats
        else:
            m.mats = np.array([[210e9, 0.3], [70e9, 0.25]])
    else:
        m = decks.plate_quad8(7, 5, E=3e10, nu=0.22)
        m.coords[:, :2] += rng.uniform(-0.1, 0.1, (m.nn, 2))
        m.mats = np.array([[3e10, 0.22], [7e10, 0.31]])
        m.thick = rng.uniform(0.01, 0.03, m.ne)
    m.emat = np.arange(m.ne) % 2
    adr, ci, a = oracle.assemble(m, sym=True)
    with mefel.stiffness_matrix(m) as K:
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, adr) and np.array_equal(g_ci, ci)
    assert np.allclose(g_a, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


@pytest.mark.gpu
@pytest.mark.parametrize("name,kind", [("hex20_cantilever", "hex20"), ("quad8_plate", "quad8")])
def test_serendipity_golden_on_device(gpu_lib, name, kind):
    from ssf_b200 import mefel
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    with mefel.stiffness_matrix(_golden_mesh(g, kind)) as K:
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, g["adr"]) and np.array_equal(g_ci, g["ci"])
    assert np.allclose(g_a, g["a"], rtol=1e-12, atol=1e-12 * np.abs(g["a"]).max())


@pytest.mark.gpu
def test_quad8_negative_jacobian_rejected_on_device(gpu_lib):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.plate_quad8(3, 2)
    e = m.elems[2].copy()
    m.elems[2] = e[[1, 0, 3, 2, 4, 7, 6, 5]]  # mirrored node order
    with pytest.raises(L.SgpuError, match="negative"):
        mefel.stiffness_matrix(m)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["hex20", "quad8"])
def test_serendipity_solve_matches_oracle(oracle, gpu_lib, kind):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.cantilever_hex20(16, 3, 3) if kind == "hex20" else decks.plate_quad8(40, 20, E=3e10, nu=0.22)
    adr, ci, a = oracle.assemble(m, sym=True)
    f = oracle.load_vector(m)
    xo, st, ani_o, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26, zero=1e-300)
    with mefel.stiffness_matrix(m) as K:
        x, r = K.pcg(f, res=1e-22, zero=1e-300, prec="jacobi", mode="fp64")
        assert r.status == L.OK
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8
        K.set_nullspace(mefel.rigid_body_modes(m))
        x, r = K.pcg(f, res=1e-22, zero=1e-300, prec="agg", mode="mixed")
        assert r.status == L.OK
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["hex8", "tet4", "hex20", "quad4", "tri3", "quad8", "hex8t"])
def test_pattern_paths_agree(gpu_lib, monkeypatch, kind):
    # the node-adjacency pattern and the element-pair sort give the same SCR
    # arrays (and therefore the same matrix), constrained DOFs included
    from ssf_b200 import mefel
    make = {"hex8": lambda: decks.cantilever_hex(7, 3, 2), "tet4": lambda: decks.cantilever_tet(5, 2, 2),
            "hex20": lambda: decks.cantilever_hex20(4, 2, 2), "quad4": lambda: decks.plate_quad(9, 5),
            "tri3": lambda: decks.plate_tri(9, 5), "quad8": lambda: decks.plate_quad8(6, 4),
            "hex8t": lambda: decks.heat_cube(6, seed=2)}[kind]
    m = make()
    fn = mefel.conductivity_matrix if kind == "hex8t" else mefel.stiffness_matrix
    with fn(m) as K:
        a1 = K.download(symmetric=1)
    monkeypatch.setenv("SGPU_PATTERN_SORT", "1")
    with fn(m) as K:
        a2 = K.download(symmetric=1)
    for u, v in zip(a1, a2):
        assert np.array_equal(u, v)
