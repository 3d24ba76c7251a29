"""The oracle against the compiled SIFEL reference on fresh decks (skipped
where oracle/_ref has not been built: the reference sources are needed)."""
import os
import tempfile

import numpy as np
import pytest

from ssf_b200 import decks


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.ref_available():
        pytest.skip("compiled reference (oracle/_ref) not built")
    return oracle


def test_random_distorted_cantilever_bit_exact(ref):
    m = decks.cantilever_hex(7, 3, 2)
    rng = np.random.default_rng(42)
    inner = ~np.isclose(m.coords[:, 0], 0.0)
    m.coords[inner] += rng.uniform(-0.01, 0.01, (inner.sum(), 3))
    m.emat = rng.integers(0, 3, m.ne)
    m.mats = np.array([[210e9, 0.3], [70e9, 0.33], [30e9, 0.2]])
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "d.in")
        decks.write_mefel_deck(m, deck)
        d = ref.run_mefel_dump(deck, td)
    adr, ci, a = ref.assemble(m, sym=True)
    assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
    assert np.array_equal(a, d["K_a"])
    f = ref.load_vector(m)
    x, st, ani, ares = ref.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert ani == d["meta"]["ani_0"] and np.array_equal(x, d["u"])


def test_random_distorted_tet_cantilever_bit_exact(ref):
    # lintet (element type 100): one integration point, weight det3d/6
    m = decks.cantilever_tet(6, 3, 2)
    rng = np.random.default_rng(43)
    inner = ~np.isclose(m.coords[:, 0], 0.0)
    m.coords[inner] += rng.uniform(-0.005, 0.005, (inner.sum(), 3))
    assert (decks.det3d(m.coords, m.elems) > 0).all()
    m.emat = rng.integers(0, 3, m.ne)
    m.mats = np.array([[210e9, 0.3], [70e9, 0.33], [30e9, 0.2]])
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "d.in")
        decks.write_mefel_deck(m, deck)
        d = ref.run_mefel_dump(deck, td)
    adr, ci, a = ref.assemble(m, sym=True)
    assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
    assert np.array_equal(a, d["K_a"])
    f = ref.load_vector(m)
    assert np.array_equal(f, d["f"][: f.size])
    x, st, ani, ares = ref.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert ani == d["meta"]["ani_0"] and np.array_equal(x, d["u"])


def test_random_distorted_tri_plate_bit_exact(ref):
    # planeelemlt (element type 20): one point at (1/3, 1/3), weight t det/2
    m = decks.plate_tri(7, 4, E=3e10, nu=0.22, t=0.02)
    rng = np.random.default_rng(44)
    m.coords[:, :2] += rng.uniform(-0.1, 0.1, (m.nn, 2))
    m.emat = rng.integers(0, 2, m.ne)
    m.mats = np.array([[3e10, 0.22], [7e10, 0.31]])
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "d.in")
        decks.write_mefel_deck(m, deck)
        d = ref.run_mefel_dump(deck, td)
    adr, ci, a = ref.assemble(m, sym=True)
    assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
    assert np.array_equal(a, d["K_a"])
    f = ref.load_vector(m)
    assert np.array_equal(f, d["f"][: f.size])
    x, st, ani, ares = ref.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert ani == d["meta"]["ani_0"] and np.array_equal(x, d["u"])


def _dump_and_compare(ref, m):
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "d.in")
        decks.write_mefel_deck(m, deck)
        d = ref.run_mefel_dump(deck, td)
    adr, ci, a = ref.assemble(m, sym=True)
    assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
    assert np.array_equal(a, d["K_a"])
    f = ref.load_vector(m)
    x, st, ani, ares = ref.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert ani == d["meta"]["ani_0"] and np.array_equal(x, d["u"])


@pytest.mark.parametrize("kind", ["hex8", "tet4"])
def test_orthotropic_material_bit_exact(ref, kind):
    # elastortomat (material type 3): local orthotropic stiffness turned into
    # the global system by lg_tens4transf with a constant rotation; two
    # instances with different axes
    m = decks.cantilever_hex(6, 2, 2) if kind == "hex8" else decks.cantilever_tet(5, 2, 2)
    rng = np.random.default_rng(45)
    inner = ~np.isclose(m.coords[:, 0], 0.0)
    m.coords[inner] += rng.uniform(-0.004, 0.004, (inner.sum(), 3))
    Dl = decks.orthotropic_local(150e9, 10e9, 9e9, 0.3, 0.28, 0.45, 3.5e9, 5e9, 5.5e9)
    rows = [np.concatenate([Dl.ravel(), decks.rotation(a).ravel()]) for a in ((0.0, 0.0, 0.0), (0.3, -0.5, 0.9))]
    m.mtype, m.mats = "ortho", np.array(rows)
    m.emat = rng.integers(0, 2, m.ne)
    _dump_and_compare(ref, m)


def test_general_anisotropic_material_bit_exact(ref):
    # elastgmat3d (material type 2): the 21 entries of a symmetric 6 x 6 D
    m = decks.cantilever_hex(6, 2, 2)
    Dl = decks.orthotropic_local(150e9, 10e9, 9e9, 0.3, 0.28, 0.45, 3.5e9, 5e9, 5.5e9)
    m.mtype = "gen3d"
    m.mats = np.array([Dl[np.triu_indices(6)], (1.5 * Dl)[np.triu_indices(6)]])
    m.emat = np.arange(m.ne) % 2
    _dump_and_compare(ref, m)


@pytest.mark.parametrize("kind", ["hex20", "quad8"])
def test_serendipity_elements_match_reference(ref, kind):
    # quadhex (type 103, 3x3x3 Gauss) and planeelemqq (type 24, 3x3 Gauss):
    # the oracle writes the serendipity derivatives from the corner and
    # mid-edge formulas instead of the reference's per-node expressions, so
    # the pin is to rounding (1e-13 of the largest entry), with the same
    # pattern, loads and CG iteration count
    if kind == "hex20":
        m = decks.cantilever_hex20(5, 2, 2)
        inner = ~np.isclose(m.coords[:, 0], 0.0)
        m.coords[inner] += np.random.default_rng(46).uniform(-0.004, 0.004, (inner.sum(), 3))
    else:
        m = decks.plate_quad8(6, 4, E=3e10, nu=0.22, t=0.02)
        m.coords[:, :2] += np.random.default_rng(47).uniform(-0.1, 0.1, (m.nn, 2))
    m.emat = np.arange(m.ne) % 2
    m.mats = np.array([[m.mats[0, 0], m.mats[0, 1]], [0.5 * m.mats[0, 0], 0.27]])
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "d.in")
        decks.write_mefel_deck(m, deck)
        d = ref.run_mefel_dump(deck, td)
    adr, ci, a = ref.assemble(m, sym=True)
    assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
    assert np.abs(a - d["K_a"]).max() <= 1e-13 * np.abs(d["K_a"]).max()
    f = ref.load_vector(m)
    assert np.allclose(f, d["f"][: f.size], rtol=1e-15, atol=0)
    x, st, ani, ares = ref.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20, zero=1e-300)
    xr, _, _, _ = ref.scr_cg_prec(d["K_adr"], d["K_ci"], d["K_a"], d["f"][: f.size], ni=20000, res=1e-20,
                                  zero=1e-300)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)


def test_reference_solver_library_matches_oracle(ref):
    """libsifelref.so runs the reference's own symcomprow::cg_prec."""
    m = decks.cantilever_hex(10, 2, 2)
    adr, ci, a = ref.assemble(m, sym=True)
    f = ref.load_vector(m)
    x_o, _, ani_o, ares_o = ref.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    x_r, ani_r, ares_r = ref.ref_scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert ani_r == ani_o and ares_r == ares_o and np.array_equal(x_r, x_o)


@pytest.mark.parametrize("form", ["d", "v"])
def test_trfel_random_cube_bit_exact(ref, form):
    # trapezoidd (linear_nonstat_solv_dform) and trapezoidv
    # (nonstat_solv_vform_comp) decks through the compiled reference
    m = decks.heat_cube(3, seed=77)
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "c.in")
        decks.write_trfel_deck(m, deck, dt=25.0, nsteps=2, alpha=0.5, form=form)
        d = ref.run_trfel_dump(deck, td)
    T, V, its = ref.trfel_steps(m, 2, 25.0, alpha=0.5, iv=1, form=form)
    assert np.array_equal(T, d["T"]) and np.array_equal(V, d["V"])


def test_trfel_density_and_distortion_bit_exact(ref):
    # a cross-section density other than 1 (crsec3dt) scales the capacity
    # matrix; distorted nodes exercise the Jacobians; several prescribed
    # values; the deck reader's view of the same file gives the same matrices
    from ssf_b200 import mefel
    m = decks.heat_cube(4, seed=21, T_left=3.5)
    rng = np.random.default_rng(5)
    inner = ~np.isclose(m.coords[:, 0], 0.0)
    m.coords[inner] += rng.uniform(-0.02, 0.02, (inner.sum(), 3))
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "c.in")
        decks.write_trfel_deck(m, deck, dt=15.0, nsteps=3, alpha=0.75, rho=2.5)
        d = ref.run_trfel_dump(deck, td)
        with mefel.Deck(deck, front="trfel") as dk:
            r = dk.mesh()
    rho = np.full(m.ne, 2.5)
    assert np.array_equal(r.meta["rho"], rho)
    _, _, ka = ref.assemble(m, sym=True, kind="hex8t_k")
    _, _, ca = ref.assemble(m, sym=True, kind="hex8t_c", rho=rho)
    assert np.array_equal(ka, d["K_a"]) and np.array_equal(ca, d["C_a"])
    _, _, ca_r = ref.assemble(r, sym=True, kind="hex8t_c", rho=r.meta["rho"])
    assert np.array_equal(ca_r, d["C_a"])
    T, V, _ = ref.trfel_steps(m, 3, 15.0, alpha=0.75, iv=1, rho=rho)
    assert np.array_equal(T, d["T"]) and np.array_equal(V, d["V"])


@pytest.mark.parametrize("kind", ["tet4", "tri3", "hex20"])
def test_cr_storage_of_the_added_elements(ref, kind):
    # compressed_rows (storage 10) + no preconditioner, the reference's CR
    # path: the full-row storage and the CG on it
    m = {"tet4": lambda: decks.cantilever_tet(4, 2, 2), "tri3": lambda: decks.plate_tri(6, 3, E=3e10, nu=0.22),
         "hex20": lambda: decks.cantilever_hex20(3, 2, 2)}[kind]()
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "d.in")
        decks.write_mefel_deck(m, deck, storage=10, precond=0, res=1e-10)
        d = ref.run_mefel_dump(deck, td)
    adr, ci, a = ref.assemble(m, sym=False)
    assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
    if kind == "hex20":
        assert np.abs(a - d["K_a"]).max() <= 1e-14 * np.abs(d["K_a"]).max()
        return
    assert np.array_equal(a, d["K_a"])
    f = ref.load_vector(m)
    x, st, ani, ares = ref.cr_cg_prec(adr, ci, a, f, ni=20000, res=1e-10, zero=1e-300)
    assert ani == d["meta"]["ani_0"] and np.array_equal(x, d["u"])


def test_thickness_sets_and_load_cases_bit_exact(ref):
    # plane stress with two cross-section thickness sets, and a cantilever
    # with three load cases: K, every right-hand side and every solution
    q = decks.plate_quad(6, 4, E=3e10, nu=0.22)
    q.meta["tvals"] = [0.01, 0.03]
    q.meta["tset"] = list(np.arange(q.ne) % 2)
    q.thick = np.array([0.01, 0.03])[np.arange(q.ne) % 2]
    c = decks.cantilever_top_loads(decks.cantilever_hex(5, 2, 2), 3, seed=9)
    for m in (q, c):
        with tempfile.TemporaryDirectory() as td:
            deck = os.path.join(td, "d.in")
            decks.write_mefel_deck(m, deck)
            d = ref.run_mefel_dump(deck, td)
        adr, ci, a = ref.assemble(m, sym=True)
        assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
        assert np.array_equal(a, d["K_a"])
        n = adr.size - 1
        for lc in range(m.loads.shape[0]):
            f = ref.load_vector(m, lc)
            assert np.array_equal(f, d["f"][lc * n:(lc + 1) * n])
            x, st, ani, ares = ref.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
            assert ani == d["meta"][f"ani_{lc}"] and np.array_equal(x, d["u"][lc * n:(lc + 1) * n])


def _run_and_compare(ref, m):
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "d.in")
        decks.write_mefel_deck(m, deck)
        d = ref.run_mefel_dump(deck, td)
    adr, ci, a = ref.assemble(m, sym=True)
    assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
    assert np.array_equal(a, d["K_a"])
    f = ref.load_vector(m)
    assert np.array_equal(f, d["f"][: f.size])
    x, st, ani, ares = ref.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert ani == d["meta"]["ani_0"] and np.array_equal(x, d["u"][: f.size])
    return f, d


def test_surface_traction_as_element_loads_bit_exact(ref):
    # the 1 MPa end traction of the cantilever as hexahedron surface loads
    # (linhex::node_forces_surf) on distorted faces; same f and u
    m = decks.cantilever_surface_traction(decks.cantilever_hex(6, 2, 3))
    rng = np.random.default_rng(44)
    inner = ~np.isclose(m.coords[:, 0], 0.0)
    m.coords = m.coords.copy()
    m.coords[inner] += rng.uniform(-0.01, 0.01, (inner.sum(), 3))
    f, _ = _run_and_compare(ref, m)
    # the consistent forces of a uniform traction on the undistorted face
    # equal the nodal loads cantilever_hex lumps by hand
    u = decks.cantilever_hex(6, 2, 3)
    assert np.allclose(ref.load_vector(decks.cantilever_surface_traction(u)), ref.load_vector(u), rtol=1e-12,
                       atol=1e-9)


def test_edge_load_and_prescribed_displacements_bit_exact(ref):
    # quad edge loads on every edge kind, a second load case, and prescribed
    # displacements on part of the clamped edge
    m = decks.plate_quad(6, 4)
    rng = np.random.default_rng(45)
    m.coords = m.coords.copy()
    m.coords[:, :2] += rng.uniform(-0.1, 0.1, (m.nn, 2))
    rec = []
    for e in range(m.ne):
        flags = [int(v) for v in rng.integers(0, 2, 4)]
        rec.append((e, flags, rng.standard_normal(16)))
    m.eloads = [rec[: m.ne // 2], rec[m.ne // 2:]]
    m.loads = np.concatenate([m.loads, rng.standard_normal((1, m.nn, 2))])
    left = np.nonzero(np.isclose(decks.plate_quad(6, 4).coords[:, 0], 0.0))[0]
    m = decks.prescribe(m, left[1:3], 0, [1e-4, -2e-4])
    m = decks.prescribe(m, left[3:4], 1, [5e-5])
    m.pd[1] *= -3.0
    f, d = _run_and_compare(ref, m)
    assert d["meta"]["nlc"] == 2
    assert np.array_equal(ref.load_vector(m, 1), d["f"][f.size: 2 * f.size])


def test_hex_prescribed_displacements_bit_exact(ref):
    m = decks.cantilever_hex(5, 2, 2)
    base = np.nonzero(np.isclose(m.coords[:, 0], 0.0))[0]
    m = decks.prescribe(m, base[:4], 2, np.linspace(1e-5, 4e-5, 4))
    _run_and_compare(ref, m)
