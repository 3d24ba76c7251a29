"""Element loads and prescribed displacements on the GPU path against the
oracle (pinned bit-exact to the compiled reference on the same decks:
tests/test_oracle_vs_reference.py).  The right-hand side of a load case is
loadcase::assemble (MEFEL/SRC/loadcase.cpp:400): nodal loads, the element
loads' consistent nodal forces (linhex::node_forces_surf,
planeelemlq::nodeforces) and -K_e r_e of the elements with prescribed
displacements (prdisplcontrib), the last formed on the GPU from the
assembled matrix (sgpu_assembly_lift)."""
import numpy as np
import pytest

from ssf_b200 import _lib as L
from ssf_b200 import decks, mefel

pytestmark = pytest.mark.gpu


def _cases():
    # the cantilever's 1 MPa end traction as element surface loads, its
    # clamped face partly replaced by prescribed displacements
    hx = decks.cantilever_surface_traction(decks.cantilever_hex(12, 3, 3))
    base = np.nonzero(np.isclose(hx.coords[:, 0], 0.0))[0]
    hx = decks.prescribe(hx, base[::3], 2, np.linspace(-2e-5, 3e-5, base[::3].size))
    hx = decks.prescribe(hx, base[1::5], 0, 1e-5)
    yield "hex8", hx
    # a distorted plate: random edge loads on every edge kind, two load
    # cases, prescribed displacements on the left edge
    q = decks.plate_quad(10, 6, E=3e10, nu=0.22)
    rng = np.random.default_rng(21)
    q.coords = q.coords.copy()
    q.coords[:, :2] += rng.uniform(-0.08, 0.08, (q.nn, 2))
    # forces of 1e4 N per unit length keep |d.p| far above the absolute
    # computer zero 1e-30 of the reference's breakdown test down to 1e-11
    recs = [(e, [int(v) for v in rng.integers(0, 2, 4)], 1e4 * rng.standard_normal(16)) for e in range(q.ne)]
    q.eloads = [recs[::2], recs[1::2]]
    q.loads = np.concatenate([q.loads, np.zeros_like(q.loads)])
    left = np.nonzero(np.isclose(decks.plate_quad(10, 6).coords[:, 0], 0.0))[0]
    q = decks.prescribe(q, left[2:5], 0, [1e-5, -2e-5, 3e-5])
    q.pd[1] *= -2.0
    yield "quad4", q


@pytest.mark.parametrize("name,m", list(_cases()))
def test_right_hand_side_and_solution(oracle, gpu_lib, name, m):
    adr, ci, a = oracle.assemble(m, sym=True)
    nlc = m.loads.shape[0]
    with mefel.stiffness_matrix(m) as K:
        for lc in range(nlc):
            fo = oracle.load_vector(m, lc)
            f = mefel.mefel_right_hand_side(m, lc, K)
            # element loads bit-exact (host), the GPU lifting to rounding
            assert np.allclose(f, fo, rtol=1e-12, atol=1e-12 * np.abs(fo).max())
    X, res = mefel.solve_linear_statics(m, res=1e-22, batched=False)
    for lc in range(nlc):
        fo = oracle.load_vector(m, lc)
        xo, st, _, _ = oracle.scr_cg_prec(adr, ci, a, fo, ni=200000, res=1e-26)
        assert res[lc].status == L.OK
        assert np.linalg.norm(X[lc] - xo) / np.linalg.norm(xo) <= 1e-8


def test_lifting_skips_elements_without_prescribed_values(oracle, gpu_lib):
    # r = 0 everywhere: the lifting adds nothing (not even rounding)
    m = decks.cantilever_hex(6, 2, 2)
    with mefel.stiffness_matrix(m) as K:
        f = np.arange(K.n, dtype=np.float64)
        g = f.copy()
        L.check(L.lib().sgpu_assembly_lift(K.h, np.zeros(m.nn * 3), g))
    assert np.array_equal(f, g)


@pytest.mark.parametrize("name,m", list(_cases()))
def test_deck_with_element_loads_end_to_end(oracle, gpu_lib, tmp_path, name, m):
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p, res=1e-22)
    X, results, info = mefel.solve_deck(p, mode="fp64")
    adr, ci, a = oracle.assemble(m, sym=True)
    for lc in range(m.loads.shape[0]):
        fo = oracle.load_vector(m, lc)
        xo, st, _, _ = oracle.scr_cg_prec(adr, ci, a, fo, ni=200000, res=1e-26)
        assert results[lc].status == L.OK
        assert np.linalg.norm(X[lc] - xo) / np.linalg.norm(xo) <= 1e-8


def test_surface_traction_reproduces_the_lumped_cantilever(oracle, gpu_lib):
    # the headline cantilever's load written as element surface loads gives
    # the same solution as its hand-lumped nodal forces
    m0 = decks.cantilever_hex(20, 4, 4)
    m1 = decks.cantilever_surface_traction(m0)
    X0, r0 = mefel.solve_linear_statics(m0, res=1e-22)
    X1, r1 = mefel.solve_linear_statics(m1, res=1e-22)
    assert r0[0].status == r1[0].status == L.OK
    assert np.linalg.norm(X1[0] - X0[0]) / np.linalg.norm(X0[0]) <= 1e-9
