"""TRFEL linear transient conduction on the GPU against the oracle:
Dirichlet lifting (assemble_init), and steps of the d-form trapezoid
(linear_nonstat_solv_dform) with K and C assembled on the device."""
import numpy as np
import pytest

from ssf_b200 import decks

pytestmark = pytest.mark.gpu


def _cube(n=4, seed=5):
    m = decks.heat_cube(n, seed=seed)
    rng = np.random.default_rng(seed)
    m.coords = m.coords + rng.uniform(-0.01, 0.01, m.coords.shape)
    return m


def test_lifting_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import mefel
    m = _cube()
    r = m.meta["prescribed"][:, 0].copy()
    # a non-zero initial state on free nodes exercises the reference's use of
    # initial values in prescvalues() (globmatt.cpp:1069)
    r[m.dofflag[:, 0] == 1] = np.random.default_rng(1).uniform(0, 0.1, (m.dofflag[:, 0] == 1).sum())
    ref = oracle.trfel_lift(m, r)
    with mefel.conductivity_matrix(m) as K:
        got = mefel.trfel_lift(K, r)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("alpha", [1.0, 0.5])
def test_transient_steps_match_oracle(oracle, gpu_lib, alpha):
    from ssf_b200 import mefel
    m = _cube()
    d_o, v_o, its_o = oracle.trfel_steps(m, 3, 10.0, alpha=alpha, res=1e-24, iv=1)
    assert all(st == 0 for st, _ in its_o)
    d, v, its, info = mefel.linear_nonstat_solv_dform(m, 3, 10.0, alpha=alpha, res=1e-24, iv=1)
    assert np.linalg.norm(d - d_o) / np.linalg.norm(d_o) <= 1e-8
    assert np.linalg.norm(v - v_o) / np.linalg.norm(v_o) <= 1e-6
    for (st, a_o), a in zip(its_o, its):
        assert abs(int(a) - (a_o + 1)) <= 2  # GPU reports iterations done = ani + 1


def test_transient_mixed_form(oracle, gpu_lib):
    from ssf_b200 import mefel
    m = _cube(6)
    d_o, _, _ = oracle.trfel_steps(m, 2, 10.0, res=1e-24, iv=1)
    d, _, _, info = mefel.linear_nonstat_solv_dform(m, 2, 10.0, res=1e-20, iv=1, mode="mixed")
    assert np.linalg.norm(d - d_o) / np.linalg.norm(d_o) <= 1e-7


@pytest.mark.parametrize("alpha", [1.0, 0.5])
def test_vform_steps_match_oracle(oracle, gpu_lib, alpha):
    # trapezoidv: nonstat_solv_vform_comp (npsolvert.cpp:62) solves for the rates
    from ssf_b200 import mefel
    m = _cube()
    d_o, v_o, its_o = oracle.trfel_steps(m, 3, 10.0, alpha=alpha, res=1e-24, iv=1, form="v")
    assert all(st == 0 for st, _ in its_o)
    d, v, its, info = mefel.nonstat_solv_vform_comp(m, 3, 10.0, alpha=alpha, res=1e-24, iv=1)
    assert np.linalg.norm(d - d_o) / np.linalg.norm(d_o) <= 1e-8
    assert np.linalg.norm(v - v_o) / np.linalg.norm(v_o) <= 1e-8
    for (st, a_o), a in zip(its_o, its):
        assert abs(int(a) - (a_o + 1)) <= 2


@pytest.mark.parametrize("mode", ["mixed", "fp64"])
def test_transient_aggregation_preconditioner(oracle, gpu_lib, mode):
    # the aggregation hierarchy is built on the first step and reused by the
    # others; the steps still reach the oracle's states
    from ssf_b200 import mefel
    m = _cube(12, seed=9)
    d_o, v_o, _ = oracle.trfel_steps(m, 3, 10.0, res=1e-26, iv=1)
    d, v, its, info = mefel.linear_nonstat_solv_dform(m, 3, 10.0, res=1e-22, iv=1, mode=mode, prec="agg")
    assert np.linalg.norm(d - d_o) / np.linalg.norm(d_o) <= 1e-8
    assert np.linalg.norm(v - v_o) / np.linalg.norm(v_o) <= 1e-6
    assert info["precond_levels"] >= 2 and info["precond_setup_ms"] > 0.0


def test_stationary_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import mefel
    from ssf_b200 import _lib as L
    m = _cube(6, seed=8)
    xo, st, ani_o, _ = oracle.trfel_stationary(m)
    assert st == 0
    x, r = mefel.solve_stationary_problem(m)
    assert r.status == L.OK and abs(r.ani - ani_o) <= 2
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


def test_capacity_on_the_conductivity_pattern(oracle, gpu_lib):
    # sgpu_assemble_copy: C integrated on K's pattern equals C assembled on
    # its own, and the oracle's C; new element parameters are taken
    from ssf_b200 import mefel
    m = decks.heat_cube(6, seed=8)
    rho = np.random.default_rng(3).uniform(0.5, 2.0, m.ne)
    _, _, ca = oracle.assemble(m, sym=True, kind="hex8t_c", rho=rho)
    with mefel.conductivity_matrix(m) as K:
        with mefel.assemble_copy(K, "hex8t_c", rho=rho) as Cc, mefel.capacity_matrix(m, rho=rho) as Cs:
            a1, a2 = Cc.download(symmetric=1), Cs.download(symmetric=1)
        for u, v in zip(a1[:2], a2[:2]):
            assert np.array_equal(u, v)
        assert np.array_equal(a1[2], a2[2])
        assert np.allclose(a1[2], ca, rtol=1e-12, atol=1e-12 * np.abs(ca).max())
        # K itself is untouched, and a copy with new conductivities follows them
        _, _, ka = oracle.assemble(m, sym=True, kind="hex8t_k")
        assert np.allclose(K.download(symmetric=1)[2], ka, rtol=1e-12, atol=1e-12 * np.abs(ka).max())
        mats2 = m.mats[m.emat].copy()
        mats2[:, 0] *= 3.0
        with mefel.assemble_copy(K, "hex8t_k", emat=mats2) as K3:
            assert np.allclose(K3.download(symmetric=1)[2], 3.0 * ka, rtol=1e-12, atol=1e-12 * np.abs(ka).max())
