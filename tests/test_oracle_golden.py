"""The CPU oracle (oracle/sifel_oracle.c) against the golden fixtures the
compiled SIFEL reference produced (tests/golden/make_golden.py).  Pins the
restatement: integer/index work bit-exact, element matrices and solutions to
the last few ulps."""
import os

import numpy as np
import pytest

from ssf_b200 import decks

G = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return dict(np.load(os.path.join(G, name)))


def test_c1_cantilever_pattern_matrix_rhs_solution(oracle):
    g = load("c1_cantilever.npz")
    m = decks.cantilever_hex(20, 4, 4)
    adr, ci, a = oracle.assemble(m, sym=True)
    assert np.array_equal(adr, g["adr"]) and np.array_equal(ci, g["ci"])
    assert np.array_equal(a, g["a"])  # same operation order -> bit-exact
    f = oracle.load_vector(m)
    assert np.array_equal(f, g["f"])
    x, st, ani, ares = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert st == 0 and ani == int(g["ani"])
    assert np.array_equal(x, g["u"])
    assert ares == float(g["ares"])


def test_single_hex_element_matrix(oracle):
    g = load("hex8_single.npz")
    ke = oracle.hex8_ke(g["coords"][g["elems"][0]], float(g["E"]), float(g["nu"]))
    K = oracle.scr_to_dense(g["adr"], g["ci"], g["a"])
    # the deck numbers node DOFs in node order, which is the element order here
    order = np.argsort(g["elems"][0])
    perm = np.concatenate([[3 * k, 3 * k + 1, 3 * k + 2] for k in order])
    Ke_nodes = np.zeros((24, 24))
    Ke_nodes[np.ix_(np.arange(24), np.arange(24))] = ke
    # reorder the element matrix to global (node-id) DOF order
    inv = np.empty(8, dtype=int)
    inv[g["elems"][0]] = np.arange(8)
    p = np.concatenate([[3 * inv[k], 3 * inv[k] + 1, 3 * inv[k] + 2] for k in range(8)])
    Kg = ke[np.ix_(p, p)]
    assert np.allclose(Kg, K, rtol=0, atol=1e-15 * np.abs(K).max())
    # symmetric, and six rigid-body modes in the null space
    assert np.allclose(ke, ke.T, rtol=0, atol=1e-14 * np.abs(ke).max())
    xyz = g["coords"][g["elems"][0]]
    rbm = []
    for d in range(3):
        v = np.zeros((8, 3)); v[:, d] = 1.0; rbm.append(v.ravel())
    for (i, j) in ((0, 1), (1, 2), (0, 2)):
        v = np.zeros((8, 3)); v[:, i] = -xyz[:, j]; v[:, j] = xyz[:, i]; rbm.append(v.ravel())
    for v in rbm:
        assert np.abs(ke @ v).max() < 1e-6 * np.abs(ke).max()
    del order, perm, Ke_nodes


def test_quad4_plate(oracle):
    g = load("quad4_plate.npz")
    m = decks.Mesh(kind="quad4", coords=g["coords"], elems=g["elems"], dofflag=g["dofflag"], emat=g["emat"],
                   mats=g["mats"], loads=g["loads"], thick=g["thick"])
    adr, ci, a = oracle.assemble(m, sym=True)
    assert np.array_equal(adr, g["adr"]) and np.array_equal(ci, g["ci"])
    assert np.array_equal(a, g["a"])
    f = oracle.load_vector(m)
    assert np.array_equal(f, g["f"])
    x, st, ani, ares = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    # unit traction x 0.02 m thickness gives forces of 1e-2 N: |d.p| falls
    # under the absolute computer zero 1e-30 (scr.cpp:1146) before
    # (r.r)/(f.f) < 1e-20, and the reference leaves with ani = i, ares = r.h
    assert st == 2 and ani == int(g["ani"]) and ares == float(g["ares"])
    assert np.array_equal(x, g["u"])


def test_cr_storage_unpreconditioned_cg(oracle):
    g = load("cr_cantilever.npz")
    m = decks.cantilever_hex(10, 2, 2)
    adr, ci, a = oracle.assemble(m, sym=False)
    assert np.array_equal(adr, g["adr"]) and np.array_equal(ci, g["ci"])
    assert np.array_equal(a, g["a"])
    f = oracle.load_vector(m)
    x, st, ani, ares = oracle.cr_cg_prec(adr, ci, a, f, ni=20000, res=1e-10)
    assert st == 0 and ani == int(g["ani"]) and ares == float(g["ares"])
    assert np.array_equal(x, g["u"])


def test_scr_mxv_equals_dense(oracle):
    g = load("c1_cantilever.npz")
    K = oracle.scr_to_dense(g["adr"], g["ci"], g["a"])
    b = np.random.default_rng(0).standard_normal(K.shape[0])
    assert np.allclose(oracle.scr_mxv(g["adr"], g["ci"], g["a"], b), K @ b, rtol=1e-12,
                       atol=1e-12 * np.abs(K @ b).max())


def test_zero_rhs_and_breakdown_statuses(oracle):
    g = load("c1_cantilever.npz")
    f = np.zeros_like(g["f"])
    x, st, ani, ares = oracle.scr_cg_prec(g["adr"], g["ci"], g["a"], f, ni=100, res=1e-20)
    # the reference reports the zero norm and then leaves on the zero denominator
    assert st == 2 and ani == 0 and ares == 0.0 and not x.any()


def test_iteration_limit_leaves_ani_untouched(oracle):
    g = load("c1_cantilever.npz")
    x, st, ani, ares = oracle.scr_cg_prec(g["adr"], g["ci"], g["a"], g["f"], ni=5, res=1e-20)
    assert st == 1 and ani == -1


def test_trfel_cube_matrices_and_steps(oracle):
    """TRFEL conductivity/capacity (linhext, TRFEL/SRC/linhext.cpp:774/979),
    Dirichlet lifting (globmatt.cpp:1635) and the d-form trapezoid
    (npsolvert.cpp:1071): bit-exact with the compiled reference."""
    g = load("trfel_cube.npz")
    m = decks.heat_cube(4)
    adr, ci, ka = oracle.assemble(m, sym=True, kind="hex8t_k")
    assert np.array_equal(adr, g["K_adr"]) and np.array_equal(ci, g["K_ci"])
    assert np.array_equal(ka, g["K_a"])
    _, _, ca = oracle.assemble(m, sym=True, kind="hex8t_c")
    assert np.array_equal(ca, g["C_a"])
    T1, V1, _ = oracle.trfel_steps(m, 1, float(g["dt"]), iv=1)
    assert np.array_equal(T1, g["T1"]) and np.array_equal(V1, g["V1"])
    T3, V3, its = oracle.trfel_steps(m, 3, float(g["dt"]), iv=1)
    assert np.array_equal(T3, g["T3"]) and np.array_equal(V3, g["V3"])
    assert its[-1][1] == int(g["ani3"])


def test_trfel_stationary(oracle):
    """solve_stationary_problem (TRFEL/SRC/spsolvert.cpp:13): bit-exact."""
    g = load("trfel_stationary.npz")
    m = decks.heat_cube(4, seed=3)
    _, _, ka = oracle.assemble(m, sym=True, kind="hex8t_k")
    assert np.array_equal(ka, g["K_a"])
    x, st, ani, ares = oracle.trfel_stationary(m)
    assert st == 0 and ani == int(g["ani"]) and ares == float(g["ares"])
    assert np.array_equal(x, g["T"])
