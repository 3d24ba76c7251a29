"""SIFEL's own front end with the GPU solver linked in (the link-time
drop-in binding, ssf_b200/integration/sifel_gpu_shim.cpp): a deck in SIFEL's
input format runs unchanged through the compiled reference pipeline; only
symcomprow::cg_prec is replaced at link time by the C-ABI call.  Compared with the all-CPU reference run."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from ssf_b200 import decks

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def _run(exe, deck, env_extra=None):
    from oracle import oracle as O
    td = tempfile.mkdtemp()
    env = dict(os.environ, **(env_extra or {}))
    with open(os.path.join(td, "run.log"), "w") as log:
        rc = subprocess.run([os.path.join(REF, exe), deck, "."], cwd=td, stdout=log, stderr=subprocess.STDOUT,
                            env=env, timeout=300).returncode
    if rc != 0:
        tail = open(os.path.join(td, "run.log"), errors="replace").read()[-2000:]
        raise AssertionError(f"{exe} exited with {rc}; the end of its output:\n{tail}")
    return O.read_dump(td)


@pytest.fixture(scope="module")
def bins(gpu_lib):
    for exe in ("mefel_dump", "mefel_dump_gpu", "trfel_dump", "trfel_dump_gpu"):
        if not os.path.exists(os.path.join(REF, exe)):
            pytest.fail(f"{exe} not built (python oracle/build_ref.py)")
    return REF


@pytest.mark.parametrize("case", ["cantilever", "plate"])
def test_unchanged_deck_runs_with_gpu_solver(bins, case):
    if case == "cantilever":
        m = decks.cantilever_hex(20, 4, 4)
    else:
        m = decks.plate_quad(30, 12, E=3e10, nu=0.22, traction=1e6)
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "deck.in")
        decks.write_mefel_deck(m, deck)
        cpu = _run("mefel_dump", deck)
        gpu = _run("mefel_dump_gpu", deck)
        off = _run("mefel_dump_gpu", deck, {"SIFEL_GPU": "off"})
        cpu_asm = _run("mefel_dump_gpu", deck, {"SIFEL_GPU_ASSEMBLY": "off"})
    # the front end produced the same system: the hexahedral stiffness matrix
    # comes from the GPU assembly binding (same pattern, values to rounding),
    # the plate's from SIFEL's own element loop (no GPU form for it there)
    assert np.array_equal(cpu["K_adr"], gpu["K_adr"]) and np.array_equal(cpu["K_ci"], gpu["K_ci"])
    assert np.allclose(gpu["K_a"], cpu["K_a"], rtol=1e-12, atol=1e-12 * np.abs(cpu["K_a"]).max())
    assert np.array_equal(cpu["K_a"], cpu_asm["K_a"]) and np.array_equal(cpu["f"], gpu["f"])
    if case == "plate":
        assert np.array_equal(cpu["K_a"], gpu["K_a"])
    u_c, u_g = cpu["u"], gpu["u"]
    assert np.linalg.norm(u_g - u_c) / np.linalg.norm(u_c) <= 1e-8
    assert abs(gpu["meta"]["ani_0"] - cpu["meta"]["ani_0"]) <= 2
    # with the GPU switched off the binding calls the reference routine itself
    assert np.array_equal(off["u"], u_c) and off["meta"]["ani_0"] == cpu["meta"]["ani_0"]


@pytest.mark.parametrize("env", ["agg", "agg64"])
def test_unchanged_deck_with_aggregation_preconditioner(bins, env):
    # SIFEL_GPU=agg: the flexible CG with the aggregation preconditioner (its
    # near-null space from MEFEL's topology), a different iteration from the
    # reference's, so both runs solve to a tighter threshold (1e-24 on
    # (r.r)/(f.f)) and the solutions are compared
    m = decks.cantilever_hex(30, 6, 6)
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "deck.in")
        decks.write_mefel_deck(m, deck, res=1e-24)
        cpu = _run("mefel_dump", deck)
        gpu = _run("mefel_dump_gpu", deck, {"SIFEL_GPU": env})
    u_c, u_g = cpu["u"], gpu["u"]
    assert np.linalg.norm(u_g - u_c) / np.linalg.norm(u_c) <= 1e-8
    assert 0 < gpu["meta"]["ani_0"] < cpu["meta"]["ani_0"] / 3


def test_stiffness_matrix_binding_on_a_distorted_multi_material_mesh(bins):
    # stiffness_matrix wrapped at link time: SIFEL's own front end, the matrix
    # from sgpu_assemble copied into its symcomprow storage (three materials,
    # distorted elements), the solve through the solver binding; compared
    # with the all-CPU run on K and u
    m = decks.cantilever_hex(9, 3, 2)
    rng = np.random.default_rng(61)
    inner = ~np.isclose(m.coords[:, 0], 0.0)
    m.coords = m.coords.copy()
    m.coords[inner] += rng.uniform(-0.01, 0.01, (inner.sum(), 3))
    m.emat = np.arange(m.ne) % 3
    m.mats = np.array([[210e9, 0.3], [70e9, 0.33], [30e9, 0.2]])
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "deck.in")
        decks.write_mefel_deck(m, deck, res=1e-22)
        cpu = _run("mefel_dump", deck)
        gpu = _run("mefel_dump_gpu", deck)
    assert np.array_equal(cpu["K_adr"], gpu["K_adr"]) and np.array_equal(cpu["K_ci"], gpu["K_ci"])
    assert np.allclose(gpu["K_a"], cpu["K_a"], rtol=1e-12, atol=1e-12 * np.abs(cpu["K_a"]).max())
    assert np.linalg.norm(gpu["u"] - cpu["u"]) / np.linalg.norm(cpu["u"]) <= 1e-8


@pytest.mark.parametrize("form", ["d", "v"])
def test_unchanged_trfel_deck_runs_with_gpu_solver(bins, form):
    # SIFEL's own TRFEL front end (trfel_init, solve_trfel_problem: the
    # generalized trapezoid of linear_nonstat_solv_dform / vform, TRFEL/SRC/
    # npsolvert.cpp) with every time step's symcomprow::cg_prec on the GPU
    m = decks.heat_cube(8, seed=5)
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "deck.in")
        decks.write_trfel_deck(m, deck, dt=2000.0, nsteps=6, alpha=0.5 if form == "v" else 1.0, res=1e-22,
                               rho=1.0, form=form)
        cpu = _run("trfel_dump", deck)
        gpu = _run("trfel_dump_gpu", deck)
        off = _run("trfel_dump_gpu", deck, {"SIFEL_GPU": "off"})
    # the same matrices from the same front end; the temperatures of every
    # step come from the GPU solve
    assert np.array_equal(cpu["K_a"], gpu["K_a"]) and np.array_equal(cpu["C_a"], gpu["C_a"])
    for key in ("T", "V"):
        c, g = cpu[key], gpu[key]
        assert np.linalg.norm(g - c) / np.linalg.norm(c) <= 1e-8, key
    assert np.array_equal(off["T"], cpu["T"])
