"""Regenerate the golden fixtures in tests/golden/ from the compiled SIFEL
reference (oracle/_ref, built from the reference sources by
oracle/build_ref.py).

Every fixture is the reference's own output on a generated deck in SIFEL's
positional input format, run through the reference pipeline by the harnesses
oracle/ref_harness_mefel.cpp / ref_harness_trfel.cpp:

  c1_cantilever.npz   20x4x4 hex8 cantilever, SCR + Jacobi-PCG (the small case
                      of the benchmark set): SCR K, f, u, ani, ares
  hex8_single.npz     one distorted linear hexahedron, no constraints: K = Ke
  quad4_plate.npz     6x4 distorted plane-stress plate, 2 materials: K, f, u
  cr_cantilever.npz   10x2x2 cantilever, CR storage + unpreconditioned CG
                      (the reference's comprow::cg_prec path): K, f, u
  trfel_cube.npz      4^3 heat cube, lognormal k, T = 1 on x = 0, implicit
                      Euler: K, C and T after 1 and 3 steps
  tet4_cantilever.npz 5x2x2 distorted cantilever of linear tetrahedra (lintet,
                      element type 100), 2 materials, SCR + Jacobi-PCG:
                      coordinates, elements, K, f, u, ani, ares
  tri3_plate.npz      6x4 distorted plane-stress plate of constant-strain
                      triangles (planeelemlt, type 20), 2 materials: K, f, u
  hex20_cantilever.npz, quad8_plate.npz
                      the serendipity elements (quadhex, type 103;
                      planeelemqq, type 24), distorted, 2 materials: K, f, u
  reference_iterations.json
                      iteration counts and solve times of full reference runs
                      on the benchmark cantilevers (used by bench.py to scale
                      its bounded CPU sample to a full solve)

Usage: python tests/golden/make_golden.py [--big] [--elements]   (--big adds
the 1.01M-DOF run, about 2-3 minutes of CPU; --elements writes only the
tet4, tri3, hex20 and quad8 fixtures)
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from ssf_b200 import decks  # noqa: E402


def run(mesh, tag, **deck_kw):
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, f"{tag}.in")
        decks.write_mefel_deck(mesh, deck, **deck_kw)
        return O.run_mefel_dump(deck, td)


def tet4_fixture():
    t = decks.cantilever_tet(5, 2, 2)
    rng = np.random.default_rng(13)
    inner = ~np.isclose(t.coords[:, 0], 0.0)
    t.coords[inner] += rng.uniform(-0.01, 0.01, (int(inner.sum()), 3))
    t.emat = (np.arange(t.ne) % 2).astype(np.int64)
    t.mats = np.array([[210e9, 0.3], [70e9, 0.33]])
    d = run(t, "tet4")
    np.savez_compressed(os.path.join(HERE, "tet4_cantilever.npz"), coords=t.coords, elems=t.elems, emat=t.emat,
                        mats=t.mats, dofflag=t.dofflag, loads=t.loads, adr=d["K_adr"], ci=d["K_ci"], a=d["K_a"],
                        f=d["f"], u=d["u"], ani=d["meta"]["ani_0"], ares=d["meta"]["ares_0"])


def tri3_fixture():
    q = decks.plate_tri(6, 4, E=3.0e10, nu=0.22, t=0.02)
    rng = np.random.default_rng(14)
    q.coords[:, :2] += rng.uniform(-0.15, 0.15, (q.nn, 2))
    q.emat = (np.arange(q.ne) % 2).astype(np.int64)
    q.mats = np.array([[3.0e10, 0.22], [7.0e10, 0.31]])
    d = run(q, "tri3")
    np.savez_compressed(os.path.join(HERE, "tri3_plate.npz"), coords=q.coords, elems=q.elems, emat=q.emat,
                        mats=q.mats, thick=q.thick, dofflag=q.dofflag, loads=q.loads, adr=d["K_adr"],
                        ci=d["K_ci"], a=d["K_a"], f=d["f"], u=d["u"], ani=d["meta"]["ani_0"],
                        ares=d["meta"]["ares_0"])


def serendipity_fixtures():
    h = decks.cantilever_hex20(4, 2, 2)
    inner = ~np.isclose(h.coords[:, 0], 0.0)
    h.coords[inner] += np.random.default_rng(15).uniform(-0.004, 0.004, (int(inner.sum()), 3))
    q = decks.plate_quad8(5, 4, E=3.0e10, nu=0.22, t=0.02)
    q.coords[:, :2] += np.random.default_rng(16).uniform(-0.1, 0.1, (q.nn, 2))
    for m, name in ((h, "hex20_cantilever"), (q, "quad8_plate")):
        m.emat = (np.arange(m.ne) % 2).astype(np.int64)
        m.mats = np.array([[m.mats[0, 0], m.mats[0, 1]], [0.5 * m.mats[0, 0], 0.27]])
        d = run(m, name)
        extra = {"thick": m.thick} if m.thick is not None else {}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), coords=m.coords, elems=m.elems, emat=m.emat,
                            mats=m.mats, dofflag=m.dofflag, loads=m.loads, adr=d["K_adr"], ci=d["K_ci"],
                            a=d["K_a"], f=d["f"], u=d["u"], ani=d["meta"]["ani_0"], ares=d["meta"]["ares_0"],
                            **extra)


def main(big=False, elements_only=False):
    if not O.ref_available():
        raise SystemExit("build the reference first: python oracle/build_ref.py")
    tet4_fixture()
    tri3_fixture()
    serendipity_fixtures()
    if elements_only:
        return
    out = {}

    m = decks.cantilever_hex(20, 4, 4)
    d = run(m, "c1")
    np.savez_compressed(os.path.join(HERE, "c1_cantilever.npz"), adr=d["K_adr"], ci=d["K_ci"], a=d["K_a"],
                        f=d["f"], u=d["u"], ani=d["meta"]["ani_0"], ares=d["meta"]["ares_0"])
    out["cantilever_20x4x4"] = {"n": d["meta"]["n"], "iterations": d["meta"]["ani_0"],
                                "t_solve_s": d["meta"]["t_solve_0"]}

    # one distorted hexahedron, every DOF free
    h = decks.cantilever_hex(1, 1, 1, L=1.0, B=0.8, H=0.6, E=150e9, nu=0.27)
    rng = np.random.default_rng(11)
    h.coords = h.coords + rng.uniform(-0.1, 0.1, h.coords.shape)
    h.dofflag[:] = 1
    h.loads[:] = 0.0
    h.loads[0, 0, 2] = -1.0  # one nodal load so the deck has a load case
    d = run(h, "hex1", ni=10)
    np.savez_compressed(os.path.join(HERE, "hex8_single.npz"), coords=h.coords, elems=h.elems, E=150e9, nu=0.27,
                        adr=d["K_adr"], ci=d["K_ci"], a=d["K_a"])

    # distorted quad plate with two materials
    q = decks.plate_quad(6, 4, E=3.0e10, nu=0.22, t=0.02)
    rng = np.random.default_rng(12)
    q.coords[:, :2] += rng.uniform(-0.15, 0.15, (q.nn, 2))
    q.emat = (np.arange(q.ne) % 2).astype(np.int64)
    q.mats = np.array([[3.0e10, 0.22], [7.0e10, 0.31]])
    d = run(q, "quad")
    np.savez_compressed(os.path.join(HERE, "quad4_plate.npz"), coords=q.coords, elems=q.elems, emat=q.emat,
                        mats=q.mats, thick=q.thick, dofflag=q.dofflag, loads=q.loads, adr=d["K_adr"],
                        ci=d["K_ci"], a=d["K_a"], f=d["f"], u=d["u"], ani=d["meta"]["ani_0"],
                        ares=d["meta"]["ares_0"])

    # CR storage, unpreconditioned CG (comprow::cg_prec with noprecond)
    c = decks.cantilever_hex(10, 2, 2)
    d = run(c, "cr", storage=10, precond=0, res=1e-10)
    np.savez_compressed(os.path.join(HERE, "cr_cantilever.npz"), adr=d["K_adr"], ci=d["K_ci"], a=d["K_a"],
                        f=d["f"], u=d["u"], ani=d["meta"]["ani_0"], ares=d["meta"]["ares_0"])

    # TRFEL: 4^3 heat cube, lognormal conductivity per element, T = 1 on x = 0,
    # implicit Euler, dt = 10 s: K, C and (T, V) after 1 and 3 steps
    cube = decks.heat_cube(4)
    res = {}
    for nsteps in (1, 3):
        with tempfile.TemporaryDirectory() as td:
            deck = os.path.join(td, "cube.in")
            decks.write_trfel_deck(cube, deck, dt=10.0, nsteps=nsteps)
            dd = O.run_trfel_dump(deck, td)
        res[nsteps] = dd
    d1, d3 = res[1], res[3]
    np.savez_compressed(os.path.join(HERE, "trfel_cube.npz"), K_adr=d3["K_adr"], K_ci=d3["K_ci"], K_a=d3["K_a"],
                        C_adr=d3["C_adr"], C_ci=d3["C_ci"], C_a=d3["C_a"], T1=d1["T"], V1=d1["V"], T3=d3["T"],
                        V3=d3["V"], ani3=d3["meta"]["ani"], dt=10.0)

    # TRFEL stationary conduction on the same kind of cube (solve_stationary_problem)
    cube_s = decks.heat_cube(4, seed=3)
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "st.in")
        decks.write_trfel_deck(cube_s, deck, stationary=True)
        ds = O.run_trfel_dump(deck, td)
    np.savez_compressed(os.path.join(HERE, "trfel_stationary.npz"), K_a=ds["K_a"], T=ds["T"], ani=ds["meta"]["ani"],
                        ares=ds["meta"]["ares"])

    for (nx, ny, nz), key in (((100, 20, 20), "cantilever_100x20x20"),) + (
            (((200, 40, 40), "cantilever_200x40x40"),) if big else ()):
        d = run(decks.cantilever_hex(nx, ny, nz), key)
        out[key] = {"n": d["meta"]["n"], "iterations": d["meta"]["ani_0"], "t_solve_s": d["meta"]["t_solve_0"],
                    "t_stiffness_s": d["meta"]["t_stiffness"]}
        print(key, out[key], flush=True)

    path = os.path.join(HERE, "reference_iterations.json")
    old = {}
    if os.path.exists(path):
        with open(path) as fh:
            old = json.load(fh)
    old.update(out)
    with open(path, "w") as fh:
        json.dump(old, fh, indent=1, sort_keys=True)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(big="--big" in sys.argv, elements_only="--elements" in sys.argv)
