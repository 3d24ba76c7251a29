"""The library's parallel reader of MEFEL positional decks (sgpu_deck_read_mefel):
decks written by ssf_b200.decks come back array for array, the reader agrees
with the reference's own reading (the compiled reference assembles the same
K from the same file), unsupported decks fail naming the record, and on the
GPU a deck runs end to end to the oracle's solution.  The reader is host
code: the CPU tests call no GPU work."""
import os

import numpy as np
import pytest

from ssf_b200 import decks

KINDS = {
    "hex8": lambda: decks.cantilever_hex(5, 2, 2),
    "tet4": lambda: decks.cantilever_tet(3, 2, 2),
    "hex20": lambda: decks.cantilever_hex20(3, 2, 2),
    "quad4": lambda: decks.plate_quad(4, 3),
    "tri3": lambda: decks.plate_tri(4, 3),
    "quad8": lambda: decks.plate_quad8(4, 3),
}


def _ortho(m):
    Dl = decks.orthotropic_local(150e9, 10e9, 9e9, 0.3, 0.28, 0.45, 3.5e9, 5e9, 5.5e9)
    m.mtype = "ortho"
    m.mats = np.array([np.concatenate([Dl.ravel(), decks.rotation(a).ravel()]) for a in ((0, 0, 0), (0.3, -0.5, 0.9))])
    m.emat = np.arange(m.ne) % 2
    return m


def _variants():
    for k, make in KINDS.items():
        yield k, make
    yield "hex8_ortho", lambda: _ortho(decks.cantilever_hex(4, 2, 2))
    yield "tet4_gen3d", lambda: _gen3d(decks.cantilever_tet(3, 2, 2))
    yield "hex8_loadcases", lambda: decks.cantilever_top_loads(decks.cantilever_hex(6, 2, 2), 7, seed=2)
    yield "quad4_tsets", lambda: _tsets(decks.plate_quad(5, 4))


def _gen3d(m):
    Dl = decks.orthotropic_local(150e9, 10e9, 9e9, 0.3, 0.28, 0.45, 3.5e9, 5e9, 5.5e9)
    m.mtype = "gen3d"
    m.mats = np.array([Dl[np.triu_indices(6)]])
    return m


def _tsets(m):
    m.meta["tvals"] = [0.01, 0.03]
    m.meta["tset"] = list(np.arange(m.ne) % 2)
    m.thick = np.array([0.01, 0.03])[np.arange(m.ne) % 2]
    m.mats = np.array([[1e10, 0.25], [3e10, 0.2]])
    m.emat = (np.arange(m.ne) // 3) % 2
    return m


@pytest.mark.parametrize("name,make", list(_variants()))
def test_round_trip(tmp_path, name, make):
    from ssf_b200 import mefel
    m = make()
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    with mefel.Deck(p, threads=3) as d:
        r = d.mesh()
        assert d.info["n"] == m.ndof and d.info["nlc"] == m.loads.shape[0]
        for lc in range(m.loads.shape[0]):
            assert np.array_equal(d.rhs(lc), mefel.mefel_right_hand_side(m, lc))
    assert r.kind == m.kind and r.mtype == m.mtype
    for k in ("coords", "elems", "dofflag", "emat", "loads"):
        assert np.array_equal(getattr(r, k), getattr(m, k)), k
    assert np.array_equal(r.mats, np.asarray(m.mats, dtype=np.float64))
    if m.thick is not None:
        assert np.array_equal(r.thick, m.thick)
    assert np.array_equal(r.code_numbers(), m.code_numbers())


def test_records_in_any_order(tmp_path):
    # node and element records may come in any id order, as the reference
    # indexes them by id
    from ssf_b200 import mefel
    m = decks.cantilever_hex(4, 2, 2)
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    lines = open(p).read().split("\n")
    i0 = 10  # first node record
    nodes = lines[i0:i0 + m.nn]
    rng = np.random.default_rng(1)
    lines[i0:i0 + m.nn] = [nodes[k] for k in rng.permutation(m.nn)]
    ncon = int(lines[i0 + m.nn])
    e0 = i0 + m.nn + 1 + ncon + 1
    el = lines[e0:e0 + m.ne]
    lines[e0:e0 + m.ne] = [el[k] for k in rng.permutation(m.ne)]
    open(p, "w").write("\n".join(lines))
    with mefel.Deck(p) as d:
        r = d.mesh()
    assert np.array_equal(r.coords, m.coords) and np.array_equal(r.elems, m.elems)


@pytest.mark.parametrize("edit,match", [
    (lambda L: L.__setitem__(2, "2"), "problemtype"),
    (lambda L: L.__setitem__(10, L[10].replace(" 3 0 0", " 3 1 0")), "node record 1"),
    (lambda L: L.__setitem__(11, L[10]), "node record"),
    (lambda L: L.__setitem__(-1, "oops"), "integer expected"),
    (lambda L: L.append("7"), "unexpected token"),
])
def test_unsupported_or_broken_decks_fail(tmp_path, edit, match):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.cantilever_hex(3, 2, 2)
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    lines = open(p).read().rstrip("\n").split("\n")
    edit(lines)
    open(p, "w").write("\n".join(lines) + "\n")
    with pytest.raises(L.SgpuError, match=match):
        mefel.Deck(p)


def test_missing_file_fails(tmp_path):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    with pytest.raises(L.SgpuError, match="cannot open"):
        mefel.Deck(str(tmp_path / "absent.in"))


@pytest.mark.parametrize("name", ["hex8", "tet4", "quad8", "hex8_ortho"])
def test_reader_agrees_with_the_reference_reading(oracle, tmp_path, name):
    # the compiled reference reads the same file: its K is the oracle's K of
    # the mesh this reader returns, bit for bit
    from ssf_b200 import mefel
    if not oracle.ref_available():
        pytest.skip("compiled reference (oracle/_ref) not built")
    m = dict(_variants())[name]()
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    d = oracle.run_mefel_dump(p, str(tmp_path), solve=False)
    with mefel.Deck(p) as dk:
        r = dk.mesh()
        f = dk.rhs(0)
    adr, ci, a = oracle.assemble(r, sym=True)
    assert np.array_equal(adr, d["K_adr"]) and np.array_equal(ci, d["K_ci"])
    if name == "quad8":
        assert np.abs(a - d["K_a"]).max() <= 1e-14 * np.abs(d["K_a"]).max()
    else:
        assert np.array_equal(a, d["K_a"])
    assert np.array_equal(f, d["f"][: f.size])


@pytest.mark.gpu
@pytest.mark.parametrize("name,prec", [("hex8", None), ("tet4", None), ("hex8_ortho", "agg"),
                                       ("hex8_loadcases", None)])
def test_deck_end_to_end(oracle, gpu_lib, tmp_path, name, prec):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = dict(_variants())[name]()
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p, res=1e-22)
    X, results, info = mefel.solve_deck(p, prec=prec, mode="fp64")
    adr, ci, a = oracle.assemble(m, sym=True)
    for lc in range(m.loads.shape[0]):
        f = oracle.load_vector(m, lc)
        xo, st, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
        assert results[lc].status == L.OK
        assert np.linalg.norm(X[lc] - xo) / np.linalg.norm(xo) <= 1e-8
    assert info["n"] == m.ndof and info["parse_ms"] > 0.0


# ---------------------------------------------------------------------------
# TRFEL decks
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("stationary,form", [(False, "d"), (False, "v"), (True, "d")])
def test_trfel_round_trip(tmp_path, stationary, form):
    from ssf_b200 import mefel
    m = decks.heat_cube(5, seed=3)
    p = str(tmp_path / "t.in")
    decks.write_trfel_deck(m, p, dt=10.0, nsteps=3, alpha=0.5, stationary=stationary, form=form)
    with mefel.Deck(p, front="trfel", threads=3) as d:
        r = d.mesh()
        info = d.info
    assert info["problem"] == (50 if stationary else 60)
    if not stationary:
        assert info["tform"] == {"d": 1, "v": 2}[form] and info["alpha"] == 0.5
        assert info["dt"] == 10.0 and round((info["t1"] - info["t0"]) / info["dt"]) == 3
    assert np.array_equal(r.coords, m.coords) and np.array_equal(r.elems, m.elems)
    assert np.array_equal(r.dofflag, m.dofflag)
    assert np.array_equal(r.mats[r.emat], m.mats[m.emat])
    assert np.array_equal(r.meta["prescribed"], m.meta["prescribed"])
    assert np.array_equal(r.meta["rho"], np.ones(m.ne))


def test_trfel_reader_agrees_with_the_reference_reading(oracle, tmp_path):
    from ssf_b200 import mefel
    if not oracle.ref_available():
        pytest.skip("compiled reference (oracle/_ref) not built")
    m = decks.heat_cube(4, seed=11)
    p = str(tmp_path / "t.in")
    decks.write_trfel_deck(m, p, dt=25.0, nsteps=2, alpha=0.5)
    d = oracle.run_trfel_dump(p, str(tmp_path))
    with mefel.Deck(p, front="trfel") as dk:
        r = dk.mesh()
    _, _, ka = oracle.assemble(r, sym=True, kind="hex8t_k")
    _, _, ca = oracle.assemble(r, sym=True, kind="hex8t_c", rho=r.meta["rho"])
    assert np.array_equal(ka, d["K_a"]) and np.array_equal(ca, d["C_a"])
    T, V, _ = oracle.trfel_steps(r, 2, 25.0, alpha=0.5, iv=1, rnode=r.meta["rnode"])
    assert np.array_equal(T, d["T"]) and np.array_equal(V, d["V"])


@pytest.mark.gpu
@pytest.mark.parametrize("form,prec", [("d", "jacobi"), ("v", "jacobi"), ("d", "agg")])
def test_trfel_deck_end_to_end(oracle, gpu_lib, tmp_path, form, prec):
    from ssf_b200 import mefel
    m = decks.heat_cube(12, seed=5)
    p = str(tmp_path / "t.in")
    decks.write_trfel_deck(m, p, dt=10.0, nsteps=4, alpha=1.0, res=1e-24, form=form)
    d, v, its, info = mefel.solve_trfel_deck(p, prec=prec, mode="fp64")
    To, Vo, _ = oracle.trfel_steps(m, 4, 10.0, alpha=1.0, res=1e-26, form=form)
    assert info["nsteps"] == 4 and (its > 0).all()
    assert np.linalg.norm(d - To) / np.linalg.norm(To) <= 1e-8
    assert np.linalg.norm(v - Vo) / np.linalg.norm(Vo) <= 1e-6


@pytest.mark.gpu
def test_trfel_stationary_deck_end_to_end(oracle, gpu_lib, tmp_path):
    from ssf_b200 import mefel
    m = decks.heat_cube(10, seed=6)
    p = str(tmp_path / "s.in")
    decks.write_trfel_deck(m, p, stationary=True, res=1e-24)
    x, _, its, info = mefel.solve_trfel_deck(p)
    xo, st, _, _ = oracle.trfel_stationary(m, res=1e-26)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


def test_crlf_tabs_and_exponents(tmp_path):
    # the positional format is token based: CR LF line ends, tabs, upper-case
    # exponents and explicit plus signs read as the reference's xfscanf reads them
    from ssf_b200 import mefel
    m = decks.cantilever_hex(3, 2, 2)
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    text = open(p).read()
    lines = text.rstrip("\n").split("\n")
    head, rest = lines[:1], lines[1:]
    rest = [ln.replace(" ", "\t", 1).replace("e-", "E-").replace("e+", "E+") for ln in rest]
    open(p, "w", newline="").write("\r\n".join(head + rest) + "\r\n")
    with mefel.Deck(p) as d:
        r = d.mesh()
        f = d.rhs(0)
    assert np.array_equal(r.coords, m.coords) and np.array_equal(r.elems, m.elems)
    assert np.array_equal(f, mefel.mefel_right_hand_side(m, 0))


def test_integers_with_a_leading_plus(tmp_path):
    # fscanf's %ld (the reference's integer reading) accepts "+5"; a second
    # sign does not make a number
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.cantilever_hex(3, 2, 2)
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    lines = open(p).read().rstrip("\n").split("\n")
    i0 = 10  # first node record: "id x y z ndofn crst transf"
    lines[i0 - 1] = "+" + lines[i0 - 1].strip()  # the node count
    tok = lines[i0].split()
    tok[0], tok[4] = "+" + tok[0], "+" + tok[4]
    lines[i0] = " ".join(tok)
    open(p, "w").write("\n".join(lines) + "\n")
    with mefel.Deck(p) as d:
        r = d.mesh()
    assert np.array_equal(r.coords, m.coords) and np.array_equal(r.elems, m.elems)
    tok[0] = "+-" + tok[0][1:]
    lines[i0] = " ".join(tok)
    open(p, "w").write("\n".join(lines) + "\n")
    with pytest.raises(L.SgpuError, match="node record 1|integer expected"):
        mefel.Deck(p)


def _loaded_decks():
    # element loads and prescribed displacements as a SIFEL deck states them
    hx = decks.cantilever_surface_traction(decks.cantilever_hex(5, 2, 2))
    hx.coords = hx.coords + np.random.default_rng(3).uniform(-0.004, 0.004, hx.coords.shape)
    yield "hex8_surface", hx
    q = decks.plate_quad(5, 4)
    rng = np.random.default_rng(4)
    q.eloads = [[(e, [int(v) for v in rng.integers(0, 2, 4)], rng.standard_normal(16)) for e in range(q.ne)]]
    yield "quad4_edges", q
    p = decks.prescribe(decks.cantilever_hex(4, 2, 2), [0, 1, 2], 2, [1e-4, 2e-4, 3e-4])
    yield "hex8_prescribed", p


@pytest.mark.parametrize("name,m", list(_loaded_decks()))
def test_element_loads_and_prescribed_codes_read_back(oracle, tmp_path, name, m):
    # the reader's right-hand side (nodal + element loads, host code) equals
    # the oracle's loadcase::assemble bit for bit when nothing is prescribed,
    # and the prescribed values come back per DOF
    from ssf_b200 import mefel
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    with mefel.Deck(p, threads=2) as d:
        r = d.mesh()
        assert np.array_equal(r.dofflag, m.dofflag)
        assert np.array_equal(r.code_numbers(), m.code_numbers())
        f = np.zeros(d.view.n)
        from ssf_b200 import _lib as L
        L.check(L.lib().sgpu_deck_rhs(d.h, 0, f))
        rr = np.zeros(d.view.nn * d.view.ndofn)
        import ctypes as C
        cnt = C.c_int64(-1)
        L.check(L.lib().sgpu_deck_prescribed(d.h, 0, rr, C.byref(cnt)))
    want = mefel.prescribed_displacements(m, 0)
    if want is None:
        assert cnt.value == 0 and not rr.any()
        assert np.array_equal(f, oracle.load_vector(m, 0))
    else:
        assert cnt.value == int((m.dofflag < 0).sum()) and np.array_equal(rr, want.reshape(-1))
    # the mesh-level entry point adds the same element loads after the nodal
    # ones (the oracle's order): bit for bit
    if m.eloads and want is None:
        m0 = decks.Mesh(**{**m.__dict__})
        m0.eloads = None
        g = oracle.load_vector(m0, 0)
        mefel._element_loads_into(m, 0, g)
        assert np.array_equal(g, oracle.load_vector(m, 0))


@pytest.mark.parametrize("edit,match", [
    (lambda ln: ln.replace(" 3 1 ", " 3 2 ", 1), "surface flag 2"),
    (lambda ln: ln.replace(" 3 1 ", " 1 1 ", 1), "load type 1"),
])
def test_unsupported_element_loads_fail(tmp_path, edit, match):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.cantilever_surface_traction(decks.cantilever_hex(3, 2, 2))
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    lines = open(p).read().split("\n")
    first = f"{m.eloads[0][0][0] + 1} 3 1 "  # the first loaded-element record: "eid 3 1 values ..."
    k = next(i for i, ln in enumerate(lines) if ln.startswith(first))
    lines[k] = edit(lines[k])
    open(p, "w").write("\n".join(lines))
    with pytest.raises(L.SgpuError, match=match):
        mefel.Deck(p)


def test_prescribed_index_beyond_the_load_case_fails(tmp_path):
    from ssf_b200 import _lib as L
    from ssf_b200 import mefel
    m = decks.prescribe(decks.cantilever_hex(3, 2, 2), [0, 1], 2, [1e-4, 2e-4])
    m.pd = m.pd[:, :1]  # the constraints name value 2, the load case has 1
    p = str(tmp_path / "d.in")
    decks.write_mefel_deck(m, p)
    with pytest.raises(L.SgpuError, match="prescribed displacements"):
        mefel.Deck(p)
