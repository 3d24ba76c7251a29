"""GPU assembly of the hexahedral stiffness matrix in its four forms -- the
default colour-ordered element scatter on the pairs a <= b with the
isotropic P-form, the write-once gather (the 36 blocks a <= b of every
element into a buffer, then one warp per node sums its rows and writes each
entry once; SGPU_HEX8_GATHER=1), the same scatter with the full B^T D B product
(SGPU_HEX8_FULL=1), and rows (one warp per node forming its elements'
blocks; SGPU_ASSEMBLY_ROWS=1) -- against the oracle's
stiffness_matrix (MEFEL/SRC/globmat.cpp:41 with linhex::gl_stiffness_matrix
and symcomprow::localize), and against the default colour-ordered element
scatter: partially constrained nodes (the per-entry search), several
materials, distorted elements, and a node whose rows do not fit the row
kernel (the fallback to the colour-ordered scatter)."""
import os

import numpy as np
import pytest

from ssf_b200 import decks

pytestmark = pytest.mark.gpu


FORMS = {  # name: (SGPU_ASSEMBLY_ROWS, SGPU_HEX8_FULL, SGPU_HEX8_GATHER, SGPU_ASSEMBLY_SLABS)
    "gather": (None, None, "1", None),   # element blocks into a buffer, rows gathered per node
    "rows": ("1", None, None, None),     # one warp per node forms its elements' blocks, rows written once
    "iso": (None, None, None, None),     # colour-ordered, P-form on the pairs a <= b (default)
    "full": (None, "1", None, None),     # colour-ordered, full B^T D B product per block
    "slabs": (None, None, None, "3"),    # colour-ordered within three slabs of element ids
}


def _download(m, form):
    from ssf_b200 import mefel
    names = ("SGPU_ASSEMBLY_ROWS", "SGPU_HEX8_FULL", "SGPU_HEX8_GATHER", "SGPU_ASSEMBLY_SLABS")
    old = {k: os.environ.pop(k, None) for k in names}
    for k, v in zip(names, FORMS[form]):
        if v is not None:
            os.environ[k] = v
    try:
        with mefel.stiffness_matrix(m) as K:
            return K.download(symmetric=1), K.assembly
    finally:
        for k in names:
            os.environ.pop(k, None)
            if old[k] is not None:
                os.environ[k] = old[k]


def _check(oracle, m):
    adr, ci, a = oracle.assemble(m, sym=True)
    tol = 1e-12 * np.abs(a).max()
    out = {}
    for form in FORMS:
        (g_adr, g_ci, g_a), info = _download(m, form)
        assert np.array_equal(g_adr, adr) and np.array_equal(g_ci, ci)
        assert np.allclose(g_a, a, rtol=1e-12, atol=tol), form
        out[form] = g_a
    # the GPU forms differ only in rounding
    for form in ("rows", "full", "gather", "slabs"):
        assert np.allclose(out[form], out["iso"], rtol=1e-13, atol=1e-13 * np.abs(a).max()), form
    # the gather sums the same blocks as the colour-ordered scatter, in
    # ascending element order instead of colour order: rounding apart, equal
    assert np.allclose(out["gather"], out["iso"], rtol=1e-14, atol=1e-14 * np.abs(a).max())
    return out


def test_rows_on_partially_constrained_nodes(oracle, gpu_lib):
    m = decks.cantilever_hex(7, 3, 3)
    rng = np.random.default_rng(11)
    m.coords = m.coords + rng.uniform(-0.008, 0.008, m.coords.shape)
    # x = 0 face: only u fixed; y = 0 face: v fixed; one node fully free on
    # the clamped face, one node with only w free
    df = np.ones_like(m.dofflag)
    df[np.isclose(m.coords[:, 0], 0.0, atol=0.01), 0] = 0
    df[np.isclose(m.coords[:, 1], 0.0, atol=0.01), 1] = 0
    df[5] = (0, 0, 1)
    m.dofflag = df
    m.emat = np.arange(m.ne) % 3
    m.mats = np.array([[210e9, 0.3], [70e9, 0.25], [3e9, 0.45]])
    _check(oracle, m)


def test_rows_fall_back_on_a_node_of_many_elements(oracle, gpu_lib):
    # 40 unit cubes (they overlap in space, which the integration does not
    # mind) that share only their (0,0,0) corner node: that node's rows have
    # 834 entries and it has 40 elements, beyond the row kernel's shared
    # memory; the assembly must fall back to the colour-ordered scatter
    nc = 40
    rng = np.random.default_rng(12)
    coords, elems = [], []
    for k in range(nc):
        # SIFEL node order: n0 (+,+,+), n1 (-,+,+), n2 (-,-,+), n3 (+,-,+), n4..7 with z = -
        corners = [(1, 1, 1), (0, 1, 1), (0, 0, 1), (1, 0, 1), (1, 1, 0), (0, 1, 0), (0, 0, 0), (1, 0, 0)]
        ids = []
        for q, (cx, cy, cz) in enumerate(corners):
            if q == 6:
                ids.append(-1)  # the shared node
                continue
            ids.append(len(coords))
            coords.append(tuple(np.array((cx, cy, cz), dtype=float) + rng.uniform(-0.05, 0.05, 3)))
        elems.append(ids)
    shared = len(coords)
    coords.append((0.0, 0.0, 0.0))
    elems = np.array([[shared if v < 0 else v for v in e] for e in elems], dtype=np.int64)
    coords = np.array(coords, dtype=np.float64)
    nn = coords.shape[0]
    dofflag = np.ones((nn, 3), dtype=np.int64)
    dofflag[:3] = 0
    m = decks.Mesh(kind="hex8", coords=coords, elems=elems, dofflag=dofflag,
                   emat=np.zeros(nc, dtype=np.int64), mats=np.array([[1e9, 0.3]]), loads=np.zeros((1, nn, 3)))
    _check(oracle, m)


def test_rows_match_on_the_cantilever(oracle, gpu_lib):
    m = decks.cantilever_hex(20, 4, 4)
    out = _check(oracle, m)
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "c1_cantilever.npz"))
    assert np.allclose(out["iso"], g["a"], rtol=1e-12, atol=1e-12 * np.abs(g["a"]).max())
