"""GPU parity of the drop-in solvers against the oracle (CPU restatement of
GEFEL's CG routines) and the committed golden fixtures."""
import numpy as np
import pytest

from ssf_b200 import decks, gefel
from ssf_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _system(oracle, nx=20, ny=4, nz=4, sym=True):
    m = decks.cantilever_hex(nx, ny, nz)
    adr, ci, a = oracle.assemble(m, sym=sym)
    f = oracle.load_vector(m)
    return m, adr, ci, a, f


def test_scr_spmv_matches_oracle(oracle, gpu_lib):
    m, adr, ci, a, f = _system(oracle)
    rng = np.random.default_rng(0)
    b = rng.standard_normal(adr.size - 1)
    ref = oracle.scr_mxv(adr, ci, a, b)
    got = gefel.symcomprow(adr, ci, a).mxv_scr(b)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_cr_spmv_matches_oracle(oracle, gpu_lib):
    m, adr, ci, a, f = _system(oracle, sym=False)
    b = np.random.default_rng(1).standard_normal(adr.size - 1)
    ref = oracle.cr_mxv(adr, ci, a, b)
    got = gefel.comprow(adr, ci, a).mxv_cr(b)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_scr_cg_prec_fp64_parity(oracle, gpu_lib):
    m, adr, ci, a, f = _system(oracle)
    xo, st, ani_o, ares_o = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert st == 0
    x = np.zeros_like(f)
    r = gefel.symcomprow(adr, ci, a).cg_prec(x, f, 20000, 1e-20)
    assert r.status == L.OK
    # same iteration within rounding of the dot products
    assert abs(r.ani - ani_o) <= 2
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8
    assert r.info["true_relres"] < 1e-9


def test_scr_cg_prec_mixed_parity(oracle, gpu_lib):
    m, adr, ci, a, f = _system(oracle)
    xo, st, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-24)
    x = np.zeros_like(f)
    r = gefel.symcomprow(adr, ci, a).cg_prec(x, f, 20000, 1e-20, mode="mixed")
    assert r.status == L.OK
    assert r.info["true_relres"] < 1e-10
    # solution error against a tight FP64 oracle solve: the refined mixed form
    # reaches the same relative residual, so its error is bounded alike
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-7
    assert r.info["refinements"] >= 2


def test_cr_cg_noprec_parity(oracle, gpu_lib):
    m, adr, ci, a, f = _system(oracle, nx=10, ny=2, nz=2, sym=False)
    xo, st, ani_o, ares_o = oracle.cr_cg_prec(adr, ci, a, f, ni=20000, res=1e-10)
    assert st == 0
    x = np.zeros_like(f)
    r = gefel.comprow(adr, ci, a).cg_prec(x, f, 20000, 1e-10)
    assert r.status == L.OK
    assert abs(r.ani - ani_o) <= 2
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


def test_hex8_assembly_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import mefel
    m = decks.cantilever_hex(6, 3, 2)
    # distort the nodes so every element differs
    rng = np.random.default_rng(3)
    m.coords = m.coords + rng.uniform(-0.01, 0.01, m.coords.shape)
    m.emat = np.arange(m.ne) % 2
    m.mats = np.array([[210e9, 0.3], [70e9, 0.25]])
    adr, ci, a = oracle.assemble(m, sym=True)
    with mefel.stiffness_matrix(m) as K:
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, adr) and np.array_equal(g_ci, ci)
    assert np.allclose(g_a, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


def test_quad4_assembly_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import mefel
    m = decks.plate_quad(7, 5, E=3e10, nu=0.22)
    rng = np.random.default_rng(4)
    m.coords[:, :2] += rng.uniform(-0.1, 0.1, (m.nn, 2))
    adr, ci, a = oracle.assemble(m, sym=True)
    with mefel.stiffness_matrix(m) as K:
        g_adr, g_ci, g_a = K.download(symmetric=1)
    assert np.array_equal(g_adr, adr) and np.array_equal(g_ci, ci)
    assert np.allclose(g_a, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


def test_hex8t_assembly_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import mefel
    m = decks.heat_cube(4)
    rng = np.random.default_rng(5)
    m.coords = m.coords + rng.uniform(-0.02, 0.02, m.coords.shape)
    for kind, fn in (("hex8t_k", mefel.conductivity_matrix), ("hex8t_c", mefel.capacity_matrix)):
        adr, ci, a = oracle.assemble(m, sym=True, kind=kind)
        with fn(m) as K:
            g_adr, g_ci, g_a = K.download(symmetric=1)
        assert np.array_equal(g_adr, adr) and np.array_equal(g_ci, ci)
        assert np.allclose(g_a, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


def test_linear_statics_end_to_end(oracle, gpu_lib):
    from ssf_b200 import mefel
    m = decks.cantilever_hex(20, 4, 4)
    adr, ci, a = oracle.assemble(m, sym=True)
    f = oracle.load_vector(m)
    xo, st, ani_o, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    X, res = mefel.solve_linear_statics(m, res=1e-20)
    assert res[0].status == L.OK
    assert np.linalg.norm(X[0] - xo) / np.linalg.norm(xo) <= 1e-8


@pytest.mark.parametrize("fmt,variant", [(0, 4), (0, 8), (0, 16), (0, 32), (2, 32), (3, 8), (3, 16), (3, 32),
                                         (3, 132), (3, 232), (3, 116), (3, 216), (3, 108), (3, 208)])
def test_every_spmv_kernel_fp64(oracle, gpu_lib, fmt, variant):
    m, adr, ci, a, f = _system(oracle, nx=12, ny=3, nz=3)
    b = np.random.default_rng(7).standard_normal(adr.size - 1)
    ref = oracle.scr_mxv(adr, ci, a, b)
    with gefel.DeviceMatrix(adr, ci, a, 1) as d:
        d.set_spmv(64, fmt, variant)
        got = d.mxv(b)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("fmt,variant", [(0, 4), (0, 8), (0, 16), (0, 32), (3, 8), (3, 16), (3, 32), (3, 132),
                                         (3, 232), (3, 116), (3, 216), (3, 108), (3, 208)])
def test_every_spmv_kernel_fp32_scaled(oracle, gpu_lib, fmt, variant):
    import ctypes
    import torch
    m, adr, ci, a, f = _system(oracle, nx=12, ny=3, nz=3)
    K = oracle.scr_to_dense(adr, ci, a)
    s = 1.0 / np.sqrt(np.diag(K))
    Ah = K * s[:, None] * s[None, :]
    b = np.random.default_rng(8).standard_normal(K.shape[0]).astype(np.float32)
    ref = Ah @ b.astype(np.float64)
    xd = torch.from_numpy(b).cuda()
    yd = torch.empty_like(xd)
    with gefel.DeviceMatrix(adr, ci, a, 1) as d:
        d.set_spmv(32, fmt, variant)
        L.check(L.lib().sgpu_matrix_mxv32_d(d.h, ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr())))
        torch.cuda.synchronize()
    got = yd.cpu().numpy().astype(np.float64)
    # FP32 values and accumulation: a few ulps of the row's magnitude
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("nrhs,sym", [(5, True), (40, True), (7, False)])
def test_batched_load_cases_match_oracle(oracle, gpu_lib, nrhs, sym):
    from ssf_b200.gefel import DeviceMatrix, pcg_multi
    m = decks.cantilever_top_loads(decks.cantilever_hex(12, 3, 3, H=0.2), nrhs, seed=9)
    adr, ci, a = oracle.assemble(m, sym=True)
    F = np.stack([oracle.load_vector(m, lc) for lc in range(nrhs)], axis=1)
    if not sym:  # a matrix without the 3x3 block form takes the CSR product
        adr, ci, a = oracle.assemble(m, sym=False)
        with DeviceMatrix(adr, ci, a, 0) as d:
            X, res = pcg_multi(d, F, res=1e-20)
        sadr, sci, sa = oracle.assemble(m, sym=True)
    else:
        with DeviceMatrix(adr, ci, a, 1) as d:
            X, res = pcg_multi(d, F, res=1e-20)
        sadr, sci, sa = adr, ci, a
    for c in range(nrhs):
        xo, st, ani_o, _ = oracle.scr_cg_prec(sadr, sci, sa, F[:, c], ni=20000, res=1e-20)
        assert st == 0 and res[c].status == L.OK
        assert abs(res[c].ani - ani_o) <= 2
        assert np.linalg.norm(X[:, c] - xo) / np.linalg.norm(xo) <= 1e-8


def test_uneven_batch_matches_oracle(oracle, gpu_lib):
    from ssf_b200 import mefel
    rng = np.random.default_rng(21)
    plates = [decks.plate_quad(int(a), int(b), E=float(e), nu=float(v), traction=1e6)
              for a, b, e, v in zip(rng.integers(3, 12, 9), rng.integers(3, 12, 9), rng.uniform(1e9, 1e11, 9),
                                    rng.uniform(0.2, 0.35, 9))]
    xs, out = mefel.solve_batch(plates, res=1e-20, tune=True)
    for k, p in enumerate(plates):
        adr, ci, a = oracle.assemble(p, sym=True)
        f = oracle.load_vector(p)
        xo, st, ani_o, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
        assert st == 0 and out["status"][k] == L.OK
        assert abs(int(out["ani"][k]) - ani_o) <= 2
        assert np.linalg.norm(xs[k] - xo) / np.linalg.norm(xo) <= 1e-8


@pytest.mark.parametrize("form", ["persistent", "graph"])
def test_uneven_batch_forms_agree(oracle, gpu_lib, form):
    # the persistent form (one CTA per system, no launch per iteration) and
    # the segmented graph form are the same iteration per system: the same
    # statuses, iteration counts within the rounding of the dot products, and
    # the oracle's solutions; one plate carries a zero load (its own
    # zero-right-hand-side exit)
    import os
    from ssf_b200 import mefel
    rng = np.random.default_rng(22)
    plates = [decks.plate_quad(int(a), int(b), E=float(e), nu=float(v), traction=1e6)
              for a, b, e, v in zip(rng.integers(2, 30, 23), rng.integers(2, 30, 23), rng.uniform(1e9, 1e11, 23),
                                    rng.uniform(0.2, 0.35, 23))]
    plates[5].loads = np.zeros_like(plates[5].loads)
    old = os.environ.get("SGPU_BATCH_FORM")
    os.environ["SGPU_BATCH_FORM"] = form
    try:
        xs, out = mefel.solve_batch(plates, res=1e-20, tune=False)
    finally:
        if old is None:
            os.environ.pop("SGPU_BATCH_FORM", None)
        else:
            os.environ["SGPU_BATCH_FORM"] = old
    for k, p in enumerate(plates):
        adr, ci, a = oracle.assemble(p, sym=True)
        f = oracle.load_vector(p)
        xo, st, ani_o, ares_o = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-20)
        if k == 5:
            assert out["status"][k] == L.ZERO_RHS and not xs[k].any() and out["ani"][k] == ani_o == 0
            continue
        assert st == 0 and out["status"][k] == L.OK
        assert abs(int(out["ani"][k]) - ani_o) <= 2
        assert np.linalg.norm(xs[k] - xo) / np.linalg.norm(xo) <= 1e-8


def test_sliced_ell_in_the_solves(oracle, gpu_lib):
    # a scalar conduction matrix (rows of similar length): the sliced ELL
    # SpMV pinned for the FP64 Jacobi-PCG and for the transient steps' combined
    # matrix must reproduce the oracle, and survive a value update (its value
    # copy is refreshed with the CSR's)
    from ssf_b200 import mefel
    m = decks.heat_cube(10, seed=4)
    with mefel.conductivity_matrix(m) as K:
        adr, ci, a = K.download(symmetric=1)
    n = adr.size - 1
    f = np.random.default_rng(9).standard_normal(n)
    xo, st, ani_o, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-20)
    with gefel.DeviceMatrix(adr, ci, a, 1) as d:
        d.set_spmv(64, 2, 32)
        x, r = d.pcg(f, res=1e-20, prec="jacobi", mode="fp64")
        assert r.status == L.OK and abs(r.ani - ani_o) <= 2
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8
        d.update_values(3.0 * a)
        x3, r3 = d.pcg(f, res=1e-20, prec="jacobi", mode="fp64")
        assert np.linalg.norm(3.0 * x3 - xo) / np.linalg.norm(xo) <= 1e-8
    with pytest.raises(L.SgpuError):
        with gefel.DeviceMatrix(adr, ci, a, 1) as d:
            d.set_spmv(32, 2, 32)
