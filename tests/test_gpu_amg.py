"""The aggregation multilevel preconditioner (SGPU_PREC_AGG) and the flexible
CG around it.  The preconditioner changes the iteration, not the system: every
solve must reach the solution of the reference's own Jacobi-PCG on the same
inputs (the oracle, solved to a tighter residual) within the tolerance the
FP64 drop-in meets (1e-8 relative in the solution), in far fewer iterations.
"""
import numpy as np
import pytest

from ssf_b200 import decks, gefel, mefel
from ssf_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _oracle_system(oracle, m, kind=None):
    adr, ci, a = oracle.assemble(m, sym=True, kind=kind) if kind else oracle.assemble(m, sym=True)
    return adr, ci, a


@pytest.mark.parametrize("mode", ["mixed", "fp64"])
@pytest.mark.parametrize("dims,res", [((20, 4, 4), 1e-20), ((40, 8, 8), 1e-22)])
def test_cantilever_matches_oracle(oracle, gpu_lib, mode, dims, res):
    m = decks.cantilever_hex(*dims)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    xo, st, ani_jacobi, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    assert st == 0
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        x, r = dm.pcg(f, res=res, prec="agg", mode=mode)
    assert r.status == L.OK
    assert r.ani == r.info["iterations"]
    assert r.info["true_relres"] < 3.0 * np.sqrt(res)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8
    # the point of the preconditioner: a small fraction of the Jacobi iterations
    assert r.info["iterations"] * 3 < ani_jacobi
    assert r.info["precond_levels"] >= 2 and 0 < r.info["precond_coarse_n"] <= 4096


def test_plane_stress_plate(oracle, gpu_lib):
    m = decks.plate_quad(48, 24, E=3e10, nu=0.22)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    xo, st, ani_jacobi, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))  # 3 plane rigid-body modes, scalar CSR level 0
        x, r = dm.pcg(f, res=1e-22, prec="agg", mode="mixed")
    assert r.status == L.OK
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8
    assert r.info["iterations"] * 4 < ani_jacobi


def test_heterogeneous_conduction(oracle, gpu_lib):
    # lognormal conductivity, scalar problem (near-null space: constants)
    m = decks.heat_cube(14, sigma=1.0)
    with mefel.conductivity_matrix(m) as K:
        adr, ci, a = K.download(symmetric=1)
    n = adr.size - 1
    f = np.random.default_rng(7).standard_normal(n)
    xo, st, ani_jacobi, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(np.ones(n))
        for mode in ("mixed", "fp64"):
            x, r = dm.pcg(f, res=1e-22, prec="agg", mode=mode)
            assert r.status == L.OK
            assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8
            assert r.info["iterations"] * 3 < ani_jacobi


def test_translations_only_and_true_criterion(oracle, gpu_lib):
    # no near-null space given: one constant per node component
    m = decks.cantilever_hex(30, 6, 6)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    xo, _, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        x, r = dm.pcg(f, res=1e-11, crit="true", prec="agg", mode="mixed")
    assert r.status == L.OK
    assert r.info["true_relres"] < 1e-11
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


def test_deterministic_and_values_update(oracle, gpu_lib):
    m = decks.cantilever_hex(24, 6, 6)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        x1, r1 = dm.pcg(f, res=1e-20, prec="agg", mode="mixed")
        x2, r2 = dm.pcg(f, res=1e-20, prec="agg", mode="mixed")
        assert np.array_equal(x1, x2) and r1.info["iterations"] == r2.info["iterations"]
        assert r1.info["precond_setup_ms"] > 0.0 and r2.info["precond_setup_ms"] >= 0.0
        # new values on the same pattern rebuild the hierarchy: 2 K -> x / 2
        dm.update_values(2.0 * a)
        x3, r3 = dm.pcg(f, res=1e-20, prec="agg", mode="mixed")
        assert r3.status == L.OK
        assert np.linalg.norm(2.0 * x3 - x1) / np.linalg.norm(x1) <= 1e-8
        # zero right-hand side
        x0, r0 = dm.pcg(np.zeros_like(f), res=1e-20, prec="agg", mode="mixed")
        assert r0.status == L.ZERO_RHS and not np.any(x0)


def test_bad_nullspace_rejected(oracle, gpu_lib):
    m = decks.cantilever_hex(4, 2, 2)
    adr, ci, a = _oracle_system(oracle, m)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        with pytest.raises(L.SgpuError):
            dm.set_nullspace(np.ones((adr.size - 1, 2)))


@pytest.mark.parametrize("mode,nrhs", [("mixed", 5), ("fp64", 40), ("mixed", 70)])
def test_batched_load_cases(oracle, gpu_lib, mode, nrhs):
    # every load case its own flexible CG, all sharing one hierarchy and every
    # kernel: each column must reach the oracle's solution of its own system
    m = decks.cantilever_top_loads(decks.cantilever_hex(24, 6, 6), nrhs, seed=3)
    adr, ci, a = _oracle_system(oracle, m)
    F = np.stack([oracle.load_vector(m, lc) for lc in range(nrhs)], axis=1)
    F[:, 1] = 0.0  # a zero load case stops at once with its own status
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        X, res = gefel.pcg_multi(dm, F, res=1e-22, prec="agg", mode=mode)
    assert res[1].status == L.ZERO_RHS and not np.any(X[:, 1])
    for c in range(nrhs):
        if c == 1:
            continue
        xo, st, _, _ = oracle.scr_cg_prec(adr, ci, a, F[:, c], ni=200000, res=1e-26)
        assert res[c].status == L.OK and res[c].ani is not None
        assert np.linalg.norm(X[:, c] - xo) / np.linalg.norm(xo) <= 1e-8, c


@pytest.mark.parametrize("mode", ["mixed", "fp64"])
def test_uneven_batch(oracle, gpu_lib, mode):
    # independent plates of uneven size in one block-diagonal matrix: every
    # plate its own flexible CG, one shared hierarchy; each plate must reach
    # the oracle's solution of its own system
    plates = decks.plate_batch(12, seed=5, lo=8, hi=40)
    xs, o = mefel.solve_batch(plates, res=1e-22, zero=1e-300, prec="agg", mode=mode)
    assert (o["status"] == 0).all()
    for k, p in enumerate(plates):
        adr, ci, a = oracle.assemble(p, sym=True)
        f = oracle.load_vector(p)
        xo, st, ani_o, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26, zero=1e-300)
        assert np.linalg.norm(xs[k] - xo) / np.linalg.norm(xo) <= 1e-8, k
        assert o["iterations"][k] < ani_o


def test_smoothed_bottom_level(oracle, gpu_lib, monkeypatch):
    # a coarsest level above the dense limit is smoothed instead of inverted
    # (the tuning switch SGPU_AMG sets the limit to 0 here); the solve still
    # reaches the oracle's solution, single and batched
    monkeypatch.setenv("SGPU_AMG", "1,1.7,30,768,2,14,2,0")
    m = decks.cantilever_hex(24, 6, 6)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    xo, _, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        x, r = dm.pcg(f, res=1e-22, prec="agg", mode="mixed")
        assert r.status == L.OK and r.info["precond_coarse_n"] == 0
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8
        X, res = gefel.pcg_multi(dm, np.stack([f, 2.0 * f], axis=1), res=1e-22, prec="agg", mode="mixed")
        assert all(rr.status == L.OK for rr in res)
        assert np.linalg.norm(X[:, 1] - 2.0 * xo) / np.linalg.norm(2.0 * xo) <= 1e-8


@pytest.mark.parametrize("which", ["hex", "plate"])
def test_rigid_body_modes_built_on_device(oracle, gpu_lib, which):
    # sgpu_matrix_set_rigid_body_modes (coordinates and code numbers in, the
    # vectors formed on the device) preconditions like the host-built modes
    m = decks.cantilever_hex(24, 6, 6) if which == "hex" else decks.plate_quad(48, 24, E=3e10, nu=0.22)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    xo, _, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        x1, r1 = dm.pcg(f, res=1e-22, prec="agg", mode="mixed")
        dm.set_rigid_body_modes(m.coords, m.code_numbers())
        x2, r2 = dm.pcg(f, res=1e-22, prec="agg", mode="mixed")
    assert r1.status == L.OK and r2.status == L.OK
    assert abs(r1.info["iterations"] - r2.info["iterations"]) <= 1
    for x in (x1, x2):
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


def _agg_solve(dm, f, mode, tail):
    import os
    old = os.environ.get("SGPU_AMG_TAIL")
    os.environ["SGPU_AMG_TAIL"] = "1" if tail else "0"
    try:
        dm.precond_clear()
        return dm.pcg(f, res=1e-22, prec="agg", mode=mode)
    finally:
        if old is None:
            os.environ.pop("SGPU_AMG_TAIL", None)
        else:
            os.environ["SGPU_AMG_TAIL"] = old


@pytest.mark.parametrize("mode", ["mixed", "fp64"])
@pytest.mark.parametrize("case", ["cantilever", "plate", "conduction"])
def test_fused_coarse_tail_gives_the_same_bits(oracle, gpu_lib, mode, case):
    # the last smoothed level and the dense level below it, run as one
    # cluster launch per coarse correction, must give exactly the result of
    # the separate kernels (same rows, same summation order)
    if case == "cantilever":
        m = decks.cantilever_hex(60, 12, 12)
        adr, ci, a = _oracle_system(oracle, m)
        f = oracle.load_vector(m)
        B = mefel.rigid_body_modes(m)
    elif case == "plate":
        m = decks.plate_quad(96, 48, E=3e10, nu=0.22)
        adr, ci, a = _oracle_system(oracle, m)
        f = oracle.load_vector(m)
        B = mefel.rigid_body_modes(m)
    else:
        m = decks.heat_cube(40, sigma=1.0)
        with mefel.conductivity_matrix(m) as K:
            adr, ci, a = K.download(symmetric=1)
        f = np.random.default_rng(9).standard_normal(adr.size - 1)
        B = np.ones((adr.size - 1, 1))
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(B)
        x0, r0 = _agg_solve(dm, f, mode, tail=False)
        x1, r1 = _agg_solve(dm, f, mode, tail=True)
    assert r0.status == r1.status == L.OK
    assert r1.info["precond_levels"] >= 3, "the hierarchy has no coarse tail to fuse"
    assert r0.info["iterations"] == r1.info["iterations"]
    assert np.array_equal(x0, x1)


def test_overlapped_smoother_bound_gives_the_same_bits(oracle, gpu_lib):
    # the level-0 smoother bound of the FP32 cycle runs on a second stream
    # beside the aggregation set-up; the same Lanczos steps, so the same
    # hierarchy and the same solve as the serial set-up
    import os
    m = decks.cantilever_hex(40, 8, 8)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    out = []
    for serial in (True, False):
        if serial:
            os.environ["SGPU_AMG_SERIAL_BOUND"] = "1"
        try:
            with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
                dm.set_nullspace(mefel.rigid_body_modes(m))
                out.append(dm.pcg(f, res=1e-22, prec="agg", mode="mixed"))
        finally:
            os.environ.pop("SGPU_AMG_SERIAL_BOUND", None)
    (x0, r0), (x1, r1) = out
    assert r0.status == r1.status == L.OK
    assert r0.info["iterations"] == r1.info["iterations"]
    assert np.array_equal(x0, x1)


def _solve_with_env(dm, f, mode, name, value):
    import os
    old = os.environ.get(name)
    if value is None:
        os.environ.pop(name, None)
    else:
        os.environ[name] = value
    try:
        dm.precond_clear()
        return dm.pcg(f, res=1e-22, prec="agg", mode=mode)
    finally:
        if old is None:
            os.environ.pop(name, None)
        else:
            os.environ[name] = old


@pytest.mark.parametrize("case", ["cantilever", "plate", "conduction", "dense_graph"])
def test_galerkin_by_aggregate_rows_matches_the_sort_path(oracle, gpu_lib, case, capfd, monkeypatch):
    # the coarse operators built one aggregate row per warp and by the
    # global key sort are the same sums in another order: the hierarchies
    # agree to rounding, so the solves agree to the solver tolerance.  The
    # dense graph's coarse rows reach more aggregates than one warp's table
    # holds, so there the row pass hands the level to the sort path.
    if case == "cantilever":
        m = decks.cantilever_hex(48, 10, 10)
        adr, ci, a = _oracle_system(oracle, m)
        f = oracle.load_vector(m)
        B = mefel.rigid_body_modes(m)
    elif case == "plate":
        m = decks.plate_quad(48, 24, E=3e10, nu=0.22)
        adr, ci, a = _oracle_system(oracle, m)
        f = oracle.load_vector(m)
        B = mefel.rigid_body_modes(m)
    elif case == "conduction":
        m = decks.heat_cube(30, sigma=1.0)
        with mefel.conductivity_matrix(m) as K:
            adr, ci, a = K.download(symmetric=1)
        f = np.random.default_rng(11).standard_normal(adr.size - 1)
        B = np.ones((adr.size - 1, 1))
    else:
        # graph Laplacian plus the identity: a 128 x 128 five-point grid with
        # 8 random long-range edges per node, so that each small aggregate's
        # rows reach far more aggregates than a coarse row of the table holds
        rng = np.random.default_rng(5)
        side = 128
        n = side * side
        idx = np.arange(n).reshape(side, side)
        e1 = np.concatenate([np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], 1),
                             np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], 1),
                             np.stack([np.repeat(np.arange(n), 8), rng.integers(0, n, 8 * n)], 1)])
        e1 = e1[e1[:, 0] != e1[:, 1]]
        lo, hi = np.minimum(e1[:, 0], e1[:, 1]), np.maximum(e1[:, 0], e1[:, 1])
        pairs = np.unique(hi * n + lo)
        r, c = pairs // n, pairs % n  # row r > column c (lower triangle), sorted by row then column
        w = -rng.uniform(0.5, 1.5, r.size)
        d = 1.0 + np.bincount(r, -w, n) + np.bincount(c, -w, n)
        rr = np.concatenate([r, np.arange(n)])
        cc = np.concatenate([c, np.arange(n)])
        vv = np.concatenate([w, d])
        order = np.lexsort((cc, rr))  # the diagonal ends each row
        ci = cc[order].astype(np.int64)
        a = vv[order]
        adr = np.zeros(n + 1, dtype=np.int64)
        adr[1:] = np.cumsum(np.bincount(rr, minlength=n))
        f = rng.standard_normal(n)
        B = np.ones((n, 1))
    # the reference's solve to a residual below what FP64 reaches (it stops
    # at its iteration floor, as in the tests above): the solution to compare with
    xo, _, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    monkeypatch.setenv("SGPU_AMG_VERBOSE", "1")  # the set-up names the path of each level
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(B)
        x0, r0 = _solve_with_env(dm, f, "mixed", "SGPU_GALERKIN", "sort")
        log0 = capfd.readouterr().err
        x1, r1 = _solve_with_env(dm, f, "mixed", "SGPU_GALERKIN", None)
        log1 = capfd.readouterr().err
        # the by-rows values through the staging kernel instead of the
        # warp-private accumulators (the default where a coarse row fits them)
        x2, r2 = _solve_with_env(dm, f, "mixed", "SGPU_GALERKIN", "staged")
        log2 = capfd.readouterr().err
    assert "galerkin product (sort)" in log0 and "galerkin product (rows)" not in log0
    if case == "dense_graph":
        assert "galerkin product (sort)" in log1  # the row pass handed the level over
    else:
        assert "galerkin product (rows)" in log1 and "galerkin product (sort)" not in log1
        assert "galerkin product (rows)" in log2 and "galerkin product (sort)" not in log2
    assert r0.status == r1.status == r2.status == L.OK
    for r in (r1, r2):
        assert r0.info["precond_levels"] == r.info["precond_levels"]
        assert r0.info["precond_coarse_n"] == r.info["precond_coarse_n"]
        assert abs(r0.info["iterations"] - r.info["iterations"]) <= 1
    for x in (x0, x1, x2):
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


def test_streamed_level0_products_agree(oracle, gpu_lib, monkeypatch):
    # SGPU_LV0_TMA=1: the FP32 level-0 products stream tiles of 32 block rows
    # through shared memory with bulk copies; the same sums per row, so the
    # same solve to rounding (both against the FP32-valued level 0)
    monkeypatch.setenv("SGPU_LV0_H16", "0")
    m = decks.cantilever_hex(60, 12, 12)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    xo, _, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        x0, r0 = _solve_with_env(dm, f, "mixed", "SGPU_LV0_TMA", None)
        x1, r1 = _solve_with_env(dm, f, "mixed", "SGPU_LV0_TMA", "1")
    assert r0.status == r1.status == L.OK
    assert abs(r0.info["iterations"] - r1.info["iterations"]) <= 1
    for x in (x0, x1):
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


def test_device_loop_and_chunked_iterations_agree(oracle, gpu_lib):
    # the flexible CG's iterations as one graph with a device-side WHILE node
    # against graphs of 8 iterations with a host test between them: the same
    # kernels in the same order, so the same bits and iteration count
    m = decks.cantilever_hex(40, 8, 8)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        for crit in (None, "true"):
            out = []
            for loop in (None, "chunk"):
                import os
                old = os.environ.get("SGPU_FCG_LOOP")
                if loop is None:
                    os.environ.pop("SGPU_FCG_LOOP", None)
                else:
                    os.environ["SGPU_FCG_LOOP"] = loop
                try:
                    kw = {"crit": crit} if crit else {}
                    out.append(dm.pcg(f, res=1e-11 if crit else 1e-22, prec="agg", mode="mixed", **kw))
                finally:
                    if old is None:
                        os.environ.pop("SGPU_FCG_LOOP", None)
                    else:
                        os.environ["SGPU_FCG_LOOP"] = old
            (x0, r0), (x1, r1) = out
            assert r0.status == r1.status == L.OK
            assert r0.info["iterations"] == r1.info["iterations"]
            assert np.array_equal(x0, x1)


@pytest.mark.parametrize("shape", [None, "4,1", "4,2", "8,2"])
def test_half_precision_level0_values(oracle, gpu_lib, shape, monkeypatch):
    # the FP32 cycle's level 0 with binary16 values (the default for 3x3
    # block rows) against FP32 values (SGPU_LV0_H16=0): the preconditioner
    # changes by a rounding of 2^-11, the flexible CG's FP64 residual and
    # update do not, so both reach the oracle's solution within the FP64
    # drop-in's 1e-8 in about the same number of iterations; every lane shape
    # of the half-precision product does too
    if shape:
        monkeypatch.setenv("SGPU_LV0_H16_SHAPE", shape)
    m = decks.cantilever_hex(60, 12, 12)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    xo, _, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        x16, r16 = _solve_with_env(dm, f, "mixed", "SGPU_LV0_H16", None)
        x32, r32 = _solve_with_env(dm, f, "mixed", "SGPU_LV0_H16", "0")
        # a second set-up on the same handle converts the values again
        x16b, r16b = _solve_with_env(dm, f, "mixed", "SGPU_LV0_H16", None)
    assert r16.status == r32.status == r16b.status == L.OK
    assert r16.info["iterations"] <= r32.info["iterations"] + 2
    assert np.array_equal(x16, x16b)
    assert not np.array_equal(x16, x32)  # the half-precision product really ran
    for x in (x16, x32):
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


@pytest.mark.parametrize("case", ["cantilever", "plate"])
def test_cluster_independent_set_gives_the_same_bits(oracle, gpu_lib, case):
    # graphs of up to 2048 nodes (the default), of up to 32768 nodes
    # (SGPU_MIS=cluster) or none (SGPU_MIS=rounds) run all their
    # independent-set rounds in one thread-block cluster launch; the same
    # keys, maxima and decisions as the separate launches per pass (which
    # skip the nodes that take no part in a pass), so the same aggregates,
    # hierarchy and solve to the bit
    if case == "cantilever":
        m = decks.cantilever_hex(40, 8, 8)
    else:
        m = decks.plate_quad(48, 24, E=3e10, nu=0.22)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        x0, r0 = _solve_with_env(dm, f, "mixed", "SGPU_MIS", "rounds")
        x1, r1 = _solve_with_env(dm, f, "mixed", "SGPU_MIS", "cluster")
        x2, r2 = _solve_with_env(dm, f, "mixed", "SGPU_MIS", None)
    assert r0.status == r1.status == r2.status == L.OK
    assert r0.info["iterations"] == r1.info["iterations"] == r2.info["iterations"]
    assert r0.info["precond_coarse_n"] == r1.info["precond_coarse_n"] == r2.info["precond_coarse_n"]
    assert np.array_equal(x0, x1)
    assert np.array_equal(x0, x2)


@pytest.mark.parametrize("case", ["cantilever", "plate", "conduction"])
def test_pipelined_galerkin_gives_the_same_bits(oracle, gpu_lib, case):
    # the coarse operators' row walk with the next chunk's loads in flight
    # (the default) against the walk one chunk after another
    # (SGPU_GALERKIN=plain): the same sums in the same order, so the same
    # hierarchy and solve to the bit (3x3 blocks with six modes, scalar rows
    # with three, scalar rows with one)
    if case == "cantilever":
        m = decks.cantilever_hex(40, 8, 8)
        adr, ci, a = _oracle_system(oracle, m)
        f = oracle.load_vector(m)
        B = mefel.rigid_body_modes(m)
    elif case == "plate":
        m = decks.plate_quad(48, 24, E=3e10, nu=0.22)
        adr, ci, a = _oracle_system(oracle, m)
        f = oracle.load_vector(m)
        B = mefel.rigid_body_modes(m)
    else:
        m = decks.heat_cube(24, sigma=1.0)
        with mefel.conductivity_matrix(m) as K:
            adr, ci, a = K.download(symmetric=1)
        f = np.random.default_rng(11).standard_normal(adr.size - 1)
        B = np.ones((adr.size - 1, 1))
    xo, _, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(B)
        for mode in ("mixed", "fp64"):
            x0, r0 = _solve_with_env(dm, f, mode, "SGPU_GALERKIN", None)
            x1, r1 = _solve_with_env(dm, f, mode, "SGPU_GALERKIN", "plain")
            assert r0.status == r1.status == L.OK
            assert r0.info["precond_levels"] == r1.info["precond_levels"] > 1
            assert r0.info["iterations"] == r1.info["iterations"]
            assert np.array_equal(x0, x1)
            assert np.linalg.norm(x1 - xo) / np.linalg.norm(xo) <= 1e-8


@pytest.mark.parametrize("case", ["cantilever", "plate"])
def test_cluster_gauss_jordan_gives_the_same_bits(oracle, gpu_lib, case):
    # the coarsest level's blocked Gauss-Jordan inverse in one thread-block
    # cluster launch (SGPU_GJ=cluster) against four launches per pivot block:
    # the same expressions in the same order, so the same inverse, hierarchy
    # and solve to the bit
    if case == "cantilever":
        m = decks.cantilever_hex(40, 8, 8)
    else:
        m = decks.plate_quad(48, 24, E=3e10, nu=0.22)
    adr, ci, a = _oracle_system(oracle, m)
    f = oracle.load_vector(m)
    xo, _, _, _ = oracle.scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-26)
    with gefel.DeviceMatrix(adr, ci, a, 1) as dm:
        dm.set_nullspace(mefel.rigid_body_modes(m))
        for mode in ("mixed", "fp64"):
            x0, r0 = _solve_with_env(dm, f, mode, "SGPU_GJ", None)
            x1, r1 = _solve_with_env(dm, f, mode, "SGPU_GJ", "cluster")
            assert r0.status == r1.status == L.OK
            assert r0.info["precond_coarse_n"] == r1.info["precond_coarse_n"] > 0
            assert r0.info["iterations"] == r1.info["iterations"]
            assert np.array_equal(x0, x1)
            assert np.linalg.norm(x1 - xo) / np.linalg.norm(xo) <= 1e-8
