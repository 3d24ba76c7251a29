"""The no-allocation solver entry point against the oracle and the regular drop-in.

sgpu_csr_pcg_noalloc_d serves callers that cannot allocate GPU memory while
they solve (an application whose allocator owns the whole device memory pool,
or one that must not call cudaMalloc/cudaFree because they synchronise the
device).  Its work vectors live in a static device array of the library, so
this test checks, through the C ABI, that two calls in a row (the second
reusing the array the first left behind) give the oracle's solution and the
allocating drop-in sgpu_scr_cg_prec's, within the FP64 parity tolerance used
elsewhere in the tests; that sizes beyond the array, malformed rows and calls
on a capturing stream are refused without touching x; and that a zero
right-hand side ends as the drop-in's does.

This file is collected last on purpose: a run that stops at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from ssf_b200 import _lib as L
from ssf_b200 import decks

pytestmark = pytest.mark.gpu


def _full_csr(adr, ci, a):
    n = adr.size - 1
    rows = np.repeat(np.arange(n), np.diff(adr))
    r = np.concatenate([rows, ci[ci != rows]])
    c = np.concatenate([ci, rows[ci != rows]])
    v = np.concatenate([a, a[ci != rows]])
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    rowptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(rowptr, r + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), c.astype(np.int32), v


def _system(oracle):
    m = decks.cantilever_hex(20, 4, 4)
    adr, ci, a = oracle.assemble(m, sym=True)
    f = oracle.load_vector(m)
    return adr, ci, a, f


def _call(lib, n, rp_d, col_d, val_d, f_d, x_d, iv=0, stream=None):
    ani, ares, its = C.c_int64(-1), C.c_double(-7.0), C.c_int64(0)
    st = lib.sgpu_csr_pcg_noalloc_d(n, C.c_void_p(rp_d.data_ptr()), C.c_void_p(col_d.data_ptr()),
                                    C.c_void_p(val_d.data_ptr()), C.c_void_p(f_d.data_ptr()),
                                    C.c_void_p(x_d.data_ptr()), 20000, 1e-20, 1e-30, iv, stream,
                                    C.byref(ani), C.byref(ares), C.byref(its))
    return st, ani.value, ares.value, its.value


def test_no_alloc_pcg_matches_oracle_and_drop_in_twice(oracle, gpu_lib):
    import torch
    adr, ci, a, f = _system(oracle)
    n = f.size
    lib = L.lib()
    x_o, st_o, ani_o, ares_o = oracle.scr_cg_prec(adr, ci, a, f, ni=20000, res=1e-20)
    assert st_o == 0
    # the allocating drop-in
    x_ref = np.zeros(n)
    ani_r, ares_r = C.c_int64(-1), C.c_double(0.0)
    st = lib.sgpu_scr_cg_prec(n, adr, ci, a, x_ref, f, 20000, 1e-20, C.byref(ani_r), C.byref(ares_r), 1e-30, 0,
                              L.FP64, None)
    assert st == L.OK
    rowptr, col, val = _full_csr(adr, ci, a)
    dev = torch.device("cuda")
    rp_d = torch.from_numpy(rowptr).to(dev)
    col_d = torch.from_numpy(col).to(dev)
    val_d = torch.from_numpy(val).to(dev)
    f_d = torch.from_numpy(f).to(dev)
    for call in range(2):
        # the second call starts from a non-zero x and must still zero it (iv = 0)
        x_d = torch.full((n,), 1.0 if call else 0.0, dtype=torch.float64, device=dev)
        st, ani, ares, its = _call(lib, n, rp_d, col_d, val_d, f_d, x_d)
        assert st == L.OK, L.last_error()
        torch.cuda.synchronize()
        x = x_d.cpu().numpy()
        assert np.linalg.norm(x - x_o) / np.linalg.norm(x_o) <= 1e-8
        assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) <= 1e-8
        assert abs(ani - ani_o) <= 2 and abs(ani - ani_r.value) <= 2 and its == ani + 1
        assert ares == pytest.approx(ares_o, rel=0.5)
    # a start vector (iv = 1) near the solution converges in fewer iterations
    x_d = torch.from_numpy(x_o * (1 + 1e-6)).to(dev)
    st, ani, _, _ = _call(lib, n, rp_d, col_d, val_d, f_d, x_d, iv=1)
    assert st == L.OK and ani < ani_o
    assert np.linalg.norm(x_d.cpu().numpy() - x_o) / np.linalg.norm(x_o) <= 1e-8


def test_no_alloc_zero_rhs_as_the_drop_in(oracle, gpu_lib):
    import torch
    adr, ci, a, f = _system(oracle)
    n = f.size
    lib = L.lib()
    rowptr, col, val = _full_csr(adr, ci, a)
    dev = torch.device("cuda")
    x_ref = np.ones(n)
    ani_r, ares_r = C.c_int64(-1), C.c_double(-7.0)
    st_r = lib.sgpu_scr_cg_prec(n, adr, ci, a, x_ref, np.zeros(n), 20000, 1e-20, C.byref(ani_r), C.byref(ares_r),
                                1e-30, 0, L.FP64, None)
    x_d = torch.ones(n, dtype=torch.float64, device=dev)
    st, ani, ares, _ = _call(lib, n, torch.from_numpy(rowptr).to(dev), torch.from_numpy(col).to(dev),
                             torch.from_numpy(val).to(dev), torch.zeros(n, dtype=torch.float64, device=dev), x_d)
    assert st == st_r == L.ZERO_RHS
    assert (ani, ares) == (ani_r.value, ares_r.value) == (0, 0.0)
    assert not x_d.cpu().numpy().any() and not x_ref.any()


def _malformed():
    # (name, edit of (rowptr, col, val)) -- each breaks one row of the storage
    def nonmono(rp, c, v):
        rp[5] = rp[7]
    def col_out(rp, c, v):
        c[rp[3]] = 10**6
    def col_negative(rp, c, v):
        c[rp[3] + 1] = -1
    def zero_diag(rp, c, v):
        k = rp[4] + int(np.nonzero(c[rp[4]:rp[5]] == 4)[0][0])
        v[k] = 0.0
    def negative_diag(rp, c, v):
        k = rp[4] + int(np.nonzero(c[rp[4]:rp[5]] == 4)[0][0])
        v[k] = -v[k]
    def no_diag(rp, c, v):
        k = rp[4] + int(np.nonzero(c[rp[4]:rp[5]] == 4)[0][0])
        c[k] = 3
    def end_beyond(rp, c, v):
        rp[-2] = rp[-1] + 5
    return [("non_monotone_rowptr", nonmono), ("column_beyond_n", col_out), ("negative_column", col_negative),
            ("zero_diagonal", zero_diag), ("negative_diagonal", negative_diag), ("missing_diagonal", no_diag),
            ("row_end_beyond_nnz", end_beyond)]


@pytest.mark.parametrize("name,edit", _malformed())
def test_no_alloc_refuses_malformed_rows(oracle, gpu_lib, name, edit):
    import torch
    adr, ci, a, f = _system(oracle)
    n = f.size
    lib = L.lib()
    rowptr, col, val = _full_csr(adr, ci, a)
    rowptr, col, val = rowptr.copy(), col.copy(), val.copy()
    edit(rowptr, col, val)
    dev = torch.device("cuda")
    x0 = np.linspace(-1.0, 1.0, n)
    x_d = torch.from_numpy(x0).to(dev)
    st, ani, ares, _ = _call(lib, n, torch.from_numpy(rowptr).to(dev), torch.from_numpy(col).to(dev),
                             torch.from_numpy(val).to(dev), torch.from_numpy(f).to(dev), x_d)
    assert st == L.BAD_INPUT, name
    assert (ani, ares) == (-1, -7.0)
    assert np.array_equal(x_d.cpu().numpy(), x0)


def test_no_alloc_refuses_a_capturing_stream(oracle, gpu_lib):
    import torch
    adr, ci, a, f = _system(oracle)
    n = f.size
    lib = L.lib()
    rowptr, col, val = _full_csr(adr, ci, a)
    dev = torch.device("cuda")
    rp_d, col_d, val_d = torch.from_numpy(rowptr).to(dev), torch.from_numpy(col).to(dev), torch.from_numpy(val).to(dev)
    f_d = torch.from_numpy(f).to(dev)
    x_d = torch.zeros(n, dtype=torch.float64, device=dev)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            st, _, _, _ = _call(lib, n, rp_d, col_d, val_d, f_d, x_d, stream=C.c_void_p(s.cuda_stream))
        finally:
            g.capture_end()
    assert st == L.BAD_INPUT and "capture" in L.last_error()
    del g
    # the library is still usable afterwards
    st, _, _, _ = _call(lib, n, rp_d, col_d, val_d, f_d, x_d)
    assert st == L.OK


def test_no_alloc_rejects_sizes_beyond_its_array(gpu_lib):
    lib = L.lib()
    n = L.NOALLOC_MAX_N + 1
    st = lib.sgpu_csr_pcg_noalloc_d(n, None, None, None, None, None, 10, 1e-20, 1e-30, 0, None, None, None, None)
    assert st == L.BAD_INPUT
    assert "exceeds" in L.last_error()
