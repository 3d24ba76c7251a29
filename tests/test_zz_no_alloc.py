"""The no-allocation solver entry point against the regular drop-in.

sgpu_csr_pcg_noalloc_d serves callers that cannot allocate GPU memory while
they solve (an application whose allocator owns the whole device memory pool,
or one that must not call cudaMalloc/cudaFree because they synchronise the
device).  Its work vectors live in a static device array of the library, so
this test checks, through the C ABI, that two calls in a row (the second
reusing the array the first left behind) give the same solution as the
allocating drop-in sgpu_scr_cg_prec, within the FP64 parity tolerance used
elsewhere in the tests, and that sizes beyond the array are refused.

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


def test_no_alloc_pcg_matches_drop_in_twice(oracle, gpu_lib):
    import torch
    m = decks.cantilever_hex(20, 4, 4)
    adr, ci, a = oracle.assemble(m, sym=True)
    f = oracle.load_vector(m)
    n = f.size
    lib = L.lib()
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
        ani, ares, its = C.c_int64(-1), C.c_double(0.0), C.c_int64(0)
        st = lib.sgpu_csr_pcg_noalloc_d(n, C.c_void_p(rp_d.data_ptr()), C.c_void_p(col_d.data_ptr()),
                                        C.c_void_p(val_d.data_ptr()), C.c_void_p(f_d.data_ptr()),
                                        C.c_void_p(x_d.data_ptr()), 20000, 1e-20, 1e-30, 0, None,
                                        C.byref(ani), C.byref(ares), C.byref(its))
        assert st == L.OK, L.last_error()
        torch.cuda.synchronize()
        x = x_d.cpu().numpy()
        assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) <= 1e-8
        assert abs(ani.value - ani_r.value) <= 2 and its.value == ani.value + 1


def test_no_alloc_rejects_sizes_beyond_its_array(gpu_lib):
    lib = L.lib()
    n = 131072 + 1
    st = lib.sgpu_csr_pcg_noalloc_d(n, None, None, None, None, None, 10, 1e-20, 1e-30, 0, None, None, None, None)
    assert st == L.BAD_INPUT
    assert "exceeds" in L.last_error()
