"""The allocation-free residual entry point (xcal_residual_noalloc) is for
callers that cannot allocate device memory when they call it -- a host
framework that owns all device memory in its own pool, or a loop that must not
pay cudaMalloc's synchronisation.  Its partial sums live in a fixed array of the
library.  Checked through the C ABI against the allocating xcal_residual on two
calls in a row (the fixed array keeps the previous call's contents): both run
the same kernels and the same reduction tree, so the results are bitwise equal.
Also its size limit, and its own bounds checks on device CSR arrays (a column
index outside [0, n) and a row range past the end are skipped by the kernel and
reported as XCAL_ERR_ARG).  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import xcal as X
from xcal import _abi, cases

pytestmark = pytest.mark.gpu


def _system(n_side, seed):
    """A pressure system of the cavity after 3 SIMPLE iterations, as CSR.  The
    oracle stores the matrix column-compressed (the reference's CSC); its
    column pointers, row indices and values are the CSR arrays of the
    transposed matrix, which is what both entry points are given."""
    mesh, model, config, pref = cases.cavity2d(n_side, iterations=3)
    om = O.from_mesh2(mesh)
    case, keep = X.make_case(model, config, pref)
    U, p = cases.fields(model)
    out = O.run(om, case, 3, U, p, want_eqns=True)
    colptr, rowval = om.pattern()
    n = len(colptr) - 1
    rng = np.random.default_rng(seed)
    return (colptr.astype(np.int32), rowval.astype(np.int32), out["Ap"], rng.standard_normal(n),
            rng.standard_normal(n))


def test_residual_noalloc_matches_allocating_entry():
    import torch
    lib = _abi.load()
    h = C.c_void_p()
    _abi.check(lib.xcal_ctx_create(0, 0, C.byref(h)))
    try:
        for call, (side, seed) in enumerate(((40, 1), (23, 2))):   # two calls, different sizes
            rp, col, val, x, b = _system(side, seed)
            n = len(b)
            R_ref = np.zeros(1)
            _abi.check(lib.xcal_residual(h, n, _abi.i32ptr(rp), _abi.i32ptr(col), _abi.dptr(val),
                                         _abi.dptr(x), _abi.dptr(b), _abi.dptr(R_ref)), h)
            dev = torch.device("cuda", 0)
            t = {k: torch.from_numpy(v).to(dev) for k, v in
                 dict(rp=rp, col=col, val=val, x=x, b=b).items()}
            R = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            ptr = lambda a: C.c_void_p(a.data_ptr())
            _abi.check(lib.xcal_residual_noalloc(h, n, ptr(t["rp"]), ptr(t["col"]), ptr(t["val"]),
                                                 ptr(t["x"]), ptr(t["b"]), ptr(R)), h)
            got = float(R.cpu()[0])
            assert got == R_ref[0], (call, got, R_ref[0])   # same kernels, same reduction order
    finally:
        lib.xcal_ctx_destroy(h)


def test_residual_noalloc_rejects_oversized_input():
    lib = _abi.load()
    h = C.c_void_p()
    _abi.check(lib.xcal_ctx_create(0, 0, C.byref(h)))
    try:
        dummy = C.c_void_p(1)
        st = lib.xcal_residual_noalloc(h, 65536 * 256 + 1, dummy, dummy, dummy, dummy, dummy, dummy)
        assert st == -1
        buf = C.create_string_buffer(256)
        lib.xcal_last_error(h, buf, 256)
        assert b"exceeds the allocation-free limit" in buf.value
    finally:
        lib.xcal_ctx_destroy(h)


def test_residual_noalloc_reports_out_of_range_csr():
    """Device arrays cannot be validated on the host: the kernel reads only
    inside the CSR's bounds, skips what lies outside and the call returns
    XCAL_ERR_ARG; the same context then computes a valid system again."""
    import torch
    lib = _abi.load()
    h = C.c_void_p()
    _abi.check(lib.xcal_ctx_create(0, 0, C.byref(h)))
    try:
        rp, col, val, x, b = _system(12, 3)
        n = len(b)
        dev = torch.device("cuda", 0)
        ptr = lambda a: C.c_void_p(a.data_ptr())
        R = torch.zeros(1, dtype=torch.float64, device=dev)
        tv, tx, tb = (torch.from_numpy(v).to(dev) for v in (val, x, b))
        bad_col = col.copy()
        bad_col[5] = n + 1000                       # column outside [0, n)
        bad_rp = rp.copy()
        bad_rp[7] = rp[-1] + 50                     # row range past the end of the arrays
        for rpa, cola, what in ((rp, bad_col, b"column index"), (bad_rp, col, b"row_ptr range")):
            trp, tcol = torch.from_numpy(rpa).to(dev), torch.from_numpy(cola).to(dev)
            torch.cuda.synchronize()
            st = lib.xcal_residual_noalloc(h, n, ptr(trp), ptr(tcol), ptr(tv), ptr(tx), ptr(tb), ptr(R))
            assert st == -1
            buf = C.create_string_buffer(256)
            lib.xcal_last_error(h, buf, 256)
            assert what in buf.value, buf.value
        trp, tcol = torch.from_numpy(rp).to(dev), torch.from_numpy(col).to(dev)
        torch.cuda.synchronize()
        _abi.check(lib.xcal_residual_noalloc(h, n, ptr(trp), ptr(tcol), ptr(tv), ptr(tx), ptr(tb), ptr(R)), h)
        R_ref = np.zeros(1)
        _abi.check(lib.xcal_residual(h, n, _abi.i32ptr(rp), _abi.i32ptr(col), _abi.dptr(val), _abi.dptr(x),
                                     _abi.dptr(b), _abi.dptr(R_ref)), h)
        assert float(R.cpu()[0]) == R_ref[0]
    finally:
        lib.xcal_ctx_destroy(h)
