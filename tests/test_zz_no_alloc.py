"""The allocation-free residual entry point (xcal_residual_noalloc) is for
callers that cannot allocate device memory when they call it -- a host
framework that owns all device memory in its own pool, or a loop that must not
pay cudaMalloc's synchronisation.  Its partial sums live in a fixed array of the
library.  Checked through the C ABI against the allocating xcal_residual on two
calls in a row (the fixed array keeps the previous call's contents), and for
its size limit.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import xcal as X
from xcal import _abi, cases

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _system(n_side, seed):
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
            assert abs(got - R_ref[0]) <= TOL * abs(R_ref[0]), (call, got, R_ref[0])
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
