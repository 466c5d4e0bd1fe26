"""The allocation-free H_eff entry point agrees with the arena-backed one.

`nc_heff_apply_dev_noalloc` serves callers that cannot let the library
allocate device memory (fixed memory budgets, code where a cudaMalloc or
cudaFree would stall the device); it takes its scratch from a fixed 64 MiB
array compiled into the library.  Both entry points are called through the
C-ABI on the same device inputs, twice in a row with fresh inputs (the
shared array keeps the previous call's contents), and must agree to the
FP64 tolerance of the other contraction tests (1e-12 relative).  This file
is collected last so that a failure here does not hide the other tests.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _call(nb, fn, chi, op, bufs, *extra):
    d, cl, cr = op.d, op.cl, op.cr
    L, R, x, y, W, idx = bufs
    return fn(chi, chi, cl, cr, d, op.nnz, ct.c_void_p(idx.data_ptr()), ct.c_void_p(W.data_ptr()),
              ct.c_void_p(L.data_ptr()), ct.c_void_p(R.data_ptr()), ct.c_void_p(x.data_ptr()),
              ct.c_void_p(y.data_ptr()), *extra)


def test_noalloc_heff_matches_arena_path():
    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators

    stream = torch.cuda.current_stream()
    assert nb.lib.nc_set_stream(ct.c_void_p(stream.cuda_stream)) == 0
    op = operators.heisenberg(4)[1]
    W = torch.from_numpy(op.W.ravel(order="F")).cuda()
    idx = torch.from_numpy(op.idx.ravel(order="F").astype(np.int32)).cuda()
    for call, chi in enumerate((96, 160)):  # two calls in a row, different sizes and inputs
        g = torch.Generator(device="cuda").manual_seed(100 + call)
        L = torch.randn(chi * chi * op.cl, dtype=torch.complex128, device="cuda", generator=g)
        R = torch.randn(chi * chi * op.cr, dtype=torch.complex128, device="cuda", generator=g)
        x = torch.randn(chi * chi * op.d, dtype=torch.complex128, device="cuda", generator=g)
        y_arena = torch.empty_like(x)
        y_fixed = torch.full_like(x, float("nan"))
        assert _call(nb, nb.lib.nc_heff_apply_dev, chi, op, (L, R, x, y_arena, W, idx)) == 0
        st = _call(nb, nb.lib.nc_heff_apply_dev_noalloc, chi, op, (L, R, x, y_fixed, W, idx),
                   ct.c_void_p(stream.cuda_stream))
        assert st == 0, nb.lib.nc_last_error()
        torch.cuda.synchronize()
        err = (torch.linalg.norm(y_fixed - y_arena) / torch.linalg.norm(y_arena)).item()
        assert err <= TOL, err


def test_noalloc_rejects_oversized_calls():
    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators

    op = operators.heisenberg(4)[1]
    chi = 600  # needs 16*(2*chi^2*5*2) bytes = 115 MB > 64 MiB
    dummy = torch.zeros(1, dtype=torch.complex128, device="cuda")
    p = ct.c_void_p(dummy.data_ptr())
    st = nb.lib.nc_heff_apply_dev_noalloc(chi, chi, op.cl, op.cr, op.d, op.nnz, p, p, p, p, p, p, None)
    assert st != 0
    assert b"64 MiB" in nb.lib.nc_last_error()
