"""The allocation-free H_eff entry point agrees with the arena-backed one and
with the CPU oracle.

`nc_heff_apply_dev_noalloc` serves callers that cannot let the library
allocate device memory (fixed memory budgets, code where a cudaMalloc or
cudaFree would stall the device); it takes its scratch from a fixed 64 MiB
array compiled into the library.  Both entry points are called through the
C-ABI on the same device inputs, twice in a row with fresh inputs (the
shared array keeps the previous call's contents), and must agree to the
FP64 tolerance of the other contraction tests (1e-12 relative); the first
call is also checked against the oracle's restatement of the reference's
product (core.f95:2529-2556).  The capacity check is exercised at its edge:
a call that fills the array exactly runs, one that needs one more row is
rejected.  This file is collected last so that a failure here does not
hide the other tests.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12
CAPACITY = 64 << 20


def _call(fn, bl, br, cl, cr, d, nnz, bufs, *extra):
    L, R, x, y, W, idx = bufs
    return fn(bl, br, cl, cr, d, nnz, ct.c_void_p(idx.data_ptr()), ct.c_void_p(W.data_ptr()),
              ct.c_void_p(L.data_ptr()), ct.c_void_p(R.data_ptr()), ct.c_void_p(x.data_ptr()),
              ct.c_void_p(y.data_ptr()), *extra)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).cuda()


def test_noalloc_heff_matches_arena_path_and_oracle():
    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators
    from oracle import core

    stream = torch.cuda.current_stream()
    assert nb.lib.nc_set_stream(ct.c_void_p(stream.cuda_stream)) == 0
    op = operators.heisenberg(4)[1]
    W = _dev(op.W)
    idx = _dev(op.idx.astype(np.int32))
    for call, chi in enumerate((96, 160)):  # two calls in a row, different sizes and inputs
        rng = np.random.default_rng(100 + call)
        Lh = np.asfortranarray(rng.standard_normal((chi, chi, op.cl)) + 1j * rng.standard_normal((chi, chi, op.cl)))
        Rh = np.asfortranarray(rng.standard_normal((chi, chi, op.cr)) + 1j * rng.standard_normal((chi, chi, op.cr)))
        xh = np.asfortranarray(rng.standard_normal((chi, chi, op.d)) + 1j * rng.standard_normal((chi, chi, op.d)))
        L, R, x = _dev(Lh), _dev(Rh), _dev(xh)
        y_arena = torch.empty_like(x)
        y_fixed = torch.full_like(x, float("nan"))
        assert _call(nb.lib.nc_heff_apply_dev, chi, chi, op.cl, op.cr, op.d, op.nnz,
                     (L, R, x, y_arena, W, idx)) == 0
        st = _call(nb.lib.nc_heff_apply_dev_noalloc, chi, chi, op.cl, op.cr, op.d, op.nnz,
                   (L, R, x, y_fixed, W, idx), ct.c_void_p(stream.cuda_stream))
        assert st == 0, nb.lib.nc_last_error()
        torch.cuda.synchronize()
        err = (torch.linalg.norm(y_fixed - y_arena) / torch.linalg.norm(y_arena)).item()
        assert err <= TOL, err
        if call == 0:
            want = core.apply_heff(chi, chi, op.cl, op.cr, op.d, Lh, op.idx, op.W, Rh, xh).ravel(order="F")
            got = y_fixed.cpu().numpy()
            assert np.linalg.norm(got - want) <= TOL * np.linalg.norm(want)


def test_noalloc_capacity_edge():
    """bl=br=512, d=2, cl=cr=4 needs 16*512*512*2*(4+4) bytes = 64 MiB exactly."""
    import torch

    import nutcracker_b200 as nb
    from gpu_util import random_mpo_site

    rng = np.random.default_rng(7)
    cl = cr = 4
    d, nnz = 2, 6
    idx_h, W_h = random_mpo_site(rng, cl, cr, d, nnz)
    W, idx = _dev(W_h), _dev(idx_h.astype(np.int32))
    stream = torch.cuda.current_stream()
    assert nb.lib.nc_set_stream(ct.c_void_p(stream.cuda_stream)) == 0
    bl = 512
    for br, fits in ((512, True), (513, False)):
        need = 16 * br * bl * d * (cl + cr)
        assert (need <= CAPACITY) == fits and (br == 512) == (need == CAPACITY)
        g = torch.Generator(device="cuda").manual_seed(br)
        L = torch.randn(bl * bl * cl, dtype=torch.complex128, device="cuda", generator=g)
        R = torch.randn(br * br * cr, dtype=torch.complex128, device="cuda", generator=g)
        x = torch.randn(br * bl * d, dtype=torch.complex128, device="cuda", generator=g)
        y_fixed = torch.full_like(x, float("nan"))
        st = _call(nb.lib.nc_heff_apply_dev_noalloc, bl, br, cl, cr, d, nnz,
                   (L, R, x, y_fixed, W, idx), ct.c_void_p(stream.cuda_stream))
        if not fits:
            assert st != 0 and b"64 MiB" in nb.lib.nc_last_error()
            assert torch.isnan(y_fixed).all().item()   # nothing was launched
            continue
        assert st == 0, nb.lib.nc_last_error()
        y_arena = torch.empty_like(x)
        assert _call(nb.lib.nc_heff_apply_dev, bl, br, cl, cr, d, nnz, (L, R, x, y_arena, W, idx)) == 0
        torch.cuda.synchronize()
        err = (torch.linalg.norm(y_fixed - y_arena) / torch.linalg.norm(y_arena)).item()
        assert err <= TOL, err


def test_noalloc_rejects_oversized_and_wrapping_calls():
    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators

    op = operators.heisenberg(4)[1]
    dummy = torch.zeros(1, dtype=torch.complex128, device="cuda")
    p = ct.c_void_p(dummy.data_ptr())
    chi = 600  # needs 16*(2*chi^2*5*2) bytes = 115 MB > 64 MiB
    st = nb.lib.nc_heff_apply_dev_noalloc(chi, chi, op.cl, op.cr, op.d, op.nnz, p, p, p, p, p, p, None)
    assert st != 0
    assert b"64 MiB" in nb.lib.nc_last_error()
    # products that wrap a 64-bit count, or dimensions past INT_MAX, are rejected too
    for dims in ((2 ** 31, 2 ** 31, 1, 1, 4), (2 ** 32 - 1, 2 ** 32 - 1, 2 ** 32 - 1, 2 ** 32 - 1, 4),
                 (1, 1, 1, 1, 0)):
        st = nb.lib.nc_heff_apply_dev_noalloc(*[ct.c_uint32(v) for v in dims], ct.c_uint32(1),
                                              p, p, p, p, p, p, None)
        assert st != 0, dims
