"""tcgen05 3xTF32 tensor-core path against FP64.

`nc_tc_zgemm_dev` is the complex GEMM under the precision form (each operand
split into two TF32 halves, three products, FP32 accumulation in tensor
memory); `nc_heff_apply_mixed_dev` is the precision-form H_eff product.  Both
are compared with FP64 results on the same device inputs: the GEMM with
torch's complex128 matmul, the H_eff product with the FP64 entry point
`nc_heff_apply_dev` (itself pinned to the oracle in test_gpu_contract.py).
Sizes cover full tiles, ragged M/N/K edges, a single row and a long K.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_3X = 2e-6     # relative Frobenius error of 3xTF32 (chunked FP32 accumulation); measured ~7e-7
TOL_1X = 1e-2     # one TF32 product (10-bit mantissa): loose upper bound


def _p(t):
    return ct.c_void_p(t.data_ptr())


@pytest.fixture(autouse=True)
def _on_torch_stream():
    """Run the library on torch's current stream, so it sees torch's inputs."""
    import torch

    import nutcracker_b200 as nb

    assert nb.lib.nc_set_stream(ct.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    yield
    torch.cuda.synchronize()
    assert nb.lib.nc_use_own_stream() == 0


def _rel(got, want):
    import torch
    return (torch.linalg.norm(got - want) / torch.linalg.norm(want)).item()


@pytest.mark.parametrize("M,N,K", [(128, 128, 16), (256, 128, 64), (200, 70, 33), (1, 5, 3),
                                   (300, 260, 1000), (64, 1, 257)])
def test_tc_zgemm_matches_fp64(M, N, K):
    import torch

    import nutcracker_b200 as nb

    g = torch.Generator(device="cuda").manual_seed(7 * M + 3 * N + K)
    A_cm = torch.randn(K, M, dtype=torch.complex128, device="cuda", generator=g)   # column-major M x K
    B_cm = torch.randn(N, K, dtype=torch.complex128, device="cuda", generator=g)   # column-major K x N
    ref = A_cm.T @ B_cm.T
    errs = []
    for three in (1, 0):
        C_cm = torch.full((N, M), float("nan"), dtype=torch.complex128, device="cuda")
        st = nb.lib.nc_tc_zgemm_dev(M, N, K, _p(A_cm), _p(B_cm), _p(C_cm), three)
        assert st == 0, nb.lib.nc_last_error()
        errs.append(_rel(C_cm.T, ref))
    err3, err1 = errs
    assert err3 <= TOL_3X, err3
    assert err1 <= TOL_1X, err1
    assert err3 * 10 < err1, (err3, err1)   # the small halves carry real precision


@pytest.mark.parametrize("bl,br", [(96, 96), (40, 72), (130, 33)])
def test_mixed_heff_matches_fp64(bl, br):
    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators

    op = operators.heisenberg(4)[1]
    W = torch.from_numpy(op.W.ravel(order="F")).cuda()
    idx = torch.from_numpy(op.idx.ravel(order="F").astype(np.int32)).cuda()
    g = torch.Generator(device="cuda").manual_seed(bl * 1000 + br)
    L = torch.randn(bl * bl * op.cl, dtype=torch.complex128, device="cuda", generator=g)
    R = torch.randn(br * br * op.cr, dtype=torch.complex128, device="cuda", generator=g)
    x = torch.randn(br * bl * op.d, dtype=torch.complex128, device="cuda", generator=g)
    y64 = torch.empty_like(x)
    ymx = torch.full_like(x, float("nan"))
    args = (bl, br, op.cl, op.cr, op.d, op.nnz, _p(idx), _p(W), _p(L), _p(R), _p(x))
    assert nb.lib.nc_heff_apply_dev(*args, _p(y64)) == 0, nb.lib.nc_last_error()
    assert nb.lib.nc_heff_apply_mixed_dev(*args, _p(ymx)) == 0, nb.lib.nc_last_error()
    torch.cuda.synchronize()
    err = _rel(ymx, y64)
    assert err <= TOL_3X, err


@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("bl,br", [(96, 96), (40, 72), (130, 33)])
def test_mixed_environment_matches_fp64(side, bl, br):
    import torch

    import nutcracker_b200 as nb
    from nutcracker_b200 import operators

    op = operators.heisenberg(4)[1]
    W = torch.from_numpy(op.W.ravel(order="F")).cuda()
    idx = torch.from_numpy(op.idx.ravel(order="F").astype(np.int32)).cuda()
    g = torch.Generator(device="cuda").manual_seed(side * 7 + bl * 1000 + br)
    n_in, n_out = (bl * bl * op.cl, br * br * op.cr) if side == 0 else (br * br * op.cr, bl * bl * op.cl)
    env = torch.randn(n_in, dtype=torch.complex128, device="cuda", generator=g)
    psi = torch.randn(br * bl * op.d, dtype=torch.complex128, device="cuda", generator=g)
    o64 = torch.empty(n_out, dtype=torch.complex128, device="cuda")
    omx = torch.full_like(o64, float("nan"))
    args = (bl, br, op.cl, op.cr, op.d, op.nnz, _p(idx), _p(W), _p(env), _p(psi))
    assert nb.lib.nc_env_update_dev(side, 0, *args, _p(o64)) == 0, nb.lib.nc_last_error()
    assert nb.lib.nc_env_update_dev(side, 1, *args, _p(omx)) == 0, nb.lib.nc_last_error()
    torch.cuda.synchronize()
    err = _rel(omx, o64)
    assert err <= TOL_3X, err


def test_bounded_wait_reports_timeout_and_context_recovers():
    """The failure path of the tcgen05 GEMM's bounded waits, without a fault:
    with the test switch, tile (0,0,0) leaves its first K stage unloaded, its
    MMA issuer's wait runs out after the (shortened, 2 ms) limit, the kernel
    stops issuing, frees its tensor memory and returns, and the host call
    reports NC_ERR_TIMEOUT (1004).  The next GEMM on the same context, with
    the default limit restored, is correct."""
    import torch

    import nutcracker_b200 as nb

    M, N, K = 128, 128, 64
    g = torch.Generator(device="cuda").manual_seed(5)
    A_cm = torch.randn(K, M, dtype=torch.complex128, device="cuda", generator=g)
    B_cm = torch.randn(N, K, dtype=torch.complex128, device="cuda", generator=g)
    C_cm = torch.zeros((N, M), dtype=torch.complex128, device="cuda")
    assert nb.lib.nc_test_tc32_wait(ct.c_uint64(2_000_000), 1) == 0
    try:
        st = nb.lib.nc_tc_zgemm_dev(M, N, K, _p(A_cm), _p(B_cm), _p(C_cm), 1)
        msg = nb.lib.nc_last_error()   # read before the restoring call resets the status
    finally:
        assert nb.lib.nc_test_tc32_wait(ct.c_uint64(2_000_000_000), 0) == 0
    assert st == 1004, (st, msg)
    assert b"time limit" in msg
    st = nb.lib.nc_tc_zgemm_dev(M, N, K, _p(A_cm), _p(B_cm), _p(C_cm), 1)
    assert st == 0, nb.lib.nc_last_error()
    assert _rel(C_cm.T, A_cm.T @ B_cm.T) <= TOL_3X
